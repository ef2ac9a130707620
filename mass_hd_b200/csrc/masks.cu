// Division / death masks on the device: SetMasks of the lyotropic division
// models (src/models/lyotropic-with-division.cpp:35-106) with the random
// numbers drawn by the caller.
//
// The reference walks the domain in site order k = y + LY*x; every site with
// phi >= .5 (a candidate) draws one random_real() and becomes a centre when
// the draw is below rate*phi*(1 - phi/phi_critical) (division) or rate*phi
// (death); then every site within the circle test of a centre is masked.
// Here
//  1. cand_count_kernel counts the candidates per block of 1024 sites,
//  2. scan_kernel turns the counts into exclusive block offsets and the
//     total (the number of draws the caller must supply),
//  3. center_kernel gives every candidate its rank (block offset + ballot
//     prefix inside the block) and compares draws[rank] with its threshold,
//  4. stamp_kernel writes each centre's disk, offsets (dx, dy) with
//     dx^2 + dy^2 <= ceil(radius^2) on the torus (the same set as the
//     reference's minimum-image test of every site against every centre),
//  5. rate_kernel forms alpha*division_mask - beta*death_mask in the
//     source plane the step kernels read.
// Compiled with --fmad=false: the thresholds are rounded as the reference
// rounds them.
#include "masks.cuh"

#include <cmath>

namespace mlb {
namespace {

constexpr int MB = 1024;   // sites per block in the counting/ranking kernels

template<typename T>
__device__ __forceinline__ double phi_at(const MaskView<T>& v, long long k)
{
  const int x = static_cast<int>(k / v.LY), y = static_cast<int>(k % v.LY);
  return static_cast<double>(v.phi[(y + v.g) + static_cast<long long>(v.EY)*(x + v.g)]);
}

template<typename T>
__global__ void __launch_bounds__(MB)
cand_count_kernel(MaskView<T> v, int* block_cnt)
{
  const long long N = static_cast<long long>(v.LX)*v.LY;
  const long long k = static_cast<long long>(blockIdx.x)*MB + threadIdx.x;
  const int flag = k < N && phi_at(v, k) >= .5;
  const int c = __syncthreads_count(flag);
  if(threadIdx.x == 0) block_cnt[blockIdx.x] = c;
}

// one block: exclusive offsets of nb counts, and their total
__global__ void __launch_bounds__(MB)
scan_kernel(int nb, const int* __restrict__ cnt, long long* __restrict__ off, long long* total)
{
  __shared__ long long part[MB];
  const int per = (nb + MB - 1)/MB;
  const int lo = threadIdx.x*per, hi = min(nb, lo + per);
  long long s = 0;
  for(int i = lo; i < hi; ++i) s += cnt[i];
  part[threadIdx.x] = s;
  __syncthreads();
  // inclusive scan of the per-thread sums (Hillis-Steele)
  for(int d = 1; d < MB; d <<= 1)
  {
    const long long add = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for(int i = lo; i < hi; ++i)
  {
    off[i] = run;
    run += cnt[i];
  }
  if(threadIdx.x == MB - 1) *total = part[MB - 1];
}

template<typename T>
__global__ void __launch_bounds__(MB)
center_kernel(MaskView<T> v, const long long* __restrict__ off, const double* __restrict__ draws,
              long long ndraws, double coef, double phi_critical, int division,
              unsigned char* __restrict__ center)
{
  __shared__ int warp_cnt[MB/32];
  const long long N = static_cast<long long>(v.LX)*v.LY;
  const long long k = static_cast<long long>(blockIdx.x)*MB + threadIdx.x;
  const double p = k < N ? phi_at(v, k) : 0.;
  const bool flag = k < N && p >= .5;
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned ballot = __ballot_sync(0xffffffffu, flag);
  if(lane == 0) warp_cnt[warp] = __popc(ballot);
  __syncthreads();
  int before = 0;
  for(unsigned w = 0; w < warp; ++w) before += warp_cnt[w];
  before += __popc(ballot & ((1u << lane) - 1u));
  if(k >= N) return;
  unsigned char c = 0;
  if(flag)
  {
    const long long rank = off[blockIdx.x] + before;
    if(rank < ndraws)
    {
      // src/models/lyotropic-with-division.cpp:47 (division), :83 (death)
      const double thr = division ? coef*p*(1 - p/phi_critical) : coef*p;
      c = draws[rank] < thr;
    }
  }
  center[k] = c;
}

// The same centre test with the uniforms taken from a queue on the device:
// the draws of this mask start `kslot` candidate counts past the queue head
// (division first, then death, as the reference draws them). A draw past
// what the caller has supplied sets *err and makes no centre.
template<typename T>
__global__ void __launch_bounds__(MB)
center_queue_kernel(MaskView<T> v, const long long* __restrict__ off,
                    const double* __restrict__ queue, long long qcap,
                    const long long* __restrict__ head, const long long* __restrict__ total,
                    int kslot, long long supplied, double coef, double phi_critical,
                    int division, unsigned char* __restrict__ center, int* err)
{
  __shared__ int warp_cnt[MB/32];
  const long long N = static_cast<long long>(v.LX)*v.LY;
  const long long k = static_cast<long long>(blockIdx.x)*MB + threadIdx.x;
  const double p = k < N ? phi_at(v, k) : 0.;
  const bool flag = k < N && p >= .5;
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned ballot = __ballot_sync(0xffffffffu, flag);
  if(lane == 0) warp_cnt[warp] = __popc(ballot);
  __syncthreads();
  int before = 0;
  for(unsigned w = 0; w < warp; ++w) before += warp_cnt[w];
  before += __popc(ballot & ((1u << lane) - 1u));
  if(k >= N) return;
  unsigned char c = 0;
  if(flag)
  {
    const long long idx = *head + kslot*(*total) + off[blockIdx.x] + before;
    if(idx < supplied)
    {
      const double thr = division ? coef*p*(1 - p/phi_critical) : coef*p;
      c = queue[idx % qcap] < thr;
    }
    else atomicOr(err, 1);
  }
  center[k] = c;
}

__global__ void advance_head_kernel(long long* head, const long long* total, int nkinds)
{
  if(blockIdx.x == 0 && threadIdx.x == 0) *head += nkinds*(*total);
}

__global__ void stamp_kernel(int LX, int LY, const unsigned char* __restrict__ center,
                             unsigned char* __restrict__ mask, double r2, int R)
{
  const long long N = static_cast<long long>(LX)*LY;
  for(long long k = static_cast<long long>(blockIdx.x)*blockDim.x + threadIdx.x; k < N;
      k += static_cast<long long>(gridDim.x)*blockDim.x)
  {
    if(!center[k]) continue;
    const int cx = static_cast<int>(k / LY), cy = static_cast<int>(k % LY);
    for(int dx = -R; dx <= R; ++dx)
    {
      const int x = ((cx + dx) % LX + LX) % LX;
      for(int dy = -R; dy <= R; ++dy)
      {
        if(static_cast<double>(dx*dx + dy*dy) > r2) continue;
        const int y = ((cy + dy) % LY + LY) % LY;
        mask[y + static_cast<long long>(LY)*x] = 1;   // every writer stores 1
      }
    }
  }
}

template<typename T>
__global__ void rate_kernel(int LX, int LY, int g, int EY, const unsigned char* __restrict__ dm,
                            const unsigned char* __restrict__ de, double alpha, double beta,
                            T* __restrict__ src)
{
  const long long N = static_cast<long long>(LX)*LY;
  for(long long k = static_cast<long long>(blockIdx.x)*blockDim.x + threadIdx.x; k < N;
      k += static_cast<long long>(gridDim.x)*blockDim.x)
  {
    const int x = static_cast<int>(k / LY), y = static_cast<int>(k % LY);
    // alpha*division_m - beta*death_m (src/models/lyotropic-with-division.cpp:121)
    const double r = alpha*(dm[k] ? 1. : 0.) - beta*(de[k] ? 1. : 0.);
    src[(y + g) + static_cast<long long>(EY)*(x + g)] = static_cast<T>(r);
  }
}

inline int grid_for(long long n)
{
  const long long b = (n + 255)/256;
  return static_cast<int>(b < 1 ? 1 : (b > 8192 ? 8192 : b));
}

} // namespace

int mask_blocks(long long nsites) { return static_cast<int>((nsites + MB - 1)/MB); }

template<typename T>
cudaError_t mask_count(const MaskView<T>& v, const MaskScratch& s, cudaStream_t st)
{
  const long long N = static_cast<long long>(v.LX)*v.LY;
  const int nb = mask_blocks(N);
  cand_count_kernel<T><<<nb, MB, 0, st>>>(v, s.block_cnt);
  scan_kernel<<<1, MB, 0, st>>>(nb, s.block_cnt, s.block_off, s.total);
  return cudaGetLastError();
}

template<typename T>
cudaError_t mask_draw(const MaskView<T>& v, const MaskScratch& s, int kind, long long ndraws,
                      double coef, double phi_critical, double radius, cudaStream_t st)
{
  const long long N = static_cast<long long>(v.LX)*v.LY;
  const int nb = mask_blocks(N);
  center_kernel<T><<<nb, MB, 0, st>>>(v, s.block_off, s.draws, ndraws, coef, phi_critical,
                                      kind == 0 ? 1 : 0, s.center);
  unsigned char* mask = s.mask[kind];
  cudaError_t e = cudaMemsetAsync(mask, 0, N, st);
  if(e != cudaSuccess) return e;
  // ceil(radius^2) as the reference computes it (:60, :96)
  const double r2 = std::ceil(radius*radius);
  if(r2 >= 0)
  {
    const int R = static_cast<int>(std::floor(std::sqrt(r2)));
    stamp_kernel<<<grid_for(N), 256, 0, st>>>(v.LX, v.LY, s.center, mask, r2, R);
  }
  return cudaGetLastError();
}

template<typename T>
cudaError_t mask_draw_queued(const MaskView<T>& v, const MaskScratch& s, const MaskQueue& q,
                             int kind, int kslot, double coef, double phi_critical, double radius,
                             int* err, cudaStream_t st)
{
  const long long N = static_cast<long long>(v.LX)*v.LY;
  const int nb = mask_blocks(N);
  center_queue_kernel<T><<<nb, MB, 0, st>>>(v, s.block_off, q.buf, q.cap, q.head, s.total, kslot,
                                            q.supplied, coef, phi_critical, kind == 0 ? 1 : 0,
                                            s.center, err);
  unsigned char* mask = s.mask[kind];
  cudaError_t e = cudaMemsetAsync(mask, 0, N, st);
  if(e != cudaSuccess) return e;
  const double r2 = std::ceil(radius*radius);
  if(r2 >= 0)
  {
    const int R = static_cast<int>(std::floor(std::sqrt(r2)));
    stamp_kernel<<<grid_for(N), 256, 0, st>>>(v.LX, v.LY, s.center, mask, r2, R);
  }
  return cudaGetLastError();
}

cudaError_t mask_queue_advance(const MaskScratch& s, const MaskQueue& q, int nkinds,
                               cudaStream_t st)
{
  advance_head_kernel<<<1, 32, 0, st>>>(q.head, s.total, nkinds);
  return cudaGetLastError();
}

template<typename T>
cudaError_t mask_rate(int LX, int LY, int g, int EY, const MaskScratch& s, double alpha,
                      double beta, T* src, cudaStream_t st)
{
  const long long N = static_cast<long long>(LX)*LY;
  rate_kernel<T><<<grid_for(N), 256, 0, st>>>(LX, LY, g, EY, s.mask[0], s.mask[1], alpha, beta, src);
  return cudaGetLastError();
}

template cudaError_t mask_count<double>(const MaskView<double>&, const MaskScratch&, cudaStream_t);
template cudaError_t mask_count<float>(const MaskView<float>&, const MaskScratch&, cudaStream_t);
template cudaError_t mask_draw<double>(const MaskView<double>&, const MaskScratch&, int, long long,
                                       double, double, double, cudaStream_t);
template cudaError_t mask_draw<float>(const MaskView<float>&, const MaskScratch&, int, long long,
                                      double, double, double, cudaStream_t);
template cudaError_t mask_draw_queued<double>(const MaskView<double>&, const MaskScratch&,
                                              const MaskQueue&, int, int, double, double, double,
                                              int*, cudaStream_t);
template cudaError_t mask_draw_queued<float>(const MaskView<float>&, const MaskScratch&,
                                             const MaskQueue&, int, int, double, double, double,
                                             int*, cudaStream_t);
template cudaError_t mask_rate<double>(int, int, int, int, const MaskScratch&, double, double,
                                       double*, cudaStream_t);
template cudaError_t mask_rate<float>(int, int, int, int, const MaskScratch&, double, double,
                                      float*, cudaStream_t);

} // namespace mlb
