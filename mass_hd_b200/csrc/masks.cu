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
// A draw from uniforms queued on the device ahead of need
// (queued_draw_kernel) does the same in one cooperative launch.
// Compiled with --fmad=false: the thresholds are rounded as the reference
// rounds them.
#include "masks.cuh"

#include <cmath>

#include <cooperative_groups.h>

namespace mlb {
namespace {

constexpr int MB = 1024;   // sites per block in the counting/ranking kernels

template<typename T>
__device__ __forceinline__ double phi_at(const MaskView<T>& v, long long k)
{
  // without a ghost ring the plane is in site order already
  if(v.g == 0 && v.EY == v.LY) return static_cast<double>(v.phi[k]);
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

// The circle of centre site k as stamp_kernel writes it (every writer
// stores 1), by a warp: lane l takes the offsets l, l+32, ... of the
// (2R+1)^2 square.
__device__ __forceinline__ void stamp_circle_warp(int LX, int LY, long long k,
                                                  unsigned char* __restrict__ mask, double r2,
                                                  int R, unsigned lane)
{
  const int cx = static_cast<int>(k / LY), cy = static_cast<int>(k % LY);
  const int D = 2*R + 1;
  for(int o = static_cast<int>(lane); o < D*D; o += 32)
  {
    const int dx = o/D - R, dy = o - (o/D)*D - R;
    if(static_cast<double>(dx*dx + dy*dy) > r2) continue;
    const int x = ((cx + dx) % LX + LX) % LX;
    const int y = ((cy + dy) % LY + LY) % LY;
    mask[y + static_cast<long long>(LY)*x] = 1;
  }
}

// A queued draw in one cooperative launch (blocks of MB threads, each block
// walking chunks of MB sites). Phases, separated by grid barriers:
//  1. candidates per chunk; the masks being redrawn are cleared,
//  2. every block forms the exclusive chunk offsets it needs and the total
//     from all chunk counts (as scan_kernel), then the centres of its
//     chunks: a candidate's draw for kind j is the queue entry
//     head + slot_j*total + rank (division first),
//     and a centre writes its circle into the mask of its kind (as
//     stamp_kernel),
//  3. the source plane alpha*division - beta*death (as rate_kernel) and
//     head += kinds drawn * total, also written with the error flag to the
//     draw's snapshot.
template<typename T>
__global__ void __launch_bounds__(MB)
queued_draw_kernel(MaskView<T> v, MaskScratch s, const double* __restrict__ queue, long long qcap,
                   long long* head, long long supplied, QueuedDraw<T> w, double r2_0, int R0,
                   double r2_1, int R1)
{
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ int warp_cnt[MB/32];
  __shared__ long long part[MB];
  const long long N = static_cast<long long>(v.LX)*v.LY;
  const int nch = static_cast<int>((N + MB - 1)/MB);
  const int tid = threadIdx.x;
  const bool div = w.kinds & 1, dea = (w.kinds >> 1) & 1;

  for(int c = blockIdx.x; c < nch; c += gridDim.x)
  {
    const long long k = static_cast<long long>(c)*MB + tid;
    const int flag = k < N && phi_at(v, k) >= .5;
    const int n = __syncthreads_count(flag);
    if(tid == 0) s.block_cnt[c] = n;
    if(k < N)
    {
      if(div) s.mask[0][k] = 0;
      if(dea) s.mask[1][k] = 0;
    }
  }
  grid.sync();

  // inclusive prefix of the per-thread segments of the chunk counts: warp
  // scans by shuffles, then the scan of the 32 warp totals
  const int per = (nch + MB - 1)/MB;
  const unsigned lane = tid & 31u, warp = tid >> 5;
  {
    __shared__ long long wsum[MB/32];
    const int lo = tid*per, hi = min(nch, lo + per);
    long long sum = 0;
    for(int i = lo; i < hi; ++i) sum += s.block_cnt[i];
#pragma unroll
    for(int d = 1; d < 32; d <<= 1)
    {
      const long long add = __shfl_up_sync(0xffffffffu, sum, d);
      if(lane >= static_cast<unsigned>(d)) sum += add;
    }
    if(lane == 31) wsum[warp] = sum;
    __syncthreads();
    if(warp == 0)
    {
      long long ws = wsum[lane];
#pragma unroll
      for(int d = 1; d < 32; d <<= 1)
      {
        const long long add = __shfl_up_sync(0xffffffffu, ws, d);
        if(lane >= static_cast<unsigned>(d)) ws += add;
      }
      wsum[lane] = ws;
    }
    __syncthreads();
    part[tid] = sum + (warp ? wsum[warp - 1] : 0);
    __syncthreads();
  }
  const long long total = part[MB - 1], h0 = *head;
  for(int c = blockIdx.x; c < nch; c += gridDim.x)
  {
    const long long k = static_cast<long long>(c)*MB + tid;
    const double p = k < N ? phi_at(v, k) : 0.;
    const bool flag = k < N && p >= .5;
    const unsigned ballot = __ballot_sync(0xffffffffu, flag);
    __syncthreads();   // warp_cnt of the previous chunk has been read
    if(lane == 0) warp_cnt[warp] = __popc(ballot);
    __syncthreads();
    unsigned cen = 0;   // bit j: a centre of kind j
    if(flag)
    {
      // chunk offset: the segments before c's, then the chunks before c in it
      const int sg = c/per;
      long long off = sg ? part[sg - 1] : 0;
      for(int i = sg*per; i < c; ++i) off += s.block_cnt[i];
      int before = 0;
      for(unsigned i = 0; i < warp; ++i) before += warp_cnt[i];
      before += __popc(ballot & ((1u << lane) - 1u));
      const long long rank = off + before;
      int slot = 0;
      for(int j = 0; j < 2; ++j)
      {
        if(!((w.kinds >> j) & 1)) continue;
        const long long idx = h0 + slot*total + rank;
        ++slot;
        if(idx < supplied)
        {
          // src/models/lyotropic-with-division.cpp:47 (division), :83 (death)
          const double thr = j == 0 ? w.coef[0]*p*(1 - p/w.phi_critical) : w.coef[1]*p;
          if(queue[idx % qcap] < thr) cen |= 1u << j;
        }
        else atomicOr(w.err, 1);
      }
    }
    // the warp writes the circles of its centres together, one offset per lane
    for(int j = 0; j < 2; ++j)
    {
      const int R = j ? R1 : R0;
      if(!((w.kinds >> j) & 1) || R < 0) continue;
      unsigned todo = __ballot_sync(0xffffffffu, (cen >> j) & 1u);
      while(todo)
      {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        const long long kc = __shfl_sync(0xffffffffu, k, src);
        stamp_circle_warp(v.LX, v.LY, kc, s.mask[j], j ? r2_1 : r2_0, R, lane);
      }
    }
  }
  grid.sync();

  const long long stride = static_cast<long long>(gridDim.x)*MB;
  for(long long k = static_cast<long long>(blockIdx.x)*MB + tid; k < N; k += stride)
  {
    int x, y;
    if(N <= 0xffffffffll)
    {
      const unsigned ku = static_cast<unsigned>(k), ly = static_cast<unsigned>(v.LY);
      x = static_cast<int>(ku/ly);
      y = static_cast<int>(ku - static_cast<unsigned>(x)*ly);
    }
    else
    {
      x = static_cast<int>(k / v.LY);
      y = static_cast<int>(k % v.LY);
    }
    const unsigned char m0 = s.mask[0][k], m1 = s.mask[1][k];
    // alpha*division_m - beta*death_m (src/models/lyotropic-with-division.cpp:121)
    const double r = w.alpha*(m0 ? 1. : 0.) - w.beta*(m1 ? 1. : 0.);
    w.src[(y + w.g) + static_cast<long long>(w.EY)*(x + w.g)] = static_cast<T>(r);
  }
  if(blockIdx.x == 0 && tid == 0)
  {
    *head = h0 + (div + dea)*total;
    // a copy of the queue state for the host, which this draw's slot owns
    // until the host has read it (the live head moves with the next draw)
    w.snap[0] = h0 + (div + dea)*total;
    w.snap[1] = *w.err;
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
cudaError_t mask_rate(int LX, int LY, int g, int EY, const MaskScratch& s, double alpha,
                      double beta, T* src, cudaStream_t st)
{
  const long long N = static_cast<long long>(LX)*LY;
  rate_kernel<T><<<grid_for(N), 256, 0, st>>>(LX, LY, g, EY, s.mask[0], s.mask[1], alpha, beta, src);
  return cudaGetLastError();
}

template<typename T>
cudaError_t mask_draw_queued_fused(const MaskView<T>& v, const MaskScratch& s, const MaskQueue& q,
                                   const QueuedDraw<T>& w, cudaStream_t st)
{
  // resident blocks only (a cooperative launch); per device, cached
  static int grid_cache[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int& resident = grid_cache[dev & 63];
  if(!resident)
  {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, queued_draw_kernel<T>, MB, 0);
    if(e != cudaSuccess) return e;
    resident = sms*(per_sm > 0 ? per_sm : 1);
  }
  const long long N = static_cast<long long>(v.LX)*v.LY;
  const int nch = mask_blocks(N);
  const int grid = nch < resident ? nch : resident;
  // ceil(radius^2) as the reference computes it (:60, :96); R < 0: no circle
  double r2[2];
  int R[2];
  for(int j = 0; j < 2; ++j)
  {
    r2[j] = std::ceil(w.radius[j]*w.radius[j]);
    R[j] = r2[j] >= 0 ? static_cast<int>(std::floor(std::sqrt(r2[j]))) : -1;
  }
  MaskView<T> vv = v;
  MaskScratch ss = s;
  const double* qb = q.buf;
  long long qcap = q.cap;
  long long* head = q.head;
  long long supplied = q.supplied;
  QueuedDraw<T> ww = w;
  void* args[] = {&vv, &ss, &qb, &qcap, &head, &supplied, &ww, &r2[0], &R[0], &r2[1], &R[1]};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(queued_draw_kernel<T>),
                                     dim3(grid), dim3(MB), args, 0, st);
}

template cudaError_t mask_count<double>(const MaskView<double>&, const MaskScratch&, cudaStream_t);
template cudaError_t mask_count<float>(const MaskView<float>&, const MaskScratch&, cudaStream_t);
template cudaError_t mask_draw<double>(const MaskView<double>&, const MaskScratch&, int, long long,
                                       double, double, double, cudaStream_t);
template cudaError_t mask_draw<float>(const MaskView<float>&, const MaskScratch&, int, long long,
                                      double, double, double, cudaStream_t);
template cudaError_t mask_rate<double>(int, int, int, int, const MaskScratch&, double, double,
                                       double*, cudaStream_t);
template cudaError_t mask_rate<float>(int, int, int, int, const MaskScratch&, double, double,
                                      float*, cudaStream_t);

template cudaError_t mask_draw_queued_fused<double>(const MaskView<double>&, const MaskScratch&,
                                                   const MaskQueue&, const QueuedDraw<double>&,
                                                   cudaStream_t);
template cudaError_t mask_draw_queued_fused<float>(const MaskView<float>&, const MaskScratch&,
                                                  const MaskQueue&, const QueuedDraw<float>&,
                                                  cudaStream_t);

} // namespace mlb
