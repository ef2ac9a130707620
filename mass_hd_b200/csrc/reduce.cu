// FP64 compensated reductions over the lattice state.
//
// Each thread accumulates its sites with Neumaier's variant of Kahan
// summation; warps and blocks combine (sum, compensation) pairs with an
// error-free TwoSum, and a single-block pass combines the per-block pairs
// the same way. The first pass writes 5 doubles per block into the scratch
// buffer (fsum, fcomp, psum, pcomp, nonfinite count).
#include "reduce.cuh"

namespace mlb {
namespace {

constexpr int RB = 256;        // threads per block
constexpr int RBLOCKS = 592;   // 4 x 148 SMs

struct KB
{
  double s, c;
};

__device__ __forceinline__ void kb_add(KB& a, double x)
{
  const double t = a.s + x;
  if(fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x;
  else a.c += (x - t) + a.s;
  a.s = t;
}

__device__ __forceinline__ KB kb_merge(KB a, KB b)
{
  const double t = a.s + b.s;
  const double bb = t - a.s;
  const double err = (a.s - (t - bb)) + (b.s - bb);
  return KB{t, a.c + b.c + err};
}

__device__ __forceinline__ KB kb_shfl_down(KB a, int off)
{
  return KB{__shfl_down_sync(0xffffffffu, a.s, off), __shfl_down_sync(0xffffffffu, a.c, off)};
}

template<typename T>
__device__ __forceinline__ bool finite(T x) { return isfinite(x); }

template<typename T>
__global__ void __launch_bounds__(RB)
sums_pass1(SumView<T> v, double* scratch)
{
  KB fs{0.0, 0.0}, ps{0.0, 0.0};
  double bad = 0.0;
  const long long N = static_cast<long long>(v.LX)*v.LY;
  for(long long k = blockIdx.x*static_cast<long long>(RB) + threadIdx.x; k < N;
      k += static_cast<long long>(gridDim.x)*RB)
  {
    const int x = static_cast<int>(k / v.LY), y = static_cast<int>(k % v.LY);
    const long long e = (y + v.g) + static_cast<long long>(v.EY)*(x + v.g);
    double site = v.rest;
#pragma unroll
    for(int q = 0; q < 9; ++q)
    {
      const T f = v.ff[q*v.plane + e];
      if(!finite(f)) bad += 1.0;
      site += static_cast<double>(f);
    }
    kb_add(fs, site);
    if(!finite(v.Qxx[e]) || !finite(v.Qyx[e])) bad += 1.0;
    if(v.phi)
    {
      const T p = v.phi[e];
      if(!finite(p)) bad += 1.0;
      kb_add(ps, static_cast<double>(p));
    }
  }
  for(int off = 16; off > 0; off >>= 1)
  {
    fs = kb_merge(fs, kb_shfl_down(fs, off));
    ps = kb_merge(ps, kb_shfl_down(ps, off));
    bad += __shfl_down_sync(0xffffffffu, bad, off);
  }
  __shared__ double sh[RB/32][5];
  const int w = threadIdx.x/32, l = threadIdx.x%32;
  if(l == 0) { sh[w][0] = fs.s; sh[w][1] = fs.c; sh[w][2] = ps.s; sh[w][3] = ps.c; sh[w][4] = bad; }
  __syncthreads();
  if(threadIdx.x == 0)
  {
    KB F{0.0, 0.0}, Pp{0.0, 0.0};
    double B = 0.0;
    for(int i = 0; i < RB/32; ++i)
    {
      F = kb_merge(F, KB{sh[i][0], sh[i][1]});
      Pp = kb_merge(Pp, KB{sh[i][2], sh[i][3]});
      B += sh[i][4];
    }
    double* o = scratch + 5*blockIdx.x;
    o[0] = F.s; o[1] = F.c; o[2] = Pp.s; o[3] = Pp.c; o[4] = B;
  }
}

__global__ void __launch_bounds__(32)
sums_pass2(const double* scratch, int nblocks, double* out)
{
  KB F{0.0, 0.0}, Pp{0.0, 0.0};
  double B = 0.0;
  for(int i = threadIdx.x; i < nblocks; i += 32)
  {
    const double* o = scratch + 5*i;
    F = kb_merge(F, KB{o[0], o[1]});
    Pp = kb_merge(Pp, KB{o[2], o[3]});
    B += o[4];
  }
  for(int off = 16; off > 0; off >>= 1)
  {
    F = kb_merge(F, kb_shfl_down(F, off));
    Pp = kb_merge(Pp, kb_shfl_down(Pp, off));
    B += __shfl_down_sync(0xffffffffu, B, off);
  }
  if(threadIdx.x == 0)
  {
    out[0] = F.s + F.c;
    out[1] = Pp.s + Pp.c;
    out[2] = B;
  }
}

template<typename T>
cudaError_t launch(const SumView<T>& v, double* scratch, double* out, cudaStream_t st)
{
  const long long N = static_cast<long long>(v.LX)*v.LY;
  long long nb = (N + RB - 1)/RB;
  if(nb > RBLOCKS) nb = RBLOCKS;
  if(nb < 1) nb = 1;
  sums_pass1<T><<<static_cast<int>(nb), RB, 0, st>>>(v, scratch);
  sums_pass2<<<1, 32, 0, st>>>(scratch, static_cast<int>(nb), out);
  return cudaGetLastError();
}

} // namespace

int sums_scratch_doubles() { return 5*RBLOCKS; }

cudaError_t launch_sums_f64(const SumView<double>& v, double* scratch, double* out, cudaStream_t st)
{
  return launch(v, scratch, out, st);
}

cudaError_t launch_sums_f32(const SumView<float>& v, double* scratch, double* out, cudaStream_t st)
{
  return launch(v, scratch, out, st);
}

} // namespace mlb
