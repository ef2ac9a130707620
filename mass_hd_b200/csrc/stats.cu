// Flow and defect statistics of the current lattice state, on the device.
//
// The estimators are those of the reference's post-processing, so long runs
// can be compared statistically without writing frames:
//  * velocity u = j/rho from the populations
//    (plot/python/passive_q1_alpha_regime_analysis.py:137-145,
//     POST/massPy/base_modules/flow.py:7-11);
//  * vorticity w = d_x uy - d_y ux with periodic central differences
//    (passive_q1_alpha_regime_analysis.py:148-151), enstrophy density
//    0.5 <w^2> (:339-348) over the lattice and over phi > 0.5;
//  * <|u|^2>;
//  * interface length perimeter_4(phi > 0.5): exposed edges of the phi > 0.5
//    region, the lattice edge counting as exposed (:206-216);
//  * nematic defects: the director n from Q (POST/massPy/nematic/nematicPy.py:4-15),
//    the winding of n around the 8-site ring of every site with the nematic
//    fold of the angle to [-pi/2, pi/2] (POST/massPy/base_modules/defects.py:15-50),
//    sites with |charge| > 0.4 grouped into 4-connected same-sign clusters,
//    one defect each (defects.py:58-110, nematicPy.py:74-95).
// Pass 1 writes u and n per site (FP64 scratch planes). Pass 2 computes the
// sums per block (Kahan-Babuska FP64) and appends every charged site to a
// list; the host sorts and clusters that list (api.cu).
#include "stats.cuh"

#include <cmath>

namespace mlb {
namespace {

constexpr int SB = 256;

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

template<typename T>
__global__ void __launch_bounds__(SB)
stats_pass1(StatView<T> v, double* __restrict__ U, double* __restrict__ D)
{
  const long long N = static_cast<long long>(v.LX)*v.LY;
  for(long long k = blockIdx.x*static_cast<long long>(SB) + threadIdx.x; k < N;
      k += static_cast<long long>(gridDim.x)*SB)
  {
    const int x = static_cast<int>(k / v.LY), y = static_cast<int>(k % v.LY);
    const long long e = (y + v.g) + static_cast<long long>(v.EY)*(x + v.g);
    double f[9];
#pragma unroll
    for(int q = 0; q < 9; ++q) f[q] = static_cast<double>(v.ff[q*v.plane + e]);
    const double rho = v.rest + f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    const double jx = f[1] - f[2] + f[5] - f[6] - f[7] + f[8];
    const double jy = f[3] - f[4] + f[5] - f[6] + f[7] - f[8];
    U[k] = rho == 0.0 ? 0.0 : jx/rho;
    U[N + k] = rho == 0.0 ? 0.0 : jy/rho;
    const double qxx = static_cast<double>(v.Qxx[e]), qyx = static_cast<double>(v.Qyx[e]);
    const double S = sqrt(qxx*qxx + qyx*qyx);
    const double sg = qyx > 0.0 ? 1.0 : (qyx < 0.0 ? -1.0 : 0.0);
    D[k] = sqrt(.5*(1. + qxx/S));
    D[N + k] = sg*sqrt(.5*(1. - qxx/S));
  }
}

// angle between two directors folded to [-pi/2, pi/2]
__device__ __forceinline__ double wang(double a0, double a1, double b0, double b1)
{
  const double ang = atan2(a0*b1 - a1*b0, a0*b0 + a1*b1);
  if(fabs(ang) > .5*M_PI) return ang - (ang > 0 ? M_PI : -M_PI);
  return ang;
}

template<typename T>
__global__ void __launch_bounds__(SB)
stats_pass2(StatView<T> v, const double* __restrict__ U, const double* __restrict__ D,
            double* __restrict__ partial, int* __restrict__ count, int* __restrict__ list,
            int capacity, double threshold)
{
  const int LX = v.LX, LY = v.LY;
  const long long N = static_cast<long long>(LX)*LY;
  KB su2{0, 0}, sw2{0, 0}, sw2p{0, 0};
  double area = 0, perim = 0;
  for(long long k = blockIdx.x*static_cast<long long>(SB) + threadIdx.x; k < N;
      k += static_cast<long long>(gridDim.x)*SB)
  {
    const int x = static_cast<int>(k / LY), y = static_cast<int>(k % LY);
    const int xp = x + 1 == LX ? 0 : x + 1, xm = x == 0 ? LX - 1 : x - 1;
    const int yp = y + 1 == LY ? 0 : y + 1, ym = y == 0 ? LY - 1 : y - 1;
    auto at = [&](int X, int Y) { return static_cast<long long>(X)*LY + Y; };
    const double vx = U[k], vy = U[N + k];
    const double dvdx = .5*(U[N + at(xp, y)] - U[N + at(xm, y)]);
    const double dudy = .5*(U[at(x, yp)] - U[at(x, ym)]);
    const double om = dvdx - dudy;
    kb_add(su2, vx*vx + vy*vy);
    kb_add(sw2, om*om);
    if(v.phi)
    {
      auto inside = [&](int X, int Y) {
        const long long e = (Y + v.g) + static_cast<long long>(v.EY)*(X + v.g);
        return static_cast<double>(v.phi[e]) > .5;
      };
      if(inside(x, y))
      {
        area += 1;
        kb_add(sw2p, om*om);
        perim += (x + 1 >= LX || !inside(x + 1, y)) + (x == 0 || !inside(x - 1, y))
               + (y + 1 >= LY || !inside(x, y + 1)) + (y == 0 || !inside(x, y - 1));
      }
    }
    // winding of the director around the ring (x-1,y) (x-1,y-1) (x,y-1)
    // (x+1,y-1) (x+1,y) (x+1,y+1) (x,y+1) (x-1,y+1) and back
    const int rx[9] = {xm, xm, x, xp, xp, xp, x, xm, xm};
    const int ry[9] = {y, ym, ym, ym, y, yp, yp, yp, y};
    double w = 0;
    double a0 = D[at(rx[0], ry[0])], a1 = D[N + at(rx[0], ry[0])];
#pragma unroll
    for(int i = 1; i < 9; ++i)
    {
      const double b0 = D[at(rx[i], ry[i])], b1 = D[N + at(rx[i], ry[i])];
      w += wang(a0, a1, b0, b1);
      a0 = b0; a1 = b1;
    }
    w = w/(2*M_PI);
    if(fabs(w) > threshold)
    {
      const int slot = atomicAdd(count, 1);
      if(slot < capacity) list[slot] = w > 0 ? static_cast<int>(k) : -static_cast<int>(k) - 1;
    }
  }
  // block reduction
  __shared__ double sh[SB/32][8];
  for(int off = 16; off > 0; off >>= 1)
  {
    su2 = kb_merge(su2, KB{__shfl_down_sync(0xffffffffu, su2.s, off), __shfl_down_sync(0xffffffffu, su2.c, off)});
    sw2 = kb_merge(sw2, KB{__shfl_down_sync(0xffffffffu, sw2.s, off), __shfl_down_sync(0xffffffffu, sw2.c, off)});
    sw2p = kb_merge(sw2p, KB{__shfl_down_sync(0xffffffffu, sw2p.s, off), __shfl_down_sync(0xffffffffu, sw2p.c, off)});
    area += __shfl_down_sync(0xffffffffu, area, off);
    perim += __shfl_down_sync(0xffffffffu, perim, off);
  }
  const int wi = threadIdx.x/32;
  if((threadIdx.x & 31) == 0)
  {
    sh[wi][0] = su2.s; sh[wi][1] = su2.c; sh[wi][2] = sw2.s; sh[wi][3] = sw2.c;
    sh[wi][4] = sw2p.s; sh[wi][5] = sw2p.c; sh[wi][6] = area; sh[wi][7] = perim;
  }
  __syncthreads();
  if(threadIdx.x == 0)
  {
    KB a{0, 0}, b{0, 0}, c{0, 0};
    double ar = 0, pe = 0;
    for(int i = 0; i < SB/32; ++i)
    {
      a = kb_merge(a, KB{sh[i][0], sh[i][1]});
      b = kb_merge(b, KB{sh[i][2], sh[i][3]});
      c = kb_merge(c, KB{sh[i][4], sh[i][5]});
      ar += sh[i][6];
      pe += sh[i][7];
    }
    double* o = partial + 8*blockIdx.x;
    o[0] = a.s; o[1] = a.c; o[2] = b.s; o[3] = b.c; o[4] = c.s; o[5] = c.c; o[6] = ar; o[7] = pe;
  }
}

__global__ void __launch_bounds__(32)
stats_pass3(const double* __restrict__ partial, int nblocks, double* __restrict__ out)
{
  KB a{0, 0}, b{0, 0}, c{0, 0};
  double ar = 0, pe = 0;
  for(int i = threadIdx.x; i < nblocks; i += 32)
  {
    const double* o = partial + 8*i;
    a = kb_merge(a, KB{o[0], o[1]});
    b = kb_merge(b, KB{o[2], o[3]});
    c = kb_merge(c, KB{o[4], o[5]});
    ar += o[6];
    pe += o[7];
  }
  for(int off = 16; off > 0; off >>= 1)
  {
    a = kb_merge(a, KB{__shfl_down_sync(0xffffffffu, a.s, off), __shfl_down_sync(0xffffffffu, a.c, off)});
    b = kb_merge(b, KB{__shfl_down_sync(0xffffffffu, b.s, off), __shfl_down_sync(0xffffffffu, b.c, off)});
    c = kb_merge(c, KB{__shfl_down_sync(0xffffffffu, c.s, off), __shfl_down_sync(0xffffffffu, c.c, off)});
    ar += __shfl_down_sync(0xffffffffu, ar, off);
    pe += __shfl_down_sync(0xffffffffu, pe, off);
  }
  if(threadIdx.x == 0)
  {
    out[0] = a.s + a.c; out[1] = b.s + b.c; out[2] = c.s + c.c; out[3] = ar; out[4] = pe;
  }
}

template<typename T>
cudaError_t launch(const StatView<T>& v, const StatScratch& s, double threshold, cudaStream_t st)
{
  const long long N = static_cast<long long>(v.LX)*v.LY;
  long long nb = (N + SB - 1)/SB;
  if(nb > STATS_BLOCKS) nb = STATS_BLOCKS;
  if(nb < 1) nb = 1;
  cudaError_t e = cudaMemsetAsync(s.count, 0, sizeof(int), st);
  if(e != cudaSuccess) return e;
  stats_pass1<T><<<static_cast<int>(nb), SB, 0, st>>>(v, s.U, s.D);
  stats_pass2<T><<<static_cast<int>(nb), SB, 0, st>>>(v, s.U, s.D, s.partial, s.count, s.list,
                                                       s.capacity, threshold);
  stats_pass3<<<1, 32, 0, st>>>(s.partial, static_cast<int>(nb), s.out);
  return cudaGetLastError();
}

} // namespace

cudaError_t launch_stats_f64(const StatView<double>& v, const StatScratch& s, double threshold,
                             cudaStream_t st)
{
  return launch(v, s, threshold, st);
}

cudaError_t launch_stats_f32(const StatView<float>& v, const StatScratch& s, double threshold,
                             cudaStream_t st)
{
  return launch(v, s, threshold, st);
}

} // namespace mlb
