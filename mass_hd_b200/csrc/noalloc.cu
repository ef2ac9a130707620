// Allocation-free conservation sums over an FP32 device state.
//
// mass_lb_checks() reduces with a scratch buffer the handle allocated with
// cudaMalloc. Some callers cannot allocate device memory: a host program
// whose device memory is owned in full by another allocator (a framework
// that reserved the HBM up front, so a further cudaMalloc fails or forces a
// device-wide synchronization), or a monitoring path that must not pay
// cudaMalloc/cudaFree's implicit synchronization. For them,
// mass_lb_state_sums_noalloc() computes the same sums with its scratch in a
// file-scope __device__ array of fixed size, so it allocates nothing.
//
// The array: 5 doubles per block (population sum and compensation, phi sum
// and compensation, non-finite count) for up to NA_MAX_BLOCKS blocks, plus 3
// result doubles: 163,864 bytes, held by every device that loads the library
// until the process exits. Each block reduces a fixed chunk of
// NA_THREADS x NA_SITES sites, so a call handles at most
// NA_MAX_BLOCKS x NA_THREADS x NA_SITES = 67,108,864 sites (8192 x 8192);
// larger lattices are rejected.
#include "mass_lb.h"
#include "mass_lb_ext.h"

#include <cuda_runtime.h>

#include "last_error.h"

#include <cmath>
#include <mutex>
#include <string>

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_SITES = 64;                 // sites per thread
constexpr int NA_MAX_BLOCKS = 4096;
constexpr long long NA_CHUNK = static_cast<long long>(NA_THREADS)*NA_SITES;
constexpr long long NA_MAX_SITES = NA_CHUNK*NA_MAX_BLOCKS;
constexpr int NA_SLOTS = 5*NA_MAX_BLOCKS + 3;

// Shared by every call on a device; keeps the last call's contents. Each
// call writes every slot it later reads (the per-block partials of the
// blocks it launches, then the 3 results), so nothing has to start at zero.
// Calls that overlap on the GPU race on this array.
__device__ __align__(256) double g_noalloc_scratch[NA_SLOTS];

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

__device__ __forceinline__ KB kb_down(KB a, int off)
{
  return KB{__shfl_down_sync(0xffffffffu, a.s, off), __shfl_down_sync(0xffffffffu, a.c, off)};
}

// Block b sums sites [b*NA_CHUNK, (b+1)*NA_CHUNK) of the planes: populations
// are deviations from t_v*rho (sum over v of the rest part is rho).
__global__ void __launch_bounds__(NA_THREADS)
noalloc_pass1(const float* __restrict__ planes, long long plane, int has_phi,
              long long nsites, double rho, double* __restrict__ scratch)
{
  KB fs{0.0, 0.0}, ps{0.0, 0.0};
  double bad = 0.0;
  const long long base = blockIdx.x*NA_CHUNK;
  for(int j = 0; j < NA_SITES; ++j)
  {
    const long long k = base + j*NA_THREADS + threadIdx.x;
    if(k >= nsites) break;
    double site = rho;
#pragma unroll
    for(int v = 0; v < 9; ++v)
    {
      const float f = planes[v*plane + k];
      if(!isfinite(f)) bad += 1.0;
      site += static_cast<double>(f);
    }
    kb_add(fs, site);
    if(!isfinite(planes[9*plane + k]) || !isfinite(planes[10*plane + k])) bad += 1.0;
    if(has_phi)
    {
      const float p = planes[11*plane + k];
      if(!isfinite(p)) bad += 1.0;
      kb_add(ps, static_cast<double>(p));
    }
  }
  for(int off = 16; off > 0; off >>= 1)
  {
    fs = kb_merge(fs, kb_down(fs, off));
    ps = kb_merge(ps, kb_down(ps, off));
    bad += __shfl_down_sync(0xffffffffu, bad, off);
  }
  __shared__ double sh[NA_THREADS/32][5];
  const int w = threadIdx.x/32;
  if((threadIdx.x & 31) == 0)
  {
    sh[w][0] = fs.s; sh[w][1] = fs.c; sh[w][2] = ps.s; sh[w][3] = ps.c; sh[w][4] = bad;
  }
  __syncthreads();
  if(threadIdx.x == 0)
  {
    KB F{0.0, 0.0}, Pp{0.0, 0.0};
    double B = 0.0;
    for(int i = 0; i < NA_THREADS/32; ++i)
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
noalloc_pass2(double* __restrict__ scratch, int nblocks)
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
    F = kb_merge(F, kb_down(F, off));
    Pp = kb_merge(Pp, kb_down(Pp, off));
    B += __shfl_down_sync(0xffffffffu, B, off);
  }
  if(threadIdx.x == 0)
  {
    double* r = scratch + 5*NA_MAX_BLOCKS;
    r[0] = F.s + F.c;
    r[1] = Pp.s + Pp.c;
    r[2] = B;
  }
}

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {};   // device address of the array, per device

// Set-up on device `dev` (the current device), once: the array's name in
// host code is a host-side stand-in, not a device address, so the kernels
// get the address that cudaGetSymbolAddress returns for this device. The
// cached address lives as long as the device's context: a cudaDeviceReset
// ends the library's use of that device altogether (its handles' buffers
// are gone too).
cudaError_t scratch_on_current_device(int dev, double** out)
{
  if(dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  cudaError_t e = cudaSuccess;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if(!g_noalloc_ptr[dev])
  {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if(e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

int na_fail(int code, const std::string& msg)
{
  mlb_set_last_error(msg);   // read back through mass_lb_last_error()
  return code;
}

} // namespace

extern "C" int mass_lb_state_sums_noalloc(const float* planes, long long plane_stride,
                                          int nplanes, unsigned LX, unsigned LY,
                                          double rho, void* stream, double* fsum,
                                          double* phisum, int* nonfinite)
{
  if(!planes) return na_fail(MASS_LB_EINVAL, "null planes");
  if(nplanes != 11 && nplanes != 12)
    return na_fail(MASS_LB_EINVAL, "nplanes must be 11 (nematic) or 12 (lyotropic)");
  const long long nsites = static_cast<long long>(LX)*LY;
  if(nsites == 0) return na_fail(MASS_LB_EINVAL, "empty lattice");
  if(nsites > NA_MAX_SITES)
    return na_fail(MASS_LB_EINVAL,
                   "lattice of " + std::to_string(nsites) + " sites exceeds the " +
                   std::to_string(NA_MAX_SITES) + "-site limit of the static scratch");
  if(plane_stride < nsites) return na_fail(MASS_LB_EINVAL, "plane stride below LX*LY");
  // The kernels run on the current device and use that device's copy of the
  // array, so the planes and the stream must belong to it: a mismatch would
  // make the kernels read another GPU's memory or fail to launch.
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess)
    return na_fail(MASS_LB_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  cudaPointerAttributes pa{};
  e = cudaPointerGetAttributes(&pa, planes);
  if(e != cudaSuccess || pa.type != cudaMemoryTypeDevice)
  {
    cudaGetLastError();
    return na_fail(MASS_LB_EINVAL, "planes are not device memory");
  }
  if(pa.device != dev)
    return na_fail(MASS_LB_EINVAL,
                   "planes live on device " + std::to_string(pa.device) + " but device " +
                   std::to_string(dev) + " is current; make the planes' device current");
  if(stream)
  {
    int sdev = -1;
    e = cudaStreamGetDevice(static_cast<cudaStream_t>(stream), &sdev);
    if(e != cudaSuccess)
      return na_fail(MASS_LB_ECUDA, std::string("cudaStreamGetDevice: ") + cudaGetErrorString(e));
    if(sdev != dev)
      return na_fail(MASS_LB_EINVAL,
                     "stream belongs to device " + std::to_string(sdev) + " but device " +
                     std::to_string(dev) + " is current");
  }
  double* scratch = nullptr;
  e = scratch_on_current_device(dev, &scratch);
  if(e != cudaSuccess)
    return na_fail(MASS_LB_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nb = static_cast<int>((nsites + NA_CHUNK - 1)/NA_CHUNK);
  noalloc_pass1<<<nb, NA_THREADS, 0, st>>>(planes, plane_stride, nplanes == 12 ? 1 : 0,
                                           nsites, rho, scratch);
  noalloc_pass2<<<1, 32, 0, st>>>(scratch, nb);
  double r[3];
  e = cudaGetLastError();
  if(e == cudaSuccess)
    e = cudaMemcpyAsync(r, scratch + 5*NA_MAX_BLOCKS, sizeof(r), cudaMemcpyDeviceToHost, st);
  if(e == cudaSuccess) e = cudaStreamSynchronize(st);
  if(e != cudaSuccess)
    return na_fail(MASS_LB_ECUDA, std::string("noalloc sums: ") + cudaGetErrorString(e));
  if(fsum) *fsum = r[0];
  if(phisum) *phisum = r[1];
  if(nonfinite) *nonfinite = r[2] != 0.0 ? 1 : 0;
  return MASS_LB_OK;
}
