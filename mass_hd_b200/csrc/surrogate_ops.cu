// C ABI of the learned surrogate (include/mass_surrogate.h): the tensor-core
// convolutions (conv_tc.cu) plus the CUDA-core kernels around them (batch
// packing, MSE loss, bias gradients, AdamW, lattice state <-> fields).
#include "mass_lb.h"
#include "mass_surrogate.h"

#include "conv_tc.cuh"
#include "last_error.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <string>

using namespace mlb;

namespace {

int sg_fail(int code, const std::string& msg)
{
  mlb_set_last_error(msg);
  return code;
}

int sg_cuda(cudaError_t e, const char* where)
{
  if(e == cudaSuccess) return 0;
  return sg_fail(MASS_LB_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

__device__ __forceinline__ size_t pidx(int n, int yy, int xx, int H, int W)
{
  return (static_cast<size_t>(n)*(H + 2) + yy)*static_cast<size_t>(W + 2) + xx;
}

// Write the 64-channel pixel (5 values, 59 zeros) with its periodic copies.
__device__ void put5(__nv_bfloat16* base, const float* v, int n, int y, int x, int H, int W)
{
  uint4 pk[8];
  __nv_bfloat162 h[4];
  h[0] = __floats2bfloat162_rn(v[0], v[1]);
  h[1] = __floats2bfloat162_rn(v[2], v[3]);
  h[2] = __floats2bfloat162_rn(v[4], 0.f);
  h[3] = __floats2bfloat162_rn(0.f, 0.f);
  pk[0] = *reinterpret_cast<uint4*>(h);
  for(int k = 1; k < 8; ++k) pk[k] = make_uint4(0, 0, 0, 0);
  int ys[3] = {y + 1, 0, 0}, xs[3] = {x + 1, 0, 0};
  int ny = 1, nx = 1;
  if(y == 0) ys[ny++] = H + 1;
  if(y == H - 1) ys[ny++] = 0;
  if(x == 0) xs[nx++] = W + 1;
  if(x == W - 1) xs[nx++] = 0;
  for(int i = 0; i < ny; ++i)
    for(int j = 0; j < nx; ++j)
    {
      uint4* dst = reinterpret_cast<uint4*>(base + pidx(n, ys[i], xs[j], H, W)*64);
      for(int k = 0; k < 8; ++k) dst[k] = pk[k];
    }
}

__global__ void k_pack(const float* __restrict__ fields, const int* __restrict__ src,
                       const int* __restrict__ dst, int B, int H, int W,
                       __nv_bfloat16* __restrict__ x_in, float* __restrict__ xf,
                       float* __restrict__ target)
{
  const long long N = static_cast<long long>(H)*W;
  const long long total = N*B;
  for(long long i = blockIdx.x*256ll + threadIdx.x; i < total; i += 256ll*gridDim.x)
  {
    const int n = static_cast<int>(i / N);
    const long long p = i % N;
    const int y = static_cast<int>(p / W), x = static_cast<int>(p % W);
    const float* s = fields + (static_cast<long long>(src[n])*N + p)*5;
    float v[5];
    for(int c = 0; c < 5; ++c) { v[c] = s[c]; xf[5*i + c] = v[c]; }
    put5(x_in, v, n, y, x, H, W);
    if(target)
    {
      const float* t = fields + (static_cast<long long>(dst[n])*N + p)*5;
      for(int c = 0; c < 5; ++c) target[5*i + c] = t[c];
    }
  }
}

__global__ void k_mse(const float* __restrict__ pred, const float* __restrict__ target, int B,
                      int H, int W, double* sse, __nv_bfloat16* __restrict__ dout)
{
  const long long N = static_cast<long long>(H)*W;
  const long long total = N*B;
  const float g = 2.f/static_cast<float>(total*5);
  double acc = 0;
  for(long long i = blockIdx.x*256ll + threadIdx.x; i < total; i += 256ll*gridDim.x)
  {
    const int n = static_cast<int>(i / N);
    const long long p = i % N;
    const int y = static_cast<int>(p / W), x = static_cast<int>(p % W);
    float d[5];
    for(int c = 0; c < 5; ++c)
    {
      const float e = pred[5*i + c] - target[5*i + c];
      acc += static_cast<double>(e)*e;
      d[c] = g*e;
    }
    put5(dout, d, n, y, x, H, W);
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for(int s = 128; s > 0; s >>= 1)
  {
    if(threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if(threadIdx.x == 0) atomicAdd(sse, red[0]);
}

// Per-channel sums of a padded NHWC64 tensor. A warp takes whole image rows
// (W pixels x 128 bytes, contiguous in the padded layout) with 16-byte
// loads; lane l always holds channels 8(l%8)..8(l%8)+7 of pixel l/8 (mod 4)
// and keeps 8 partial sums.
__global__ void k_bias_grad(const __nv_bfloat16* __restrict__ dy, float* db, int B, int H, int W)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rows = B*H, per_row = W*8;        // 16-byte chunks per row
  float acc[8];
#pragma unroll
  for(int c = 0; c < 8; ++c) acc[c] = 0.f;
  for(int row = blockIdx.x*8 + warp; row < rows; row += gridDim.x*8)
  {
    const int n = row / H, y = row % H;
    const uint4* p = reinterpret_cast<const uint4*>(dy + pidx(n, y + 1, 1, H, W)*64);
#pragma unroll 4
    for(int k = lane; k < per_row; k += 32)
    {
      const uint4 u = __ldg(p + k);
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
      for(int c = 0; c < 4; ++c)
      {
        const float2 f = __bfloat1622float2(h[c]);
        acc[2*c] += f.x;
        acc[2*c + 1] += f.y;
      }
    }
  }
#pragma unroll
  for(int c = 0; c < 8; ++c)
  {
    acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 8);
    acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 16);
  }
  __shared__ float red[8][64];
  if(lane < 8)
#pragma unroll
    for(int c = 0; c < 8; ++c) red[warp][8*lane + c] = acc[c];
  __syncthreads();
  if(threadIdx.x < 64)
  {
    float t = 0.f;
    for(int w = 0; w < 8; ++w) t += red[w][threadIdx.x];
    atomicAdd(db + threadIdx.x, t);
  }
}

__global__ void k_adamw(float* w, float* b, float* mw, float* vw, float* mb, float* vb,
                        const float* __restrict__ dW, const float* __restrict__ db, int cout,
                        int cin, int nout_pad, float lr, float beta1, float beta2, float eps,
                        float wd_coef, float bc1, float bc2, __nv_bfloat16* wt, __nv_bfloat16* wdg)
{
  const int nw = cout*9*cin;
  for(int i = blockIdx.x*256 + threadIdx.x; i < nw + cout; i += 256*gridDim.x)
  {
    if(i < nw)
    {
      const int co = i / (9*cin), tap = (i / cin) % 9, ci = i % cin;
      const float g = dW[(tap*64 + ci)*64 + co];
      const float m = beta1*mw[i] + (1.f - beta1)*g;
      const float v = beta2*vw[i] + (1.f - beta2)*g*g;
      mw[i] = m;
      vw[i] = v;
      float x = w[i];
      x -= lr*((m/bc1)/(sqrtf(v/bc2) + eps) + wd_coef*x);
      w[i] = x;
      const __nv_bfloat16 h = __float2bfloat16_rn(x);
      wt[(tap*nout_pad + co)*64 + ci] = h;
      wdg[((8 - tap)*64 + ci)*64 + co] = h;
    }
    else
    {
      const int co = i - nw;
      const float g = db[co];
      const float m = beta1*mb[co] + (1.f - beta1)*g;
      const float v = beta2*vb[co] + (1.f - beta2)*g*g;
      mb[co] = m;
      vb[co] = v;
      b[co] -= lr*(m/bc1)/(sqrtf(v/bc2) + eps);
    }
  }
}

struct Norm
{
  float mean[5], scale[5];
};

__global__ void k_fields_from_state(const float* __restrict__ planes, long long ps, int N, float rho0,
                                    Norm nm, float* __restrict__ fields)
{
  for(int k = blockIdx.x*256 + threadIdx.x; k < N; k += 256*gridDim.x)
  {
    float g[9];
    for(int v = 0; v < 9; ++v) g[v] = planes[v*ps + k];
    float rho = rho0;
    for(int v = 0; v < 9; ++v) rho += g[v];
    const float jx = g[1] - g[2] + g[5] - g[6] - g[7] + g[8];
    const float jy = g[3] - g[4] + g[5] - g[6] + g[7] - g[8];
    const float val[5] = {planes[9*ps + k], planes[10*ps + k], planes[11*ps + k], jx/rho, jy/rho};
    for(int c = 0; c < 5; ++c) fields[5ll*k + c] = (val[c] - nm.mean[c])/nm.scale[c];
  }
}

__global__ void k_state_from_fields(const float* __restrict__ fields, int N, float rho, Norm nm,
                                    float* __restrict__ planes, long long ps)
{
  for(int k = blockIdx.x*256 + threadIdx.x; k < N; k += 256*gridDim.x)
  {
    float val[5];
    for(int c = 0; c < 5; ++c) val[c] = fields[5ll*k + c]*nm.scale[c] + nm.mean[c];
    const float vx = val[3], vy = val[4];
    const float v2 = vx*vx + vy*vy;
    // deviations fe_v - t_v*rho of the second-order equilibrium
    float g[9];
    g[1] = rho*(1.f/3.f*vx + 1.f/3.f*v2 - 0.5f*vy*vy);
    g[2] = rho*(-1.f/3.f*vx + 1.f/3.f*v2 - 0.5f*vy*vy);
    g[3] = rho*(1.f/3.f*vy - 0.5f*vx*vx + 1.f/3.f*v2);
    g[4] = rho*(-1.f/3.f*vy - 0.5f*vx*vx + 1.f/3.f*v2);
    g[5] = rho*(1.f/12.f*vx + 1.f/12.f*vy + 1.f/12.f*v2 + 0.25f*vx*vy);
    g[6] = rho*(-1.f/12.f*vx - 1.f/12.f*vy + 1.f/12.f*v2 + 0.25f*vx*vy);
    g[7] = rho*(-1.f/12.f*vx + 1.f/12.f*vy + 1.f/12.f*v2 - 0.25f*vx*vy);
    g[8] = rho*(1.f/12.f*vx - 1.f/12.f*vy + 1.f/12.f*v2 - 0.25f*vx*vy);
    g[0] = -(g[1] + g[2] + g[3] + g[4] + g[5] + g[6] + g[7] + g[8]);
    for(int v = 0; v < 9; ++v) planes[v*ps + k] = g[v];
    planes[9*ps + k] = val[0];
    planes[10*ps + k] = val[1];
    planes[11*ps + k] = val[2];
  }
}

int grid_for(long long n)
{
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255)/256, 8192)));
}

bool dims_ok(int B, int H, int W)
{
  return B >= 1 && H >= 1 && W >= 128 && W % 128 == 0;
}

Norm make_norm(const float* mean, const float* scale)
{
  Norm n;
  for(int c = 0; c < 5; ++c) { n.mean[c] = mean[c]; n.scale[c] = scale[c]; }
  return n;
}

} // namespace

extern "C" {

namespace {
int conv_call(const void* in, const void* w, int nout, int mode, int B, int H, int W,
              const float* bias, const void* resid, const void* aux, void* out, void* out2,
              const float* resid_f, float* out_f, int* err, long long* cycles, int* ncta,
              void* stream)
{
  if(!in || !w || !err) return sg_fail(MASS_LB_EINVAL, "null argument");
  if(!dims_ok(B, H, W)) return sg_fail(MASS_LB_EINVAL, "need B, H >= 1 and W a multiple of 128");
  if(mode < MASS_SG_FWD_BIAS || mode > MASS_SG_BWD_PLAIN)
    return sg_fail(MASS_LB_EINVAL, "unknown convolution mode");
  if((nout == 16) != (mode == MASS_SG_FWD_OUT) || (nout != 16 && nout != 64))
    return sg_fail(MASS_LB_EINVAL, "nout must be 16 for FWD_OUT and 64 otherwise");
  const bool need_out = mode != MASS_SG_FWD_OUT;
  if((need_out && !out) || (mode == MASS_SG_FWD_GELU && !out2) ||
     ((mode == MASS_SG_FWD_RESID || mode == MASS_SG_BWD_RESID) && !resid) ||
     (mode == MASS_SG_BWD_GELU && !aux) || (mode == MASS_SG_FWD_OUT && !out_f) ||
     (mode <= MASS_SG_FWD_OUT && !bias))
    return sg_fail(MASS_LB_EINVAL, "a buffer required by this mode is null");
  ConvArgs a{B, H, W, bias, static_cast<const __nv_bfloat16*>(resid),
             static_cast<const __nv_bfloat16*>(aux), static_cast<__nv_bfloat16*>(out),
             static_cast<__nv_bfloat16*>(out2), resid_f, out_f, err};
  a.cycles = cycles;
  return sg_cuda(conv3x3_launch(static_cast<const __nv_bfloat16*>(in),
                                static_cast<const __nv_bfloat16*>(w), nout, mode, a,
                                static_cast<cudaStream_t>(stream), ncta), "conv3x3");
}
} // namespace

int mass_sg_conv3x3(const void* in, const void* w, int nout, int mode, int B, int H, int W,
                    const float* bias, const void* resid, const void* aux, void* out, void* out2,
                    const float* resid_f, float* out_f, int* err, void* stream)
{
  return conv_call(in, w, nout, mode, B, H, W, bias, resid, aux, out, out2, resid_f, out_f, err,
                   nullptr, nullptr, stream);
}

int mass_sg_conv_strip_rows(int B, int H, int W, int nsm)
{
  return conv3x3_strip_rows(B, H, W, nsm);
}

int mass_sg_conv3x3_profile(const void* in, const void* w, int nout, int mode, int B, int H,
                            int W, const float* bias, const void* resid, const void* aux,
                            void* out, void* out2, const float* resid_f, float* out_f, int* err,
                            long long* cycles, int* ncta, void* stream)
{
  if(!cycles || !ncta) return sg_fail(MASS_LB_EINVAL, "null cycles or ncta");
  return conv_call(in, w, nout, mode, B, H, W, bias, resid, aux, out, out2, resid_f, out_f, err,
                   cycles, ncta, stream);
}

int mass_sg_conv3x3_wgrad(const void* x, const void* dy, float* dW, int B, int H, int W, int* err,
                          void* stream)
{
  if(!x || !dy || !dW || !err) return sg_fail(MASS_LB_EINVAL, "null argument");
  if(!dims_ok(B, H, W)) return sg_fail(MASS_LB_EINVAL, "need B, H >= 1 and W a multiple of 128");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if(int r = sg_cuda(cudaMemsetAsync(dW, 0, 9*64*64*sizeof(float), st), "memset")) return r;
  return sg_cuda(conv3x3_wgrad_launch(static_cast<const __nv_bfloat16*>(x),
                                      static_cast<const __nv_bfloat16*>(dy), dW, B, H, W, err, st),
                 "conv3x3 wgrad");
}

int mass_sg_bias_grad(const void* dy, float* db, int B, int H, int W, void* stream)
{
  if(!dy || !db) return sg_fail(MASS_LB_EINVAL, "null argument");
  if(!dims_ok(B, H, W)) return sg_fail(MASS_LB_EINVAL, "need B, H >= 1 and W a multiple of 128");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if(int r = sg_cuda(cudaMemsetAsync(db, 0, 64*sizeof(float), st), "memset")) return r;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::max(1, std::min((B*H + 7)/8, 4*sms));
  k_bias_grad<<<grid, 256, 0, st>>>(static_cast<const __nv_bfloat16*>(dy), db, B, H, W);
  return sg_cuda(cudaGetLastError(), "bias grad");
}

int mass_sg_pack(const float* fields, const int* src, const int* dst, int B, int H, int W,
                 void* x_in, float* xf, float* target, void* stream)
{
  if(!fields || !src || !x_in || !xf || (target && !dst)) return sg_fail(MASS_LB_EINVAL, "null argument");
  if(!dims_ok(B, H, W)) return sg_fail(MASS_LB_EINVAL, "need B, H >= 1 and W a multiple of 128");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_pack<<<grid_for(static_cast<long long>(B)*H*W), 256, 0, st>>>(
    fields, src, dst, B, H, W, static_cast<__nv_bfloat16*>(x_in), xf, target);
  return sg_cuda(cudaGetLastError(), "pack");
}

int mass_sg_mse(const float* pred, const float* target, int B, int H, int W, double* sse,
                void* dout, void* stream)
{
  if(!pred || !target || !sse || !dout) return sg_fail(MASS_LB_EINVAL, "null argument");
  if(!dims_ok(B, H, W)) return sg_fail(MASS_LB_EINVAL, "need B, H >= 1 and W a multiple of 128");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_mse<<<grid_for(static_cast<long long>(B)*H*W), 256, 0, st>>>(
    pred, target, B, H, W, sse, static_cast<__nv_bfloat16*>(dout));
  return sg_cuda(cudaGetLastError(), "mse");
}

int mass_sg_adamw(float* w, float* b, float* mw, float* vw, float* mb, float* vb, const float* dW,
                  const float* db, int cout, int cin, int nout_pad, float lr, float beta1,
                  float beta2, float eps, float weight_decay, float bc1, float bc2, void* wt,
                  void* wd, void* stream)
{
  if(!w || !b || !mw || !vw || !mb || !vb || !dW || !db || !wt || !wd)
    return sg_fail(MASS_LB_EINVAL, "null argument");
  if(cout < 1 || cout > nout_pad || cin < 1 || cin > 64 || (nout_pad != 16 && nout_pad != 64))
    return sg_fail(MASS_LB_EINVAL, "layer shape out of range");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int n = cout*9*cin + cout;
  k_adamw<<<grid_for(n), 256, 0, st>>>(w, b, mw, vw, mb, vb, dW, db, cout, cin, nout_pad, lr,
                                       beta1, beta2, eps, weight_decay, bc1, bc2,
                                       static_cast<__nv_bfloat16*>(wt),
                                       static_cast<__nv_bfloat16*>(wd));
  return sg_cuda(cudaGetLastError(), "adamw");
}

int mass_sg_fields_from_state(const float* planes, long long plane_stride, int LX, int LY,
                              double rho, const float* mean, const float* scale, float* fields,
                              void* stream)
{
  if(!planes || !mean || !scale || !fields) return sg_fail(MASS_LB_EINVAL, "null argument");
  if(LX < 1 || LY < 1 || plane_stride < static_cast<long long>(LX)*LY)
    return sg_fail(MASS_LB_EINVAL, "bad lattice size or plane stride");
  const int N = LX*LY;
  k_fields_from_state<<<grid_for(N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
    planes, plane_stride, N, static_cast<float>(rho), make_norm(mean, scale), fields);
  return sg_cuda(cudaGetLastError(), "fields from state");
}

int mass_sg_state_from_fields(const float* fields, int LX, int LY, double rho, const float* mean,
                              const float* scale, float* planes, long long plane_stride,
                              void* stream)
{
  if(!planes || !mean || !scale || !fields) return sg_fail(MASS_LB_EINVAL, "null argument");
  if(LX < 1 || LY < 1 || plane_stride < static_cast<long long>(LX)*LY)
    return sg_fail(MASS_LB_EINVAL, "bad lattice size or plane stride");
  const int N = LX*LY;
  k_state_from_fields<<<grid_for(N), 256, 0, static_cast<cudaStream_t>(stream)>>>(
    fields, N, static_cast<float>(rho), make_norm(mean, scale), planes, plane_stride);
  return sg_cuda(cudaGetLastError(), "state from fields");
}

} // extern "C"
