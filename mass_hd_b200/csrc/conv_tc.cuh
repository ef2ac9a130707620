// Tensor-core 3x3 circular convolutions of the learned surrogate (BF16
// operands, FP32 accumulation in tensor memory).
//
// Activation layout ("padded NHWC64"): bf16 [B][H+2][W+2][64]; pixel (y, x)
// of image n lives at padded (y+1, x+1) and the one-pixel ring holds the
// periodic images (row 0 = row H, row H+1 = row 1, same for columns), so a
// 3x3 tap is a plain rectangular tile. Every kernel that writes such a tensor
// writes the ring too. W must be a multiple of 128.
//
// Weights: forward bf16 [9][NOUT][64] (tap-major, then output channel, then
// input channel; tap = 3*ky + kx multiplies input (y+ky-1, x+kx-1)); the
// input-gradient pass uses the flipped transpose [9][64][64] with
// Wd[8-tap][ci][co] = W[tap][co][ci].
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace mlb {

enum ConvMode
{
  CONV_FWD_BIAS = 0,    // out = acc + bias
  CONV_FWD_GELU = 1,    // out2 = acc + bias (pre-activation), out = gelu(out2)
  CONV_FWD_RESID = 2,   // out = acc + bias + resid
  CONV_FWD_OUT = 3,     // out_f[.., c<5] = acc + bias + resid_f   (NOUT = 16)
  CONV_BWD_GELU = 4,    // out = acc * gelu'(aux)
  CONV_BWD_RESID = 5,   // out = acc + resid
  CONV_BWD_PLAIN = 6,   // out = acc
};

struct ConvArgs
{
  int B, H, W;
  const float* bias;                 // NOUT floats (forward modes)
  const __nv_bfloat16* resid;        // padded NHWC64
  const __nv_bfloat16* aux;          // padded NHWC64 (pre-activation, BWD_GELU)
  __nv_bfloat16* out;                // padded NHWC64
  __nv_bfloat16* out2;               // padded NHWC64 (FWD_GELU pre-activation)
  const float* resid_f;              // [B][H][W][5] (FWD_OUT)
  float* out_f;                      // [B][H][W][5] (FWD_OUT)
  int* err;                          // bit 1: a bounded wait gave up
  int rows = 0;                      // strip height; conv3x3_launch sets it
  // optional, 4 per CTA (grid = min(strips, SMs)): the MMA thread's cycles
  // from start to done, to its last issue, waiting for input slabs, waiting
  // for drained accumulators
  long long* cycles = nullptr;
};

// in: padded NHWC64; w: forward weights [9][nout][64] (nout 64 or 16) or the
// input-gradient weights [9][64][64] (nout 64).
// Strip height the forward / input-gradient kernel uses for B images of H x
// W on a GPU with nsm SMs (host arithmetic only; MASS_SG_CONV_ROWS, which
// conv3x3_launch honours, is not read here).
int conv3x3_strip_rows(int B, int H, int W, int nsm);

// *ncta (if given) receives the number of CTAs launched.
cudaError_t conv3x3_launch(const __nv_bfloat16* in, const __nv_bfloat16* w, int nout, int mode,
                           const ConvArgs& a, cudaStream_t st, int* ncta = nullptr);

// dW[tap][ci][co] += sum over pixels of x(p + tap offset)[ci] * dy(p)[co];
// x and dy padded NHWC64; dW fp32 [9][64][64], accumulated with atomics
// (the caller zeroes it).
cudaError_t conv3x3_wgrad_launch(const __nv_bfloat16* x, const __nv_bfloat16* dy, float* dW,
                                 int B, int H, int W, int* err, cudaStream_t st);

} // namespace mlb
