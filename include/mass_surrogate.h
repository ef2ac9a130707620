/* Learned surrogate of the lyotropic Step(): C ABI of the device kernels.
 *
 * The reference has no surrogate, so none of these entry points replaces a
 * reference interface. They are the convolution, loss, optimizer and
 * state-conversion kernels of a residual CNN that maps the lattice fields
 * (Qxx, Qyx, phi, ux, uy) forward by a fixed number of LB steps; the driver
 * (mass_hd_b200/surrogate.py) owns the buffers and calls them in order.
 *
 * Conventions: every pointer is a DEVICE pointer unless stated; `stream` is
 * a cudaStream_t (NULL = default stream); calls are asynchronous and return
 * 0 or a negative mass_lb_status (text in mass_lb_last_error()).
 *
 * Layouts:
 *  - padded NHWC64: bf16 [B][H+2][W+2][64]; pixel (y, x) at (y+1, x+1); the
 *    one-pixel ring holds the periodic images. W must be a multiple of 128.
 *    Every call that writes such a tensor writes its ring too.
 *  - fields: fp32 [B][H][W][5], channels (Qxx, Qyx, phi, ux, uy), each
 *    normalised as (value - mean[c]) / scale[c].
 *  - forward weights: bf16 [9][nout][64] (tap = 3*ky + kx multiplies input
 *    pixel (y+ky-1, x+kx-1)); input-gradient weights: bf16 [9][64][64],
 *    Wd[8-tap][ci][co] = W[tap][co][ci].
 *  - master weights: fp32 [cout][9][cin]; weight gradients from
 *    mass_sg_conv3x3_wgrad: fp32 [9][64 ci][64 co].
 */
#ifndef MASS_SURROGATE_H
#define MASS_SURROGATE_H

#ifdef __cplusplus
extern "C" {
#endif

enum mass_sg_conv_mode {
  MASS_SG_FWD_BIAS = 0,   /* out = conv + bias */
  MASS_SG_FWD_GELU = 1,   /* out2 = conv + bias; out = gelu(out2) (tanh form) */
  MASS_SG_FWD_RESID = 2,  /* out = conv + bias + resid */
  MASS_SG_FWD_OUT = 3,    /* out_f[c < 5] = conv + bias + resid_f (nout = 16) */
  MASS_SG_BWD_GELU = 4,   /* out = conv * gelu'(aux) */
  MASS_SG_BWD_RESID = 5,  /* out = conv + resid */
  MASS_SG_BWD_PLAIN = 6   /* out = conv */
};

/* 3x3 circular convolution of a padded NHWC64 tensor on the tensor cores
 * (BF16 operands, FP32 accumulation), with the fused epilogue of `mode`.
 * bias: nout floats (forward modes). err: device int, bit 1 set if a
 * bounded wait inside the kernel gave up. */
int mass_sg_conv3x3(const void* in, const void* w, int nout, int mode, int B, int H, int W,
                    const float* bias, const void* resid, const void* aux, void* out, void* out2,
                    const float* resid_f, float* out_f, int* err, void* stream);

/* mass_sg_conv3x3 that also writes the cycle counters of each CTA's MMA
 * thread to `cycles` (device, 4 long longs per CTA, at most 4 x the SM
 * count): cycles from start to done, to the last MMA issue, waiting for
 * input slabs, waiting for drained accumulators. *ncta receives the
 * number of CTAs launched. A profiling aid; same results as
 * mass_sg_conv3x3. */
int mass_sg_conv3x3_profile(const void* in, const void* w, int nout, int mode, int B, int H,
                            int W, const float* bias, const void* resid, const void* aux,
                            void* out, void* out2, const float* resid_f, float* out_f, int* err,
                            long long* cycles, int* ncta, void* stream);

/* The strip height mass_sg_conv3x3 uses for B images of H x W on a GPU
 * with nsm SMs: each CTA marches down strips of that many output rows (a
 * divisor of H, at most 16), loading each input row once per strip. Host
 * arithmetic, no GPU needed; the environment variable MASS_SG_CONV_ROWS,
 * which mass_sg_conv3x3 honours, is not read here. */
int mass_sg_conv_strip_rows(int B, int H, int W, int nsm);

/* dW[tap][ci][co] = sum_p x(p + tap)[ci] * dy(p)[co] (zeroes dW first). */
int mass_sg_conv3x3_wgrad(const void* x, const void* dy, float* dW, int B, int H, int W,
                          int* err, void* stream);

/* db[c] = sum over pixels of dy[c], c < 64 (zeroes db first). */
int mass_sg_bias_grad(const void* dy, float* db, int B, int H, int W, void* stream);

/* Network input from stored fields: for each batch item b, x_in[b] (padded
 * NHWC64, channels 5..63 zero) and xf[b] from fields[src[b]], and
 * target[b] from fields[dst[b]] (target may be NULL). src/dst: device ints. */
int mass_sg_pack(const float* fields, const int* src, const int* dst, int B, int H, int W,
                 void* x_in, float* xf, float* target, void* stream);

/* Mean squared error over B*H*W*5 values: accumulates sum (pred-target)^2
 * into *sse (device double, not zeroed) and writes dout = d(mean)/d(pred) as
 * padded NHWC64 (channels 5..63 zero). */
int mass_sg_mse(const float* pred, const float* target, int B, int H, int W, double* sse,
                void* dout, void* stream);

/* One AdamW step of a layer: master w [cout][9][cin], bias b [cout], moments
 * (same shapes); gradients dW [9][64][64] and db [64]; writes the bf16
 * forward weights wt [9][nout_pad][64] and input-gradient weights wd
 * [9][64][64] (entries outside cout x cin are left as they are). bc1, bc2:
 * 1 - beta1^t, 1 - beta2^t. */
int mass_sg_adamw(float* w, float* b, float* mw, float* vw, float* mb, float* vb,
                  const float* dW, const float* db, int cout, int cin, int nout_pad,
                  float lr, float beta1, float beta2, float eps, float weight_decay,
                  float bc1, float bc2, void* wt, void* wd, void* stream);

/* Lattice state <-> fields. planes: the FP32 fused state of a lattice
 * (mass_lb_device_state: g0..g8 as deviations from t_v*rho, Qxx, Qyx, phi,
 * plane_stride floats apart), LX x LY sites; the field image has H = LX rows
 * and W = LY columns (site k = y + LY*x is pixel k). mean/scale: 5 floats
 * each, HOST pointers. fields_from_state: velocity = first moment / density. */
int mass_sg_fields_from_state(const float* planes, long long plane_stride, int LX, int LY,
                              double rho, const float* mean, const float* scale, float* fields,
                              void* stream);
/* state_from_fields: populations at equilibrium with density rho and the
 * fields' velocity (the second-order equilibrium of src/lb.hpp:24-41), Q and
 * phi from the fields. */
int mass_sg_state_from_fields(const float* fields, int LX, int LY, double rho, const float* mean,
                              const float* scale, float* planes, long long plane_stride,
                              void* stream);

#ifdef __cplusplus
}
#endif
#endif
