// Implicit-GEMM 3x3 circular convolutions on the sm_100a tensor cores.
//
// Forward and input-gradient pass (conv3x3_kernel): D[128 pixels][NOUT] =
// sum over 9 taps of A_tap[128 pixels][64 ci] * B_tap[NOUT][64 ci]^T. One
// output tile is half a row of one image (128 consecutive x). A CTA marches
// down strips of R output rows of one image half (R a divisor of H, up to
// 16). For each padded input row of a strip (R + 2 of them), one TMA load
// (128-byte swizzle) brings a slab of 136 pixels; the three taps of that
// row are the slab read from pixel 0, 1 and 2 (descriptor start 128 bytes
// apart). The slab feeds up to three output rows (tap rows ky = 0, 1, 2 of
// output rows j, j-1, j-2), so each A operand (slab, tap column, 16-channel
// step) goes once through the tensor core's A collector buffer and meets
// the weights of every tap row that needs it: shared-memory operand reads
// per output row drop from 36 A + 36 B to 12 A + 36 B. All 9 weight taps
// stay in shared memory for the whole persistent kernel. Warp roles: warp
// 0 issues TMA loads into a 5-slab ring, warp 1 issues tcgen05.mma into
// four TMEM accumulators (output rows in flight, one per row modulo 4), and
// warps 2-17 form two epilogue groups that take alternate output rows, so
// two rows' epilogues run at once. An epilogue drains its accumulator
// (tcgen05.ld), applies the fused bias / GELU / residual / GELU' epilogue
// in packed FP32x2, stages the bf16 tile in swizzled shared memory and
// writes it (and its periodic ring row) with TMA stores; residual and
// pre-activation inputs arrive as TMA tiles.
//
// Weight gradient (conv3x3_wgrad_kernel): dW_tap[ci][co] = sum over pixels of
// x(p + tap)[ci] * dy(p)[co]. K runs over pixels, so both operands are read
// MN-major straight from the NHWC tiles. A CTA computes all 9 taps (five tap
// pairs, M = 2 x 64 input channels, the pair's tiles LBO apart in the three
// input slabs of a block) for a contiguous range of 128-pixel blocks,
// accumulates in TMEM and adds its partial sums to dW with vector
// reductions.
//
// Every mbarrier wait is bounded (about a second); on time-out the role sets
// an error bit, the others stop at their next wait, outstanding MMAs are
// awaited (bounded) and TMEM is freed before the CTA exits.
#include "conv_tc.cuh"
#include "tc_ptx.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

namespace mlb {

using namespace tc;

namespace {

constexpr int EPI_WARPS = 16;         // epilogue warps of the forward / input-gradient kernel
constexpr int CONV_THREADS = 64 + 32*EPI_WARPS;   // + TMA warp + MMA warp
constexpr int WG_THREADS = 192;       // weight gradient: TMA, MMA, 4 x epilogue
constexpr int SLAB_PX = 136;                 // 128 outputs + 2 halo pixels, rounded to 8 rows
constexpr uint32_t SLAB_BYTES = SLAB_PX*128u;   // multiple of 1024
constexpr uint32_t TILE_BYTES = 128u*128u;   // 128 pixels x 64 bf16 (weight-gradient tiles)

template<int NOUT>
struct ConvSmem
{
  // 64-channel outputs go out through a staging tile and a TMA store; an
  // epilogue input (residual, pre-activation) comes in as a TMA tile, or the
  // second staging tile holds the pre-activation output of FWD_GELU.
  // Two epilogue groups (one per TMEM accumulator) each own an output
  // staging tile and an aux tile.
  static constexpr int NSTAGE = NOUT == 64 ? 5 : 8;
  static constexpr uint32_t W_BYTES = 9u*NOUT*128u;          // multiple of 1024
  static constexpr uint32_t A_OFF = W_BYTES;
  static constexpr uint32_t OUT_OFF = A_OFF + NSTAGE*SLAB_BYTES;          // [group]
  static constexpr uint32_t AUX_OFF = OUT_OFF + (NOUT == 64 ? 2*TILE_BYTES : 0u);  // [group]
  static constexpr uint32_t BAR_OFF = AUX_OFF + (NOUT == 64 ? 2*TILE_BYTES : 0u);
  static constexpr int NACC = 4;             // TMEM accumulators (output rows in flight), a power of 2
  static constexpr int NBAR = 2*NSTAGE + 2*NACC + 4;  // full, empty, w, tfull[NACC], tempty[NACC], done, aux[2]
  static constexpr uint32_t MISC_OFF = BAR_OFF + NBAR*8;
  static constexpr uint32_t BIAS_OFF = MISC_OFF + 16;
  static constexpr uint32_t BYTES = BIAS_OFF + 64*4;
  static constexpr uint32_t ALLOC = BYTES + 1024;            // room to align the base
  static constexpr uint32_t TMEM_COLS = NACC*NOUT;          // 256 or 64 columns
  static_assert(ALLOC <= 232448, "shared memory per CTA");
};

__device__ __forceinline__ uint8_t* align1024(uint8_t* p)
{
  const uint32_t a = smem_u32(p);
  return p + ((1024u - (a & 1023u)) & 1023u);
}

__device__ __forceinline__ size_t padded_index(int n, int yy, int xx, int H, int W)
{
  return (static_cast<size_t>(n)*(H + 2) + yy)*static_cast<size_t>(W + 2) + xx;
}

// GELU in its tanh form (Hendrycks & Gimpel, "Gaussian Error Linear Units",
// 2016): gelu(x) = x/2 (1 + tanh(u)), u = sqrt(2/pi) (x + 0.044715 x^3),
// with the hardware tanh estimate (tanh.approx.f32). Pairs of channels go
// through the packed FP32x2 pipe.
constexpr float GELU_C = 0.7978845608028654f;    // sqrt(2/pi)
constexpr float GELU_A = 0.044715f;

__device__ __forceinline__ float tanh_approx(float x)
{
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2s(float s) { return make_float2(s, s); }

// tanh(u) of a pair, with u = C x (1 + A x^2)
__device__ __forceinline__ float2 gelu_t(float2 x, float2& x2)
{
  x2 = f2mul(x, x);
  const float2 u = f2mul(f2mul(f2s(GELU_C), x), f2fma(f2s(GELU_A), x2, f2s(1.f)));
  return make_float2(tanh_approx(u.x), tanh_approx(u.y));
}
__device__ __forceinline__ float2 gelu2(float2 x)
{
  float2 x2;
  const float2 t = gelu_t(x, x2);
  const float2 hx = f2mul(f2s(0.5f), x);
  return f2fma(hx, t, hx);                                   // x/2 (1 + t)
}
// d gelu / dx = (1 + t)/2 + x/2 (1 - t^2) C (1 + 3 A x^2)
__device__ __forceinline__ float2 gelu_grad2(float2 x)
{
  float2 x2;
  const float2 t = gelu_t(x, x2);
  const float2 sech2 = f2fma(make_float2(-t.x, -t.y), t, f2s(1.f));          // 1 - t^2
  const float2 du = f2mul(f2s(GELU_C), f2fma(f2s(3.f*GELU_A), x2, f2s(1.f))); // du/dx
  const float2 a = f2fma(f2s(0.5f), t, f2s(0.5f));                          // (1 + t)/2
  return f2fma(f2mul(f2mul(f2s(0.5f), x), sech2), du, a);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ void unpack8(const uint4& u, float* f)
{
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
  for(int i = 0; i < 4; ++i)
  {
    const float2 t = __bfloat1622float2(h[i]);
    f[2*i] = t.x;
    f[2*i + 1] = t.y;
  }
}

// Output rows of one CTA: the CTA takes strips (image n, half-row column
// xt, R consecutive rows from y0) item = blockIdx.x, + gridDim.x, ...; its
// t-th output row is row t % R of its (t / R)-th strip. The coordinates are
// recomputed from the kernel parameters where they are needed, so the
// epilogue keeps no extra registers live (at 576 threads it has 96).
__device__ __forceinline__ void strip_item(const ConvArgs& a, int it, int& n, int& x0, int& y0)
{
  const int xt_n = a.W >> 7, spi = a.H / a.rows;
  const int xt = it % xt_n, s = it / xt_n;
  x0 = xt << 7;
  y0 = (s % spi)*a.rows;
  n = s / spi;
}
__device__ __forceinline__ int strip_items(const ConvArgs& a)
{
  return a.B*(a.W >> 7)*(a.H / a.rows);
}
__device__ __forceinline__ void strip_row(const ConvArgs& a, int t, int& n, int& x0, int& y)
{
  int y0;
  strip_item(a, static_cast<int>(blockIdx.x) + (t / a.rows)*static_cast<int>(gridDim.x), n, x0, y0);
  y = y0 + t % a.rows;
}

// The MMAs of one input slab (padded row y0 + j of a strip) inside a strip:
// the slab feeds output rows j, j-1, j-2 with tap rows ky = 0, 1, 2. For
// each tap column kx and 16-channel step k, the slab's A operand goes once
// through the collector buffer (fill, use, lastuse) and meets the weights
// of the three tap rows. d0, d1, d2 are the accumulators of output rows j,
// j-1, j-2.
template<int NOUT>
__device__ __forceinline__ void slab_mmas(uint32_t d0, uint32_t d1, uint32_t d2, uint64_t da,
                                          uint64_t db, uint32_t idesc)
{
#pragma unroll
  for(int kx = 0; kx < 3; ++kx)
  {
#pragma unroll
    for(int k = 0; k < 4; ++k)
    {
      const uint64_t a = da + ((kx*128 + 32*k) >> 4);
      const uint64_t b = db + ((kx*NOUT*128 + 32*k) >> 4);
      // the first contribution to an output row (tap 0, first K step)
      // overwrites the accumulator
      mma_bf16_coll<1>(d0, a, b, idesc, (kx | k) != 0);
      mma_bf16_coll<2>(d1, a, b + ((3*NOUT*128) >> 4), idesc, 1u);
      mma_bf16_coll<3>(d2, a, b + ((6*NOUT*128) >> 4), idesc, 1u);
    }
  }
}

template<int NOUT, int MODE>
__global__ void __launch_bounds__(CONV_THREADS, 1)
conv3x3_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmW,
               const __grid_constant__ CUtensorMap tmO, const __grid_constant__ CUtensorMap tmO2,
               const __grid_constant__ CUtensorMap tmR, const ConvArgs a)
{
  using L = ConvSmem<NOUT>;
  constexpr int STAGES = L::NSTAGE;
  constexpr int NACC = L::NACC;
  constexpr bool HAS_AUX = MODE == CONV_FWD_RESID || MODE == CONV_BWD_RESID || MODE == CONV_BWD_GELU;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = align1024(smem_raw);
  uint8_t* Wsm = sm;
  uint8_t* Asm = sm + L::A_OFF;
  uint8_t* outS0 = sm + L::OUT_OFF;
  uint8_t* auxS0 = sm + L::AUX_OFF;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + L::BAR_OFF);
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* wbar = bars + 2*STAGES;
  uint64_t* tfull = wbar + 1;              // [NACC]
  uint64_t* tempty = tfull + NACC;         // [NACC]
  uint64_t* done = tempty + NACC;
  uint64_t* abar0 = done + 1;              // [group]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + L::MISC_OFF);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + L::MISC_OFF + 4);
  float* bias_sm = reinterpret_cast<float*>(sm + L::BIAS_OFF);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int H = a.H, W = a.W, R = a.rows;
  const int nitems = strip_items(a);
  // this CTA's output rows
  const int nrows = static_cast<int>(blockIdx.x) < nitems
                  ? ((nitems - static_cast<int>(blockIdx.x) + static_cast<int>(gridDim.x) - 1)/
                     static_cast<int>(gridDim.x))*R : 0;

  if(threadIdx.x == 0)
  {
    for(int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(wbar, 1);
    // 64-channel kernels: one epilogue group of EPI_WARPS/2 warps releases
    // each accumulator; the output layer: every epilogue warp
    const uint32_t releases = NOUT == 64 ? EPI_WARPS/2 : EPI_WARPS;
    for(int c = 0; c < NACC; ++c) { mbar_init(&tfull[c], 1); mbar_init(&tempty[c], releases); }
    mbar_init(done, 1);
    mbar_init(&abar0[0], 1);
    mbar_init(&abar0[1], 1);
    *abort_flag = 0;
    fence_barrier_init();
    fence_proxy_async();
  }
  if(warp == 1) tmem_alloc(tmem_slot, L::TMEM_COLS);
  if(threadIdx.x >= 64 && threadIdx.x < 64 + NOUT)
    bias_sm[threadIdx.x - 64] = (MODE <= CONV_FWD_OUT && a.bias) ? a.bias[threadIdx.x - 64] : 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;

  auto give_up = [&]() {
    *abort_flag = 1;
    atomicOr(a.err, 2);
  };

  if(warp == 0)
  {
    if(lane == 0)
    {
      prefetch_map(&tmX);
      prefetch_map(&tmW);
      mbar_expect_tx(wbar, L::W_BYTES);
      for(int t = 0; t < 9; ++t) tma_load_3d(Wsm + t*NOUT*128, &tmW, 0, 0, t, wbar);
      uint32_t it = 0;
      bool ok = true;
      for(int item = blockIdx.x; ok && item < nitems && !*abort_flag; item += gridDim.x)
      {
        int n, x0, y0;
        strip_item(a, item, n, x0, y0);
        // padded input rows y0 .. y0 + R + 1 feed output rows y0 .. y0 + R - 1
        for(int j = 0; j < R + 2; ++j, ++it)
        {
          const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
          if(!mbar_wait(&empty[s], ph ^ 1u)) { give_up(); ok = false; break; }
          mbar_expect_tx(&full[s], SLAB_BYTES);
          tma_load_4d(Asm + s*SLAB_BYTES, &tmX, 0, x0, y0 + j, n, &full[s]);
        }
      }
      // loads still in flight after an abort land before the CTA exits
      if(*abort_flag)
        for(uint32_t k = 0; k < STAGES && k < it; ++k)
        {
          const uint32_t j = it - 1 - k;
          mbar_wait(&full[j % STAGES], (j / STAGES) & 1u);
        }
    }
  }
  else if(warp == 1)
  {
    if(lane == 0)
    {
      constexpr uint32_t IDESC = idesc_bf16_f32(128, NOUT, 0, 0);
      bool ok = mbar_wait(wbar, 0);
      if(!ok) give_up();
      const uint32_t wbase = smem_u32(Wsm), abase = smem_u32(Asm);
      const uint64_t db = sw128_desc(wbase, 16, 1024);
      // cycle counters of this thread (ConvArgs::cycles): waits for input
      // slabs and for drained accumulators, and the span to the last issue
      long long w_slab = 0, w_acc = 0;
      const long long c_start = clock64();
      uint32_t it = 0;
      int t0 = 0;                    // this CTA's index of the strip's first output row
      for(int item = blockIdx.x; ok && item < nitems && !*abort_flag; item += gridDim.x, t0 += R)
      {
        for(int j = 0; j < R + 2; ++j, ++it)
        {
          if(j < R)
          {
            // output row j starts here: its accumulator must be drained
            const int t = t0 + j;
            const uint32_t acc = t % NACC, use = t / NACC;
            const long long c0 = clock64();
            const bool got = mbar_wait(&tempty[acc], (use & 1u) ^ 1u);
            w_acc += clock64() - c0;
            if(!got) { give_up(); ok = false; break; }
            tc_fence_after();
          }
          const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
          const long long c0 = clock64();
          const bool got = mbar_wait(&full[s], ph);
          w_slab += clock64() - c0;
          if(!got) { give_up(); ok = false; break; }
          tc_fence_after();
          // slab j feeds output rows j - ky for ky in [lo, hi]
          const int lo = j >= R ? j - R + 1 : 0;
          const int hi = j < 2 ? j : 2;
          const uint32_t d0 = tbase + ((t0 + j) & (NACC - 1))*NOUT;
          const uint32_t d1 = tbase + ((t0 + j - 1) & (NACC - 1))*NOUT;
          const uint32_t d2 = tbase + ((t0 + j - 2) & (NACC - 1))*NOUT;
          const uint64_t da = sw128_desc(abase + s*SLAB_BYTES, 16, 1024);
          // the weight descriptor base, opaque to the compiler inside the
          // loop: otherwise it hoists all 36 loop-invariant B descriptors
          // into registers, and the kernel (96 registers at 576 threads)
          // spills
          uint64_t dbs;
          asm volatile("mov.b64 %0, %1;" : "=l"(dbs) : "l"(db));
          if(lo == 0 && hi == 2) slab_mmas<NOUT>(d0, d1, d2, da, dbs, IDESC);
          else
          {
            // a strip's first two and last two slabs feed only the one or
            // two output rows inside the strip: a compact loop without the
            // collector (an unrolled variant per case costs registers)
#pragma unroll 1
            for(int ky = lo; ky <= hi; ++ky)
            {
              const uint32_t d = tbase + ((t0 + j - ky) & (NACC - 1))*NOUT;
              const uint64_t dbk = sw128_desc(wbase + 3*ky*NOUT*128, 16, 1024);
#pragma unroll
              for(int kx = 0; kx < 3; ++kx)
              {
#pragma unroll
                for(int k = 0; k < 4; ++k)
                  mma_bf16(d, da + ((kx*128 + 32*k) >> 4), dbk + ((kx*NOUT*128 + 32*k) >> 4), IDESC,
                           (ky | kx | k) != 0);
              }
            }
          }
          mma_commit(&empty[s]);
          // output row j - 2 has all its contributions
          if(j >= 2) mma_commit(&tfull[(t0 + j - 2) & (NACC - 1)]);
        }
      }
      mma_commit(done);
      const long long c_issue = clock64() - c_start;
      if(!mbar_wait(done, 0)) give_up();
      if(a.cycles)
      {
        long long* c = a.cycles + 4*blockIdx.x;
        c[0] = clock64() - c_start;
        c[1] = c_issue;
        c[2] = w_slab;
        c[3] = w_acc;
      }
    }
  }
  else if constexpr(NOUT == 16)
  {
    // output layer: 5 fp32 channels per pixel, stored directly; the warps of
    // the first 16-column slice hold all 16 columns, the others only release
    const int q = warp & 3;
    const int c0 = ((warp - 2) >> 2)*16;
    for(int t = 0; t < nrows; ++t)
    {
      if(__any_sync(0xffffffffu, *abort_flag != 0)) break;
      const uint32_t acc = t & (NACC - 1), use = t / NACC;
      int n, x0, y;
      strip_row(a, t, n, x0, y);
      const int x = x0 + q*32 + lane;
      if(!__all_sync(0xffffffffu, mbar_wait(&tfull[acc], use & 1u)))
      {
        if(lane == 0) give_up();
        break;
      }
      tc_fence_after();
      float v[16];
      if(c0 == 0) tmem_ld16(tbase + (static_cast<uint32_t>(q*32) << 16) + acc*NOUT, v);
      tc_fence_before();
      __syncwarp();
      if(lane == 0) mbar_arrive(&tempty[acc]);
      if(c0 == 0)
      {
        const size_t p = (static_cast<size_t>(n)*H + y)*W + x;
#pragma unroll
        for(int c = 0; c < 5; ++c)
          a.out_f[5*p + c] = v[c] + bias_sm[c] + (a.resid_f ? a.resid_f[5*p + c] : 0.f);
      }
    }
  }
  else
  {
    // Two groups of 8 epilogue warps; group g drains the output rows t = g,
    // g + 2, ... of this CTA (accumulator t % NACC), so two rows' epilogues
    // run at once. Within a group thread = pixel p = 32q + lane of the tile,
    // channels c0..c0+31 (two warps per TMEM lane quarter). The output tile
    // is staged in shared memory in the 128-byte-swizzled layout and written
    // by TMA stores (row y and, on the first / last image row, the periodic
    // ring row); the two ring columns are written directly by the threads of
    // pixels 0 and W-1. Every branch that leaves the loop is agreed by all
    // 256 threads of the group (named_and), so the group's named barrier is
    // always met by all.
    constexpr int GROUP_N = 32*EPI_WARPS/2;
    const int e = warp - 2;
    const int g = e / (EPI_WARPS/2);
    const int bar_id = 1 + g;
    const int q = warp & 3;
    const int c0 = ((e % (EPI_WARPS/2)) >> 2)*32;
    const int p = q*32 + lane;
    const bool leader = (e % (EPI_WARPS/2)) == 0 && lane == 0;
    uint8_t* outS = outS0 + g*TILE_BYTES;
    uint8_t* auxS = auxS0 + g*TILE_BYTES;
    uint64_t* abar = &abar0[g];
    // the four 16-byte chunks of channels c0..c0+31 in this pixel's swizzled row
    uint32_t off[4];
#pragma unroll
    for(int k = 0; k < 4; ++k) off[k] = p*128u + ((((c0 >> 3) + k) ^ (p & 7)) << 4);
    bool aux_pending = false;
    if constexpr(HAS_AUX)
    {
      if(leader && g < nrows)
      {
        int n, x0, y;
        strip_row(a, g, n, x0, y);
        mbar_expect_tx(abar, TILE_BYTES);
        tma_load_4d(auxS, &tmR, 0, x0 + 1, y + 1, n, abar);
        aux_pending = true;
      }
    }
    uint32_t k = 0;
    for(int t = g; t < nrows; t += 2, ++k)
    {
      int n, x0, y;
      strip_row(a, t, n, x0, y);
      const int x = x0 + p;
      const uint32_t acc = t & (NACC - 1), use = t / NACC;
      bool ok = *abort_flag == 0 && mbar_wait(&tfull[acc], use & 1u);
      if constexpr(HAS_AUX) ok = ok && mbar_wait(abar, k & 1u);
      if(!named_and(bar_id, GROUP_N, ok))
      {
        if(leader) give_up();
        break;
      }
      if constexpr(HAS_AUX) if(leader) aux_pending = false;
      tc_fence_after();
      float v[32];
      const uint32_t taddr = tbase + (static_cast<uint32_t>(q*32) << 16) + acc*NOUT + c0;
      tmem_ld16(taddr, v);
      tmem_ld16(taddr + 16, v + 16);
      tc_fence_before();
      __syncwarp();
      if(lane == 0) mbar_arrive(&tempty[acc]);
      float r[32];
      if constexpr(HAS_AUX)
      {
#pragma unroll
        for(int c = 0; c < 4; ++c) unpack8(*reinterpret_cast<const uint4*>(auxS + off[c]), r + 8*c);
      }
      float2* v2 = reinterpret_cast<float2*>(v);
      const float2* r2 = reinterpret_cast<const float2*>(r);
      if constexpr(MODE == CONV_FWD_BIAS || MODE == CONV_FWD_GELU || MODE == CONV_FWD_RESID)
      {
        const float2* b2 = reinterpret_cast<const float2*>(bias_sm + c0);
#pragma unroll
        for(int c = 0; c < 16; ++c) v2[c] = f2add(v2[c], b2[c]);
      }
      uint4 pre[4];
      if constexpr(MODE == CONV_FWD_GELU)
      {
#pragma unroll
        for(int c = 0; c < 4; ++c)
          pre[c] = make_uint4(pack_bf16x2(v[8*c], v[8*c + 1]), pack_bf16x2(v[8*c + 2], v[8*c + 3]),
                              pack_bf16x2(v[8*c + 4], v[8*c + 5]), pack_bf16x2(v[8*c + 6], v[8*c + 7]));
#pragma unroll
        for(int c = 0; c < 16; ++c) v2[c] = gelu2(v2[c]);
      }
      if constexpr(MODE == CONV_FWD_RESID || MODE == CONV_BWD_RESID)
      {
#pragma unroll
        for(int c = 0; c < 16; ++c) v2[c] = f2add(v2[c], r2[c]);
      }
      if constexpr(MODE == CONV_BWD_GELU)
      {
#pragma unroll
        for(int c = 0; c < 16; ++c) v2[c] = f2mul(v2[c], gelu_grad2(r2[c]));
      }
      uint4 pk[4];
#pragma unroll
      for(int c = 0; c < 4; ++c)
        pk[c] = make_uint4(pack_bf16x2(v[8*c], v[8*c + 1]), pack_bf16x2(v[8*c + 2], v[8*c + 3]),
                           pack_bf16x2(v[8*c + 4], v[8*c + 5]), pack_bf16x2(v[8*c + 6], v[8*c + 7]));
      // the group's previous stores must have read its staging tiles before
      // they are rewritten
      if(leader) bulk_wait_read_all();
      // (A) every thread of the group has read this tile's aux tile, and the
      // staging tiles are free
      named_sync(bar_id, GROUP_N);
      if constexpr(HAS_AUX)
      {
        if(leader && t + 2 < nrows)
        {
          int nn, nx0, ny;
          strip_row(a, t + 2, nn, nx0, ny);
          mbar_expect_tx(abar, TILE_BYTES);
          tma_load_4d(auxS, &tmR, 0, nx0 + 1, ny + 1, nn, abar);
          aux_pending = true;
        }
      }
#pragma unroll
      for(int c = 0; c < 4; ++c) *reinterpret_cast<uint4*>(outS + off[c]) = pk[c];
      if constexpr(MODE == CONV_FWD_GELU)
      {
#pragma unroll
        for(int c = 0; c < 4; ++c) *reinterpret_cast<uint4*>(auxS + off[c]) = pre[c];
      }
      // the two periodic ring columns (and the four corners) directly
      if(x == 0 || x == W - 1)
      {
        const int xs = x == 0 ? W + 1 : 0;
        int ys[3] = {y + 1, 0, 0}, ny = 1;
        if(y == 0) ys[ny++] = H + 1;
        if(y == H - 1) ys[ny++] = 0;
        for(int i2 = 0; i2 < ny; ++i2)
        {
          uint4* dst = reinterpret_cast<uint4*>(a.out + padded_index(n, ys[i2], xs, H, W)*64 + c0);
#pragma unroll
          for(int c = 0; c < 4; ++c) dst[c] = pk[c];
        }
      }
      fence_proxy_async();
      // (B) the staging tiles are complete
      named_sync(bar_id, GROUP_N);
      if(leader)
      {
        tma_store_4d(&tmO, 0, x0 + 1, y + 1, n, outS);
        if(y == 0) tma_store_4d(&tmO, 0, x0 + 1, H + 1, n, outS);
        if(y == H - 1) tma_store_4d(&tmO, 0, x0 + 1, 0, n, outS);
        if constexpr(MODE == CONV_FWD_GELU) tma_store_4d(&tmO2, 0, x0 + 1, y + 1, n, auxS);
        bulk_commit();
      }
    }
    if(leader)
    {
      bulk_wait_all();
      // an aux tile requested for a tile that was never processed lands
      // before the CTA exits
      if(aux_pending) mbar_wait(abar, k & 1u);
    }
  }

  tc_fence_before();
  __syncthreads();
  if(warp == 1)
  {
    tc_fence_after();
    tmem_dealloc(tbase, L::TMEM_COLS);
    tmem_relinquish();
  }
}

// ---- weight gradient ---------------------------------------------------------
//
// A CTA computes all 9 taps for a contiguous range of 128-pixel blocks. Per
// block one stage holds the three 136-pixel input slabs of padded rows y,
// y+1, y+2 (tap (ky, kx) of the block is slab ky read from pixel kx) and the
// dy tile: 68 KB of TMA writes for 40 MMAs, instead of 48 KB for every 8
// when a CTA owned one tap pair. A = two taps' input tiles, MN-major (M = 2
// x 64 input channels, the second group LBO bytes after the first, K =
// pixels), B = the dy tile; five tap pairs, five accumulators:
//   (0,0)+(0,1) and (1,0)+(1,1) and (2,0)+(2,1): one slab, LBO 128 B;
//   (0,2)+(1,2): slabs 0 and 1, LBO one slab;
//   (2,2) + a second group that is read but not kept (LBO 128 B, pixels
//   3..130 of slab 2, inside the slab).

constexpr int WG_STAGES = 3;
constexpr uint32_t WG_SLABS = 3*SLAB_BYTES;
constexpr uint32_t WG_STAGE = WG_SLABS + TILE_BYTES;     // three x slabs, dy
constexpr uint32_t WG_BAR_OFF = WG_STAGES*WG_STAGE;
constexpr uint32_t WG_MISC_OFF = WG_BAR_OFF + (2*WG_STAGES + 1)*8;
constexpr uint32_t WG_ALLOC = WG_MISC_OFF + 16 + 1024;
constexpr int WG_PAIRS = 5;
static_assert(WG_ALLOC <= 232448, "shared memory per CTA");

struct WgradArgs
{
  int B, H, W, nchunks;
  float* dW;
  int* err;
};

// tap of M group h (0 or 1) of pair p; -1: read but not kept
__device__ __forceinline__ int wg_tap(int p, int h)
{
  switch(p)
  {
    case 0: return h;          // (0,0), (0,1)
    case 1: return 3 + h;      // (1,0), (1,1)
    case 2: return 6 + h;      // (2,0), (2,1)
    case 3: return h ? 5 : 2;  // (0,2), (1,2)
    default: return h ? -1 : 8;
  }
}

__device__ __forceinline__ void red_add4(float* p, float a, float b, float c, float d)
{
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};"
               :: "l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

__global__ void __launch_bounds__(WG_THREADS, 1)
conv3x3_wgrad_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmD,
                     const WgradArgs a)
{
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = align1024(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + WG_BAR_OFF);
  uint64_t* empty = full + WG_STAGES;
  uint64_t* done = full + 2*WG_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + WG_MISC_OFF);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + WG_MISC_OFF + 4);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int chunk = blockIdx.x;
  const int xt_n = a.W >> 7;
  const long long nblocks = static_cast<long long>(a.B)*a.H*xt_n;
  const int b0 = static_cast<int>(chunk*nblocks/a.nchunks);
  const int b1 = static_cast<int>((chunk + 1)*nblocks/a.nchunks);

  if(threadIdx.x == 0)
  {
    for(int s = 0; s < WG_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(done, 1);
    *abort_flag = 0;
    fence_barrier_init();
    fence_proxy_async();
  }
  if(warp == 1) tmem_alloc(tmem_slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;
  auto give_up = [&]() {
    *abort_flag = 1;
    atomicOr(a.err, 2);
  };

  if(warp == 0)
  {
    if(lane == 0)
    {
      prefetch_map(&tmX);
      prefetch_map(&tmD);
      uint32_t it = 0;
      for(int blk = b0; blk < b1 && !*abort_flag; ++blk, ++it)
      {
        const int xt = blk % xt_n, row = blk / xt_n;
        const int y = row % a.H, n = row / a.H, x0 = xt << 7;
        const uint32_t s = it % WG_STAGES, ph = (it / WG_STAGES) & 1u;
        if(!mbar_wait(&empty[s], ph ^ 1u)) { give_up(); break; }
        uint8_t* st = sm + s*WG_STAGE;
        mbar_expect_tx(&full[s], WG_STAGE);
        for(int ky = 0; ky < 3; ++ky) tma_load_4d(st + ky*SLAB_BYTES, &tmX, 0, x0, y + ky, n, &full[s]);
        tma_load_4d(st + WG_SLABS, &tmD, 0, x0 + 1, y + 1, n, &full[s]);
      }
      if(*abort_flag)
        for(uint32_t k = 0; k < WG_STAGES && k < it; ++k)
        {
          const uint32_t j = it - 1 - k;
          mbar_wait(&full[j % WG_STAGES], (j / WG_STAGES) & 1u);
        }
    }
  }
  else if(warp == 1)
  {
    if(lane == 0)
    {
      // both operands MN-major: K = pixels in 8-row groups 1024 B apart
      constexpr uint32_t IDESC = idesc_bf16_f32(128, 64, 1, 1);
      const uint32_t base = smem_u32(sm);
      uint32_t it = 0;
      for(int blk = b0; blk < b1 && !*abort_flag; ++blk, ++it)
      {
        const uint32_t s = it % WG_STAGES, ph = (it / WG_STAGES) & 1u;
        if(!mbar_wait(&full[s], ph)) { give_up(); break; }
        tc_fence_after();
        const uint32_t st = base + s*WG_STAGE;
        const uint64_t db = sw128_desc(st + WG_SLABS, 1024, 1024);
        const uint64_t da[WG_PAIRS] = {
          sw128_desc(st, 128, 1024),
          sw128_desc(st + SLAB_BYTES, 128, 1024),
          sw128_desc(st + 2*SLAB_BYTES, 128, 1024),
          sw128_desc(st + 256, SLAB_BYTES, 1024),
          sw128_desc(st + 2*SLAB_BYTES + 256, 128, 1024)};
        const uint32_t first = blk == b0;
#pragma unroll
        for(int p = 0; p < WG_PAIRS; ++p)
        {
#pragma unroll
          for(int kk = 0; kk < 8; ++kk)
            mma_bf16(tbase + p*64, da[p] + ((kk*2048) >> 4), db + ((kk*2048) >> 4), IDESC,
                     !(first && kk == 0));
        }
        mma_commit(&empty[s]);
      }
      mma_commit(done);
      if(!mbar_wait(done, 0)) give_up();
    }
  }
  else if(b1 > b0)
  {
    // warps 2-5: TMEM lane quarter q = warp % 4 holds M rows 32q .. 32q+31
    const int q = warp & 3;
    if(!__all_sync(0xffffffffu, mbar_wait(done, 0)))
    {
      if(lane == 0) give_up();
    }
    else
    {
      tc_fence_after();
      const int m = q*32 + lane;
      const int h = m >> 6, ci = m & 63;
      const bool aborted = __any_sync(0xffffffffu, *abort_flag != 0);
      const uint32_t taddr = tbase + (static_cast<uint32_t>(q*32) << 16);
      for(int p = 0; p < WG_PAIRS; ++p)
      {
        float v[64];
        tmem_ld32(taddr + p*64, v);
        tmem_ld32(taddr + p*64 + 32, v + 32);
        const int tap = wg_tap(p, h);
        if(tap >= 0 && !aborted)
        {
          float* dst = a.dW + (static_cast<size_t>(tap)*64 + ci)*64;
#pragma unroll
          for(int co = 0; co < 64; co += 4) red_add4(dst + co, v[co], v[co + 1], v[co + 2], v[co + 3]);
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if(warp == 1)
  {
    tc_fence_after();
    tmem_dealloc(tbase, 512);
    tmem_relinquish();
  }
}

// ---- host side ------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
       q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// padded NHWC64 bf16 [B][H+2][W+2][64], box 64 channels x box_px pixels
// (a box reaching past the row's end is filled with zeros)
bool map_activation(CUtensorMap* m, const void* base, int B, int H, int W, int box_px)
{
  auto fn = encode_fn();
  if(!fn) return false;
  const cuuint64_t dims[4] = {64, static_cast<cuuint64_t>(W + 2), static_cast<cuuint64_t>(H + 2),
                              static_cast<cuuint64_t>(B)};
  const cuuint64_t strides[3] = {128, static_cast<cuuint64_t>(W + 2)*128,
                                 static_cast<cuuint64_t>(H + 2)*(W + 2)*128};
  const cuuint32_t box[4] = {64, static_cast<cuuint32_t>(box_px), 1, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// weights bf16 [9][nout][64], box 64 x nout
bool map_weights(CUtensorMap* m, const void* base, int nout)
{
  auto fn = encode_fn();
  if(!fn) return false;
  const cuuint64_t dims[3] = {64, static_cast<cuuint64_t>(nout), 9};
  const cuuint64_t strides[2] = {128, static_cast<cuuint64_t>(nout)*128};
  const cuuint32_t box[3] = {64, static_cast<cuuint32_t>(nout), 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int sm_count()
{
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

// the dynamic shared-memory opt-in, once per kernel and device
template<typename K>
cudaError_t smem_attr(K kern, unsigned long long& set_mask, int bytes)
{
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if(set_mask & bit) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if(e == cudaSuccess) set_mask |= bit;
  return e;
}

template<int NOUT, int MODE>
cudaError_t launch_mode(const CUtensorMap& tx, const CUtensorMap& tw, const CUtensorMap& to,
                        const CUtensorMap& to2, const CUtensorMap& tr, const ConvArgs& a,
                        cudaStream_t st, int* ncta)
{
  static unsigned long long attr = 0;
  auto kern = conv3x3_kernel<NOUT, MODE>;
  const cudaError_t e = smem_attr(kern, attr, static_cast<int>(ConvSmem<NOUT>::ALLOC));
  if(e != cudaSuccess) return e;
  const int nitems = a.B*(a.W >> 7)*(a.H / a.rows);
  const int grid = std::min(nitems, sm_count());
  if(ncta) *ncta = grid;
  kern<<<grid, CONV_THREADS, ConvSmem<NOUT>::ALLOC, st>>>(tx, tw, to, to2, tr, a);
  return cudaGetLastError();
}

// Strip height R of the forward / input-gradient kernel: a divisor of H of
// at most 16, so that every strip is whole. Each input slab serves up to
// three output rows of its strip, so taller strips load fewer slabs per
// output row (R + 2 per R rows), but they make fewer, longer work items.
// R minimises the busiest CTA's time: its output rows (whole strips per CTA
// times R) times the cost of a row, 0.724 + 0.245 (R + 2)/R, a fit to the
// measured time per row on B200 (strips of 1, 4, 8 and 16 rows at 32 x 256
// x 256: 1.46, 1.07, 1.02 and 1.00). At 32 x 256 x 256 that is 16 rows; at
// 16 x 256 x 256, 8 rows (56 rows per CTA against 64 with 16-row strips).
// MASS_SG_CONV_ROWS, a divisor of H from 1 to 64, fixes R.
int strip_rows(int B, int H, int W)
{
  if(const char* e = std::getenv("MASS_SG_CONV_ROWS"))
  {
    const int r = std::atoi(e);
    if(r >= 1 && r <= 64 && H % r == 0) return r;
  }
  return conv3x3_strip_rows(B, H, W, sm_count());
}

} // namespace

int conv3x3_strip_rows(int B, int H, int W, int nsm)
{
  if(B < 1 || H < 1 || W < 128 || nsm < 1) return 1;
  const long long halves = static_cast<long long>(B)*(W >> 7);
  const long long sms = nsm;
  int best = 1;
  double best_cost = -1.0;
  for(int r = 1; r <= std::min(16, H); ++r)
  {
    if(H % r) continue;
    const long long items = halves*(H / r);
    const double rows = static_cast<double>((items + sms - 1)/sms*r);
    const double cost = rows*(0.724 + 0.245*(r + 2)/r);
    if(best_cost < 0.0 || cost <= best_cost) { best = r; best_cost = cost; }
  }
  return best;
}

cudaError_t conv3x3_launch(const __nv_bfloat16* in, const __nv_bfloat16* w, int nout, int mode,
                           const ConvArgs& args, cudaStream_t st, int* ncta)
{
  if(args.B < 1 || args.H < 1 || args.W < 128 || (args.W & 127)) return cudaErrorInvalidValue;
  if((nout == 16) != (mode == CONV_FWD_OUT) || (nout != 16 && nout != 64))
    return cudaErrorInvalidValue;
  ConvArgs a = args;
  a.rows = strip_rows(a.B, a.H, a.W);
  CUtensorMap tx, tw, to, to2, tr;
  if(!map_activation(&tx, in, a.B, a.H, a.W, SLAB_PX) || !map_weights(&tw, w, nout))
    return cudaErrorInvalidValue;
  // output, pre-activation output and epilogue input tiles (128 pixels);
  // maps a mode does not use repeat one it does
  const void* out = mode == CONV_FWD_OUT ? static_cast<const void*>(in) : a.out;
  const void* out2 = mode == CONV_FWD_GELU ? static_cast<const void*>(a.out2) : out;
  const void* res = (mode == CONV_FWD_RESID || mode == CONV_BWD_RESID) ? static_cast<const void*>(a.resid)
                  : mode == CONV_BWD_GELU ? static_cast<const void*>(a.aux) : out;
  if(!map_activation(&to, out, a.B, a.H, a.W, 128) || !map_activation(&to2, out2, a.B, a.H, a.W, 128) ||
     !map_activation(&tr, res, a.B, a.H, a.W, 128))
    return cudaErrorInvalidValue;
  switch(mode)
  {
    case CONV_FWD_BIAS: return launch_mode<64, CONV_FWD_BIAS>(tx, tw, to, to2, tr, a, st, ncta);
    case CONV_FWD_GELU: return launch_mode<64, CONV_FWD_GELU>(tx, tw, to, to2, tr, a, st, ncta);
    case CONV_FWD_RESID: return launch_mode<64, CONV_FWD_RESID>(tx, tw, to, to2, tr, a, st, ncta);
    case CONV_FWD_OUT: return launch_mode<16, CONV_FWD_OUT>(tx, tw, to, to2, tr, a, st, ncta);
    case CONV_BWD_GELU: return launch_mode<64, CONV_BWD_GELU>(tx, tw, to, to2, tr, a, st, ncta);
    case CONV_BWD_RESID: return launch_mode<64, CONV_BWD_RESID>(tx, tw, to, to2, tr, a, st, ncta);
    case CONV_BWD_PLAIN: return launch_mode<64, CONV_BWD_PLAIN>(tx, tw, to, to2, tr, a, st, ncta);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t conv3x3_wgrad_launch(const __nv_bfloat16* x, const __nv_bfloat16* dy, float* dW,
                                 int B, int H, int W, int* err, cudaStream_t st)
{
  if(B < 1 || H < 1 || W < 128 || (W & 127)) return cudaErrorInvalidValue;
  CUtensorMap tx, td;
  if(!map_activation(&tx, x, B, H, W, SLAB_PX) || !map_activation(&td, dy, B, H, W, 128))
    return cudaErrorInvalidValue;
  static unsigned long long attr = 0;
  const cudaError_t e = smem_attr(conv3x3_wgrad_kernel, attr, static_cast<int>(WG_ALLOC));
  if(e != cudaSuccess) return e;
  const long long nblocks = static_cast<long long>(B)*H*(W >> 7);
  // one CTA per SM (one fits), each a contiguous range of blocks
  const int nchunks = static_cast<int>(std::max<long long>(1, std::min<long long>(nblocks, sm_count())));
  WgradArgs a{B, H, W, nchunks, dW, err};
  conv3x3_wgrad_kernel<<<nchunks, WG_THREADS, WG_ALLOC, st>>>(tx, td, a);
  return cudaGetLastError();
}

} // namespace mlb
