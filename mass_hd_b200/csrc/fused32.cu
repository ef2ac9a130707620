// FP32 fused periodic step kernel for sm_100a.
//
// One launch performs a whole Model::Step() (src/models/lyotropic.cpp:500-525,
// src/models/nematic.cpp:370-395) with npc = 1:
//   B  UpdateQuantities (predictor)   src/models/lyotropic.cpp:168-247
//   C  UpdateFields(true)             src/models/lyotropic.cpp:249-330
//      Move                           src/models/lyotropic.cpp:371-386
//   D  UpdateQuantities (corrector)
//   E  UpdateFields(false)            src/models/lyotropic.cpp:331-340
//
// Work decomposition. A CTA of NT threads owns a strip of NT lattice columns
// (y, the contiguous index): NT - 8 output columns plus a 4-column halo on
// each side, because each of the four stages reads its y-neighbours. The
// CTA marches down a chunk of rows (x) of that strip, one row per iteration;
// the stages run 0, 1, 3 and 4 rows behind the newest row, so every value a
// stage needs from a neighbouring row was produced by this thread in an
// earlier iteration (kept in registers) and every value it needs from a
// neighbouring column was published to shared memory before the single
// __syncthreads() that ends each iteration. Nothing is recomputed along x
// except 8 warm-up rows per chunk; along y the halo costs 8 of NT columns.
//
// Input rows arrive by 1D bulk copies (cp.async.bulk, TMA) into a ring of
// RING rows in shared memory, completion tracked by one mbarrier per slot;
// the copies for a row are issued RING-3 rows ahead of use. Every wait is
// bounded: on time-out the CTA records bit 0 in *err, drains the copies it
// issued (again bounded) and returns.
//
// Storage: populations as deviations g_v = f_v - t_v*rho from the rest
// state (t = 4/9, 1/9, 1/36), so FP32 keeps the O(1e-3) flow signal that
// rho = 40 would otherwise swamp; Q and phi as they are. Planes of LX*LY
// floats in the reference's site order (k = y + LY*x).
#include "fused32.cuh"

#include <cstdint>

namespace mlb {
namespace {

constexpr int RING = 6;   // input rows resident in shared memory
constexpr int PADY = 4;   // floats of padding on each side of a ring row

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
               :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 1D bulk copy global -> this CTA's shared memory (no multicast)
__device__ __forceinline__ void bulk_load(void* dst, const void* src,
                                          uint32_t bytes, uint64_t* bar)
{
  asm volatile(
    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
    " [%0], [%1], %2, [%3];"
    :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
    : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}"
    : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}

// Wait for phase `parity` of `bar`; false after ~2^31 cycles (about a second).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
  if(mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while(!mbar_try_wait(bar, parity))
    if(clock64() - t0 > (1ll << 31)) return false;
  return true;
}

// ---------------------------------------------------------------------------
// Per-site physics in FP32 (deviation storage). Same equations as the
// reference; the operand order is free here (FMA contraction allowed).

struct UQOut
{
  float dn, ux, uy, uxp, uyp, MU, Hxx, Hyx;
  float dxQxx, dyQxx, dxQyx, dyQyx, sXX, sYY, sXY, sYX;
};

// UpdateQuantitiesAtNode. Neighbour order for Q/phi: center, +x, -x, +y, -y.
template<int MODEL>
__device__ __forceinline__ void uq_site(const P32& P, const float g[9],
                                        const float Qa[5], const float Qb[5],
                                        const float Ph[5], UQOut& o,
                                        float dg[7])
{
  const float dn = ((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7])) + g[8];
  const float nn = P.rho + dn;
  const float inv = __frcp_rn(nn);
  const float jx = (g[1] - g[2]) + (g[5] - g[6]) + (g[8] - g[7]);
  const float jy = (g[3] - g[4]) + (g[5] - g[6]) + (g[7] - g[8]);
  const float vx = jx*inv, vy = jy*inv;

  const float Qxx = Qa[0], Qyx = Qb[0];
  const float lQxx = (Qa[1] + Qa[2]) + (Qa[3] + Qa[4]) - 4.f*Qxx;
  const float lQyx = (Qb[1] + Qb[2]) + (Qb[3] + Qb[4]) - 4.f*Qyx;
  const float dxQxx = 0.5f*(Qa[1] - Qa[2]), dyQxx = 0.5f*(Qa[3] - Qa[4]);
  const float dxQyx = 0.5f*(Qb[1] - Qb[2]), dyQyx = 0.5f*(Qb[3] - Qb[4]);
  const float S2 = Qxx*Qxx + Qyx*Qyx;
  const float term = MODEL == LYO ? -S2 : 1.f - S2;
  const float cterm = P.CC*term;
  const float Hxx = cterm*Qxx + P.LL*lQxx;
  const float Hyx = cterm*Qyx + P.LL*lQyx;
  const float el = P.LL*((dyQxx*dyQxx + dyQyx*dyQyx) - (dxQxx*dxQxx + dxQyx*dxQyx));
  const float elS = -2.f*P.LL*(dxQxx*dyQxx + dxQyx*dyQyx);
  const float xi2 = 2.f*P.xi;
  const float sigmaA = 2.f*(Qxx*Hyx - Qyx*Hxx);
  const float flowF = xi2*((Qxx*Qxx - 1.f)*Hxx + Qxx*Qyx*Hyx);
  const float flowS = xi2*(Qyx*Qxx*Hxx + (Qyx*Qyx - 1.f)*Hyx);

  o.dn = dn; o.ux = vx; o.uy = vy;
  o.Hxx = Hxx; o.Hyx = Hyx;
  o.dxQxx = dxQxx; o.dyQxx = dyQxx; o.dxQyx = dxQyx; o.dyQyx = dyQyx;

  if constexpr (MODEL == LYO)
  {
    const float p = Ph[0];
    const float omp = 1.f - p;
    const float lp = (Ph[1] + Ph[2]) + (Ph[3] + Ph[4]) - 4.f*p;
    const float dxPhi = 0.5f*(Ph[1] - Ph[2]), dyPhi = 0.5f*(Ph[3] - Ph[4]);
    const float mu = P.AA*p*omp*(1.f - 2.f*p) - P.KK*lp;
    const float pq = p*omp;
    const float sigmaB = 0.5f*P.AA*pq*pq + 0.5f*cterm*term - mu*p;
    const float act = P.zeta*omp;
    const float pf = 0.5f*P.KK*(dyPhi*dyPhi - dxPhi*dxPhi);
    const float pfS = -P.KK*dxPhi*dyPhi;
    const float sigmaF = flowF - act*Qxx + pf + el;
    const float sigmaS = flowS - act*Qyx + pfS + elS;
    const float iso = P.zetaI*(P.conc - p);
    o.uxp = vx*p; o.uyp = vy*p; o.MU = mu;
    o.sXX = sigmaF + sigmaB + iso;
    o.sYY = -sigmaF + sigmaB + iso;
    o.sXY = sigmaS + sigmaA;
    o.sYX = sigmaS - sigmaA;
    if(dg)
    {
      dg[0] = sigmaB + iso;
      dg[1] = sigmaF - pf + act*Qxx;
      // the reference uses zeta*Qxx in the yx component as well
      // (src/models/lyotropic.cpp:242)
      dg[2] = sigmaS - pfS + act*Qxx;
      dg[3] = pf;
      dg[4] = pfS;
      dg[5] = -act*Qxx;
      dg[6] = -act*Qyx;
    }
  }
  else
  {
    const float sigmaB = 0.5f*cterm*term;
    const float sigmaF = flowF - P.zeta*Qxx + el;
    const float sigmaS = flowS - P.zeta*Qyx + elS;
    o.uxp = 0.f; o.uyp = 0.f; o.MU = 0.f;
    o.sXX = sigmaF + sigmaB;
    o.sYY = -sigmaF + sigmaB;
    o.sXY = sigmaS + sigmaA;
    o.sYX = sigmaS - sigmaA;
  }
}

// y-neighbour values of the UQ outputs a UF site reads, in this order
enum { Y_UX_P, Y_UX_M, Y_UY_P, Y_UY_M, Y_SXY_P, Y_SXY_M, Y_SYY_P, Y_SYY_M,
       Y_UYP_P, Y_UYP_M, Y_MU_P, Y_MU_M, NYV };

// UpdateFieldsAtNode. c: this site's UQ outputs, xp/xm: the x-neighbours'.
// FIRST: (Qxx, Qyx, p, g) is the state before the step; writes the
//   predictor fn and the updated g, QN/phn and Q'/phi'.
// !FIRST: (Qxx, Qyx, p) is the predicted state, (QN, phn, fn) the
//   predictor values; g is the streamed population, updated in place.
template<int MODEL, bool FIRST>
__device__ __forceinline__ void uf_site(const P32& P, const UQOut& c,
                                        const UQOut& xp, const UQOut& xm,
                                        const float yv[NYV],
                                        float Qxx, float Qyx, float p,
                                        float QNxx, float QNyx, float phn,
                                        float g[9], float fn[9],
                                        float& Qxx_o, float& Qyx_o, float& p_o,
                                        float& QNxx_o, float& QNyx_o, float& phn_o)
{
  const float dxux = 0.5f*(xp.ux - xm.ux), dyux = 0.5f*(yv[Y_UX_P] - yv[Y_UX_M]);
  const float dxuy = 0.5f*(xp.uy - xm.uy), dyuy = 0.5f*(yv[Y_UY_P] - yv[Y_UY_M]);
  const float dxSxx = 0.5f*(xp.sXX - xm.sXX), dySxy = 0.5f*(yv[Y_SXY_P] - yv[Y_SXY_M]);
  const float dxSyx = 0.5f*(xp.sYX - xm.sYX), dySyy = 0.5f*(yv[Y_SYY_P] - yv[Y_SYY_M]);

  const float expansion = dxux + dyuy;
  const float shear = 0.5f*(dxuy + dyux);
  const float vorticity = 0.5f*(dxuy - dyux);
  const float traceQL = Qxx*(dxux - dyuy) + 2.f*Qyx*shear;
  const float vx = c.ux, vy = c.uy;

  const float Dxx = P.GammaQ*c.Hxx - vx*c.dxQxx - vy*c.dyQxx - 2.f*vorticity*Qyx
    + P.xi*((Qxx + 1.f)*(2.f*dxux - traceQL) + 2.f*Qyx*shear - expansion);
  const float Dyx = P.GammaQ*c.Hyx - vx*c.dxQyx - vy*c.dyQyx + 2.f*vorticity*Qxx
    + P.xi*(Qyx*(expansion - traceQL) + 2.f*shear);

  const float Fx = dxSxx + dySxy - P.friction*vx;
  const float Fy = dxSyx + dySyy - P.friction*vy;

  float Dp = 0.f, tau;
  if constexpr (MODEL == LYO)
  {
    const float lMU = (xp.MU + xm.MU) + (yv[Y_MU_P] + yv[Y_MU_M]) - 4.f*c.MU;
    const float pFlux = 0.5f*(xp.uxp - xm.uxp) + 0.5f*(yv[Y_UYP_P] - yv[Y_UYP_M]);
    Dp = P.GammaP*lMU - pFlux;
    tau = P.tauNem*p + P.tauIso*(1.f - p);
  }
  else tau = P.tauNem;
  const float itau = __frcp_rn(tau);

  // equilibrium deviation from t_v*rho (src/lb.hpp:24-41 minus t_v*rho)
  const float dn = c.dn;
  const float nn = P.rho + dn;
  const float jx = nn*vx, jy = nn*vy;
  const float kxx = jx*vx, kyy = jy*vy, kxy = jx*vy, k2 = kxx + kyy;
  const float dn9 = dn*(1.f/9.f), dn36 = dn*(1.f/36.f);
  float fe[9];
  fe[1] = dn9 + (k2 + jx)*(1.f/3.f) - 0.5f*kyy;
  fe[2] = dn9 + (k2 - jx)*(1.f/3.f) - 0.5f*kyy;
  fe[3] = dn9 + (k2 + jy)*(1.f/3.f) - 0.5f*kxx;
  fe[4] = dn9 + (k2 - jy)*(1.f/3.f) - 0.5f*kxx;
  fe[5] = dn36 + (k2 + jx + jy)*(1.f/12.f) + 0.25f*kxy;
  fe[6] = dn36 + (k2 - jx - jy)*(1.f/12.f) + 0.25f*kxy;
  fe[7] = dn36 + (k2 - jx + jy)*(1.f/12.f) - 0.25f*kxy;
  fe[8] = dn36 + (k2 + jx - jy)*(1.f/12.f) - 0.25f*kxy;
  fe[0] = dn - (((fe[1] + fe[2]) + (fe[3] + fe[4])) + ((fe[5] + fe[6]) + (fe[7] + fe[8])));

  float F[9];
  F[0] = 0.f;
  F[1] = Fx*(1.f/3.f); F[2] = -F[1];
  F[3] = Fy*(1.f/3.f); F[4] = -F[3];
  F[5] = (Fx + Fy)*(1.f/12.f); F[6] = -F[5];
  F[7] = (Fy - Fx)*(1.f/12.f); F[8] = -F[7];

  if constexpr (FIRST)
  {
#pragma unroll
    for(int v = 0; v < 9; ++v)
    {
      const float coll = (fe[v] - g[v])*itau + F[v];
      if constexpr (MODEL == LYO)
      {
        fn[v] = g[v] + 0.5f*coll;
        g[v] = g[v] + coll;
      }
      else
      {
        fn[v] = g[v] + 0.5f*coll;
        g[v] = fn[v] + 0.5f*coll;
      }
    }
    QNxx_o = Qxx + 0.5f*Dxx;
    QNyx_o = Qyx + 0.5f*Dyx;
    if constexpr (MODEL == LYO)
    {
      Qxx_o = Qxx + Dxx;
      Qyx_o = Qyx + Dyx;
      phn_o = p + 0.5f*Dp;
      p_o = p + Dp;
    }
    else
    {
      Qxx_o = QNxx_o + 0.5f*Dxx;
      Qyx_o = QNyx_o + 0.5f*Dyx;
      phn_o = 0.f;
      p_o = 0.f;
    }
  }
  else
  {
#pragma unroll
    for(int v = 0; v < 9; ++v)
      g[v] = fn[v] + 0.5f*((fe[v] - g[v])*itau + F[v]);
    Qxx_o = QNxx + 0.5f*Dxx;
    Qyx_o = QNyx + 0.5f*Dyx;
    p_o = MODEL == LYO ? phn + 0.5f*Dp : 0.f;
  }
}

template<int NT, int MODEL>
struct Layout
{
  static constexpr int NP = MODEL == LYO ? 12 : 11;  // state planes
  static constexpr int RW = NT + 2*PADY;            // ring row stride
  static constexpr int XW = NT + 2;                 // exchange row stride
  static constexpr int NX = MODEL == LYO ? 6 : 4;    // y-exchanged UQ fields
  static constexpr int NQ = MODEL == LYO ? 3 : 2;    // y-exchanged Q', phi'
  static constexpr int RING_F = RING*NP*RW;
  static constexpr int XQ_F = 2*NX*XW;
  static constexpr int XC_F = 3*NQ*XW;
  static constexpr int XP_F = 4*18*XW;
  static constexpr int FLOATS = RING_F + 2*XQ_F + XC_F + XP_F;
  static constexpr size_t BYTES = ((FLOATS*sizeof(float) + 15)/16)*16 + RING*sizeof(uint64_t);
};

template<int NT, int MODEL, bool DIAG>
__global__ void __launch_bounds__(NT, NT <= 128 ? 2 : 1)
fused_step_kernel(const FusedArgs a)
{
  using L = Layout<NT, MODEL>;
  constexpr int NP = L::NP, RW = L::RW, XW = L::XW, NX = L::NX, NQ = L::NQ;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* ring = reinterpret_cast<float*>(smem_raw);
  float* xq1 = ring + L::RING_F;
  float* xq2 = xq1 + L::XQ_F;
  float* xc = xq2 + L::XQ_F;
  float* xp = xc + L::XC_F;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(
    smem_raw + ((L::FLOATS*sizeof(float) + 15)/16)*16);
  __shared__ volatile int s_abort;

  const int t = threadIdx.x;
  constexpr int W = NT - 8;
  const int strip = blockIdx.x % a.nstrips;
  const int chunk = blockIdx.x / a.nstrips;
  const int y0 = strip*W;
  const int x0 = a.xbase + chunk*a.rows;
  const int rows = min(a.rows, a.xbase + a.xcount - x0);
  const int LX = a.LX, LY = a.LY;
  const int nload = rows + 9;          // input rows x0-4 .. x0+rows+4
  const int ystart = (y0 - 4 + LY) % LY;
  const P32 P = a.p;

  if(t == 0)
  {
    for(int s = 0; s < RING; ++s) mbar_init(&mbar[s], 1);
    s_abort = 0;
    fence_barrier_init();
  }
  __syncthreads();

  // thread 0: bulk-copy input row rr (lattice row x0 - 4 + rr) into its slot
  auto issue = [&](int rr) {
    const int slot = rr % RING;
    uint64_t* bar = &mbar[slot];
    mbar_expect_tx(bar, NP*NT*4);
    const int gx = ((x0 - 4 + rr) % LX + LX) % LX;
    for(int p = 0; p < NP; ++p)
    {
      const float* src = a.in + p*a.plane + static_cast<long long>(gx)*LY;
      float* dst = ring + (slot*NP + p)*RW + PADY;
      int start = ystart, rem = NT;
      while(rem > 0)
      {
        const int len = min(rem, LY - start);
        bulk_load(dst, src + start, static_cast<uint32_t>(len*4), bar);
        dst += len;
        rem -= len;
        start = 0;
      }
    }
  };

  int issued = 0;
  if(t == 0)
  {
    const int n0 = min(RING, nload);
    for(int rr = 0; rr < n0; ++rr) issue(rr);
    issued = n0;
  }
  if(!mbar_wait_bounded(&mbar[0], 0) || !mbar_wait_bounded(&mbar[1], 0)) s_abort = 1;

  UQOut q1c{}, q1m{};          // UQ1 rows b-1 and b-2
  UQOut q2c{}, q2m{};          // UQ2 rows b-4 and b-5
  float qa1[3] = {0.f, 0.f, 0.f}, qa2[3] = {0.f, 0.f, 0.f}, qa3[3] = {0.f, 0.f, 0.f};
  float qn1[3] = {0.f, 0.f, 0.f}, qn2[3] = {0.f, 0.f, 0.f}, qn3[3] = {0.f, 0.f, 0.f};
  float ffs[9], fns[9];
#pragma unroll
  for(int v = 0; v < 9; ++v) { ffs[v] = 0.f; fns[v] = 0.f; }
  int s3 = 0, s4 = 0;
  const int yg = y0 + t - 4;                       // global column (pre-wrap)
  const bool col_out = t >= 4 && t < NT - 4 && yg < LY;

  const int nit = rows + 7;
  int i = 0;
  for(; i < nit; ++i)
  {
    if(i + 2 < nload && !s_abort)
    {
      const int rr = i + 2;
      if(!mbar_wait_bounded(&mbar[rr % RING], (rr / RING) & 1)) s_abort = 1;
    }
    const float* Rm = ring + ((i    ) % RING)*NP*RW + PADY + t;   // row b-1
    const float* R0 = ring + ((i + 1) % RING)*NP*RW + PADY + t;   // row b
    const float* Rp = ring + ((i + 2) % RING)*NP*RW + PADY + t;   // row b+1

    // ---- B: predictor UpdateQuantities at row b ----
    UQOut nq1;
    {
      float g[9];
#pragma unroll
      for(int v = 0; v < 9; ++v) g[v] = R0[v*RW];
      float Qa[5], Qb[5], Ph[5];
      Qa[0] = R0[9*RW];  Qa[1] = Rp[9*RW];  Qa[2] = Rm[9*RW];  Qa[3] = R0[9*RW + 1];  Qa[4] = R0[9*RW - 1];
      Qb[0] = R0[10*RW]; Qb[1] = Rp[10*RW]; Qb[2] = Rm[10*RW]; Qb[3] = R0[10*RW + 1]; Qb[4] = R0[10*RW - 1];
      if constexpr (MODEL == LYO)
      {
        Ph[0] = R0[11*RW]; Ph[1] = Rp[11*RW]; Ph[2] = Rm[11*RW]; Ph[3] = R0[11*RW + 1]; Ph[4] = R0[11*RW - 1];
      }
      else
      {
#pragma unroll
        for(int k = 0; k < 5; ++k) Ph[k] = 0.f;
      }
      uq_site<MODEL>(P, g, Qa, Qb, Ph, nq1, nullptr);
      float* X = xq1 + (i & 1)*NX*XW + 1 + t;
      X[0*XW] = nq1.ux; X[1*XW] = nq1.uy; X[2*XW] = nq1.sXY; X[3*XW] = nq1.sYY;
      if constexpr (MODEL == LYO) { X[4*XW] = nq1.uyp; X[5*XW] = nq1.MU; }
    }

    // ---- C: predictor UpdateFields at row b-1, then publish for Move ----
    float nQ[3], nQN[3];
    {
      float yv[NYV];
      const float* Y = xq1 + ((i + 1) & 1)*NX*XW + 1 + t;
      yv[Y_UX_P] = Y[0*XW + 1]; yv[Y_UX_M] = Y[0*XW - 1];
      yv[Y_UY_P] = Y[1*XW + 1]; yv[Y_UY_M] = Y[1*XW - 1];
      yv[Y_SXY_P] = Y[2*XW + 1]; yv[Y_SXY_M] = Y[2*XW - 1];
      yv[Y_SYY_P] = Y[3*XW + 1]; yv[Y_SYY_M] = Y[3*XW - 1];
      if constexpr (MODEL == LYO)
      {
        yv[Y_UYP_P] = Y[4*XW + 1]; yv[Y_UYP_M] = Y[4*XW - 1];
        yv[Y_MU_P] = Y[5*XW + 1]; yv[Y_MU_M] = Y[5*XW - 1];
      }
      else yv[Y_UYP_P] = yv[Y_UYP_M] = yv[Y_MU_P] = yv[Y_MU_M] = 0.f;
      float g[9], fn[9];
#pragma unroll
      for(int v = 0; v < 9; ++v) g[v] = Rm[v*RW];
      const float Qxx = Rm[9*RW], Qyx = Rm[10*RW];
      const float p = MODEL == LYO ? Rm[11*RW] : 0.f;
      uf_site<MODEL, true>(P, q1c, nq1, q1m, yv, Qxx, Qyx, p, 0.f, 0.f, 0.f,
                           g, fn, nQ[0], nQ[1], nQ[2], nQN[0], nQN[1], nQN[2]);
      float* XC = xc + s3*NQ*XW + 1 + t;
      XC[0] = nQ[0]; XC[XW] = nQ[1];
      if constexpr (MODEL == LYO) XC[2*XW] = nQ[2];
      float* XP = xp + s4*18*XW + 1 + t;
#pragma unroll
      for(int v = 0; v < 9; ++v) { XP[v*XW] = g[v]; XP[(9 + v)*XW] = fn[v]; }
    }

    // ---- D: corrector UpdateQuantities at row s = b-3 ----
    UQOut nq2;
    float ffn[9], fnn[9];
    {
      // streamed populations: value of direction v at (s, t) left
      // (s - cx, t - cy) in iteration i - 2 - cx
#pragma unroll
      for(int v = 0; v < 9; ++v)
      {
        const int slot = (s4 + 6 - CXv(v)) & 3;   // (i - 2 - cx) mod 4
        const float* src = xp + slot*18*XW + 1 + t - CYv(v);
        ffn[v] = src[v*XW];
        fnn[v] = src[(9 + v)*XW];
      }
      const float* YC = xc + ((s3 + 1) % 3)*NQ*XW + 1 + t;   // (i - 2) mod 3
      float Qa[5], Qb[5], Ph[5];
      Qa[0] = qa2[0]; Qa[1] = qa1[0]; Qa[2] = qa3[0]; Qa[3] = YC[1];      Qa[4] = YC[-1];
      Qb[0] = qa2[1]; Qb[1] = qa1[1]; Qb[2] = qa3[1]; Qb[3] = YC[XW + 1]; Qb[4] = YC[XW - 1];
      if constexpr (MODEL == LYO)
      {
        Ph[0] = qa2[2]; Ph[1] = qa1[2]; Ph[2] = qa3[2]; Ph[3] = YC[2*XW + 1]; Ph[4] = YC[2*XW - 1];
      }
      else
      {
#pragma unroll
        for(int k = 0; k < 5; ++k) Ph[k] = 0.f;
      }
      float dg[7];
      uq_site<MODEL>(P, ffn, Qa, Qb, Ph, nq2, DIAG ? dg : nullptr);
      float* X = xq2 + (i & 1)*NX*XW + 1 + t;
      X[0*XW] = nq2.ux; X[1*XW] = nq2.uy; X[2*XW] = nq2.sXY; X[3*XW] = nq2.sYY;
      if constexpr (MODEL == LYO) { X[4*XW] = nq2.uyp; X[5*XW] = nq2.MU; }
      if constexpr (DIAG)
      {
        const int xs = x0 - 6 + i;
        if(col_out && xs >= x0 && xs < x0 + rows)
        {
          float* o = a.diag + static_cast<long long>(xs)*LY + yg;
          const long long pl = a.plane;
          o[0*pl] = P.rho + nq2.dn; o[1*pl] = nq2.ux; o[2*pl] = nq2.uy;
          o[3*pl] = nq2.uxp; o[4*pl] = nq2.uyp; o[5*pl] = nq2.Hxx; o[6*pl] = nq2.Hyx;
          o[7*pl] = nq2.MU; o[8*pl] = nq2.dxQxx; o[9*pl] = nq2.dyQxx;
          o[10*pl] = nq2.dxQyx; o[11*pl] = nq2.dyQyx; o[12*pl] = nq2.sXX;
          o[13*pl] = nq2.sYY; o[14*pl] = nq2.sYX; o[15*pl] = nq2.sXY;
          if constexpr (MODEL == LYO)
          {
#pragma unroll
            for(int k = 0; k < 7; ++k) o[(16 + k)*pl] = dg[k];
          }
        }
      }
    }

    // ---- E: corrector UpdateFields at row b-4, store ----
    {
      float yv[NYV];
      const float* Y = xq2 + ((i + 1) & 1)*NX*XW + 1 + t;
      yv[Y_UX_P] = Y[0*XW + 1]; yv[Y_UX_M] = Y[0*XW - 1];
      yv[Y_UY_P] = Y[1*XW + 1]; yv[Y_UY_M] = Y[1*XW - 1];
      yv[Y_SXY_P] = Y[2*XW + 1]; yv[Y_SXY_M] = Y[2*XW - 1];
      yv[Y_SYY_P] = Y[3*XW + 1]; yv[Y_SYY_M] = Y[3*XW - 1];
      if constexpr (MODEL == LYO)
      {
        yv[Y_UYP_P] = Y[4*XW + 1]; yv[Y_UYP_M] = Y[4*XW - 1];
        yv[Y_MU_P] = Y[5*XW + 1]; yv[Y_MU_M] = Y[5*XW - 1];
      }
      else yv[Y_UYP_P] = yv[Y_UYP_M] = yv[Y_MU_P] = yv[Y_MU_M] = 0.f;
      float Qo[3], dummy[3];
      uf_site<MODEL, false>(P, q2c, nq2, q2m, yv, qa3[0], qa3[1], qa3[2],
                            qn3[0], qn3[1], qn3[2], ffs, fns,
                            Qo[0], Qo[1], Qo[2], dummy[0], dummy[1], dummy[2]);
      const int xo = x0 - 7 + i;
      // the diagnostic replay re-runs a step only for the D-stage outputs;
      // it leaves the state untouched (its rounding may differ)
      if(!DIAG && col_out && i >= 7)
      {
        float* o = a.out + static_cast<long long>(xo)*LY + yg;
        const long long pl = a.plane;
#pragma unroll
        for(int v = 0; v < 9; ++v) o[v*pl] = ffs[v];
        o[9*pl] = Qo[0];
        o[10*pl] = Qo[1];
        if constexpr (MODEL == LYO) o[11*pl] = Qo[2];
      }
    }

    // ---- shift the per-thread row windows ----
    q1m = q1c; q1c = nq1;
    q2m = q2c; q2c = nq2;
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
      qa3[k] = qa2[k]; qa2[k] = qa1[k]; qa1[k] = nQ[k];
      qn3[k] = qn2[k]; qn2[k] = qn1[k]; qn1[k] = nQN[k];
    }
#pragma unroll
    for(int v = 0; v < 9; ++v) { ffs[v] = ffn[v]; fns[v] = fnn[v]; }
    s3 = s3 == 2 ? 0 : s3 + 1;
    s4 = (s4 + 1) & 3;

    __syncthreads();
    if(s_abort) break;
    if(t == 0 && issued < nload && issued <= i + RING)
    {
      fence_proxy_async();
      issue(issued);
      ++issued;
    }
  }

  if(s_abort && t == 0)
  {
    atomicOr(a.err, 1);
    // let every copy this CTA issued land before the CTA's shared memory
    // is released
    for(int rr = 0; rr < issued; ++rr)
      mbar_wait_bounded(&mbar[rr % RING], (rr / RING) & 1);
  }
}

template<int NT, int MODEL, bool DIAG>
cudaError_t launch_t(const FusedArgs& a, int rows, cudaStream_t st)
{
  using L = Layout<NT, MODEL>;
  auto kern = fused_step_kernel<NT, MODEL, DIAG>;
  // the shared-memory opt-in is per device; remember which devices have it
  static unsigned long long attr_set = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if(!(attr_set & bit))
  {
    const cudaError_t e = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(L::BYTES));
    if(e != cudaSuccess) return e;
    attr_set |= bit;
  }
  const int nchunks = (a.xcount + rows - 1)/rows;
  FusedArgs b = a;
  b.rows = rows;
  b.nstrips = (a.LY + (NT - 8) - 1)/(NT - 8);
  const dim3 grid(b.nstrips*nchunks);
  kern<<<grid, NT, L::BYTES, st>>>(b);
  return cudaGetLastError();
}

template<int NT>
cudaError_t launch_nt(const FusedArgs& a, int model, int rows, bool diag, cudaStream_t st)
{
  if(model == LYO)
    return diag ? launch_t<NT, LYO, true>(a, rows, st) : launch_t<NT, LYO, false>(a, rows, st);
  return diag ? launch_t<NT, NEM, true>(a, rows, st) : launch_t<NT, NEM, false>(a, rows, st);
}

} // namespace

cudaError_t launch_fused_step(const FusedArgs& a, int model, FusedConfig cfg,
                              bool diag, cudaStream_t st)
{
  if((a.src || a.pred) && cfg.nt != 32) return cudaErrorInvalidValue;
  switch(cfg.nt)
  {
    case 32:  return launch_fused_warp_step(a, model, cfg.rows, diag, st);
    case 64:  return launch_nt<64>(a, model, cfg.rows, diag, st);
    case 128: return launch_nt<128>(a, model, cfg.rows, diag, st);
    case 256: return launch_nt<256>(a, model, cfg.rows, diag, st);
    default:  return cudaErrorInvalidValue;
  }
}

size_t fused_smem_bytes(int nt, int model)
{
  if(model == LYO)
    return nt == 64 ? Layout<64, LYO>::BYTES : nt == 128 ? Layout<128, LYO>::BYTES : Layout<256, LYO>::BYTES;
  return nt == 64 ? Layout<64, NEM>::BYTES : nt == 128 ? Layout<128, NEM>::BYTES : Layout<256, NEM>::BYTES;
}

bool fused_supported(int LX, int LY, int nt)
{
  return LX >= 1 && LY % 4 == 0 && LY >= nt && LY >= 64 &&
         (nt == 32 || nt == 64 || nt == 128 || nt == 256);
}

} // namespace mlb
