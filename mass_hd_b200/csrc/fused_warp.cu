// FP32 fused periodic step, warp-strip variant (two lattice columns per
// lane, packed FP32x2 arithmetic).
//
// Same algorithm as fused32.cu - one launch is one Model::Step() with npc = 1
// (src/models/lyotropic.cpp:500-525, src/models/nematic.cpp:370-395) - with a
// different decomposition:
//  * every warp owns an independent strip of 64 columns (56 output columns
//    and a 4-column halo on each side) and marches along x on its own; there
//    is no CTA-wide barrier,
//  * lane l holds columns 2l and 2l+1 as one float2 and computes both with
//    the sm_100 packed FFMA2/FADD2/FMUL2 instructions,
//  * y-neighbours of computed values come from the adjacent lane by
//    __shfl_up/down; x-neighbours are rows this lane produced earlier,
//  * stages run 0 (B: predictor UpdateQuantities), 1 (C: predictor
//    UpdateFields + y-part of Move), 2 (D: corrector UpdateQuantities, x-part
//    of Move) and 3 (E: corrector UpdateFields) rows behind the newest row,
//  * D folds the corrector's fn - ff/(2 tau) per population one row early,
//    so E carries 9 instead of 18 values per site,
//  * input rows arrive in a per-warp ring by 1D bulk copies (TMA) with one
//    mbarrier per slot; every wait is bounded (bit 0 of *err on time-out).
#include "fused32.cuh"

#include <algorithm>
#include <cstdint>

namespace mlb {
namespace {

constexpr int RING = 4;     // input rows per warp in shared memory (power of 2)
constexpr int PADY = 4;     // ring row padding (floats, each side)
constexpr int COLS = 64;    // columns per warp strip
constexpr int WOUT = COLS - 8;
// ring row stride (floats): a 16-byte-aligned left pad, then the strip. The
// lane holding columns 62-63 reads one value past its row (its +y
// neighbour, a halo column whose result is never stored); that read stays
// inside this warp's shared memory.
constexpr int RWW = COLS + PADY;
constexpr int WPB = 4;      // warps per CTA
constexpr int PW = COLS + 4;         // stride of a delayed-population row
constexpr int NDP = 12;              // delayed populations (see below)

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
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
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
  asm volatile(
    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
    :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
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
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
  if(mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while(!mbar_try_wait(bar, parity))
    if(clock64() - t0 > (1ll << 31)) return false;
  return true;
}

// ---------------------------------------------------------------------------
// packed pair arithmetic (columns 2l and 2l+1)

struct f2 { float2 v; };
__device__ __forceinline__ f2 mk(float a, float b) { return f2{make_float2(a, b)}; }
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return f2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2 operator*(f2 a, f2 b) { return f2{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) { return f2{__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return f2{__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
// a literal pair: the compiler keeps these out of the registers the
// parameter pairs would take
#define KC(c) (f2{make_float2((c), (c))})
__device__ __forceinline__ f2 W2(const float2& c) { return f2{c}; }

__device__ __forceinline__ float rcp_approx(float x)
{
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
// 1/x from the hardware estimate (relative error within about 1 ulp of
// FP32 for the normal range used here: densities near rho, tau in [0.5, 10])
__device__ __forceinline__ f2 rcp2(f2 x, const PairParams& P)
{
  (void)P;
  return mk(rcp_approx(x.v.x), rcp_approx(x.v.y));
}

__device__ __forceinline__ f2 lds2(const float* p) { return f2{*reinterpret_cast<const float2*>(p)}; }

// neighbour along +y / -y of a pair held by every lane
__device__ __forceinline__ f2 yplus(f2 a)
{
  return mk(a.v.y, __shfl_down_sync(0xffffffffu, a.v.x, 1));
}
__device__ __forceinline__ f2 yminus(f2 a)
{
  return mk(__shfl_up_sync(0xffffffffu, a.v.y, 1), a.v.x);
}

using PP = PairParams;

__host__ PairParams make_pp(const P32& p, int model)
{
  auto b = [](float x) { return make_float2(x, x); };
  const bool lyo = model != NEM;      // lyotropic and go-or-grow: tau(phi)
  const bool gog = model == GOG;
  PairParams q;
  q.rho = b(p.rho); q.GammaQ = b(p.GammaQ); q.GammaP = b(p.GammaP);
  q.xi2 = b(2.f*p.xi); q.hxi = b(.5f*p.xi);
  // tau(phi) = tauIso + (tauNem - tauIso) phi (lyotropic), tau (nematic)
  q.tauIso = b(lyo ? p.tauIso : p.tauNem);
  q.dtau = b(lyo ? p.tauNem - p.tauIso : 0.f);
  q.itau = b(1.f/(lyo ? p.tauIso : p.tauNem));
  q.n2fric = b(-2.f*p.friction);
  q.AA = b(p.AA); q.hAA = b(.5f*p.AA);
  // the bulk factor of H minus 4 LL, as -nCC*S2 + c4k: CC*(-S2) (lyotropic),
  // CC*(1 - S2) (nematic), 2 CC*(Snem - S2) (go-or-grow)
  q.nCC = b(gog ? -2.f*p.CC : -p.CC); q.hCC = b(.5f*p.CC);
  q.c4k = b(gog ? 2.f*p.CC*p.Snem - 4.f*p.LL : lyo ? -4.f*p.LL : p.CC - 4.f*p.LL);
  q.LL = b(p.LL);
  q.q4LL = b(.25f*p.LL); q.nh2LL = b(-.5f*p.LL);
  q.nKK = b(-p.KK); q.KK8 = b(.125f*p.KK); q.nKK4 = b(-.25f*p.KK);
  q.zeta = b(p.zeta); q.nzeta = b(-p.zeta); q.zetaI = b(p.zetaI); q.conc = b(p.conc);
  q.Snem = b(p.Snem); q.phic = b(p.phi_critical); q.Bc = b(p.B); q.hB = b(.5f*p.B);
  q.hGP = b(.5f*p.GammaP); q.hDchi = b(.5f*p.Dchi); q.A2chi = b(2.f*p.Achi);
  q.Ochi = b(p.Ochi); q.phisw = b(p.phiswitch); q.gt = b(p.growTogether ? 1.f : 0.f);
  return q;
}

// ---------------------------------------------------------------------------
// The arithmetic of one step, restated for FP32 with fewer operations than
// the reference's expression order (the FP64 mode keeps that order; FP32 is
// held to tolerances against it):
//  * central differences are kept as raw differences (twice the
//    derivative) and their factors 1/2, 1/4 folded into the constants they
//    meet (P.q4LL, P.nh2LL, P.KK8, P.nKK4, hxi, ...);
//  * H = CC*term*Q + LL*lap(Q) is formed as (CC*term - 4 LL)*Q + LL*s, with
//    s the sum of the four neighbours, and the antisymmetric stress
//    Qxx*Hyx - Qyx*Hxx as LL*(Qxx*s_yx - Qyx*s_xx) (the bulk terms cancel);
//  * the centre-only part of the Beris-Edwards rate, Gamma*H - u.grad(Q),
//    is formed in UpdateQuantities, so UpdateFields carries 2 values
//    instead of 6 per site;
//  * the forcing term w_v*(F.c_v) is folded into the equilibrium: with
//    j' = j + tau*F, fe'_v(j') = fe_v(j) + tau*w_v*(F.c_v), so
//    (fe_v - f_v)/tau + F_v = (fe'_v - f_v)/tau, and the rest population
//    is the closed form fe_0 = 4/9 dn - 2/3 k2 (dn and k2 = n|u|^2 as
//    below), which is what nn - sum(fe_1..8) evaluates to;
//  * y-neighbour differences and sums come from two shuffles and two scalar
//    adds per pair, with no register repacking.

// Values of one site after UpdateQuantities that a later UpdateFields reads
// (centre, and through the neighbour sets). BEx/BEy: Gamma*H - u.grad(Q).
// Go-or-grow also carries chi = m/phi, phi and u*m (its phenotype update
// reads them at the neighbours); the other models leave them zero.
struct UQc
{
  f2 dn, ux, uy, BEx, BEy, MU, uxp, uyp, sXX, sYY, sXY, sYX;
  f2 chi, p, uxm, uym;
};
// x-neighbour set: what UpdateFields reads from the rows x +- 1
struct UQx
{
  f2 ux, uy, sXX, sYX, uxp, MU, chi, p, uxm;
};
__device__ __forceinline__ UQx xset(const UQc& a)
{
  return UQx{a.ux, a.uy, a.sXX, a.sYX, a.uxp, a.MU, a.chi, a.p, a.uxm};
}
// Derived fields of the diagnostic replay (DIAG launches only)
struct UQd
{
  f2 Hxx, Hyx, XA, YA, XB, YB, bi, sigmaF, sigmaS, pf, pfS, nact;
};

// (v(y+1) + v(y-1), v(y+1) - v(y-1)) for both columns of every lane's pair:
// lane l holds columns 2l, 2l+1; columns 2l-1 and 2l+2 come from the
// neighbouring lanes.
__device__ __forceinline__ void yboth(f2 a, f2& sum, f2& diff)
{
  const float lo = __shfl_up_sync(0xffffffffu, a.v.y, 1);
  const float hi = __shfl_down_sync(0xffffffffu, a.v.x, 1);
  sum = mk(a.v.y + lo, hi + a.v.x);
  diff = mk(a.v.y - lo, hi - a.v.x);
}
__device__ __forceinline__ f2 ydiff(f2 a)
{
  const float lo = __shfl_up_sync(0xffffffffu, a.v.y, 1);
  const float hi = __shfl_down_sync(0xffffffffu, a.v.x, 1);
  return mk(a.v.y - lo, hi - a.v.x);
}
__device__ __forceinline__ f2 ysum(f2 a)
{
  const float lo = __shfl_up_sync(0xffffffffu, a.v.y, 1);
  const float hi = __shfl_down_sync(0xffffffffu, a.v.x, 1);
  return mk(a.v.y + lo, hi + a.v.x);
}

// Neighbour stencil of one scalar field at a site: s = sum of the four
// neighbours, X = (+x) - (-x), Y = (+y) - (-y).
struct Stn
{
  f2 c, s, X, Y;
};

// UpdateQuantities of one row pair (src/models/lyotropic.cpp:168-247,
// src/models/nematic.cpp:76-131).
template<int MODEL, bool DIAG>
__device__ __forceinline__ void uq2(const PP& P, const f2 g[9], const Stn& A, const Stn& B,
                                    const Stn& Ph, const f2 m, UQc& o, UQd& d)
{
  const f2 dn = ((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7])) + g[8];
  const f2 inv = rcp2(W2(P.rho) + dn, P);
  const f2 d56 = g[5] - g[6], d87 = g[8] - g[7];
  const f2 jx = (g[1] - g[2]) + (d56 + d87);
  const f2 jy = (g[3] - g[4]) + (d56 - d87);
  const f2 vx = jx*inv, vy = jy*inv;

  const f2 Qxx = A.c, Qyx = B.c;
  const f2 S2 = fma(Qxx, Qxx, Qyx*Qyx);
  // CC*term - 4*LL, term = -S2 (lyotropic) or 1 - S2 (nematic)
  const f2 c4 = fma(W2(P.nCC), S2, W2(P.c4k));
  const f2 LsA = W2(P.LL)*A.s, LsB = W2(P.LL)*B.s;
  const f2 Hxx = fma(c4, Qxx, LsA);
  const f2 Hyx = fma(c4, Qyx, LsB);
  // Qxx*Hyx - Qyx*Hxx
  const f2 aQ = Qxx*LsB - Qyx*LsA;
  // 4/LL times the elastic normal stress, -2/LL times the shear one
  const f2 elr = fma(A.Y, A.Y, B.Y*B.Y) - fma(A.X, A.X, B.X*B.X);
  const f2 elSr = fma(A.X, A.Y, B.X*B.Y);
  const f2 QQ = Qxx*Qyx;
  const f2 fF = fma(fma(Qxx, Qxx, KC(-1.f)), Hxx, QQ*Hyx);
  const f2 fS = fma(QQ, Hxx, fma(Qyx, Qyx, KC(-1.f))*Hyx);
  f2 sigmaF, sigmaS, bi, pf = KC(0.f), pfS = KC(0.f), nact;

  if constexpr (MODEL == LYO)
  {
    const f2 p = Ph.c;
    nact = fma(W2(P.zeta), p, W2(P.nzeta));              // -zeta*(1 - p)
    pf = W2(P.KK8)*((Ph.Y - Ph.X)*(Ph.Y + Ph.X));       // .5 KK (dyPhi^2 - dxPhi^2)
    pfS = W2(P.nKK4)*(Ph.X*Ph.Y);                        // -KK dxPhi dyPhi
    sigmaF = fma(W2(P.xi2), fF, fma(nact, Qxx, fma(W2(P.q4LL), elr, pf)));
    sigmaS = fma(W2(P.xi2), fS, fma(nact, Qyx, fma(W2(P.nh2LL), elSr, pfS)));
    const f2 pq = p*(KC(1.f) - p);
    const f2 lp = fma(KC(-4.f), p, Ph.s);
    const f2 mu = fma(W2(P.AA)*pq, fma(KC(-2.f), p, KC(1.f)), W2(P.nKK)*lp);
    // .5 AA (p(1-p))^2 + .5 CC term^2 - mu p, term^2 = S2^2
    const f2 y = fma(W2(P.hCC)*S2, S2, (W2(P.hAA)*pq)*pq);
    bi = fma(W2(P.zetaI), W2(P.conc) - p, y - mu*p);
    o.MU = mu;
    o.uxp = vx*p;
    o.uyp = vy*p;
    o.chi = o.p = o.uxm = o.uym = KC(0.f);
  }
  else if constexpr (MODEL == GOG)
  {
    // GoOrGrow::UpdateQuantitiesAtNode (src/models/go-or-grow.cpp:230-308):
    // H and the bulk stress with term = Snem - q^2 (H's factor 2 CC is in
    // nCC and c4k), the crowding penalty B above phi_critical, and the
    // active stress weighted by the go fraction 1 - chi, chi = m/phi
    const f2 p = Ph.c;
    const f2 mp = m*rcp2(p, P);
    const f2 chi = mk(p.v.x > 1e-12f ? mp.v.x : 0.f, p.v.y > 1e-12f ? mp.v.y : 0.f);
    nact = (W2(P.nzeta)*p)*(KC(1.f) - chi);             // -zeta*phi*(1 - chi)
    pf = W2(P.KK8)*((Ph.Y - Ph.X)*(Ph.Y + Ph.X));
    pfS = W2(P.nKK4)*(Ph.X*Ph.Y);
    sigmaF = fma(W2(P.xi2), fF, fma(nact, Qxx, fma(W2(P.q4LL), elr, pf)));
    sigmaS = fma(W2(P.xi2), fS, fma(nact, Qyx, fma(W2(P.nh2LL), elSr, pfS)));
    const f2 pq = p*(KC(1.f) - p);
    const f2 lp = fma(KC(-4.f), p, Ph.s);
    const f2 dpc = p - W2(P.phic);
    const f2 pos = mk(fmaxf(dpc.v.x, 0.f), fmaxf(dpc.v.y, 0.f));
    const f2 mu = fma(W2(P.AA)*pq, fma(KC(-2.f), p, KC(1.f)),
                      fma(W2(P.Bc), pos, W2(P.nKK)*lp));
    // .5 AA (p(1-p))^2 + .5 B pos^2 + .5 CC term^2 - mu p
    const f2 term = W2(P.Snem) - S2;
    const f2 y = fma(W2(P.hCC)*term, term, fma(W2(P.hAA)*pq, pq, (W2(P.hB)*pos)*pos));
    bi = fma(W2(P.zetaI), W2(P.conc) - p, y - mu*p);
    o.MU = mu;
    o.uxp = vx*p;
    o.uyp = vy*p;
    o.chi = chi;
    o.p = p;
    o.uxm = vx*m;
    o.uym = vy*m;
  }
  else
  {
    nact = W2(P.nzeta);
    sigmaF = fma(W2(P.xi2), fF, fma(nact, Qxx, W2(P.q4LL)*elr));
    sigmaS = fma(W2(P.xi2), fS, fma(nact, Qyx, W2(P.nh2LL)*elSr));
    const f2 term = KC(1.f) - S2;
    bi = W2(P.hCC)*(term*term);
    o.MU = o.uxp = o.uyp = KC(0.f);
    o.chi = o.p = o.uxm = o.uym = KC(0.f);
  }
  o.dn = dn;
  o.ux = vx;
  o.uy = vy;
  o.sXX = bi + sigmaF;
  o.sYY = bi - sigmaF;
  o.sXY = fma(KC(2.f), aQ, sigmaS);
  o.sYX = fma(KC(-2.f), aQ, sigmaS);
  o.BEx = fma(W2(P.GammaQ), Hxx, KC(-.5f)*fma(vx, A.X, vy*A.Y));
  o.BEy = fma(W2(P.GammaQ), Hyx, KC(-.5f)*fma(vx, B.X, vy*B.Y));
  if constexpr (DIAG)
  {
    d.Hxx = Hxx; d.Hyx = Hyx;
    d.XA = A.X; d.YA = A.Y; d.XB = B.X; d.YB = B.Y;
    d.bi = bi; d.sigmaF = sigmaF; d.sigmaS = sigmaS;
    d.pf = pf; d.pfS = pfS; d.nact = nact;
  }
}

// y-neighbour differences (and the MU sum) of a row's UpdateQuantities
// (go-or-grow: the y+-1 values of chi, phi and MU themselves, and the
// y-difference of uy*m)
struct YD
{
  f2 ux, uy, sXY, sYY, uyp, MUs;
  f2 chip, chim, pp, pm, MUp, MUm, uym;
};
template<int MODEL>
__device__ __forceinline__ YD ydiffs(const UQc& c)
{
  YD y;
  y.ux = ydiff(c.ux);
  y.uy = ydiff(c.uy);
  y.sXY = ydiff(c.sXY);
  y.sYY = ydiff(c.sYY);
  if constexpr (MODEL == LYO)
  {
    y.uyp = ydiff(c.uyp);
    y.MUs = ysum(c.MU);
  }
  else if constexpr (MODEL == GOG)
  {
    y.uyp = ydiff(c.uyp);
    y.MUp = yplus(c.MU); y.MUm = yminus(c.MU);
    y.MUs = y.MUp + y.MUm;
    y.chip = yplus(c.chi); y.chim = yminus(c.chi);
    y.pp = yplus(c.p); y.pm = yminus(c.p);
    y.uym = ydiff(c.uym);
  }
  else y.uyp = y.MUs = KC(0.f);
  return y;
}

// Go-or-grow's rate of change of m (src/models/go-or-grow.cpp:331-362)
// and its growth term R = chi*phi*rate, at a site whose UpdateQuantities
// values are c, with the x-neighbour sets xp, xm and the y-neighbours in y.
// Dm = GammaP*sum_n .5(chi_n + chi)(MU_n - MU) + Dchi*sum_n .5(phi_n + phi)(chi_n - chi)
//      - div(u m) - phi*V'(chi) + (growTogether ? chi R : R)
__device__ __forceinline__ void pheno_rate(const PP& P, const UQc& c, const UQx& xp,
                                           const UQx& xm, const YD& y, const f2 rate,
                                           f2& Dm, f2& R)
{
  const f2 chi = c.chi, MU = c.MU, p = c.p;
  f2 dmf = (xp.chi + chi)*(xp.MU - MU);
  f2 pd = (xp.p + p)*(xp.chi - chi);
  dmf = fma(xm.chi + chi, xm.MU - MU, dmf);
  pd = fma(xm.p + p, xm.chi - chi, pd);
  dmf = fma(y.chip + chi, y.MUp - MU, dmf);
  pd = fma(y.pp + p, y.chip - chi, pd);
  dmf = fma(y.chim + chi, y.MUm - MU, dmf);
  pd = fma(y.pm + p, y.chim - chi, pd);
  // twice the divergence of u m
  const f2 mF2 = (xp.uxm - xm.uxm) + y.uym;
  // V'(chi) = 2 Achi chi (1 - chi)(1 - 2 chi) + Ochi (phi - phiswitch)
  const f2 dV = fma(W2(P.A2chi)*chi, (KC(1.f) - chi)*fma(KC(-2.f), chi, KC(1.f)),
                    W2(P.Ochi)*(p - W2(P.phisw)));
  R = (chi*p)*rate;
  // growTogether: chi R, else R
  const f2 mG = fma(W2(P.gt), chi - KC(1.f), KC(1.f))*R;
  Dm = fma(W2(P.hGP), dmf, W2(P.hDchi)*pd);
  Dm = fma(KC(-.5f), mF2, Dm) - p*dV;
  Dm = Dm + mG;
}

// m after a sub-step clamped to [0, max(phi after the sub-step, 0)]
// (src/models/go-or-grow.cpp:378-383)
__device__ __forceinline__ f2 clamp_m(f2 mt, f2 pt)
{
  return mk(fminf(fmaxf(mt.v.x, 0.f), fmaxf(pt.v.x, 0.f)),
            fminf(fmaxf(mt.v.y, 0.f), fmaxf(pt.v.y, 0.f)));
}

template<int MODEL>
__device__ __forceinline__ f2 itau_of(const PP& P, f2 p)
{
  return MODEL != NEM ? rcp2(fma(W2(P.dtau), p, W2(P.tauIso)), P) : W2(P.itau);
}

// UpdateFields of one row pair up to the node update
// (src/models/lyotropic.cpp:249-306, src/models/nematic.cpp:132-199):
// Beris-Edwards rates Dxx, Dyx, the Cahn-Hilliard rate Dp, and the
// equilibrium fe' with the forcing folded in (see above), so that the
// collision is (fe'_v - f_v)*itau. itau = 1/tau(phi).
template<int MODEL>
__device__ __forceinline__ void uf2(const PP& P, const UQc& c, const UQx& xp, const UQx& xm,
                                    const YD& y, f2 Qxx, f2 Qyx, f2 itau, f2 tau, f2 fe[9],
                                    f2& Dxx, f2& Dyx, f2& Dp)
{
  const f2 Dxux = xp.ux - xm.ux, Dxuy = xp.uy - xm.uy;
  const f2 E2 = Dxux + y.uy;          // 2 expansion
  const f2 S4 = Dxuy + y.ux;          // 4 shear
  const f2 V4 = Dxuy - y.ux;          // 4 vorticity
  const f2 QS = Qyx*S4;
  const f2 T2 = fma(Qxx, Dxux - y.uy, QS);     // 2 traceQL
  // xi*((Qxx+1)(2dxux - trQL) + 2Qyx shear - expansion) = hxi*bx2
  const f2 bx2 = fma(Qxx + KC(1.f), KC(2.f)*Dxux - T2, QS - E2);
  // xi*(Qyx(expansion - trQL) + 2 shear) = hxi*by2
  const f2 by2 = fma(Qyx, E2 - T2, S4);
  Dxx = fma(W2(P.hxi), bx2, fma(KC(-.5f)*V4, Qyx, c.BEx));
  Dyx = fma(W2(P.hxi), by2, fma(KC(.5f)*V4, Qxx, c.BEy));
  // twice the force: (d_x s_xx + d_y s_xy - friction u_x), ...
  const f2 Fx2 = fma(W2(P.n2fric), c.ux, (xp.sXX - xm.sXX) + y.sXY);
  const f2 Fy2 = fma(W2(P.n2fric), c.uy, (xp.sYX - xm.sYX) + y.sYY);
  if constexpr (MODEL != NEM)
  {
    const f2 lMU = fma(KC(-4.f), c.MU, (xp.MU + xm.MU) + y.MUs);
    Dp = fma(W2(P.GammaP), lMU, KC(-.5f)*((xp.uxp - xm.uxp) + y.uyp));
  }
  else Dp = KC(0.f);

  const f2 dn = c.dn;
  const f2 nn = W2(P.rho) + dn;
  const f2 jx = nn*c.ux, jy = nn*c.uy;
  const f2 kxx = jx*c.ux, kyy = jy*c.uy, kxy = jx*c.uy, k2 = kxx + kyy;
  const f2 th = KC(.5f)*tau;
  const f2 jxF = fma(th, Fx2, jx), jyF = fma(th, Fy2, jy);
  const f2 A = fma(KC((1.f/3.f)), k2, KC((1.f/9.f))*dn);
  const f2 E1 = fma(KC(-.5f), kyy, A), E3 = fma(KC(-.5f), kxx, A);
  fe[1] = fma(KC((1.f/3.f)), jxF, E1);
  fe[2] = fma(KC((-1.f/3.f)), jxF, E1);
  fe[3] = fma(KC((1.f/3.f)), jyF, E3);
  fe[4] = fma(KC((-1.f/3.f)), jyF, E3);
  const f2 B = fma(KC((1.f/12.f)), k2, KC((1.f/36.f))*dn);
  const f2 Bp = fma(KC(.25f), kxy, B), Bm = fma(KC(-.25f), kxy, B);
  const f2 s = jxF + jyF, d = jxF - jyF;
  fe[5] = fma(KC((1.f/12.f)), s, Bp);
  fe[6] = fma(KC((-1.f/12.f)), s, Bp);
  fe[7] = fma(KC((-1.f/12.f)), d, Bm);
  fe[8] = fma(KC((1.f/12.f)), d, Bm);
  fe[0] = fma(KC((4.f/9.f)), dn, KC((-2.f/3.f))*k2);
  (void)itau;
}

// One lattice as one work item sees it.
struct ItemView
{
  const float* in;
  float* out;
  float* diag;
  int* err;
  int LX, LY;
  long long plane;
  int rows;
  const float* src;   // per-site phi source rate (SRC launches)
  float* pred;        // PRED launches: fn (9 planes), QNxx, QNyx[, phn] per site
  int xbase, xcount;  // the rows stepped: [xbase, xbase + xcount)
};

// Per-warp shared memory: input ring | delayed populations (3 rows) |
// fn - ff/(2 tau) (2 rows); then the ring's mbarriers after all warps.
template<int MODEL>
struct WarpSmem
{
  static constexpr int NP = MODEL == NEM ? 11 : MODEL == LYO ? 12 : 13;
  static constexpr int FLOATS = RING*NP*RWW + 3*NDP*PW + 2*9*COLS;
};

// Advance one strip chunk (strip `strip`, rows chunk*a.rows ..) of one
// lattice by a full step. `rowbase` counts the input rows this warp has
// copied through its ring so far (mbarrier phases continue across items).
// Returns false if a bounded wait gave up. SRC adds the division models'
// phi source, phi_tmp += phi*r after each UpdateFields
// (src/models/lyotropic-with-division.cpp:121), in C and E.
template<int MODEL, bool DIAG, bool SRC, bool PRED = false>
__device__ __forceinline__ bool warp_item(const ItemView& a, const PairParams& P, const int strip,
                                          const int chunk, float* ring, float* dpop, float* hrow,
                                          uint64_t* mbar, const int lane, unsigned& rowbase)
{
  constexpr int NP = MODEL == NEM ? 11 : MODEL == LYO ? 12 : 13;
  const int y0 = strip*WOUT;
  const int x0 = a.xbase + chunk*a.rows;
  const int rows = min(a.rows, a.xbase + a.xcount - x0);
  const int LX = a.LX, LY = a.LY;
  const int nload = rows + 8;            // rows x0-4 .. x0+rows+3
  const int ystart = (y0 - 4 + LY) % LY;
  const unsigned rb = rowbase;

  // Bulk-copy input row rr (lattice row x0 - 4 + rr) into its ring slot:
  // lane 0 posts the byte count, then lanes 0..NP-1 copy one plane each
  // (called by the whole warp).
  const float* plane_in = a.in + static_cast<long long>(lane < NP ? lane : 0)*a.plane;
  int gx_next = ((x0 - 4) % LX + LX) % LX;   // lattice row of the next copy
  auto issue = [&](int rr) {
    const int slot = (rb + rr) & (RING - 1);
    uint64_t* bar = &mbar[slot];
    if(lane == 0) mbar_expect_tx(bar, NP*COLS*4);
    __syncwarp();
    const int gx = gx_next;
    gx_next = gx_next + 1 == LX ? 0 : gx_next + 1;
    if(lane < NP)
    {
      const float* src = plane_in + static_cast<long long>(gx)*LY;
      float* dst = ring + (slot*NP + lane)*RWW + PADY;
      int start = ystart, rem = COLS;
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

  const int n0 = min(RING, nload);
  for(int rr = 0; rr < n0; ++rr) issue(rr);
  int issued = n0;
  bool abort = !mbar_wait_bounded(&mbar[rb & (RING - 1)], (rb / RING) & 1) ||
               !mbar_wait_bounded(&mbar[(rb + 1) & (RING - 1)], ((rb + 1) / RING) & 1);

  const int cl = PADY + 2*lane;            // this lane's first column in a ring row
  const int yg = y0 - 4 + 2*lane;          // global column of .x (pre-wrap)
  const bool lane_out = lane >= 2 && lane < 30;
  const bool colx_ok = lane_out && yg < LY;
  const bool coly_ok = lane_out && yg + 1 < LY;
  // source-rate pair of this lane at lattice row x (any row of the window)
  const int yw = yg < 0 ? yg + LY : (yg >= LY ? yg - LY : yg);
  auto src_at = [&](int x) {
    x = x < 0 ? x + LX : (x >= LX ? x - LX : x);
    return f2{__ldg(reinterpret_cast<const float2*>(a.src + static_cast<long long>(x)*LY + yw))};
  };

  UQc q1c{}, q2c{};
  UQx q1m{}, q2m{};
  UQd dq{};
  // predicted (Qxx, Qyx, phi, m) and QN (QNxx, QNyx, phn, mN) of the rows
  // one and two iterations back; m only in go-or-grow
  f2 qa1[4], qa2[4], qn1[4], qn2[4];
  // Delayed populations live in shared memory: row slot s (the row C
  // produced s iterations ago, mod 3), array k: ff v = 0,3,4 (k = 0..2),
  // fn v = 0,3,4 (3..5), ff v = 1,5,8 (6..8), fn v = 1,5,8 (9..11). C writes
  // them already shifted along y (column + cy); D reads its own columns.
#pragma unroll
  for(int k = 0; k < 4; ++k) { qa1[k] = qa2[k] = qn1[k] = qn2[k] = KC(0.f); }
  int s3 = 0;                              // i mod 3
  float* orow = a.out + static_cast<long long>(x0 - 6)*LY + yg;   // E's output row

  // stencil of plane q at ring row R0 (centre), Rp (+x), Rm (-x)
  auto ring_stn = [&](const float* Rm, const float* R0, const float* Rp, int q) {
    const float* c = R0 + q*RWW + cl;
    Stn t;
    t.c = lds2(c);
    const f2 xp = lds2(Rp + q*RWW + cl), xm = lds2(Rm + q*RWW + cl);
    const float lo = c[-1], hi = c[2];
    t.s = (xp + xm) + mk(t.c.v.y + lo, hi + t.c.v.x);
    t.X = xp - xm;
    t.Y = mk(t.c.v.y - lo, hi - t.c.v.x);
    return t;
  };
  // stencil from register rows: centre (held by this lane), +x, -x
  auto reg_stn = [&](f2 cen, f2 xp, f2 xm) {
    Stn t;
    t.c = cen;
    f2 ys;
    yboth(cen, ys, t.Y);
    t.s = (xp + xm) + ys;
    t.X = xp - xm;
    return t;
  };

  const int nit = rows + 6;
  for(int i = 0; i < nit; ++i)
  {
    if(i + 2 < nload)
    {
      const int rr = i + 2;
      if(!mbar_wait_bounded(&mbar[(rb + rr) & (RING - 1)], ((rb + rr) / RING) & 1)) abort = true;
    }
    if(__any_sync(0xffffffffu, abort)) break;
    const float* Rm = ring + ((rb + i    ) & (RING - 1))*NP*RWW;   // row b-1
    const float* R0 = ring + ((rb + i + 1) & (RING - 1))*NP*RWW;   // row b
    const float* Rp = ring + ((rb + i + 2) & (RING - 1))*NP*RWW;   // row b+1
    float* dp_now = dpop + s3*NDP*PW + 2 + 2*lane;                    // row of C, this iteration
    const float* dp_1 = dpop + (s3 == 0 ? 2 : s3 - 1)*NDP*PW + 2 + 2*lane;   // one iteration ago
    const float* dp_2 = dpop + (s3 == 2 ? 0 : s3 + 1)*NDP*PW + 2 + 2*lane;   // two iterations ago

    // ---- B: predictor UpdateQuantities at row b ----
    UQc nq1;
    {
      f2 g[9];
#pragma unroll
      for(int v = 0; v < 9; ++v) g[v] = lds2(R0 + v*RWW + cl);
      const Stn A = ring_stn(Rm, R0, Rp, 9), B = ring_stn(Rm, R0, Rp, 10);
      Stn Ph{};
      if constexpr (MODEL != NEM) Ph = ring_stn(Rm, R0, Rp, 11);
      const f2 m0 = MODEL == GOG ? lds2(R0 + 12*RWW + cl) : KC(0.f);
      UQd unused;
      uq2<MODEL, false>(P, g, A, B, Ph, m0, nq1, unused);
    }

    // ---- C: predictor UpdateFields at row b-1, then y-part of Move ----
    f2 nQ[4], nQN[4], pf[9], pn[9];
    {
      const YD y = ydiffs<MODEL>(q1c);
      const f2 Qxx = lds2(Rm + 9*RWW + cl), Qyx = lds2(Rm + 10*RWW + cl);
      const f2 p = MODEL != NEM ? lds2(Rm + 11*RWW + cl) : KC(0.f);
      const f2 tau = MODEL != NEM ? fma(W2(P.dtau), p, W2(P.tauIso)) : W2(P.tauIso);
      const f2 itau = MODEL != NEM ? rcp2(tau, P) : W2(P.itau);
      const f2 hitau = KC(.5f)*itau;
      f2 fe[9], Dxx, Dyx, Dp;
      uf2<MODEL>(P, q1c, xset(nq1), q1m, y, Qxx, Qyx, itau, tau, fe, Dxx, Dyx, Dp);
#pragma unroll
      for(int v = 0; v < 9; ++v)
      {
        const f2 g = lds2(Rm + v*RWW + cl);
        const f2 dv = fe[v] - g;
        pn[v] = fma(hitau, dv, g);
        pf[v] = fma(itau, dv, g);
      }
      nQN[0] = fma(KC(.5f), Dxx, Qxx);
      nQN[1] = fma(KC(.5f), Dyx, Qyx);
      if constexpr (MODEL == LYO)
      {
        nQ[0] = Qxx + Dxx;
        nQ[1] = Qyx + Dyx;
        nQN[2] = fma(KC(.5f), Dp, p);
        nQ[2] = p + Dp;
        if constexpr (SRC) nQ[2] = fma(p, src_at(x0 - 4 + i), nQ[2]);
        nQN[3] = nQ[3] = KC(0.f);
      }
      else if constexpr (MODEL == GOG)
      {
        f2 Dm, R;
        pheno_rate(P, q1c, xset(nq1), q1m, y, src_at(x0 - 4 + i), Dm, R);
        const f2 me = lds2(Rm + 12*RWW + cl);
        nQ[0] = Qxx + Dxx;
        nQ[1] = Qyx + Dyx;
        nQN[2] = fma(KC(.5f), Dp, p);
        nQ[2] = (p + Dp) + R;
        nQN[3] = fma(KC(.5f), Dm, me);
        nQ[3] = clamp_m(me + Dm, nQ[2]);
      }
      else
      {
        nQ[0] = Qxx + Dxx;
        nQ[1] = Qyx + Dyx;
        nQN[2] = nQ[2] = nQN[3] = nQ[3] = KC(0.f);
      }
      // stream along y. Directions with cx = -1 (2, 6, 7) are used by D in
      // this same iteration: shift them by shuffles. The others go to the
      // delayed-population rows in shared memory, written at column + cy.
      pf[6] = yplus(pf[6]); pn[6] = yplus(pn[6]);
      pf[7] = yminus(pf[7]); pn[7] = yminus(pn[7]);
      const int dv[6] = {0, 3, 4, 1, 5, 8};
#pragma unroll
      for(int k = 0; k < 6; ++k)
      {
        const int v = dv[k];
        float* d0 = dp_now + (k < 3 ? k : k + 3)*PW + CYv(v);
        float* d1p = dp_now + (k < 3 ? k + 3 : k + 6)*PW + CYv(v);
        if(CYv(v) == 0)
        {
          *reinterpret_cast<float2*>(d0) = pf[v].v;
          *reinterpret_cast<float2*>(d1p) = pn[v].v;
        }
        else
        {
          d0[0] = pf[v].v.x; d0[1] = pf[v].v.y;
          d1p[0] = pn[v].v.x; d1p[1] = pn[v].v.y;
        }
      }
    }

    // ---- D: corrector UpdateQuantities at row s = b-2 (x-part of Move) ----
    UQc nq2;
    {
      // direction v at (s, y) left row s - cx: cx = -1 is the row C just
      // produced, cx = 0 the previous one, cx = +1 the one before that
      f2 fs[9], ns[9];
      fs[2] = pf[2]; fs[6] = pf[6]; fs[7] = pf[7];
      ns[2] = pn[2]; ns[6] = pn[6]; ns[7] = pn[7];
      fs[0] = lds2(dp_1 + 0*PW); fs[3] = lds2(dp_1 + 1*PW); fs[4] = lds2(dp_1 + 2*PW);
      ns[0] = lds2(dp_1 + 3*PW); ns[3] = lds2(dp_1 + 4*PW); ns[4] = lds2(dp_1 + 5*PW);
      fs[1] = lds2(dp_2 + 6*PW); fs[5] = lds2(dp_2 + 7*PW); fs[8] = lds2(dp_2 + 8*PW);
      ns[1] = lds2(dp_2 + 9*PW); ns[5] = lds2(dp_2 + 10*PW); ns[8] = lds2(dp_2 + 11*PW);
      const Stn A = reg_stn(qa1[0], nQ[0], qa2[0]);
      const Stn B = reg_stn(qa1[1], nQ[1], qa2[1]);
      Stn Ph{};
      if constexpr (MODEL != NEM) Ph = reg_stn(qa1[2], nQ[2], qa2[2]);
      uq2<MODEL, DIAG>(P, fs, A, B, Ph, qa1[3], nq2, dq);
      const f2 hitau = KC(-.5f)*itau_of<MODEL>(P, qa1[2]);
#pragma unroll
      for(int v = 0; v < 9; ++v)
        *reinterpret_cast<float2*>(hrow + ((i & 1)*9 + v)*COLS + 2*lane) = fma(hitau, fs[v], ns[v]).v;
      if constexpr (PRED)
      {
        // what every further corrector of the step reads (npc > 1): the
        // moved predictor populations fn and the half-step fields QN of
        // this row, in the sweeps' plane order
        const int xs = x0 - 5 + i;
        if(xs >= x0 && xs < x0 + rows)
        {
          const long long pl = a.plane;
          float* o = a.pred + static_cast<long long>(xs)*LY + yg;
          constexpr int NPRED = MODEL == NEM ? 11 : 12;
          f2 w[12];
#pragma unroll
          for(int v = 0; v < 9; ++v) w[v] = ns[v];
          w[9] = qn1[0];
          w[10] = qn1[1];
          w[11] = qn1[2];
          if(colx_ok && coly_ok)
          {
#pragma unroll
            for(int k = 0; k < NPRED; ++k) *reinterpret_cast<float2*>(o + k*pl) = w[k].v;
          }
          else if(colx_ok)
          {
#pragma unroll
            for(int k = 0; k < NPRED; ++k) o[k*pl] = w[k].v.x;
          }
        }
      }
      if constexpr (DIAG)
      {
        const int xs = x0 - 5 + i;
        if(xs >= x0 && xs < x0 + rows)
        {
          const long long pl = a.plane;
          float* o = a.diag + static_cast<long long>(xs)*LY + yg;
          const f2 vals[16] = {W2(P.rho) + nq2.dn, nq2.ux, nq2.uy, nq2.uxp, nq2.uyp, dq.Hxx,
                               dq.Hyx, nq2.MU, KC(.5f)*dq.XA, KC(.5f)*dq.YA, KC(.5f)*dq.XB,
                               KC(.5f)*dq.YB, nq2.sXX, nq2.sYY, nq2.sYX, nq2.sXY};
#pragma unroll
          for(int k = 0; k < 16; ++k)
          {
            if(colx_ok) o[k*pl] = vals[k].v.x;
            if(coly_ok) o[k*pl + 1] = vals[k].v.y;
          }
          if constexpr (MODEL != NEM)
          {
            const f2 aQxx = dq.nact*qa1[0], aQyx = dq.nact*qa1[1];
            // the lyotropic elastic yx stress carries +zeta*Qxx*(1-phi) as
            // the reference has it (src/models/lyotropic.cpp:242); the
            // go-or-grow one the Qyx term (src/models/go-or-grow.cpp:300)
            const f2 dg[7] = {dq.bi, (dq.sigmaF - dq.pf) - aQxx,
                              (dq.sigmaS - dq.pfS) - (MODEL == GOG ? aQyx : aQxx),
                              dq.pf, dq.pfS, aQxx, aQyx};
#pragma unroll
            for(int k = 0; k < 7; ++k)
            {
              if(colx_ok) o[(16 + k)*pl] = dg[k].v.x;
              if(coly_ok) o[(16 + k)*pl + 1] = dg[k].v.y;
            }
          }
        }
      }
    }

    // ---- E: corrector UpdateFields at row b-3, store ----
    if constexpr (!DIAG)
    {
      const YD y = ydiffs<MODEL>(q2c);
      const f2 tau = MODEL != NEM ? fma(W2(P.dtau), qa2[2], W2(P.tauIso)) : W2(P.tauIso);
      const f2 itau = MODEL != NEM ? rcp2(tau, P) : W2(P.itau);
      const f2 hitau = KC(.5f)*itau;
      f2 fe[9], Dxx, Dyx, Dp;
      uf2<MODEL>(P, q2c, xset(nq2), q2m, y, qa2[0], qa2[1], itau, tau, fe, Dxx, Dyx, Dp);
      f2 gout[9];
#pragma unroll
      for(int v = 0; v < 9; ++v)
        gout[v] = fma(hitau, fe[v], lds2(hrow + (((i + 1) & 1)*9 + v)*COLS + 2*lane));
      const f2 Qo0 = fma(KC(.5f), Dxx, qn2[0]);
      const f2 Qo1 = fma(KC(.5f), Dyx, qn2[1]);
      f2 Qo2 = fma(KC(.5f), Dp, qn2[2]);
      // corrector source with the predicted phi of this row
      if constexpr (SRC) Qo2 = fma(qa2[2], src_at(x0 - 6 + i), Qo2);
      f2 Qo3 = KC(0.f);
      if constexpr (MODEL == GOG)
      {
        f2 Dm, R;
        pheno_rate(P, q2c, xset(nq2), q2m, y, src_at(x0 - 6 + i), Dm, R);
        Qo2 = Qo2 + R;
        Qo3 = clamp_m(fma(KC(.5f), Dm, qn2[3]), Qo2);
      }
      if(i >= 6)
      {
        const long long pl = a.plane;
        float* o = orow;
        if(colx_ok && coly_ok)
        {
#pragma unroll
          for(int v = 0; v < 9; ++v) *reinterpret_cast<float2*>(o + v*pl) = gout[v].v;
          *reinterpret_cast<float2*>(o + 9*pl) = Qo0.v;
          *reinterpret_cast<float2*>(o + 10*pl) = Qo1.v;
          if constexpr (MODEL != NEM) *reinterpret_cast<float2*>(o + 11*pl) = Qo2.v;
          if constexpr (MODEL == GOG) *reinterpret_cast<float2*>(o + 12*pl) = Qo3.v;
        }
        else if(colx_ok)
        {
#pragma unroll
          for(int v = 0; v < 9; ++v) o[v*pl] = gout[v].v.x;
          o[9*pl] = Qo0.v.x;
          o[10*pl] = Qo1.v.x;
          if constexpr (MODEL != NEM) o[11*pl] = Qo2.v.x;
          if constexpr (MODEL == GOG) o[12*pl] = Qo3.v.x;
        }
      }
    }

    // ---- advance the row windows ----
    q1m = xset(q1c); q1c = nq1;
    q2m = xset(q2c); q2c = nq2;
#pragma unroll
    for(int k = 0; k < 4; ++k)
    {
      qa2[k] = qa1[k]; qa1[k] = nQ[k];
      qn2[k] = qn1[k]; qn1[k] = nQN[k];
    }
    s3 = s3 == 2 ? 0 : s3 + 1;
    orow += LY;

    __syncwarp();
    if(issued < nload && issued <= i + RING)
    {
      fence_proxy_async();
      issue(issued);
      ++issued;
    }
  }

  rowbase = rb + issued;
  if(abort)
  {
    if(lane == 0) atomicOr(a.err, 1);
    // let every copy this warp issued land before its shared memory is
    // released
    for(int rr = 0; rr < issued; ++rr)
      mbar_wait_bounded(&mbar[(rb + rr) & (RING - 1)], ((rb + rr) / RING) & 1);
    return false;
  }
  return true;
}

template<int MODEL>
__device__ __forceinline__ void warp_smem(float*& ring, float*& dpop, float*& hrow,
                                          uint64_t*& mbar, const int warp, const int lane)
{
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int NP = WarpSmem<MODEL>::NP;
  ring = reinterpret_cast<float*>(smem_raw) + warp*WarpSmem<MODEL>::FLOATS;
  dpop = ring + RING*NP*RWW;
  hrow = dpop + 3*NDP*PW;
  mbar = reinterpret_cast<uint64_t*>(
    smem_raw + WPB*WarpSmem<MODEL>::FLOATS*sizeof(float)) + warp*RING;
  if(lane == 0)
  {
    for(int s = 0; s < RING; ++s) mbar_init(&mbar[s], 1);
    fence_barrier_init();
  }
  __syncwarp();
}

// One lattice: work item = blockIdx.x*WPB + warp.
template<int MODEL, bool DIAG, bool SRC, bool PRED>
__global__ void __launch_bounds__(32*WPB, 2)
fused_warp_kernel(const __grid_constant__ FusedArgs a, const int nitems)
{
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x*WPB + warp;
  if(item >= nitems) return;
  float *ring, *dpop, *hrow;
  uint64_t* mbar;
  warp_smem<MODEL>(ring, dpop, hrow, mbar, warp, lane);
  const ItemView v{a.in, a.out, a.diag, a.err, a.LX, a.LY, a.plane, a.rows, a.src, a.pred,
                   a.xbase, a.xcount};
  unsigned rowbase = 0;
  // chunk-major: the warps in flight together work down a few strips at
  // every height of the lattice (about 4 % faster than strip-major at 4096^2)
  const int nchunks = (a.xcount + a.rows - 1)/a.rows;
  warp_item<MODEL, DIAG, SRC, PRED>(v, a.pp, item / nchunks, item % nchunks, ring, dpop, hrow,
                                     mbar, lane, rowbase);
}

// Ensemble: persistent warps take (run, strip, chunk) items from a packed
// list through an atomic counter until it runs out. Per-run physics is in
// constant memory (a slot range per ensemble).
__constant__ PairParams c_ens_pp[ENS_MAX_RUNS];

template<int MODEL>
__global__ void __launch_bounds__(32*WPB, 2)
fused_warp_ensemble_kernel(const EnsRun* __restrict__ runs, const int* __restrict__ item_run,
                           const int nitems, int* __restrict__ counter, int* err, const int parity)
{
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float *ring, *dpop, *hrow;
  uint64_t* mbar;
  warp_smem<MODEL>(ring, dpop, hrow, mbar, warp, lane);
  unsigned rowbase = 0;
  for(;;)
  {
    int item = 0;
    if(lane == 0) item = atomicAdd(counter, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if(item >= nitems) break;
    const int r = item_run[item];
    const EnsRun& R = runs[r];
    const int local = item - R.item0;
    const ItemView v{parity ? R.b : R.a, parity ? R.a : R.b, nullptr, err, R.LX, R.LY,
                     R.plane, R.rows, nullptr, nullptr, 0, R.LX};
    const int nchunks = (R.LX + R.rows - 1)/R.rows;   // chunk-major, as fused_warp_kernel
    if(!warp_item<MODEL, false, false>(v, c_ens_pp[R.slot], local / nchunks, local % nchunks,
                                ring, dpop, hrow, mbar, lane, rowbase))
      break;
  }
}

template<int MODEL>
constexpr size_t smem_bytes()
{
  return static_cast<size_t>(WPB)*WarpSmem<MODEL>::FLOATS*sizeof(float) +
         static_cast<size_t>(WPB)*RING*sizeof(uint64_t);
}

template<int MODEL, bool DIAG, bool SRC, bool PRED = false>
cudaError_t launch_t(const FusedArgs& a, int rows, cudaStream_t st)
{
  auto kern = fused_warp_kernel<MODEL, DIAG, SRC, PRED>;
  static unsigned long long attr_set = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if(!(attr_set & bit))
  {
    const cudaError_t e = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_bytes<MODEL>()));
    if(e != cudaSuccess) return e;
    attr_set |= bit;
  }
  FusedArgs b = a;
  b.rows = rows;
  b.nstrips = (a.LY + WOUT - 1)/WOUT;
  b.pp = make_pp(a.p, MODEL);
  const int nchunks = (a.xcount + rows - 1)/rows;
  const int nitems = b.nstrips*nchunks;
  const dim3 grid((nitems + WPB - 1)/WPB);
  kern<<<grid, 32*WPB, smem_bytes<MODEL>(), st>>>(b, nitems);
  return cudaGetLastError();
}

template<int MODEL>
cudaError_t ens_attr()
{
  static unsigned long long attr_set = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if(!(attr_set & bit))
  {
    const cudaError_t e = cudaFuncSetAttribute(fused_warp_ensemble_kernel<MODEL>,
      cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_bytes<MODEL>()));
    if(e != cudaSuccess) return e;
    attr_set |= bit;
  }
  return cudaSuccess;
}

template<int MODEL>
cudaError_t launch_ens(const EnsRun* runs, const int* item_run, int nitems, int* counter,
                       int* err, int parity, int grid, cudaStream_t st)
{
  const cudaError_t e = ens_attr<MODEL>();
  if(e != cudaSuccess) return e;
  fused_warp_ensemble_kernel<MODEL><<<grid, 32*WPB, smem_bytes<MODEL>(), st>>>(
    runs, item_run, nitems, counter, err, parity);
  return cudaGetLastError();
}

template<int MODEL>
int ens_grid()
{
  if(ens_attr<MODEL>() != cudaSuccess) return 0;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_warp_ensemble_kernel<MODEL>,
                                                   32*WPB, smem_bytes<MODEL>()) != cudaSuccess)
    return 0;
  return sms*std::max(per_sm, 1);
}

} // namespace

cudaError_t ensemble_set_params(int slot, const P32& p, int model, cudaStream_t st)
{
  if(slot < 0 || slot >= ENS_MAX_RUNS) return cudaErrorInvalidValue;
  static thread_local PairParams staging[ENS_MAX_RUNS];
  staging[slot] = make_pp(p, model);
  const cudaError_t e = cudaMemcpyToSymbolAsync(c_ens_pp, &staging[slot], sizeof(PairParams),
                                                slot*sizeof(PairParams), cudaMemcpyHostToDevice, st);
  if(e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}

cudaError_t launch_fused_warp_ensemble(const EnsRun* runs, const int* item_run, int nitems,
                                       int* counter, int* err, int parity, int model, int grid,
                                       cudaStream_t st)
{
  return model == LYO ? launch_ens<LYO>(runs, item_run, nitems, counter, err, parity, grid, st)
                      : launch_ens<NEM>(runs, item_run, nitems, counter, err, parity, grid, st);
}

int ensemble_grid(int model)
{
  return model == LYO ? ens_grid<LYO>() : ens_grid<NEM>();
}

cudaError_t launch_fused_warp_step(const FusedArgs& a, int model, int rows, bool diag,
                                   cudaStream_t st)
{
  // a non-diagnostic launch with a.pred set also writes the predictor
  // values the further correctors of npc > 1 read (lyotropic, nematic)
  const bool pred = !diag && a.pred;
  if(model == LYO)
  {
    if(a.src)
    {
      if(pred) return launch_t<LYO, false, true, true>(a, rows, st);
      return diag ? launch_t<LYO, true, true>(a, rows, st) : launch_t<LYO, false, true>(a, rows, st);
    }
    if(pred) return launch_t<LYO, false, false, true>(a, rows, st);
    return diag ? launch_t<LYO, true, false>(a, rows, st) : launch_t<LYO, false, false>(a, rows, st);
  }
  if(model == GOG)
  {
    // the growth-rate plane is part of every go-or-grow step
    if(!a.src) return cudaErrorInvalidValue;
    return diag ? launch_t<GOG, true, false>(a, rows, st) : launch_t<GOG, false, false>(a, rows, st);
  }
  if(pred) return launch_t<NEM, false, false, true>(a, rows, st);
  return diag ? launch_t<NEM, true, false>(a, rows, st) : launch_t<NEM, false, false>(a, rows, st);
}

} // namespace mlb
