// Unfused step kernels: one sweep per reference loop.
//
//   UpdateQuantities  -> uq_kernel   (src/models/lyotropic.cpp:168-247,
//                                     src/models/nematic.cpp:76-130)
//   UpdateFields      -> uf_kernel   (src/models/lyotropic.cpp:249-341,
//                                     src/models/nematic.cpp:132-226)
//   Move              -> move_kernel (src/models/lyotropic.cpp:371-386),
//                        written as a pull over the extended torus, which
//                        assigns every target exactly the value the
//                        reference's push assigns it
//   BoundaryConditions*-> bc_*_kernel (src/fields.hpp:620-930)
//   periodic lattices -> substep_kernel: UpdateQuantities on a tile plus a
//                        one-site ring in shared memory, then UpdateFields
//                        (and, in the predictor, Move) in the same launch
//
// Two instantiations, built as two objects (MLB_UNFUSED_PART = 64 / 32):
//   T = double, DEV = false : the FP64 oracle mode. Its object is compiled
//     with --fmad=false and every expression keeps the reference's operand
//     order, so each value is rounded exactly as the reference's x86-64
//     build rounds it.
//   T = float,  DEV = true  : FP32 for go-or-grow, wall lattices and shapes
//     the fused kernels do not take. Populations are stored as deviations
//     g_v = f_v - t_v*rho from the rest state, so the O(1e-3) flow signal is
//     not lost against rho = 40 in a 24-bit mantissa. Its object contracts
//     multiply-adds, and it multiplies by 1/tau and 1/n where FP64 divides.
#include "lb_common.cuh"
#include "unfused.h"

#include <atomic>
#include <type_traits>
#include <utility>

namespace mlb {
namespace {

template<typename T>
struct Nbr
{
  long long e, e1, e2, e3, e4;  // self, +x, -x, +y, -y
};

template<typename T>
__device__ __forceinline__ Nbr<T> neighbours(const Dims& d, int X, int Y)
{
  Nbr<T> n;
  const int Xp = X + 1 == d.EX ? 0 : X + 1, Xm = X == 0 ? d.EX - 1 : X - 1;
  const int Yp = Y + 1 == d.EY ? 0 : Y + 1, Ym = Y == 0 ? d.EY - 1 : Y - 1;
  n.e  = Y  + (long long)d.EY*X;
  n.e1 = Y  + (long long)d.EY*Xp;
  n.e2 = Y  + (long long)d.EY*Xm;
  n.e3 = Yp + (long long)d.EY*X;
  n.e4 = Ym + (long long)d.EY*X;
  return n;
}

// 5-point stencils (src/lb.hpp:79, :89, :134); `+0*stencil` adds +0
template<typename T>
__device__ __forceinline__ T dX(const T* __restrict__ a, const Nbr<T>& n)
{ return T(.5)*(a[n.e1]-a[n.e2]) + T(0); }
template<typename T>
__device__ __forceinline__ T dY(const T* __restrict__ a, const Nbr<T>& n)
{ return T(.5)*(a[n.e3]-a[n.e4]) + T(0); }
template<typename T>
__device__ __forceinline__ T lap(const T* __restrict__ a, const Nbr<T>& n)
{ return a[n.e1]+a[n.e2]+a[n.e3]+a[n.e4] - T(4)*a[n.e] + T(0); }

// Equilibrium (src/lb.hpp:24-41). DEV: deviation from t_v*rho, given the
// density deviation dn = nn - rho (t_v*dn + the velocity terms times nn).
template<typename T, bool DEV>
__device__ __forceinline__ void equilibrium(T vx, T vy, T nn, T dn, T fe[9])
{
  const T v2 = vx*vx + vy*vy;
  if constexpr (!DEV)
  {
    fe[1] = nn*(T(1./9.) + T(1./3.)*vx + T(1./3.)*v2 - T(1./2.)*vy*vy);
    fe[2] = nn*(T(1./9.) - T(1./3.)*vx + T(1./3.)*v2 - T(1./2.)*vy*vy);
    fe[3] = nn*(T(1./9.) + T(1./3.)*vy - T(1./2.)*vx*vx + T(1./3.)*v2);
    fe[4] = nn*(T(1./9.) - T(1./3.)*vy - T(1./2.)*vx*vx + T(1./3.)*v2);
    fe[5] = nn*(T(1./36.) + T(1./12.)*vx + T(1./12.)*vy + T(1./12.)*v2 + T(1./4.)*vx*vy);
    fe[6] = nn*(T(1./36.) - T(1./12.)*vx - T(1./12.)*vy + T(1./12.)*v2 + T(1./4.)*vx*vy);
    fe[7] = nn*(T(1./36.) - T(1./12.)*vx + T(1./12.)*vy + T(1./12.)*v2 - T(1./4.)*vx*vy);
    fe[8] = nn*(T(1./36.) + T(1./12.)*vx - T(1./12.)*vy + T(1./12.)*v2 - T(1./4.)*vx*vy);
    fe[0] = nn-fe[1]-fe[2]-fe[3]-fe[4]-fe[5]-fe[6]-fe[7]-fe[8];
  }
  else
  {
    fe[1] = T(1./9.)*dn + nn*( T(1./3.)*vx + T(1./3.)*v2 - T(1./2.)*vy*vy);
    fe[2] = T(1./9.)*dn + nn*(-T(1./3.)*vx + T(1./3.)*v2 - T(1./2.)*vy*vy);
    fe[3] = T(1./9.)*dn + nn*( T(1./3.)*vy - T(1./2.)*vx*vx + T(1./3.)*v2);
    fe[4] = T(1./9.)*dn + nn*(-T(1./3.)*vy - T(1./2.)*vx*vx + T(1./3.)*v2);
    fe[5] = T(1./36.)*dn + nn*( T(1./12.)*vx + T(1./12.)*vy + T(1./12.)*v2 + T(1./4.)*vx*vy);
    fe[6] = T(1./36.)*dn + nn*(-T(1./12.)*vx - T(1./12.)*vy + T(1./12.)*v2 + T(1./4.)*vx*vy);
    fe[7] = T(1./36.)*dn + nn*(-T(1./12.)*vx + T(1./12.)*vy + T(1./12.)*v2 - T(1./4.)*vx*vy);
    fe[8] = T(1./36.)*dn + nn*( T(1./12.)*vx - T(1./12.)*vy + T(1./12.)*v2 - T(1./4.)*vx*vy);
    fe[0] = dn-fe[1]-fe[2]-fe[3]-fe[4]-fe[5]-fe[6]-fe[7]-fe[8];
  }
}

// The values one UpdateQuantities leaves at a site (src/models/lyotropic.cpp:
// 215-247): density (n, or its deviation in DEV mode), velocity, phi flux,
// molecular field, chemical potential, Q derivatives, stresses, and the
// seven diagnostic stresses (DIAG).
template<typename T>
struct UQOut
{
  T n, ux, uy, uxp, uyp, Hxx, Hyx, MU, dxQxx, dyQxx, dxQyx, dyQyx, sXX, sYY, sXY, sYX;
  T dg[7];
};

// UpdateQuantities of one site (the outputs in `o`)
template<typename T, bool DEV, int MODEL, bool DIAG>
__device__ __forceinline__ void uq_site(const Params& P, const State<T>& s, const Nbr<T>& nb,
                                        const long long NE, UQOut<T>& o)
{
  const long long e = nb.e;
  const T* __restrict__ F = s.ff;
  const T f0 = F[e], f1 = F[NE+e], f2 = F[2*NE+e], f3 = F[3*NE+e], f4 = F[4*NE+e],
          f5 = F[5*NE+e], f6 = F[6*NE+e], f7 = F[7*NE+e], f8 = F[8*NE+e];
  const T Qxx = s.Qxx[e], Qyx = s.Qyx[e];

  T nn, dn;
  if constexpr (DEV) { dn = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8; nn = T(P.rho) + dn; }
  else { nn = f0 + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8; dn = nn; }
  T vx, vy;
  if constexpr (DEV)
  {
    const T inn = T(1)/nn;
    vx = (f1 - f2 + f5 - f6 - f7 + f8)*inn;
    vy = (f3 - f4 + f5 - f6 + f7 - f8)*inn;
  }
  else
  {
    vx = (f1 - f2 + f5 - f6 - f7 + f8)/nn;
    vy = (f3 - f4 + f5 - f6 + f7 - f8)/nn;
  }

  const T del2Qxx = lap(s.Qxx, nb);
  const T dxQxx = dX(s.Qxx, nb);
  const T dyQxx = dY(s.Qxx, nb);
  const T del2Qyx = lap(s.Qyx, nb);
  const T dxQyx = dX(s.Qyx, nb);
  const T dyQyx = dY(s.Qyx, nb);

  const T CC = T(P.CC), LL = T(P.LL), xi = T(P.xi), zeta = T(P.zeta);

  o.n = DEV ? dn : nn;   // DEV mode keeps the density deviation
  o.ux = vx;
  o.uy = vy;
  o.dxQxx = dxQxx;
  o.dxQyx = dxQyx;
  o.dyQxx = dyQxx;
  o.dyQyx = dyQyx;

  if constexpr (MODEL == LYO)
  {
    const T AA = T(P.AA), KK = T(P.KK), zetaI = T(P.zetaI), conc = T(P.conc);
    const T p = s.phi[e];
    const T del2p = lap(s.phi, nb);
    const T dxPhi = dX(s.phi, nb);
    const T dyPhi = dY(s.phi, nb);
    const T term = T(0) - Qxx*Qxx - Qyx*Qyx;
    const T Hxx = CC*term*Qxx + LL*del2Qxx;
    const T Hyx = CC*term*Qyx + LL*del2Qyx;
    const T mu = AA*p*(T(1)-p)*(T(1)-T(2)*p) + T(0)*CC*term - KK*del2p;
    const T sigmaB = T(.5)*AA*p*p*(T(1)-p)*(T(1)-p) + T(.5)*CC*term*term - mu*p;
    const T sigmaF = T(2)*xi*( (Qxx*Qxx-T(1))*Hxx + Qxx*Qyx*Hyx )
      - zeta*Qxx*(T(1)-p) + T(.5)*KK*(dyPhi*dyPhi-dxPhi*dxPhi)
      + LL*(dyQxx*dyQxx+dyQyx*dyQyx-dxQxx*dxQxx-dxQyx*dxQyx);
    const T sigmaS = T(2)*xi*(Qyx*Qxx*Hxx + (Qyx*Qyx-T(1))*Hyx)
      - zeta*Qyx*(T(1)-p) - KK*dxPhi*dyPhi
      - T(2)*LL*(dxQxx*dyQxx+dxQyx*dyQyx);
    const T sigmaA = T(2)*(Qxx*Hyx - Qyx*Hxx);

    o.uxp = vx*p;
    o.uyp = vy*p;
    o.Hxx = Hxx;
    o.Hyx = Hyx;
    o.MU = mu;
    o.sXX = sigmaF + sigmaB + zetaI*(conc-p);
    o.sYY = -sigmaF + sigmaB + zetaI*(conc-p);
    o.sXY = sigmaS + sigmaA;
    o.sYX = sigmaS - sigmaA;
    if constexpr (DIAG)
    {
      o.dg[0] = sigmaB + zetaI*(conc-p);
      o.dg[1] = sigmaF - T(.5)*KK*(dyPhi*dyPhi-dxPhi*dxPhi) + zeta*Qxx*(T(1)-p);
      // the reference uses zeta*Qxx here too (src/models/lyotropic.cpp:242)
      o.dg[2] = sigmaS + KK*dxPhi*dyPhi + zeta*Qxx*(T(1)-p);
      o.dg[3] = T(.5)*KK*(dyPhi*dyPhi-dxPhi*dxPhi);
      o.dg[4] = -KK*dxPhi*dyPhi;
      o.dg[5] = -zeta*Qxx*(T(1)-p);
      o.dg[6] = -zeta*Qyx*(T(1)-p);
    }
  }
  else if constexpr (MODEL == GOG)
  {
    // GoOrGrow::UpdateQuantitiesAtNode (src/models/go-or-grow.cpp:230-308):
    // preferred order Snem, crowding penalty B above phi_critical, and an
    // active stress weighted by the go fraction 1 - chi
    const T AA = T(P.AA), KK = T(P.KK), zetaI = T(P.zetaI), conc = T(P.conc);
    const T B = T(s.ph.B), Snem = T(s.ph.Snem), phic = T(s.ph.phi_critical);
    const T p = s.phi[e];
    const T del2p = lap(s.phi, nb);
    const T dxPhi = dX(s.phi, nb);
    const T dyPhi = dY(s.phi, nb);
    const T q2 = Qxx*Qxx + Qyx*Qyx;
    const T term = Snem - q2;
    const T Hxx = T(2)*CC*term*Qxx + LL*del2Qxx;
    const T Hyx = T(2)*CC*term*Qyx + LL*del2Qyx;
    const T dpc = p - phic;
    const T f_compress = dpc > T(0) ? T(.5)*B*dpc*dpc : T(0);
    const T mu_compress = dpc > T(0) ? B*dpc : T(0);
    const T mu = AA*p*(T(1)-p)*(T(1)-T(2)*p) + mu_compress - KK*del2p;
    const T sigmaB = T(.5)*AA*p*p*(T(1)-p)*(T(1)-p)
      + f_compress + T(.5)*CC*term*term - mu*p;
    const T ap = zeta*p*(T(1)-s.chi[e]);
    const T sigmaF = T(2)*xi*( (Qxx*Qxx-T(1))*Hxx + Qxx*Qyx*Hyx )
      - ap*Qxx + T(.5)*KK*(dyPhi*dyPhi-dxPhi*dxPhi)
      + LL*(dyQxx*dyQxx+dyQyx*dyQyx-dxQxx*dxQxx-dxQyx*dxQyx);
    const T sigmaS = T(2)*xi*(Qyx*Qxx*Hxx + (Qyx*Qyx-T(1))*Hyx)
      - ap*Qyx - KK*dxPhi*dyPhi
      - T(2)*LL*(dxQxx*dyQxx+dxQyx*dyQyx);
    const T sigmaA = T(2)*(Qxx*Hyx - Qyx*Hxx);

    o.uxp = vx*p;
    o.uyp = vy*p;
    o.Hxx = Hxx;
    o.Hyx = Hyx;
    o.MU = mu;
    o.sXX = sigmaF + sigmaB + zetaI*(conc-p);
    o.sYY = -sigmaF + sigmaB + zetaI*(conc-p);
    o.sXY = sigmaS + sigmaA;
    o.sYX = sigmaS - sigmaA;
    if constexpr (DIAG)
    {
      o.dg[0] = sigmaB + zetaI*(conc-p);
      o.dg[1] = sigmaF - T(.5)*KK*(dyPhi*dyPhi-dxPhi*dxPhi) + ap*Qxx;
      o.dg[2] = sigmaS + KK*dxPhi*dyPhi + ap*Qyx;
      o.dg[3] = T(.5)*KK*(dyPhi*dyPhi-dxPhi*dxPhi);
      o.dg[4] = -KK*dxPhi*dyPhi;
      o.dg[5] = -ap*Qxx;
      o.dg[6] = -ap*Qyx;
    }
  }
  else
  {
    const T term = T(1.) - Qxx*Qxx - Qyx*Qyx;
    const T Hxx = CC*term*Qxx + LL*del2Qxx;
    const T Hyx = CC*term*Qyx + LL*del2Qyx;
    const T sigmaB = T(.5)*CC*term*term;
    const T sigmaF = T(2)*xi*( (Qxx*Qxx-T(1.))*Hxx + Qxx*Qyx*Hyx )
      - zeta*Qxx
      + LL*(dyQxx*dyQxx+dyQyx*dyQyx-dxQxx*dxQxx-dxQyx*dxQyx);
    const T sigmaS = T(2)*xi*(Qyx*Qxx*Hxx + (Qyx*Qyx-T(1))*Hyx) - zeta*Qyx
      - T(2)*LL*(dxQxx*dyQxx+dxQyx*dyQyx);
    const T sigmaA = T(2)*(Qxx*Hyx - Qyx*Hxx);
    o.Hxx = Hxx;
    o.Hyx = Hyx;
    o.sXX = sigmaF + sigmaB;
    o.sYY = -sigmaF + sigmaB;
    o.sXY = sigmaS + sigmaA;
    o.sYX = sigmaS - sigmaA;
  }
}

template<typename T, int MODEL, bool DIAG>
__device__ __forceinline__ void store_uq(const State<T>& s, const long long e, const UQOut<T>& o)
{
  s.n[e] = o.n; s.ux[e] = o.ux; s.uy[e] = o.uy;
  s.dxQxx[e] = o.dxQxx; s.dxQyx[e] = o.dxQyx; s.dyQxx[e] = o.dyQxx; s.dyQyx[e] = o.dyQyx;
  s.Hxx[e] = o.Hxx; s.Hyx[e] = o.Hyx;
  s.sXX[e] = o.sXX; s.sYY[e] = o.sYY; s.sXY[e] = o.sXY; s.sYX[e] = o.sYX;
  if constexpr (MODEL != NEM)
  {
    s.uxp[e] = o.uxp; s.uyp[e] = o.uyp; s.MU[e] = o.MU;
    if constexpr (DIAG)
    {
#pragma unroll
      for(int k = 0; k < 7; ++k) s.diag[k][e] = o.dg[k];
    }
  }
}

template<typename T, bool DEV, int MODEL, bool DIAG>
__global__ void __launch_bounds__(256)
uq_kernel(Dims d, Params P, State<T> s)
{
  const int y = blockIdx.x*blockDim.x + threadIdx.x;
  const int x = blockIdx.y*blockDim.y + threadIdx.y;
  if(x >= d.LX || y >= d.LY) return;
  const Nbr<T> nb = neighbours<T>(d, x + d.g, y + d.g);
  UQOut<T> o;
  uq_site<T, DEV, MODEL, DIAG>(P, s, nb, d.NE, o);
  store_uq<T, MODEL, DIAG>(s, nb.e, o);
}

// PUSH (periodic lattices without a ghost ring, predictor only): the new ff
// and fn of direction v go straight to the site they stream to, in the
// ff_tmp/fn_tmp planes, which is Move (:371-386) fused into UpdateFields;
// the same values land where move_kernel would put them.
// UpdateQuantities fields, in the order of UQOut
enum { Q_N = 0, Q_UX, Q_UY, Q_UXP, Q_UYP, Q_HXX, Q_HYX, Q_MU, Q_DXQXX, Q_DYQXX, Q_DXQYX,
       Q_DYQYX, Q_SXX, Q_SYY, Q_SXY, Q_SYX, NUQ };
// state scalars UpdateFields reads around a site (phi, and m and chi for
// go-or-grow), after the UpdateQuantities values in the tile
enum { S_PHI = NUQ, S_CHI, S_M, NTILE };

// The UpdateQuantities values of a site (w = 0) and its neighbours +x, -x,
// +y, -y (w = 1..4), with the stencils of src/lb.hpp in their operand order.
template<typename T, class Derived>
struct UQStencil
{
  __device__ __forceinline__ T dx(int f) const
  { const Derived& a = static_cast<const Derived&>(*this); return T(.5)*(a.at(f, 1)-a.at(f, 2)) + T(0); }
  __device__ __forceinline__ T dy(int f) const
  { const Derived& a = static_cast<const Derived&>(*this); return T(.5)*(a.at(f, 3)-a.at(f, 4)) + T(0); }
  __device__ __forceinline__ T lap(int f) const
  {
    const Derived& a = static_cast<const Derived&>(*this);
    return a.at(f, 1)+a.at(f, 2)+a.at(f, 3)+a.at(f, 4) - T(4)*a.at(f, 0) + T(0);
  }
};

// ... read from the global planes of the state
template<typename T>
struct GlobalUQ : UQStencil<T, GlobalUQ<T>>
{
  const T* p[NTILE];
  long long k[5];
  __device__ __forceinline__ GlobalUQ(const State<T>& s, const Nbr<T>& nb)
  {
    p[S_PHI] = s.phi; p[S_CHI] = s.chi; p[S_M] = s.m;
    p[Q_N] = s.n; p[Q_UX] = s.ux; p[Q_UY] = s.uy; p[Q_UXP] = s.uxp; p[Q_UYP] = s.uyp;
    p[Q_HXX] = s.Hxx; p[Q_HYX] = s.Hyx; p[Q_MU] = s.MU; p[Q_DXQXX] = s.dxQxx;
    p[Q_DYQXX] = s.dyQxx; p[Q_DXQYX] = s.dxQyx; p[Q_DYQYX] = s.dyQyx; p[Q_SXX] = s.sXX;
    p[Q_SYY] = s.sYY; p[Q_SXY] = s.sXY; p[Q_SYX] = s.sYX;
    k[0] = nb.e; k[1] = nb.e1; k[2] = nb.e2; k[3] = nb.e3; k[4] = nb.e4;
  }
  __device__ __forceinline__ T at(int f, int w) const { return __ldg(p[f] + k[w]); }
};

// UpdateFields of one site. `U` gives the UpdateQuantities values at the
// site and its four neighbours (global planes, or a shared-memory tile).
// SEP: the new Q goes to Qxx_tmp/Qyx_tmp and the corrector's populations to
// ff_tmp (the sub-step kernel, whose blocks read Q and ff around their tile
// while other blocks update theirs); otherwise both are updated in place.
template<typename T, bool DEV, int MODEL, bool FIRST, bool PUSH, class UQA, bool SEP = false>
__device__ __forceinline__ void uf_site(const Dims& d, const Params& P, const State<T>& s,
                                        const Nbr<T>& nb, const int x, const int y, const UQA& U)
{
  const long long e = nb.e, NE = d.NE;
  T* const QXo = SEP ? s.Qxx_tmp : s.Qxx;
  T* const QYo = SEP ? s.Qyx_tmp : s.Qyx;
  // where direction v streams to (PUSH)
  auto dest = [&](int v) {
    const int X = wrapi(x + d.g + CXv(v), d.EX), Y = wrapi(y + d.g + CYv(v), d.EY);
    return Y + static_cast<long long>(d.EY)*X;
  };

  const T nstore = U.at(Q_N, 0);
  const T nn = DEV ? T(P.rho) + nstore : nstore;
  const T dn = nstore;
  const T vx = U.at(Q_UX, 0);
  const T vy = U.at(Q_UY, 0);
  const T Qxx = s.Qxx[e];
  const T Qyx = s.Qyx[e];
  const T Hxx = U.at(Q_HXX, 0);
  const T Hyx = U.at(Q_HYX, 0);
  const T dxQxx = U.at(Q_DXQXX, 0);
  const T dyQxx = U.at(Q_DYQXX, 0);
  const T dxQyx = U.at(Q_DXQYX, 0);
  const T dyQyx = U.at(Q_DYQYX, 0);

  const T dxux = U.dx(Q_UX);
  const T dyux = U.dy(Q_UX);
  const T dxuy = U.dx(Q_UY);
  const T dyuy = U.dy(Q_UY);
  const T dxSxx = U.dx(Q_SXX);
  const T dySxy = U.dy(Q_SXY);
  const T dxSyx = U.dx(Q_SYX);
  const T dySyy = U.dy(Q_SYY);

  const T GammaQ = T(P.GammaQ), xi = T(P.xi), friction = T(P.friction);

  const T expansion = dxux + dyuy;
  const T shear     = T(.5)*(dxuy + dyux);
  const T vorticity = T(.5)*(dxuy - dyux);
  const T traceQL   = Qxx*(dxux - dyuy) + T(2)*Qyx*shear;

  const T Dxx = GammaQ*Hxx - vx*dxQxx - vy*dyQxx - T(2)*vorticity*Qyx
    + xi*((Qxx+T(1))*(T(2)*dxux-traceQL) +T(2)*Qyx*shear -expansion);
  const T Dyx = GammaQ*Hyx - vx*dxQyx - vy*dyQyx + T(2)*vorticity*Qxx
    + xi*( Qyx*(expansion-traceQL) + T(2)*shear);

  const T Fx = dxSxx + dySxy - friction*vx;
  const T Fy = dxSyx + dySyy - friction*vy;

  T fe[9];
  equilibrium<T, DEV>(vx, vy, nn, dn, fe);

  T* __restrict__ FF = s.ff;
  T* __restrict__ FN = s.fn;

  if constexpr (MODEL != NEM)
  {
    const T p = U.at(S_PHI, 0);
    // go-or-grow phenotype update (src/models/go-or-grow.cpp:331-362): the
    // growth R = chi*phi*(alpha*division_mask - beta*death_mask) and the
    // rate of change Dm of m = phi*chi
    T R = T(0), Dm = T(0);
    if constexpr (MODEL == GOG)
    {
      const T rate = s.src ? s.src[e] : T(0);
      const T chi_eff = U.at(S_CHI, 0);
      R = chi_eff*p*rate;
      const T mFlux = T(.5)*(U.at(Q_UX, 1)*U.at(S_M, 1) - U.at(Q_UX, 2)*U.at(S_M, 2))
                    + T(.5)*(U.at(Q_UY, 3)*U.at(S_M, 3) - U.at(Q_UY, 4)*U.at(S_M, 4));
      const T chi_px = U.at(S_CHI, 1), chi_mx = U.at(S_CHI, 2);
      const T chi_py = U.at(S_CHI, 3), chi_my = U.at(S_CHI, 4);
      const T MUe = U.at(Q_MU, 0);
      const T diffusiveMFlux =
        T(.5)*(chi_px + chi_eff)*(U.at(Q_MU, 1) - MUe)
      - T(.5)*(chi_eff + chi_mx)*(MUe - U.at(Q_MU, 2))
      + T(.5)*(chi_py + chi_eff)*(U.at(Q_MU, 3) - MUe)
      - T(.5)*(chi_eff + chi_my)*(MUe - U.at(Q_MU, 4));
      const T phenotypeDiffusion =
        T(.5)*(U.at(S_PHI, 1) + p)*(chi_px - chi_eff)
      - T(.5)*(p + U.at(S_PHI, 2))*(chi_eff - chi_mx)
      + T(.5)*(U.at(S_PHI, 3) + p)*(chi_py - chi_eff)
      - T(.5)*(p + U.at(S_PHI, 4))*(chi_eff - chi_my);
      const T Achi = T(s.ph.Achi);
      const T dVdChi = T(2)*Achi*chi_eff*(T(1)-chi_eff)*(T(1)-T(2)*chi_eff)
                     + T(s.ph.Ochi)*(p-T(s.ph.phiswitch));
      const T Sswitch = -p*dVdChi;
      const T mGrowth = s.ph.growTogether ? chi_eff*R : R;
      Dm = T(P.GammaP)*diffusiveMFlux + T(s.ph.Dchi)*phenotypeDiffusion - mFlux + Sswitch + mGrowth;
    }
    // m after the sub-step, clamped to [0, max(phi, 0)], and chi = m/phi
    // (src/models/go-or-grow.cpp:364-384, :208-216)
    auto phenotype_out = [&](T pt, T mt) {
      const T upper = pt > T(0) ? pt : T(0);
      if(mt < T(0)) mt = T(0);
      else if(mt > upper) mt = upper;
      s.m_tmp[e] = mt;
      s.chi_tmp[e] = pt > T(1e-12) ? mt/pt : T(0);
    };
    const T del2mu = U.lap(Q_MU);
    const T pFlux = U.dx(Q_UXP) + U.dy(Q_UYP);
    // conserve_phi is false for Lyotropic (src/models/lyotropic.hpp:46) and
    // set by the division models when division and death are off
    // (src/models/lyotropic-with-division.cpp:30)
    const T corr = s.conserve_phi ? T((*s.phisum - s.totalphi)/static_cast<double>(d.LX*d.LY))
                                  : T(0);
    const T Dp = T(P.GammaP)*del2mu - pFlux - corr;
    const T tau = T(P.tauNem)*p + T(P.tauIso)*(T(1)-p);
    // FP32 multiplies by 1/tau; FP64 divides as the reference does
    const T itau = DEV ? T(1)/tau : T(0);
    auto over_tau = [&](T a) { return DEV ? a*itau : a/tau; };
    if constexpr (FIRST)
    {
      s.QNxx[e] = s.Qxx[e] + T(.5)*Dxx;
      s.QNyx[e] = s.Qyx[e] + T(.5)*Dyx;
      s.phn[e]  = p + T(.5)*Dp;
      QXo[e]  = s.Qxx[e] + Dxx;
      QYo[e]  = s.Qyx[e] + Dyx;
      T pt = p + Dp;
      if constexpr (MODEL == GOG)
      {
        pt = pt + R;
        const T me = U.at(S_M, 0);
        s.mN[e] = me + T(.5)*Dm;
        phenotype_out(pt, me + Dm);
      }
      // division source, added after the node update as the division model
      // does (src/models/lyotropic-with-division.cpp:121)
      else if(s.src) pt = pt + p*s.src[e];
      s.phi_tmp[e] = pt;
#pragma unroll
      for(int v=0; v<9; ++v)
      {
        const T f = FF[v*NE+e];
        const T force = T(Wv(v))*(Fx*T(CXv(v)) + Fy*T(CYv(v)));
        const long long o = PUSH ? dest(v) : e;
        T* fn_out = PUSH ? s.fn_tmp : FN;
        T* ff_out = PUSH ? s.ff_tmp : FF;
        fn_out[v*NE+o] = f + T(.5)*(over_tau(fe[v]-f) + force);
        ff_out[v*NE+o] = f +      (over_tau(fe[v]-f) + force);
      }
    }
    else
    {
      QXo[e] = s.QNxx[e] + T(.5)*Dxx;
      QYo[e] = s.QNyx[e] + T(.5)*Dyx;
      T pt = s.phn[e] + T(.5)*Dp;
      if constexpr (MODEL == GOG)
      {
        pt = pt + R;
        phenotype_out(pt, s.mN[e] + T(.5)*Dm);
      }
      else if(s.src) pt = pt + p*s.src[e];
      s.phi_tmp[e] = pt;
#pragma unroll
      for(int v=0; v<9; ++v)
      {
        const T f = FF[v*NE+e];
        const T force = T(Wv(v))*(Fx*T(CXv(v)) + Fy*T(CYv(v)));
        (SEP ? s.ff_tmp : FF)[v*NE+e] = FN[v*NE+e] + T(.5)*(over_tau(fe[v]-f) + force);
      }
    }
  }
  else
  {
    const T tau = T(P.tauNem);
    // FP32 multiplies by 1/tau; FP64 divides as the reference does
    const T itau = DEV ? T(1)/tau : T(0);
    auto over_tau = [&](T a) { return DEV ? a*itau : a/tau; };
    if constexpr (FIRST)
    {
      const T qn_xx = s.Qxx[e] + T(.5)*Dxx + T(0);
      const T qn_yx = s.Qyx[e] + T(.5)*Dyx + T(0);
      s.QNxx[e] = qn_xx;
      s.QNyx[e] = qn_yx;
      QXo[e] = qn_xx + T(.5)*Dxx;
      QYo[e] = qn_yx + T(.5)*Dyx;
#pragma unroll
      for(int v=0; v<9; ++v)
      {
        const T f = FF[v*NE+e];
        const T force = T(Wv(v))*(Fx*T(CXv(v)) + Fy*T(CYv(v)));
        const T fnv = f + T(.5)*(over_tau(fe[v]-f) + force) + T(0);
        const long long o = PUSH ? dest(v) : e;
        T* fn_out = PUSH ? s.fn_tmp : FN;
        T* ff_out = PUSH ? s.ff_tmp : FF;
        fn_out[v*NE+o] = fnv;
        ff_out[v*NE+o] = fnv + T(.5)*(over_tau(fe[v]-f) + force);
      }
    }
    else
    {
      QXo[e] = s.QNxx[e] + T(.5)*Dxx;
      QYo[e] = s.QNyx[e] + T(.5)*Dyx;
#pragma unroll
      for(int v=0; v<9; ++v)
      {
        const T f = FF[v*NE+e];
        const T force = T(Wv(v))*(Fx*T(CXv(v)) + Fy*T(CYv(v)));
        (SEP ? s.ff_tmp : FF)[v*NE+e] = FN[v*NE+e] + T(.5)*(over_tau(fe[v]-f) + force);
      }
    }
  }
}

template<typename T, bool DEV, int MODEL, bool FIRST, bool PUSH = false>
__global__ void __launch_bounds__(256)
uf_kernel(Dims d, Params P, State<T> s)
{
  const int y = blockIdx.x*blockDim.x + threadIdx.x;
  const int x = blockIdx.y*blockDim.y + threadIdx.y;
  if(x >= d.LX || y >= d.LY) return;
  const Nbr<T> nb = neighbours<T>(d, x + d.g, y + d.g);
  const GlobalUQ<T> U(s, nb);
  uf_site<T, DEV, MODEL, FIRST, PUSH>(d, P, s, nb, x, y, U);
}

// One predictor or corrector sub-step on a periodic lattice in one launch:
// UpdateQuantities over the block's tile plus a one-site ring into shared
// memory, then UpdateFields over the tile reading its stencils from there.
// The ring sites are computed by both neighbouring blocks with the same
// expressions, so the values equal the two-sweep form's. Nothing derived is
// written to HBM unless storeq is set, which leaves the planes the two
// sweeps leave (the library replays them on demand instead). Blocks read Q, phi, chi and
// ff around their tile, so the new Q and (corrector) ff are written beside
// them (SEP) and the host swaps the planes after the launch.
// One thread per site of the tile and its ring (32 x 10 threads, a warp per
// x row): every thread computes one UpdateQuantities, the 30 x 8 inner ones
// then one UpdateFields.
constexpr int SUB_TY = 30, SUB_TX = 8;                 // tile: y (contiguous) x x
constexpr int SUB_HY = SUB_TY + 2, SUB_HX = SUB_TX + 2;
constexpr int SUB_HS = SUB_HY*SUB_HX;

__device__ __forceinline__ void prefetch_l2(const void* p)
{
  asm volatile("prefetch.global.L2 [%0];" :: "l"(p));
}

template<typename T>
struct TileUQ : UQStencil<T, TileUQ<T>>
{
  const T (*a)[SUB_HS];
  int c;
  __device__ __forceinline__ T at(int f, int w) const
  {
    const int off = w == 0 ? 0 : w == 1 ? SUB_HY : w == 2 ? -SUB_HY : w == 3 ? 1 : -1;
    return a[f][c + off];
  }
};

template<typename T, bool DEV, int MODEL, bool FIRST, bool DIAG>
__global__ void __launch_bounds__(SUB_HY*SUB_HX)
substep_kernel(Dims d, Params P, State<T> s, int storeq, int prefetch)
{
  extern __shared__ __align__(16) unsigned char sub_smem[];
  T (*uq_s)[SUB_HS] = reinterpret_cast<T (*)[SUB_HS]>(sub_smem);
  const int y0 = blockIdx.x*SUB_TY, x0 = blockIdx.y*SUB_TX;
  const int i = threadIdx.y*SUB_HY + threadIdx.x;          // this thread's tile site
  const int X = x0 - 1 + static_cast<int>(threadIdx.y), Y = y0 - 1 + static_cast<int>(threadIdx.x);
  const bool inner = threadIdx.x >= 1 && threadIdx.x <= SUB_TY && threadIdx.y >= 1 &&
                     threadIdx.y <= SUB_TX && X < d.LX && Y < d.LY;
  if constexpr (!FIRST)
  {
    // the corrector's own-site inputs (fn, QN, phi_N, m_N) start towards L2
    // while the tile's UpdateQuantities runs (states larger than L2)
    if(prefetch && inner)
    {
      const long long e = Y + static_cast<long long>(d.EY)*X;
#pragma unroll
      for(int v = 0; v < 9; ++v) prefetch_l2(s.fn + v*d.NE + e);
      prefetch_l2(s.QNxx + e);
      prefetch_l2(s.QNyx + e);
      if constexpr (MODEL != NEM) prefetch_l2(s.phn + e);
      if constexpr (MODEL == GOG) prefetch_l2(s.mN + e);
    }
  }
  // the ring one past the lattice's end is the periodic image of site 0
  if(X <= d.LX && Y <= d.LY)
  {
    const Nbr<T> nb = neighbours<T>(d, wrapi(X, d.LX), wrapi(Y, d.LY));
    UQOut<T> o;
    uq_site<T, DEV, MODEL, DIAG>(P, s, nb, d.NE, o);
    uq_s[Q_N][i] = o.n; uq_s[Q_UX][i] = o.ux; uq_s[Q_UY][i] = o.uy;
    uq_s[Q_HXX][i] = o.Hxx; uq_s[Q_HYX][i] = o.Hyx;
    uq_s[Q_DXQXX][i] = o.dxQxx; uq_s[Q_DYQXX][i] = o.dyQxx;
    uq_s[Q_DXQYX][i] = o.dxQyx; uq_s[Q_DYQYX][i] = o.dyQyx;
    uq_s[Q_SXX][i] = o.sXX; uq_s[Q_SYY][i] = o.sYY; uq_s[Q_SXY][i] = o.sXY; uq_s[Q_SYX][i] = o.sYX;
    if constexpr (MODEL != NEM)
    {
      uq_s[Q_UXP][i] = o.uxp; uq_s[Q_UYP][i] = o.uyp; uq_s[Q_MU][i] = o.MU;
      uq_s[S_PHI][i] = s.phi[nb.e];
    }
    if constexpr (MODEL == GOG)
    {
      uq_s[S_CHI][i] = s.chi[nb.e];
      uq_s[S_M][i] = s.m[nb.e];
    }
    if(storeq && inner) store_uq<T, MODEL, DIAG>(s, nb.e, o);
  }
  __syncthreads();
  if(!inner) return;
  const Nbr<T> nb = neighbours<T>(d, X, Y);
  TileUQ<T> U;
  U.a = uq_s;
  U.c = i;
  uf_site<T, DEV, MODEL, FIRST, FIRST, TileUQ<T>, true>(d, P, s, nb, X, Y, U);
}

// Launch a sub-step; its tile needs NTILE*SUB_HS values of shared memory,
// above the 48 KB default for larger tiles in FP64.
template<typename T, bool DEV, int MODEL, bool FIRST, bool DIAG>
void launch_substep(const Dims& d, const Params& P, const State<T>& s, int storeq,
                    cudaStream_t st)
{
  constexpr size_t bytes = sizeof(T)*NTILE*SUB_HS;
  if constexpr (bytes > 48*1024)
  {
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if(!(done.load() & bit))
    {
      cudaFuncSetAttribute(substep_kernel<T, DEV, MODEL, FIRST, DIAG>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
      done.fetch_or(bit);
    }
  }
  const dim3 blk(SUB_HY, SUB_HX);
  const dim3 grd((d.LY + SUB_TY - 1)/SUB_TY, (d.LX + SUB_TX - 1)/SUB_TX);
  // about 60 planes of state and sweep fields; L2 holds 126 MB
  const int prefetch = static_cast<double>(d.NE)*sizeof(T)*60 > 96e6 ? 1 : 0;
  substep_kernel<T, DEV, MODEL, FIRST, DIAG><<<grd, blk, bytes, st>>>(d, P, s, storeq, prefetch);
}

// Streaming as a pull over every extended site.
template<typename T>
__global__ void __launch_bounds__(256)
move_kernel(Dims d, const T* __restrict__ ff, const T* __restrict__ fn,
            T* __restrict__ ff_out, T* __restrict__ fn_out)
{
  const int Y = blockIdx.x*blockDim.x + threadIdx.x;
  const int X = blockIdx.y*blockDim.y + threadIdx.y;
  if(X >= d.EX || Y >= d.EY) return;
  const long long e = Y + (long long)d.EY*X, NE = d.NE;
#pragma unroll
  for(int v=0; v<9; ++v)
  {
    const int Xs = wrapi(X - CXv(v), d.EX), Ys = wrapi(Y - CYv(v), d.EY);
    const long long src = Ys + (long long)d.EY*Xs;
    ff_out[v*NE+e] = ff[v*NE+src];
    fn_out[v*NE+e] = fn[v*NE+src];
  }
}

// ---------------------------------------------------------------------------
// Wall boundary conditions on the ghost ring (g = 1), src/fields.hpp:620-930.
// Wall and corner ids are their direction numbers (src/geometry.hpp:146-193).

enum { W_RIGHT = 1, W_LEFT = 2, W_BACK = 3, W_FRONT = 4 };
enum { C_RIGHTBACK = 5, C_LEFTFRONT = 6, C_LEFTBACK = 7, C_RIGHTFRONT = 8 };

__constant__ int c_refl[9][9] = {
  {0, 2, 1, 4, 3, 6, 5, 8, 7},
  {0, 2, 1, 3, 4, 7, 8, 5, 6},
  {0, 2, 1, 3, 4, 7, 8, 5, 6},
  {0, 1, 2, 4, 3, 8, 7, 6, 5},
  {0, 1, 2, 4, 3, 8, 7, 6, 5},
  {0, 4, 3, 2, 1, 6, 5, 7, 8},
  {0, 4, 3, 2, 1, 6, 5, 7, 8},
  {0, 3, 4, 1, 2, 5, 6, 8, 7},
  {0, 3, 4, 1, 2, 5, 6, 8, 7}};
__constant__ int c_proj[9][9] = {
  {0, 0, 0, 0, 0, 0, 0, 0, 0},
  {0, 0, 0, 3, 4, 3, 4, 3, 4},
  {0, 0, 0, 3, 4, 3, 4, 3, 4},
  {0, 1, 2, 0, 0, 1, 2, 2, 1},
  {0, 1, 2, 0, 0, 1, 2, 2, 1},
  {0, 5, 6, 5, 6, 5, 6, 0, 0},
  {0, 1, 2, 4, 3, 8, 7, 6, 5},
  {0, 8, 7, 7, 8, 0, 0, 7, 8},
  {0, 8, 7, 7, 8, 0, 0, 7, 8}};

struct XY { int X, Y; };

__device__ __forceinline__ XY wall_xy(const Dims& d, int w, int k)
{
  switch(w)
  {
    case W_LEFT:  return {0, k + 1};
    case W_RIGHT: return {d.EX - 1, k + 1};
    case W_FRONT: return {k + 1, 0};
    default:      return {k + 1, d.EY - 1};
  }
}
__device__ __forceinline__ XY corner_xy(const Dims& d, int c)
{
  switch(c)
  {
    case C_LEFTFRONT:  return {0, 0};
    case C_RIGHTFRONT: return {d.EX - 1, 0};
    case C_LEFTBACK:   return {0, d.EY - 1};
    default:           return {d.EX - 1, d.EY - 1};
  }
}
__device__ __forceinline__ XY step_xy(const Dims& d, XY a, int v)
{
  return {wrapi(a.X + CXv(v), d.EX), wrapi(a.Y + CYv(v), d.EY)};
}
__device__ __forceinline__ long long at(const Dims& d, XY a)
{
  return a.Y + (long long)d.EY*a.X;
}
__device__ __forceinline__ bool incoming(int v, int w)
{
  return CXv(w)*CXv(v) == -1 || CYv(w)*CYv(v) == -1;
}

// one scalar ghost value from inward direction `in`
template<typename T>
__device__ __forceinline__ void s_apply(const Dims& d, T* a, XY i, int in, int kind)
{
  const XY j = step_xy(d, i, in);
  if(kind == BC_NEUMANN) a[at(d, i)] = a[at(d, j)];
  else if(kind == BC_DIRICHLET0) a[at(d, i)] = T(2)*T(0) - a[at(d, j)];
  else a[at(d, i)] = T(2)*a[at(d, j)] - a[at(d, step_xy(d, j, in))];
}

// Scalar fields, in two launches: the walls (they read domain values only),
// then the corners (channel corners read the left/right ghosts the walls
// wrote). Every ghost value is a copy, a negation or a 2a - b of values the
// launch before has settled, so the grid's layout does not change a bit.
template<typename T>
__global__ void __launch_bounds__(256)
bc_scalar_walls(Dims d, ScalarBC<T> job)
{
  const int LX = d.LX, LY = d.LY;
  const int nwall = 2*LY + 2*LX;
  // one thread per (ghost site, field)
  for(int t = blockIdx.x*blockDim.x + threadIdx.x; t < nwall*job.nf; t += blockDim.x*gridDim.x)
  {
    const int f = t / nwall, idx = t - f*nwall;
    int w, k;
    if(idx < LY) { w = W_LEFT; k = idx; }
    else if(idx < 2*LY) { w = W_RIGHT; k = idx - LY; }
    else if(idx < 2*LY + LX) { w = W_FRONT; k = idx - 2*LY; }
    else { w = W_BACK; k = idx - 2*LY - LX; }
    const XY i = wall_xy(d, w, k);
    const bool pbc = job.mode == BCM_PBC ||
                     (job.mode == BCM_CHANNEL && (w == W_LEFT || w == W_RIGHT));
    T* a = job.f[f];
    if(pbc)
    {
      const XY o = wall_xy(d, OPPv(w), k);
      a[at(d, i)] = a[at(d, step_xy(d, o, w))];
    }
    else s_apply(d, a, i, OPPv(w), job.kind[f]);
  }
}

template<typename T>
__global__ void __launch_bounds__(64)
bc_scalar_corners(Dims d, ScalarBC<T> job)
{
  // one thread per (corner, field); the order of the reference's corner
  // calls does not matter: each corner reads a wall ghost or a domain site,
  // never another corner
  const int t = threadIdx.x;
  if(t >= 4*job.nf) return;
  const int cs[4] = {C_RIGHTBACK, C_RIGHTFRONT, C_LEFTBACK, C_LEFTFRONT};
  const int c = cs[t & 3], f = t >> 2;
  const XY i = corner_xy(d, c);
  T* a = job.f[f];
  if(job.mode == BCM_PBC)
    a[at(d, i)] = a[at(d, step_xy(d, corner_xy(d, OPPv(c)), c))];
  else if(job.mode == BCM_CHANNEL)
  {
    const int w = (c == C_RIGHTBACK || c == C_LEFTBACK) ? W_BACK : W_FRONT;
    s_apply(d, a, i, OPPv(w), job.kind[f]);
  }
  else s_apply(d, a, i, OPPv(c), job.kind[f]);
}

template<typename T>
void launch_bc_scalar(const Dims& d, const ScalarBC<T>& j, cudaStream_t st)
{
  const int n = (2*d.LY + 2*d.LX)*j.nf;
  bc_scalar_walls<T><<<(n + 255)/256, 256, 0, st>>>(d, j);
  bc_scalar_corners<T><<<1, 64, 0, st>>>(d, j);
}

template<typename T>
__device__ __forceinline__ void f_pbc_node(const Dims& d, T* f, XY dst, XY src)
{
  const long long a = at(d, dst), b = at(d, src);
#pragma unroll
  for(int v=0; v<9; ++v) f[v*d.NE + a] = f[v*d.NE + b];
}

template<typename T>
__device__ __forceinline__ void f_wall(const Dims& d, T* f, int w, int k, bool noslip)
{
  const XY i = wall_xy(d, w, k);
  const long long ki = at(d, i);
#pragma unroll
  for(int v=0; v<9; ++v)
    if(incoming(v, w))
    {
      if(noslip) f[v*d.NE + ki] = f[OPPv(v)*d.NE + at(d, step_xy(d, i, v))];
      else f[v*d.NE + ki] = f[c_refl[w][v]*d.NE + at(d, step_xy(d, i, OPPv(w)))];
    }
}

// Population fields ff and fn, in up to three launches: (1) left/right
// walls, and every wall whose update reads domain values only (a no-slip
// box's left/right walls read the front/back ghosts as the last Move left
// them, the reference's order); (2) front/back no-slip walls, whose
// diagonal bounce reads the left/right ghosts (1) wrote; (3) the corners.
template<typename T>
__global__ void __launch_bounds__(256)
bc_lb_walls(Dims d, T* ff, T* fn, int kind)
{
  const int LX = d.LX, LY = d.LY;
  const int nwall = 2*LY + 2*LX;
  // one thread per (ghost site, population array)
  for(int t = blockIdx.x*blockDim.x + threadIdx.x; t < 2*nwall; t += blockDim.x*gridDim.x)
  {
    const int a = t / nwall, idx = t - a*nwall;
    T* f = a ? fn : ff;
    int w, k;
    if(idx < LY) { w = W_LEFT; k = idx; }
    else if(idx < 2*LY) { w = W_RIGHT; k = idx - LY; }
    else if(idx < 2*LY + LX) { w = W_FRONT; k = idx - 2*LY; }
    else { w = W_BACK; k = idx - 2*LY - LX; }
    const bool lr = (w == W_LEFT || w == W_RIGHT);
    if(kind == LBK_PBC || ((kind == LBK_FREESLIP_CHANNEL || kind == LBK_NOSLIP_CHANNEL) && lr))
      f_pbc_node(d, f, wall_xy(d, w, k), step_xy(d, wall_xy(d, OPPv(w), k), w));
    else if(kind == LBK_FREESLIP_CHANNEL || kind == LBK_FREESLIP_BOX)
      f_wall(d, f, w, k, false);
    else if(kind == LBK_NOSLIP_BOX && lr)
      f_wall(d, f, w, k, true);
  }
}

template<typename T>
__global__ void __launch_bounds__(256)
bc_lb_noslip_fb(Dims d, T* ff, T* fn)
{
  const int LX = d.LX;
  for(int t = blockIdx.x*blockDim.x + threadIdx.x; t < 4*LX; t += blockDim.x*gridDim.x)
  {
    const int a = t / (2*LX), idx = t - a*2*LX;
    const int w = idx < LX ? W_FRONT : W_BACK;
    const int k = idx < LX ? idx : idx - LX;
    f_wall(d, a ? fn : ff, w, k, true);
  }
}

template<typename T>
__global__ void __launch_bounds__(32)
bc_lb_corners(Dims d, T* ff, T* fn, int kind)
{
  // one thread per (corner, population array)
  const int t = threadIdx.x;
  if(t >= 8) return;
  T* f = (t >> 2) ? fn : ff;
  const int cs[4] = {C_RIGHTBACK, C_RIGHTFRONT, C_LEFTBACK, C_LEFTFRONT};
  const int c = cs[t & 3];
  const XY i = corner_xy(d, c);
  if(kind == LBK_PBC)
    f_pbc_node(d, f, i, step_xy(d, corner_xy(d, OPPv(c)), c));
  else if(kind == LBK_FREESLIP_CHANNEL)
  {
    const int w = (c == C_RIGHTBACK || c == C_LEFTBACK) ? W_BACK : W_FRONT;
    const int p = c_proj[w][c];
    const int v = OPPv(c);
    const XY l = step_xy(d, corner_xy(d, c_refl[p][c]), p);
    f[v*d.NE + at(d, i)] = f[v*d.NE + at(d, l)];
  }
  else
  {
    const int v = OPPv(c);
    f[v*d.NE + at(d, i)] = f[c*d.NE + at(d, step_xy(d, i, v))];
  }
}

bool lb_noslip(int kind) { return kind == LBK_NOSLIP_CHANNEL || kind == LBK_NOSLIP_BOX; }

template<typename T>
void launch_bc_lb(const Dims& d, T* ff, T* fn, int kind, cudaStream_t st)
{
  const int n = 2*(2*d.LY + 2*d.LX);
  bc_lb_walls<T><<<(n + 255)/256, 256, 0, st>>>(d, ff, fn, kind);
  if(lb_noslip(kind)) bc_lb_noslip_fb<T><<<(4*d.LX + 255)/256, 256, 0, st>>>(d, ff, fn);
  bc_lb_corners<T><<<1, 32, 0, st>>>(d, ff, fn, kind);
}

inline dim3 site_grid(int nx, int ny, dim3 blk)
{
  return dim3((ny + blk.x - 1)/blk.x, (nx + blk.y - 1)/blk.y);
}

// countphi of UpdateQuantities (src/models/lyotropic.cpp:343-360) summed in
// site order k = y + LY*x by one thread, so that the FP64 result is the
// serial reference's bit for bit.
template<typename T>
__global__ void phi_sum_serial(Dims d, const T* __restrict__ phi, double* out)
{
  if(blockIdx.x != 0 || threadIdx.x != 0) return;
  double sum = 0;
  for(int x = 0; x < d.LX; ++x)
  {
    const T* row = phi + static_cast<long long>(d.EY)*(x + d.g) + d.g;
    for(int y = 0; y < d.LY; ++y) sum = sum + static_cast<double>(row[y]);
  }
  *out = sum;
}

// countphi for the FP32 sweeps, which do not reproduce the reference's
// rounding anyway: per-block FP64 partial sums (PHI_PARTS blocks), then one
// block adds the partials. Writes out[0]; out[1 .. PHI_PARTS] is scratch.
template<typename T>
__global__ void __launch_bounds__(256)
phi_sum_partial(Dims d, const T* __restrict__ phi, double* __restrict__ out)
{
  __shared__ double red[256];
  const long long N = static_cast<long long>(d.LX)*d.LY;
  double s = 0;
  for(long long k = static_cast<long long>(blockIdx.x)*256 + threadIdx.x; k < N;
      k += static_cast<long long>(gridDim.x)*256)
  {
    const int x = static_cast<int>(k / d.LY), y = static_cast<int>(k % d.LY);
    s += static_cast<double>(phi[(y + d.g) + static_cast<long long>(d.EY)*(x + d.g)]);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for(int w = 128; w > 0; w >>= 1)
  {
    if(threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if(threadIdx.x == 0) out[1 + blockIdx.x] = red[0];
}

template<typename T>
__global__ void __launch_bounds__(256)
phi_sum_final(int nparts, double* __restrict__ out)
{
  __shared__ double red[256];
  double s = 0;
  for(int i = threadIdx.x; i < nparts; i += 256) s += out[1 + i];
  red[threadIdx.x] = s;
  __syncthreads();
  for(int w = 128; w > 0; w >>= 1)
  {
    if(threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if(threadIdx.x == 0) out[0] = red[0];
}

// countphi before an UpdateFields: the serial site-order sum in FP64 (the
// reference's rounding), a parallel sum in FP32
template<typename T>
void phi_sum(const Dims& d, const T* phi, double* out, cudaStream_t st)
{
  if constexpr (std::is_same<T, float>::value)
  {
    phi_sum_partial<T><<<PHI_PARTS, 256, 0, st>>>(d, phi, out);
    phi_sum_final<T><<<1, 256, 0, st>>>(PHI_PARTS, out);
  }
  else phi_sum_serial<T><<<1, 1, 0, st>>>(d, phi, out);
}

// GoOrGrow::RelaxFreeEnergy (src/models/go-or-grow.cpp:42-119): dry
// free-energy descent of phi (Cahn-Hilliard) and Q (molecular field) before
// the dynamics. First sweep: H and mu at every site.
template<typename T>
__global__ void __launch_bounds__(256)
relax_mu_kernel(Dims d, Params P, State<T> s)
{
  const int y = blockIdx.x*blockDim.x + threadIdx.x;
  const int x = blockIdx.y*blockDim.y + threadIdx.y;
  if(x >= d.LX || y >= d.LY) return;
  const Nbr<T> nb = neighbours<T>(d, x + d.g, y + d.g);
  const long long e = nb.e;
  const T CC = T(P.CC), LL = T(P.LL), AA = T(P.AA), KK = T(P.KK);
  const T B = T(s.ph.B), Snem = T(s.ph.Snem), phic = T(s.ph.phi_critical);
  const T Qxx = s.Qxx[e];
  const T Qyx = s.Qyx[e];
  const T p = s.phi[e];
  const T q2 = Qxx*Qxx + Qyx*Qyx;
  const T term = Snem - q2;
  const T dpc = p - phic;
  const T mu_compress = dpc > T(0) ? B*dpc : T(0);
  s.Hxx[e] = T(2)*CC*term*Qxx + LL*lap(s.Qxx, nb);
  s.Hyx[e] = T(2)*CC*term*Qyx + LL*lap(s.Qyx, nb);
  s.MU[e] = AA*p*(T(1)-p)*(T(1)-T(2)*p) + mu_compress - KK*lap(s.phi, nb);
}

// Second sweep: explicit descent step into phi_tmp and QN (swapped in after).
template<typename T>
__global__ void __launch_bounds__(256)
relax_update_kernel(Dims d, Params P, State<T> s, double dt, int relax_phi, int relax_Q)
{
  const int y = blockIdx.x*blockDim.x + threadIdx.x;
  const int x = blockIdx.y*blockDim.y + threadIdx.y;
  if(x >= d.LX || y >= d.LY) return;
  const Nbr<T> nb = neighbours<T>(d, x + d.g, y + d.g);
  const long long e = nb.e;
  const T rdt = T(dt);
  if(relax_phi) s.phi_tmp[e] = s.phi[e] + rdt*T(P.GammaP)*lap(s.MU, nb);
  else s.phi_tmp[e] = s.phi[e];
  if(relax_Q)
  {
    s.QNxx[e] = s.Qxx[e] + rdt*T(P.GammaQ)*s.Hxx[e];
    s.QNyx[e] = s.Qyx[e] + rdt*T(P.GammaQ)*s.Hyx[e];
  }
  else
  {
    s.QNxx[e] = s.Qxx[e];
    s.QNyx[e] = s.Qyx[e];
  }
}

// chi = m/phi where phi > 1e-12, else 0, at every domain site
// (GoOrGrow::UpdatePhenotypeQuantities, src/models/go-or-grow.cpp:208-216)
template<typename T>
__global__ void __launch_bounds__(256)
chi_kernel(Dims d, State<T> s)
{
  const int y = blockIdx.x*blockDim.x + threadIdx.x;
  const int x = blockIdx.y*blockDim.y + threadIdx.y;
  if(x >= d.LX || y >= d.LY) return;
  const long long e = (y + d.g) + static_cast<long long>(d.EY)*(x + d.g);
  const T p = s.phi[e];
  s.chi[e] = p > T(1e-12) ? s.m[e]/p : T(0);
}

template<typename T>
int relax_impl(const Dims& d, const Params& P, State<T>& s, int bc, unsigned nsteps,
               double dt, int relax_phi, int relax_Q, double* sum_out, cudaStream_t st)
{
  const dim3 blk(64, 4);
  const dim3 grd = site_grid(d.LX, d.LY, blk);
  const int bcm = bc_mode(GOG, bc);
  // Lyotropic::BoundaryConditionsFields (Q, phi) and the mu walls of :70-83
  auto scalar_bc = [&](T* a, T* b, T* c) {
    if(!bc) return;
    ScalarBC<T> j{};
    j.mode = bcm;
    j.f[0] = a; j.f[1] = b; j.f[2] = c;
    j.nf = c ? 3 : 1;
    for(int i = 0; i < j.nf; ++i) j.kind[i] = BC_NEUMANN;
    launch_bc_scalar<T>(d, j, st);
  };
  if(nsteps > 0 && (relax_phi || relax_Q))
  {
    for(unsigned it = 0; it < nsteps; ++it)
    {
      scalar_bc(s.Qxx, s.Qyx, s.phi);
      relax_mu_kernel<T><<<grd, blk, 0, st>>>(d, P, s);
      scalar_bc(s.MU, nullptr, nullptr);
      relax_update_kernel<T><<<grd, blk, 0, st>>>(d, P, s, dt, relax_phi, relax_Q);
      std::swap(s.phi, s.phi_tmp);
      std::swap(s.Qxx, s.QNxx);
      std::swap(s.Qyx, s.QNyx);
    }
    scalar_bc(s.Qxx, s.Qyx, s.phi);
  }
  // the relaxed total of phi, summed in site order (:114-118)
  phi_sum_serial<T><<<1, 1, 0, st>>>(d, s.phi, sum_out);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template<typename T, bool DEV, int MODEL>
int step_impl(const Dims& d, const Params& P, State<T>& s, int bc,
              unsigned nsteps, bool diag_last, cudaStream_t st)
{
  const dim3 blk(64, 4);
  const dim3 grd = site_grid(d.LX, d.LY, blk);
  const dim3 egrd = site_grid(d.EX, d.EY, blk);
  const int lbk = lb_kind(MODEL, bc);
  const int bcm_fields = bc_mode(MODEL, bc);

  auto fields_bc = [&]() {
    if(!bc) return;
    ScalarBC<T> j{};
    j.mode = bcm_fields;
    j.f[0] = s.Qxx; j.f[1] = s.Qyx; j.nf = 2;
    if(MODEL != NEM) { j.f[2] = s.phi; j.nf = 3; }
    // go-or-grow walls treat m and chi as phi (src/models/go-or-grow.cpp:393-418)
    if(MODEL == GOG) { j.f[3] = s.m; j.f[4] = s.chi; j.nf = 5; }
    for(int i = 0; i < j.nf; ++i) j.kind[i] = BC_NEUMANN;
    launch_bc_scalar<T>(d, j, st);
  };
  auto fields2_bc = [&]() {
    if(!bc) return;
    ScalarBC<T> j{};
    j.mode = bcm_fields;
    if(MODEL != NEM)
    {
      T* fs[9] = {s.uy, s.ux, s.uyp, s.uxp, s.MU, s.sXX, s.sYY, s.sYX, s.sXY};
      const int ks[9] = {BC_COPYDERIV, BC_COPYDERIV, BC_DIRICHLET0, BC_DIRICHLET0,
                         BC_NEUMANN, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN, BC_NEUMANN};
      for(int i = 0; i < 9; ++i) { j.f[i] = fs[i]; j.kind[i] = ks[i]; }
      j.nf = 9;
    }
    else
    {
      // nematic walls use Neumann for u as well (src/models/nematic.cpp:338-357)
      T* fs[6] = {s.ux, s.uy, s.sXX, s.sYY, s.sYX, s.sXY};
      for(int i = 0; i < 6; ++i) { j.f[i] = fs[i]; j.kind[i] = BC_NEUMANN; }
      j.nf = 6;
    }
    launch_bc_scalar<T>(d, j, st);
  };

  // after UpdateFields: the new phi (and, for go-or-grow, m and chi =
  // m/phi, UpdatePhenotypeQuantities of src/models/go-or-grow.cpp:208-216)
  auto swap_fields = [&]() {
    if(MODEL != NEM) std::swap(s.phi, s.phi_tmp);
    if(MODEL == GOG) { std::swap(s.m, s.m_tmp); std::swap(s.chi, s.chi_tmp); }
  };

  if(substep_path(d, P, bc))
  {
    // periodic: one launch per sub-step
    auto swap_sub = [&]() {
      swap_fields();
      std::swap(s.Qxx, s.Qxx_tmp);
      std::swap(s.Qyx, s.Qyx_tmp);
      std::swap(s.ff, s.ff_tmp);
    };
    for(unsigned it = 0; it < nsteps; ++it)
    {
      if(MODEL != NEM && s.conserve_phi) phi_sum<T>(d, s.phi, s.phisum, st);
      launch_substep<T, DEV, MODEL, true, false>(d, P, s, 0, st);
      swap_sub();
      std::swap(s.fn, s.fn_tmp);
      for(unsigned c = 1; c <= P.npc; ++c)
      {
        // diag_last: the last sub-step also stores what its UpdateQuantities
        // computed (else replay_derived recomputes it when it is asked for)
        const bool last = diag_last && it + 1 == nsteps && c == P.npc;
        if(MODEL != NEM && s.conserve_phi) phi_sum<T>(d, s.phi, s.phisum, st);
        if(last) launch_substep<T, DEV, MODEL, false, true>(d, P, s, 1, st);
        else launch_substep<T, DEV, MODEL, false, false>(d, P, s, 0, st);
        swap_sub();
      }
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }

  for(unsigned it = 0; it < nsteps; ++it)
  {
    fields_bc();
    uq_kernel<T, DEV, MODEL, false><<<grd, blk, 0, st>>>(d, P, s);
    fields2_bc();
    if(MODEL != NEM && s.conserve_phi) phi_sum<T>(d, s.phi, s.phisum, st);
    if(bc)
    {
      uf_kernel<T, DEV, MODEL, true><<<grd, blk, 0, st>>>(d, P, s);
      swap_fields();
      launch_bc_lb<T>(d, s.ff, s.fn, lbk, st);
      move_kernel<T><<<egrd, blk, 0, st>>>(d, s.ff, s.fn, s.ff_tmp, s.fn_tmp);
    }
    else
    {
      // no walls: Move happens inside UpdateFields
      uf_kernel<T, DEV, MODEL, true, true><<<grd, blk, 0, st>>>(d, P, s);
      swap_fields();
    }
    std::swap(s.ff, s.ff_tmp);
    std::swap(s.fn, s.fn_tmp);
    for(unsigned c = 1; c <= P.npc; ++c)
    {
      const bool diag = diag_last && it + 1 == nsteps && c == P.npc;
      fields_bc();
      if(diag) uq_kernel<T, DEV, MODEL, true><<<grd, blk, 0, st>>>(d, P, s);
      else uq_kernel<T, DEV, MODEL, false><<<grd, blk, 0, st>>>(d, P, s);
      fields2_bc();
      if(MODEL != NEM && s.conserve_phi) phi_sum<T>(d, s.phi, s.phisum, st);
      uf_kernel<T, DEV, MODEL, false><<<grd, blk, 0, st>>>(d, P, s);
      swap_fields();
    }
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// The derived fields of the last sub-step-kernel step: its last
// UpdateQuantities again, on the state that sub-step read, which the step
// leaves in the spare planes (ff_tmp, Qxx_tmp, Qyx_tmp, phi_tmp, chi_tmp).
template<typename T, bool DEV>
int replay_impl(const Dims& d, const Params& P, const State<T>& s, cudaStream_t st)
{
  State<T> r = s;
  r.ff = s.ff_tmp;
  r.Qxx = s.Qxx_tmp;
  r.Qyx = s.Qyx_tmp;
  r.phi = s.phi_tmp;
  r.chi = s.chi_tmp;
  const dim3 blk(64, 4);
  const dim3 grd = site_grid(d.LX, d.LY, blk);
  switch(P.model)
  {
    case LYO: uq_kernel<T, DEV, LYO, true><<<grd, blk, 0, st>>>(d, P, r); break;
    case GOG: uq_kernel<T, DEV, GOG, true><<<grd, blk, 0, st>>>(d, P, r); break;
    default: uq_kernel<T, DEV, NEM, true><<<grd, blk, 0, st>>>(d, P, r); break;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

} // namespace

#ifndef MLB_UNFUSED_PART
#define MLB_UNFUSED_PART 0   // both precisions in one object
#endif

#if MLB_UNFUSED_PART != 32
bool substep_path(const Dims& d, const Params& P, int bc)
{
  return !bc && d.g == 0 && P.npc >= 1;
}

int replay_derived_f64(const Dims& d, const Params& P, const State<double>& s, cudaStream_t st)
{
  return replay_impl<double, false>(d, P, s, st);
}

int lb_kind(int model, int bc)
{
  if(model != NEM)
  {
    switch(bc)
    {
      case 1: return LBK_FREESLIP_CHANNEL;
      case 2: return LBK_NOSLIP_CHANNEL;
      case 3: return LBK_FREESLIP_BOX;
      case 4: return LBK_NOSLIP_BOX;
      default: return LBK_PBC;
    }
  }
  return bc == 1 ? LBK_FREESLIP_CHANNEL : LBK_PBC;
}

int bc_mode(int model, int bc)
{
  if(model != NEM)
    return (bc == 1 || bc == 2) ? BCM_CHANNEL : (bc == 3 || bc == 4) ? BCM_BOX : BCM_PBC;
  return bc == 1 ? BCM_CHANNEL : BCM_PBC;
}

int launches_unfused(int model, int bc, unsigned npc)
{
  // periodic: one sub-step kernel per predictor and corrector; walls:
  // predictor [bc] uq [bc] uf [bc] move, corrector [bc] uq [bc] uf, where
  // a scalar [bc] is two launches and the populations' two or three
  if(!bc) return 1 + (int)npc;
  const int lb = lb_noslip(lb_kind(model, bc)) ? 3 : 2;
  return (2 + 1 + 2 + 1 + lb + 1) + (int)npc*6;
}

int step_unfused_f64(const Dims& d, const Params& P, State<double>& s, int bc,
                     unsigned nsteps, bool diag_last, cudaStream_t st)
{
  switch(P.model)
  {
    case LYO: return step_impl<double, false, LYO>(d, P, s, bc, nsteps, diag_last, st);
    case GOG: return step_impl<double, false, GOG>(d, P, s, bc, nsteps, diag_last, st);
    default: return step_impl<double, false, NEM>(d, P, s, bc, nsteps, diag_last, st);
  }
}

int relax_unfused_f64(const Dims& d, const Params& P, State<double>& s, int bc,
                      unsigned nsteps, double dt, int relax_phi, int relax_Q,
                      double* sum_out, cudaStream_t st)
{
  return relax_impl<double>(d, P, s, bc, nsteps, dt, relax_phi, relax_Q, sum_out, st);
}

int update_chi_f64(const Dims& d, State<double>& s, cudaStream_t st)
{
  const dim3 blk(64, 4);
  chi_kernel<double><<<site_grid(d.LX, d.LY, blk), blk, 0, st>>>(d, s);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

#endif

#if MLB_UNFUSED_PART != 64
int replay_derived_f32(const Dims& d, const Params& P, const State<float>& s, cudaStream_t st)
{
  return replay_impl<float, true>(d, P, s, st);
}

int step_unfused_f32(const Dims& d, const Params& P, State<float>& s, int bc,
                     unsigned nsteps, bool diag_last, cudaStream_t st)
{
  switch(P.model)
  {
    case LYO: return step_impl<float, true, LYO>(d, P, s, bc, nsteps, diag_last, st);
    case GOG: return step_impl<float, true, GOG>(d, P, s, bc, nsteps, diag_last, st);
    default: return step_impl<float, true, NEM>(d, P, s, bc, nsteps, diag_last, st);
  }
}

int relax_unfused_f32(const Dims& d, const Params& P, State<float>& s, int bc,
                      unsigned nsteps, double dt, int relax_phi, int relax_Q,
                      double* sum_out, cudaStream_t st)
{
  return relax_impl<float>(d, P, s, bc, nsteps, dt, relax_phi, relax_Q, sum_out, st);
}

int corrector_substep_f32(const Dims& d, const Params& P, const State<float>& s, bool diag,
                          cudaStream_t st)
{
  switch(P.model)
  {
    case LYO:
      if(diag) launch_substep<float, true, LYO, false, true>(d, P, s, 1, st);
      else launch_substep<float, true, LYO, false, false>(d, P, s, 0, st);
      break;
    case NEM:
      if(diag) launch_substep<float, true, NEM, false, true>(d, P, s, 1, st);
      else launch_substep<float, true, NEM, false, false>(d, P, s, 0, st);
      break;
    default:
      return -1;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int update_chi_f32(const Dims& d, State<float>& s, cudaStream_t st)
{
  const dim3 blk(64, 4);
  chi_kernel<float><<<site_grid(d.LX, d.LY, blk), blk, 0, st>>>(d, s);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

#endif

} // namespace mlb
