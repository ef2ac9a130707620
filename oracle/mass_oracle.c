/* CPU oracle: FP64 restatement of the MASS lyotropic / nematic Step().
 *
 * TEST INFRASTRUCTURE ONLY (see mass_oracle.h). Parity is pinned against the
 * reference's own sources compiled in oracle/_ref, through the golden
 * fixtures in tests/golden/.
 *
 * Layout. The state lives on an "extended" torus of EX x EY sites,
 * EX = LX + 2g, EY = LY + 2g, with g = 0 for bc = 0 (src/geometry.cpp:100-111,
 * no ghost cells) and g = 1 otherwise (the ghost ring of GridType::Layer,
 * src/geometry.cpp:141-183, whose neighbour table is the periodic table of
 * the (LX+2) x (LY+2) grid). Site (X, Y) has index Y + EY*X; domain site
 * (x, y) is (x+g, y+g). Populations are stored site-major f[9*e + v].
 *
 * Reference correspondence:
 *   D2Q9 directions        src/geometry.hpp:17-27
 *   forcing weights w[]    src/lb.hpp:15-16
 *   equilibrium            src/lb.hpp:24-41
 *   derivX/derivY/laplacian (5-point) src/lb.hpp:73-90, :127-136
 *   lyotropic UQ / UF      src/models/lyotropic.cpp:168-247 / :249-341
 *   lyotropic Step         src/models/lyotropic.cpp:500-525
 *   nematic UQ / UF / Step src/models/nematic.cpp:76-130 / :132-226 / :370-395
 *   Move (push streaming)  src/models/lyotropic.cpp:371-386
 *   wall BCs               src/fields.hpp:620-930, dispatch
 *                          src/models/lyotropic.cpp:388-498,
 *                          src/models/nematic.cpp:259-368
 */
#include "mass_oracle.h"

#include <stdlib.h>
#include <string.h>

static const int CX[9] = {0, 1, -1, 0, 0, 1, -1, -1, 1};
static const int CY[9] = {0, 0, 0, 1, -1, 1, -1, 1, -1};
static const double W[9] = {0, 1/3., 1/3., 1/3., 1/3.,
                            1/12., 1/12., 1/12., 1/12.};
/* opposite direction (bounce back) */
static const int OPP[9] = {0, 2, 1, 4, 3, 6, 5, 8, 7};
/* reflection of direction v about the plane whose normal is direction a
 * (a = 1..4 are the wall normals), src/geometry.hpp:41-60 */
static const int REFL[9][9] = {
  {0, 2, 1, 4, 3, 6, 5, 8, 7},
  {0, 2, 1, 3, 4, 7, 8, 5, 6},
  {0, 2, 1, 3, 4, 7, 8, 5, 6},
  {0, 1, 2, 4, 3, 8, 7, 6, 5},
  {0, 1, 2, 4, 3, 8, 7, 6, 5},
  {0, 4, 3, 2, 1, 6, 5, 7, 8},
  {0, 4, 3, 2, 1, 6, 5, 7, 8},
  {0, 3, 4, 1, 2, 5, 6, 8, 7},
  {0, 3, 4, 1, 2, 5, 6, 8, 7}};
/* projection table, src/geometry.hpp:67-86 */
static const int PROJ[9][9] = {
  {0, 0, 0, 0, 0, 0, 0, 0, 0},
  {0, 0, 0, 3, 4, 3, 4, 3, 4},
  {0, 0, 0, 3, 4, 3, 4, 3, 4},
  {0, 1, 2, 0, 0, 1, 2, 2, 1},
  {0, 1, 2, 0, 0, 1, 2, 2, 1},
  {0, 5, 6, 5, 6, 5, 6, 0, 0},
  {0, 1, 2, 4, 3, 8, 7, 6, 5},
  {0, 8, 7, 7, 8, 0, 0, 7, 8},
  {0, 8, 7, 7, 8, 0, 0, 7, 8}};

/* wall / corner ids are their direction numbers (src/geometry.hpp:146-193) */
enum { W_RIGHT = 1, W_LEFT = 2, W_BACK = 3, W_FRONT = 4 };
enum { C_RIGHTBACK = 5, C_LEFTFRONT = 6, C_LEFTBACK = 7, C_RIGHTFRONT = 8 };

struct mo_state {
  mo_params p;
  unsigned LX, LY, BC, g, EX, EY;
  size_t NE;
  double *ff, *fn, *ff_tmp, *fn_tmp;
  double *Qxx, *Qyx, *QNxx, *QNyx, *phi, *phn, *phi_tmp;
  double *n, *ux, *uy, *uxp, *uyp, *Hxx, *Hyx, *MU;
  double *dxQxx, *dyQxx, *dxQyx, *dyQyx;
  double *sXX, *sYY, *sYX, *sXY;
  double *s_bulk, *s_el_xx, *s_el_yx, *s_pf_xx, *s_pf_yx, *s_act_xx, *s_act_yx;
};

/* ------------------------------------------------------------------------ */
/* neighbours on the extended torus */

static size_t nb(const mo_state* s, size_t e, int v)
{
  const long X = (long)(e / s->EY), Y = (long)(e % s->EY);
  const long EX = s->EX, EY = s->EY;
  const long Xn = (X + CX[v] + EX) % EX, Yn = (Y + CY[v] + EY) % EY;
  return (size_t)(Yn + EY*Xn);
}

static size_t dom(const mo_state* s, unsigned x, unsigned y)
{
  return (size_t)(y + s->g) + (size_t)s->EY*(x + s->g);
}

/* 5-point stencils exactly as written in src/lb.hpp:79, :89, :134
 * (the `+0*stencil` term adds +0.0) */
static double dX(const double* a, const size_t* d) { return .5*(a[d[1]]-a[d[2]]) + 0.0; }
static double dY(const double* a, const size_t* d) { return .5*(a[d[3]]-a[d[4]]) + 0.0; }
static double lap(const double* a, const size_t* d)
{
  return a[d[1]]+a[d[2]]+a[d[3]]+a[d[4]] - 4*a[d[0]] + 0.0;
}

static void equilibrium(double vx, double vy, double nn, double fe[9])
{
  const double v2 = vx*vx + vy*vy;
  fe[1] = nn*(1./9. + 1./3.*vx + 1./3.*v2 - 1./2.*vy*vy);
  fe[2] = nn*(1./9. - 1./3.*vx + 1./3.*v2 - 1./2.*vy*vy);
  fe[3] = nn*(1./9. + 1./3.*vy - 1./2.*vx*vx + 1./3.*v2);
  fe[4] = nn*(1./9. - 1./3.*vy - 1./2.*vx*vx + 1./3.*v2);
  fe[5] = nn*(1./36. + 1./12.*vx + 1./12.*vy + 1./12.*v2 + 1./4.*vx*vy);
  fe[6] = nn*(1./36. - 1./12.*vx - 1./12.*vy + 1./12.*v2 + 1./4.*vx*vy);
  fe[7] = nn*(1./36. - 1./12.*vx + 1./12.*vy + 1./12.*v2 - 1./4.*vx*vy);
  fe[8] = nn*(1./36. + 1./12.*vx - 1./12.*vy + 1./12.*v2 - 1./4.*vx*vy);
  fe[0] = nn-fe[1]-fe[2]-fe[3]-fe[4]-fe[5]-fe[6]-fe[7]-fe[8];
}

static void neighbours(const mo_state* s, size_t e, size_t d[9])
{
  for(int v=0; v<9; ++v) d[v] = nb(s, e, v);
}

/* ------------------------------------------------------------------------ */
/* UpdateQuantities */

static void uq_site(mo_state* s, size_t e)
{
  const mo_params* P = &s->p;
  size_t d[9];
  neighbours(s, e, d);
  const double* f = s->ff + 9*e;
  const double Qxx = s->Qxx[e], Qyx = s->Qyx[e];

  const double nn = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  const double vx = (f[1] - f[2] + f[5] - f[6] - f[7] + f[8])/nn;
  const double vy = (f[3] - f[4] + f[5] - f[6] + f[7] - f[8])/nn;

  const double del2Qxx = lap(s->Qxx, d);
  const double dxQxx = dX(s->Qxx, d);
  const double dyQxx = dY(s->Qxx, d);
  const double del2Qyx = lap(s->Qyx, d);
  const double dxQyx = dX(s->Qyx, d);
  const double dyQyx = dY(s->Qyx, d);

  s->n[e] = nn;
  s->ux[e] = vx;
  s->uy[e] = vy;
  s->dxQxx[e] = dxQxx;
  s->dxQyx[e] = dxQyx;
  s->dyQxx[e] = dyQxx;
  s->dyQyx[e] = dyQyx;

  if(P->model == MO_LYOTROPIC)
  {
    const double p = s->phi[e];
    const double del2p = lap(s->phi, d);
    const double dxPhi = dX(s->phi, d);
    const double dyPhi = dY(s->phi, d);
    const double term = 0 - Qxx*Qxx - Qyx*Qyx;
    const double Hxx = P->CC*term*Qxx + P->LL*del2Qxx;
    const double Hyx = P->CC*term*Qyx + P->LL*del2Qyx;
    const double mu = P->AA*p*(1-p)*(1-2*p) + 0*P->CC*term - P->KK*del2p;
    const double sigmaB = .5*P->AA*p*p*(1-p)*(1-p) + .5*P->CC*term*term - mu*p;
    const double sigmaF = 2*P->xi*( (Qxx*Qxx-1)*Hxx + Qxx*Qyx*Hyx )
      - P->zeta*Qxx*(1-p) + .5*P->KK*(dyPhi*dyPhi-dxPhi*dxPhi)
      + P->LL*(dyQxx*dyQxx+dyQyx*dyQyx-dxQxx*dxQxx-dxQyx*dxQyx);
    const double sigmaS = 2*P->xi*(Qyx*Qxx*Hxx + (Qyx*Qyx-1)*Hyx)
      - P->zeta*Qyx*(1-p) - P->KK*dxPhi*dyPhi
      - 2*P->LL*(dxQxx*dyQxx+dxQyx*dyQyx);
    const double sigmaA = 2*(Qxx*Hyx - Qyx*Hxx);

    s->uxp[e] = vx*p;
    s->uyp[e] = vy*p;
    s->Hxx[e] = Hxx;
    s->Hyx[e] = Hyx;
    s->MU[e] = mu;
    s->sXX[e] = sigmaF + sigmaB + P->zetaI*(P->conc-p);
    s->sYY[e] = -sigmaF + sigmaB + P->zetaI*(P->conc-p);
    s->sXY[e] = sigmaS + sigmaA;
    s->sYX[e] = sigmaS - sigmaA;
    s->s_bulk[e] = sigmaB + P->zetaI*(P->conc-p);
    s->s_el_xx[e] = sigmaF - .5*P->KK*(dyPhi*dyPhi-dxPhi*dxPhi) + P->zeta*Qxx*(1-p);
    s->s_el_yx[e] = sigmaS + P->KK*dxPhi*dyPhi + P->zeta*Qxx*(1-p);
    s->s_pf_xx[e] = .5*P->KK*(dyPhi*dyPhi-dxPhi*dxPhi);
    s->s_pf_yx[e] = -P->KK*dxPhi*dyPhi;
    s->s_act_xx[e] = -P->zeta*Qxx*(1-p);
    s->s_act_yx[e] = -P->zeta*Qyx*(1-p);
  }
  else
  {
    const double term = 1. - Qxx*Qxx - Qyx*Qyx;
    const double Hxx = P->CC*term*Qxx + P->LL*del2Qxx;
    const double Hyx = P->CC*term*Qyx + P->LL*del2Qyx;
    const double sigmaB = .5*P->CC*term*term;
    const double sigmaF = 2*P->xi*( (Qxx*Qxx-1.)*Hxx + Qxx*Qyx*Hyx )
      - P->zeta*Qxx
      + P->LL*(dyQxx*dyQxx+dyQyx*dyQyx-dxQxx*dxQxx-dxQyx*dxQyx);
    const double sigmaS = 2*P->xi*(Qyx*Qxx*Hxx + (Qyx*Qyx-1)*Hyx) - P->zeta*Qyx
      - 2*P->LL*(dxQxx*dyQxx+dxQyx*dyQyx);
    const double sigmaA = 2*(Qxx*Hyx - Qyx*Hxx);
    s->Hxx[e] = Hxx;
    s->Hyx[e] = Hyx;
    s->sXX[e] = sigmaF + sigmaB;
    s->sYY[e] = -sigmaF + sigmaB;
    s->sXY[e] = sigmaS + sigmaA;
    s->sYX[e] = sigmaS - sigmaA;
  }
}

/* ------------------------------------------------------------------------ */
/* UpdateFields */

static void uf_site(mo_state* s, size_t e, int first)
{
  const mo_params* P = &s->p;
  size_t d[9];
  neighbours(s, e, d);

  const double nn = s->n[e];
  const double vx = s->ux[e];
  const double vy = s->uy[e];
  const double Qxx = s->Qxx[e];
  const double Qyx = s->Qyx[e];
  const double Hxx = s->Hxx[e];
  const double Hyx = s->Hyx[e];
  const double dxQxx = s->dxQxx[e];
  const double dyQxx = s->dyQxx[e];
  const double dxQyx = s->dxQyx[e];
  const double dyQyx = s->dyQyx[e];

  const double dxux = dX(s->ux, d);
  const double dyux = dY(s->ux, d);
  const double dxuy = dX(s->uy, d);
  const double dyuy = dY(s->uy, d);
  const double dxSxx = dX(s->sXX, d);
  const double dySxy = dY(s->sXY, d);
  const double dxSyx = dX(s->sYX, d);
  const double dySyy = dY(s->sYY, d);

  const double expansion = dxux + dyuy;
  const double shear     = .5*(dxuy + dyux);
  const double vorticity = .5*(dxuy - dyux);
  const double traceQL   = Qxx*(dxux - dyuy) + 2*Qyx*shear;

  const double Dxx = P->GammaQ*Hxx - vx*dxQxx - vy*dyQxx - 2*vorticity*Qyx
    + P->xi*((Qxx+1)*(2*dxux-traceQL) +2*Qyx*shear -expansion);
  const double Dyx = P->GammaQ*Hyx - vx*dxQyx - vy*dyQyx + 2*vorticity*Qxx
    + P->xi*( Qyx*(expansion-traceQL) + 2*shear);

  const double Fx = dxSxx + dySxy - P->friction*vx;
  const double Fy = dxSyx + dySyy - P->friction*vy;

  double* ff = s->ff + 9*e;
  double* fn = s->fn + 9*e;
  double fe[9];

  if(P->model == MO_LYOTROPIC)
  {
    const double p = s->phi[e];
    const double del2mu = lap(s->MU, d);
    const double pFlux = dX(s->uxp, d) + dY(s->uyp, d);
    /* conserve_phi is false (src/models/lyotropic.hpp:46): `- 0` */
    const double Dp = P->GammaP*del2mu - pFlux - 0.0;
    const double tau = P->tauNem*p + P->tauIso*(1-p);
    equilibrium(vx, vy, nn, fe);
    if(first)
    {
      s->QNxx[e] = s->Qxx[e] + .5*Dxx;
      s->QNyx[e] = s->Qyx[e] + .5*Dyx;
      s->phn[e]  = s->phi[e] + .5*Dp;
      s->Qxx[e]  = s->Qxx[e] + Dxx;
      s->Qyx[e]  = s->Qyx[e] + Dyx;
      s->phi_tmp[e] = s->phi[e] + Dp;
      for(int v=0; v<9; ++v)
      {
        const double cx = CX[v], cy = CY[v];
        fn[v] = ff[v] + .5*((fe[v]-ff[v])/tau + W[v]*(Fx*cx + Fy*cy));
        ff[v] = ff[v] +    ((fe[v]-ff[v])/tau + W[v]*(Fx*cx + Fy*cy));
      }
    }
    else
    {
      s->Qxx[e] = s->QNxx[e] + .5*Dxx;
      s->Qyx[e] = s->QNyx[e] + .5*Dyx;
      s->phi_tmp[e] = s->phn[e] + .5*Dp;
      for(int v=0; v<9; ++v)
      {
        const double cx = CX[v], cy = CY[v];
        ff[v] = fn[v] + .5*((fe[v]-ff[v])/tau + W[v]*(Fx*cx + Fy*cy));
      }
    }
  }
  else
  {
    const double tau = P->tauNem;
    equilibrium(vx, vy, nn, fe);
    if(first)
    {
      /* thermal noise terms are zero (Q_kBT = u_kBT = 0) */
      s->QNxx[e] = s->Qxx[e] + .5*Dxx + 0.0;
      s->QNyx[e] = s->Qyx[e] + .5*Dyx + 0.0;
      s->Qxx[e] = s->QNxx[e] + .5*Dxx;
      s->Qyx[e] = s->QNyx[e] + .5*Dyx;
      for(int v=0; v<9; ++v)
      {
        const double cx = CX[v], cy = CY[v];
        const double fold = ff[v];
        fn[v] = fold + .5*((fe[v]-fold)/tau + W[v]*(Fx*cx + Fy*cy)) + 0.0;
        ff[v] = fn[v] + .5*((fe[v]-fold)/tau + W[v]*(Fx*cx + Fy*cy));
      }
    }
    else
    {
      s->Qxx[e] = s->QNxx[e] + .5*Dxx;
      s->Qyx[e] = s->QNyx[e] + .5*Dyx;
      for(int v=0; v<9; ++v)
      {
        const double cx = CX[v], cy = CY[v];
        ff[v] = fn[v] + .5*((fe[v]-ff[v])/tau + W[v]*(Fx*cx + Fy*cy));
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Boundary conditions on the ghost ring (g = 1 only) */

/* extended index of ghost k on wall w (k = 0..LY-1 for Left/Right, 0..LX-1
 * for Front/Back), and of a corner */
static size_t wall_site(const mo_state* s, int w, unsigned k)
{
  const unsigned EX = s->EX, EY = s->EY;
  switch(w)
  {
    case W_LEFT:  return (size_t)(k+1) + (size_t)EY*0;
    case W_RIGHT: return (size_t)(k+1) + (size_t)EY*(EX-1);
    case W_FRONT: return (size_t)0 + (size_t)EY*(k+1);
    default:      return (size_t)(EY-1) + (size_t)EY*(k+1); /* W_BACK */
  }
}
static unsigned wall_len(const mo_state* s, int w)
{
  return (w == W_LEFT || w == W_RIGHT) ? s->LY : s->LX;
}
static size_t corner_site(const mo_state* s, int c)
{
  const unsigned EX = s->EX, EY = s->EY;
  switch(c)
  {
    case C_LEFTFRONT:  return 0;
    case C_RIGHTFRONT: return (size_t)EY*(EX-1);
    case C_LEFTBACK:   return (size_t)(EY-1);
    default:           return (size_t)(EY-1) + (size_t)EY*(EX-1);
  }
}
static int incoming(int v, int w)
{
  return CX[w]*CX[v] == -1 || CY[w]*CY[v] == -1;
}

/* scalar fields */
static void s_pbc_wall(const mo_state* s, double* a, int w)
{
  for(unsigned k=0; k<wall_len(s, w); ++k)
    a[wall_site(s, w, k)] = a[nb(s, wall_site(s, OPP[w], k), w)];
}
static void s_pbc_corner(const mo_state* s, double* a, int c)
{
  a[corner_site(s, c)] = a[nb(s, corner_site(s, OPP[c]), c)];
}
static void s_pbc(const mo_state* s, double* a)
{
  s_pbc_wall(s, a, W_LEFT); s_pbc_wall(s, a, W_RIGHT);
  s_pbc_wall(s, a, W_FRONT); s_pbc_wall(s, a, W_BACK);
  s_pbc_corner(s, a, C_LEFTFRONT); s_pbc_corner(s, a, C_RIGHTFRONT);
  s_pbc_corner(s, a, C_LEFTBACK); s_pbc_corner(s, a, C_RIGHTBACK);
}

enum { S_NEUMANN = 0, S_DIRICHLET0 = 1, S_COPYDERIV = 2 };

/* one ghost value i from the inward direction `in` */
static void s_apply(const mo_state* s, double* a, size_t i, int in, int kind)
{
  const size_t j = nb(s, i, in);
  if(kind == S_NEUMANN) a[i] = a[j];
  else if(kind == S_DIRICHLET0) a[i] = 2*0.0 - a[j];
  else a[i] = 2*a[j]-a[nb(s, j, in)];
}
static void s_wall(const mo_state* s, double* a, int w, int kind)
{
  for(unsigned k=0; k<wall_len(s, w); ++k)
    s_apply(s, a, wall_site(s, w, k), OPP[w], kind);
}
/* fields.hpp:858-900: pbc left/right, kind on front/back, corners along
 * the front/back walls */
static void s_channel(const mo_state* s, double* a, int kind)
{
  s_pbc_wall(s, a, W_LEFT); s_pbc_wall(s, a, W_RIGHT);
  s_wall(s, a, W_FRONT, kind); s_wall(s, a, W_BACK, kind);
  s_apply(s, a, corner_site(s, C_RIGHTBACK), OPP[W_BACK], kind);
  s_apply(s, a, corner_site(s, C_RIGHTFRONT), OPP[W_FRONT], kind);
  s_apply(s, a, corner_site(s, C_LEFTBACK), OPP[W_BACK], kind);
  s_apply(s, a, corner_site(s, C_LEFTFRONT), OPP[W_FRONT], kind);
}
/* fields.hpp:779-829: kind on all four walls, corners along the diagonal */
static void s_box(const mo_state* s, double* a, int kind)
{
  s_wall(s, a, W_LEFT, kind); s_wall(s, a, W_RIGHT, kind);
  s_wall(s, a, W_FRONT, kind); s_wall(s, a, W_BACK, kind);
  const int cs[4] = {C_LEFTFRONT, C_RIGHTFRONT, C_LEFTBACK, C_RIGHTBACK};
  for(int i=0; i<4; ++i) s_apply(s, a, corner_site(s, cs[i]), OPP[cs[i]], kind);
}

/* lattice-Boltzmann fields */
static void f_pbc_wall(const mo_state* s, double* f, int w)
{
  for(unsigned k=0; k<wall_len(s, w); ++k)
    memcpy(f + 9*wall_site(s, w, k), f + 9*nb(s, wall_site(s, OPP[w], k), w),
           9*sizeof(double));
}
static void f_pbc(const mo_state* s, double* f)
{
  f_pbc_wall(s, f, W_LEFT); f_pbc_wall(s, f, W_RIGHT);
  f_pbc_wall(s, f, W_FRONT); f_pbc_wall(s, f, W_BACK);
  const int cs[4] = {C_LEFTFRONT, C_RIGHTFRONT, C_LEFTBACK, C_RIGHTBACK};
  for(int i=0; i<4; ++i)
    memcpy(f + 9*corner_site(s, cs[i]), f + 9*nb(s, corner_site(s, OPP[cs[i]]), cs[i]),
           9*sizeof(double));
}
static void f_freeslip_wall(const mo_state* s, double* f, int w)
{
  for(unsigned i=0; i<wall_len(s, w); ++i)
  {
    const size_t k = wall_site(s, w, i);
    for(int v=0; v<9; ++v)
      if(incoming(v, w))
        f[9*k+v] = f[9*nb(s, k, OPP[w]) + REFL[w][v]];
  }
}
static void f_noslip_wall(const mo_state* s, double* f, int w)
{
  for(unsigned i=0; i<wall_len(s, w); ++i)
  {
    const size_t k = wall_site(s, w, i);
    for(int v=0; v<9; ++v)
      if(incoming(v, w))
        f[9*k+v] = f[9*nb(s, k, v) + OPP[v]];
  }
}
/* corner c along wall w (free-slip channel), fields.hpp:677-688 */
static void f_freeslip_corner_wall(const mo_state* s, double* f, int c, int w)
{
  const int p = PROJ[w][c];
  const size_t k = corner_site(s, c);
  const int v = OPP[c];
  const size_t l = nb(s, corner_site(s, REFL[p][c]), p);
  f[9*k+v] = f[9*l+v];
}
/* simple bounce back in a corner, fields.hpp:690-702 */
static void f_bounce_corner(const mo_state* s, double* f, int c)
{
  const size_t k = corner_site(s, c);
  f[9*k+OPP[c]] = f[9*nb(s, k, OPP[c]) + c];
}
static void f_freeslip_channel(const mo_state* s, double* f)
{
  f_pbc_wall(s, f, W_LEFT); f_pbc_wall(s, f, W_RIGHT);
  f_freeslip_wall(s, f, W_FRONT); f_freeslip_wall(s, f, W_BACK);
  f_freeslip_corner_wall(s, f, C_RIGHTBACK, W_BACK);
  f_freeslip_corner_wall(s, f, C_RIGHTFRONT, W_FRONT);
  f_freeslip_corner_wall(s, f, C_LEFTBACK, W_BACK);
  f_freeslip_corner_wall(s, f, C_LEFTFRONT, W_FRONT);
}
static void f_noslip_channel(const mo_state* s, double* f)
{
  f_pbc_wall(s, f, W_LEFT); f_pbc_wall(s, f, W_RIGHT);
  f_noslip_wall(s, f, W_FRONT); f_noslip_wall(s, f, W_BACK);
  f_bounce_corner(s, f, C_RIGHTBACK); f_bounce_corner(s, f, C_RIGHTFRONT);
  f_bounce_corner(s, f, C_LEFTBACK); f_bounce_corner(s, f, C_LEFTFRONT);
}
static void f_box(const mo_state* s, double* f, int noslip)
{
  const int ws[4] = {W_LEFT, W_RIGHT, W_FRONT, W_BACK};
  for(int i=0; i<4; ++i)
  {
    if(noslip) f_noslip_wall(s, f, ws[i]);
    else f_freeslip_wall(s, f, ws[i]);
  }
  const int cs[4] = {C_LEFTFRONT, C_RIGHTFRONT, C_LEFTBACK, C_RIGHTBACK};
  for(int i=0; i<4; ++i) f_bounce_corner(s, f, cs[i]);
}

/* BoundaryConditionsFields / Fields2 / LB, per model and bc */
static void bc_fields(mo_state* s)
{
  const unsigned bc = s->BC;
  if(bc == 0) return;
  const int lyo = s->p.model == MO_LYOTROPIC;
  if(lyo)
  {
    double* a[3] = {s->Qxx, s->Qyx, s->phi};
    for(int i=0; i<3; ++i)
    {
      if(bc == 1 || bc == 2) s_channel(s, a[i], S_NEUMANN);
      else if(bc == 3 || bc == 4) s_box(s, a[i], S_NEUMANN);
      else s_pbc(s, a[i]);
    }
  }
  else
  {
    double* a[2] = {s->Qxx, s->Qyx};
    for(int i=0; i<2; ++i)
    {
      if(bc == 1) s_channel(s, a[i], S_NEUMANN);
      else s_pbc(s, a[i]);
    }
  }
}

static void bc_fields2(mo_state* s)
{
  const unsigned bc = s->BC;
  if(bc == 0) return;
  if(s->p.model == MO_LYOTROPIC)
  {
    double* nm[5] = {s->MU, s->sXX, s->sYY, s->sYX, s->sXY};
    if(bc == 1 || bc == 2)
    {
      s_channel(s, s->uy, S_COPYDERIV); s_channel(s, s->ux, S_COPYDERIV);
      s_channel(s, s->uyp, S_DIRICHLET0); s_channel(s, s->uxp, S_DIRICHLET0);
      for(int i=0; i<5; ++i) s_channel(s, nm[i], S_NEUMANN);
    }
    else if(bc == 3 || bc == 4)
    {
      s_box(s, s->uy, S_COPYDERIV); s_box(s, s->ux, S_COPYDERIV);
      s_box(s, s->uyp, S_DIRICHLET0); s_box(s, s->uxp, S_DIRICHLET0);
      for(int i=0; i<5; ++i) s_box(s, nm[i], S_NEUMANN);
    }
    else
    {
      double* a[9] = {s->ux, s->uy, s->uxp, s->uyp, s->MU,
                      s->sXX, s->sYY, s->sYX, s->sXY};
      for(int i=0; i<9; ++i) s_pbc(s, a[i]);
    }
  }
  else
  {
    double* a[6] = {s->ux, s->uy, s->sXX, s->sYY, s->sYX, s->sXY};
    for(int i=0; i<6; ++i)
    {
      if(bc == 1) s_channel(s, a[i], S_NEUMANN);
      else s_pbc(s, a[i]);
    }
  }
}

static void bc_lb(mo_state* s)
{
  const unsigned bc = s->BC;
  if(bc == 0) return;
  double* fs[2] = {s->ff, s->fn};
  for(int i=0; i<2; ++i)
  {
    if(s->p.model == MO_LYOTROPIC)
    {
      if(bc == 1) f_freeslip_channel(s, fs[i]);
      else if(bc == 2) f_noslip_channel(s, fs[i]);
      else if(bc == 3) f_box(s, fs[i], 0);
      else if(bc == 4) f_box(s, fs[i], 1);
      else f_pbc(s, fs[i]);
    }
    else
    {
      if(bc == 1) f_freeslip_channel(s, fs[i]);
      else f_pbc(s, fs[i]);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* sweeps */

static void update_quantities(mo_state* s)
{
  for(unsigned x=0; x<s->LX; ++x)
    for(unsigned y=0; y<s->LY; ++y)
      uq_site(s, dom(s, x, y));
}

static void update_fields(mo_state* s, int first)
{
  for(unsigned x=0; x<s->LX; ++x)
    for(unsigned y=0; y<s->LY; ++y)
      uf_site(s, dom(s, x, y), first);
  if(s->p.model == MO_LYOTROPIC)
  {
    double* t = s->phi; s->phi = s->phi_tmp; s->phi_tmp = t;
  }
}

/* push streaming over every extended site, then swap */
static void move(mo_state* s)
{
  for(size_t e=0; e<s->NE; ++e)
    for(int v=0; v<9; ++v)
    {
      const size_t t = nb(s, e, v);
      s->ff_tmp[9*t+v] = s->ff[9*e+v];
      s->fn_tmp[9*t+v] = s->fn[9*e+v];
    }
  double* t = s->ff; s->ff = s->ff_tmp; s->ff_tmp = t;
  t = s->fn; s->fn = s->fn_tmp; s->fn_tmp = t;
}

void mo_step(mo_state* s, unsigned nsteps)
{
  for(unsigned it=0; it<nsteps; ++it)
  {
    bc_fields(s);
    update_quantities(s);
    bc_fields2(s);
    update_fields(s, 1);
    bc_lb(s);
    move(s);
    for(unsigned c=1; c<=s->p.npc; ++c)
    {
      bc_fields(s);
      update_quantities(s);
      bc_fields2(s);
      update_fields(s, 0);
    }
  }
}

/* ------------------------------------------------------------------------ */

mo_state* mo_new(const mo_params* p, unsigned LX, unsigned LY, unsigned BC)
{
  if(LX == 0 || LY == 0) return NULL;
  mo_state* s = (mo_state*)calloc(1, sizeof(mo_state));
  if(!s) return NULL;
  s->p = *p;
  s->LX = LX; s->LY = LY; s->BC = BC;
  s->g = BC ? 1 : 0;
  s->EX = LX + 2*s->g; s->EY = LY + 2*s->g;
  s->NE = (size_t)s->EX*s->EY;
  double** lbs[4] = {&s->ff, &s->fn, &s->ff_tmp, &s->fn_tmp};
  for(int i=0; i<4; ++i) *lbs[i] = (double*)calloc(9*s->NE, sizeof(double));
  double** sc[] = {&s->Qxx, &s->Qyx, &s->QNxx, &s->QNyx, &s->phi, &s->phn,
    &s->phi_tmp, &s->n, &s->ux, &s->uy, &s->uxp, &s->uyp, &s->Hxx, &s->Hyx,
    &s->MU, &s->dxQxx, &s->dyQxx, &s->dxQyx, &s->dyQyx, &s->sXX, &s->sYY,
    &s->sYX, &s->sXY, &s->s_bulk, &s->s_el_xx, &s->s_el_yx, &s->s_pf_xx,
    &s->s_pf_yx, &s->s_act_xx, &s->s_act_yx};
  for(size_t i=0; i<sizeof(sc)/sizeof(sc[0]); ++i)
    *sc[i] = (double*)calloc(s->NE, sizeof(double));
  return s;
}

void mo_free(mo_state* s)
{
  if(!s) return;
  double* all[] = {s->ff, s->fn, s->ff_tmp, s->fn_tmp, s->Qxx, s->Qyx,
    s->QNxx, s->QNyx, s->phi, s->phn, s->phi_tmp, s->n, s->ux, s->uy, s->uxp,
    s->uyp, s->Hxx, s->Hyx, s->MU, s->dxQxx, s->dyQxx, s->dxQyx, s->dyQyx,
    s->sXX, s->sYY, s->sYX, s->sXY, s->s_bulk, s->s_el_xx, s->s_el_yx,
    s->s_pf_xx, s->s_pf_yx, s->s_act_xx, s->s_act_yx};
  for(size_t i=0; i<sizeof(all)/sizeof(all[0]); ++i) free(all[i]);
  free(s);
}

static double* scalar_by_name(mo_state* s, const char* n)
{
#define F(name, member) if(strcmp(n, name) == 0) return s->member;
  F("QQxx", Qxx) F("QQyx", Qyx) F("QNxx", QNxx) F("QNyx", QNyx) F("phi", phi)
  F("phn", phn) F("n", n) F("ux", ux) F("uy", uy) F("ux_phi", uxp)
  F("uy_phi", uyp) F("HHxx", Hxx) F("HHyx", Hyx) F("MU", MU)
  F("dxQQxx", dxQxx) F("dyQQxx", dyQxx) F("dxQQyx", dxQyx) F("dyQQyx", dyQyx)
  F("sigmaXX", sXX) F("sigmaYY", sYY) F("sigmaYX", sYX) F("sigmaXY", sXY)
  F("sigma_bulk", s_bulk) F("sigma_elastic_xx", s_el_xx)
  F("sigma_elastic_yx", s_el_yx) F("sigma_phase_field_xx", s_pf_xx)
  F("sigma_phase_field_yx", s_pf_yx) F("sigma_active_xx", s_act_xx)
  F("sigma_active_yx", s_act_yx)
#undef F
  return NULL;
}

int mo_set_field(mo_state* s, const char* name, const double* src)
{
  double* lbf = strcmp(name, "ff") == 0 ? s->ff : strcmp(name, "fn") == 0 ? s->fn : NULL;
  for(unsigned x=0; x<s->LX; ++x)
    for(unsigned y=0; y<s->LY; ++y)
    {
      const size_t k = (size_t)y + (size_t)s->LY*x, e = dom(s, x, y);
      if(lbf) memcpy(lbf + 9*e, src + 9*k, 9*sizeof(double));
      else
      {
        double* a = scalar_by_name(s, name);
        if(!a) return -1;
        a[e] = src[k];
      }
    }
  return 0;
}

int mo_get_field(mo_state* s, const char* name, double* dst)
{
  double* lbf = strcmp(name, "ff") == 0 ? s->ff : strcmp(name, "fn") == 0 ? s->fn : NULL;
  double* a = lbf ? NULL : scalar_by_name(s, name);
  if(!lbf && !a) return -1;
  for(unsigned x=0; x<s->LX; ++x)
    for(unsigned y=0; y<s->LY; ++y)
    {
      const size_t k = (size_t)y + (size_t)s->LY*x, e = dom(s, x, y);
      if(lbf) memcpy(dst + 9*k, lbf + 9*e, 9*sizeof(double));
      else dst[k] = a[e];
    }
  return 0;
}

void mo_totals(mo_state* s, double* fsum, double* phisum)
{
  double f = 0, p = 0;
  for(unsigned x=0; x<s->LX; ++x)
    for(unsigned y=0; y<s->LY; ++y)
    {
      const size_t e = dom(s, x, y);
      for(int v=0; v<9; ++v) f += s->ff[9*e+v];
      p += s->phi[e];
    }
  *fsum = f;
  *phisum = p;
}
