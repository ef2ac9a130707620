// Shared definitions for the sm_100a MASS step kernels.
//
// Lattice: site (x, y), x the slow index, y contiguous (the reference's
// k = y + LY*x, src/geometry.hpp:430). The device arrays live on an
// "extended" torus of EX x EY sites with a ghost ring of width g (g = 0 for
// periodic lattices, g = 1 for the reference's GridType::Layer walls,
// src/geometry.cpp:141-183). Every field is one plane of NE = EX*EY values;
// populations are 9 planes, plane v holding direction v
// (D2Q9 order of src/geometry.hpp:17-27).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "mass_lb.h"

namespace mlb {

enum { LYO = 0, NEM = 1, GOG = 2 };   // GOG: go-or-grow (lyotropic + phenotype)

// D2Q9 velocity set, src/geometry.hpp:17-27
__host__ __device__ constexpr int CXv(int v)
{
  return v == 1 || v == 5 || v == 8 ? 1 : (v == 2 || v == 6 || v == 7 ? -1 : 0);
}
__host__ __device__ constexpr int CYv(int v)
{
  return v == 3 || v == 5 || v == 7 ? 1 : (v == 4 || v == 6 || v == 8 ? -1 : 0);
}
// forcing weights w[], src/lb.hpp:15-16
__host__ __device__ constexpr double Wv(int v)
{
  return v == 0 ? 0.0 : (v <= 4 ? 1/3. : 1/12.);
}
// rest-state equilibrium weights t_v (fe at u = 0 is t_v * rho,
// src/lb.hpp:29-38): 4/9, 1/9 (axis), 1/36 (diagonal)
__host__ __device__ constexpr double Tv(int v)
{
  return v == 0 ? 4/9. : (v <= 4 ? 1/9. : 1/36.);
}
__host__ __device__ constexpr int OPPv(int v)
{
  return v == 0 ? 0 : (v % 2 == 1 ? v + 1 : v - 1);
}

struct Dims
{
  int LX, LY, g, EX, EY;
  long long NE;
};

// Model parameters (runcard names; nematic: Gamma -> GammaQ, tau -> tauNem)
struct Params
{
  int model;
  double GammaQ, GammaP, xi, tauNem, tauIso, rho, friction;
  double AA, CC, LL, KK, zeta, zetaI, conc;
  unsigned npc;
};

// Go-or-grow parameters (runcard names, src/models/go-or-grow.hpp:9-20;
// phi_critical is LyotropicWithDivision's, src/models/lyotropic-with-division.hpp:34)
struct Pheno
{
  double B, Snem, Dchi, Achi, Ochi, phiswitch, phi_critical;
  int growTogether;
};

// Every device array of one lattice (unfused kernels).
template<typename T>
struct State
{
  T *ff, *fn, *ff_tmp, *fn_tmp;               // 9 planes each
  T *Qxx, *Qyx, *QNxx, *QNyx, *phi, *phn, *phi_tmp;
  T *Qxx_tmp, *Qyx_tmp;  // the next Q, written beside Q by the sub-step kernel
  T *n, *ux, *uy, *uxp, *uyp, *Hxx, *Hyx, *MU;
  T *dxQxx, *dyQxx, *dxQyx, *dyQyx;
  T *sXX, *sYY, *sYX, *sXY;
  T *diag[7];  // sigma_bulk, elastic_xx, elastic_yx, phase_field_xx,
               // phase_field_yx, active_xx, active_yx
  // division models (src/models/lyotropic-with-division.cpp:111-124): a
  // per-site phi source rate r (phi_tmp += phi*r after each UpdateFields),
  // and the conserve_phi correction Dp -= (sum phi - totalphi)/DomainSize
  // (src/models/lyotropic.cpp:299) with the sum taken serially in site order
  const T* src;        // null: no source
  double* phisum;      // device scalar written before each UpdateFields
  double totalphi;
  int conserve_phi;
  // go-or-grow (src/models/go-or-grow.cpp): the phenotype density m, its
  // predictor mN, the next m, and chi = m/phi (plus the next chi)
  T *m, *mN, *m_tmp, *chi, *chi_tmp;
  Pheno ph;
};

__host__ __device__ inline int wrapi(int a, int n)
{
  return a < 0 ? a + n : (a >= n ? a - n : a);
}

} // namespace mlb
