// FP32 fused periodic step: one kernel launch advances the whole lattice by
// one Model::Step() (predictor UpdateQuantities + UpdateFields, Move, and
// npc = 1 corrector UpdateQuantities + UpdateFields).
#pragma once

#include "lb_common.cuh"

namespace mlb {

// Parameters in FP32 (nematic: Gamma -> GammaQ, tau -> tauNem = tauIso).
struct P32
{
  float rho, GammaQ, GammaP, xi, tauNem, tauIso, friction;
  float AA, CC, LL, KK, zeta, zetaI, conc;
  // go-or-grow phenotype terms (Pheno)
  float B, Snem, Dchi, Achi, Ochi, phiswitch, phi_critical;
  int growTogether;
};

// Diagnostic outputs of the corrector UpdateQuantities (the values the
// reference holds in n, ux, ..., sigma_active_yx after Step()), written only
// by the replay launch. Planes of LX*LY floats, in mass_lb_field order
// MASS_LB_N .. MASS_LB_SIGMA_ACTIVE_YX (23 planes).
enum { NDIAG = 23 };

// Parameters and literals pre-broadcast to pairs for the packed FP32x2
// kernel (read straight from the constant bank as 64-bit operands).
struct PairParams
{
  float2 rho, GammaQ, GammaP, xi2, hxi, tauIso, dtau, itau, n2fric;
  float2 AA, hAA, nCC, hCC, c4k, LL, q4LL, nh2LL;
  float2 nKK, KK8, nKK4, zeta, nzeta, zetaI, conc;
  // go-or-grow: Snem, phi_critical, B, B/2, GammaP/2, Dchi/2, 2 Achi, Ochi,
  // phiswitch, growTogether (0 or 1)
  float2 Snem, phic, Bc, hB, hGP, hDchi, A2chi, Ochi, phisw, gt;
};

struct FusedArgs
{
  const float* in;     // NP planes of LX*LY: g0..g8, Qxx, Qyx[, phi]
  float* out;          // same layout
  float* diag;         // NDIAG planes (DIAG launches only)
  int* err;            // bit 0: a bounded wait gave up
  int LX, LY;
  long long plane;     // LX*LY
  int nstrips;         // ceil(LY / (NT - 8))
  int rows;            // rows per CTA chunk
  P32 p;
  PairParams pp;       // filled by the warp-strip launcher
  const float* src;    // per-site phi source rate (LX*LY) or null; warp-strip kernel only
                       // (go-or-grow: the growth rate, always present)
  float* pred;         // or null; warp-strip kernel, lyotropic and nematic: fn (9 planes),
                       // QNxx, QNyx[, phn] of the step, for the further correctors of npc > 1
  int xbase, xcount;   // the rows stepped, [xbase, xbase + xcount) with xcount >= 1; the
                       // others are not written (inputs still wrap periodically over LX)
};

// Tile shapes the autotuner may pick.
//   nt = 64, 128, 256: CTA-strip kernel (fused32.cu), nt threads = nt
//        columns per strip, one column per thread;
//   nt = 32: warp-strip kernel (fused_warp.cu), every warp an independent
//        64-column strip, two columns per lane in packed FP32x2.
struct FusedConfig
{
  int nt;
  int rows;  // rows per CTA (or warp) chunk
};

// Warp-strip kernel launch (fused_warp.cu).
cudaError_t launch_fused_warp_step(const FusedArgs& a, int model, int rows, bool diag,
                                   cudaStream_t st);

// Ensembles: many lattices advanced by one persistent warp-strip launch.
constexpr int ENS_MAX_RUNS = 192;     // constant-memory parameter slots per device
constexpr int ENS_WOUT = 56;          // output columns per warp strip

struct EnsRun
{
  float* a;            // state buffers (ping-pong); parity 0 reads a, writes b
  float* b;
  int LX, LY;
  long long plane;
  int nstrips, rows;   // strips of ENS_WOUT columns, rows per chunk
  int item0;           // first item of this run in the packed list
  int slot;            // constant-memory parameter slot
};

cudaError_t ensemble_set_params(int slot, const P32& p, int model, cudaStream_t st);
cudaError_t launch_fused_warp_ensemble(const EnsRun* runs, const int* item_run, int nitems,
                                       int* counter, int* err, int parity, int model, int grid,
                                       cudaStream_t st);
int ensemble_grid(int model);   // resident CTAs on this device (0 on error)

// Launch one fused step (template dispatch on nt / model / diag).
cudaError_t launch_fused_step(const FusedArgs& a, int model, FusedConfig cfg,
                              bool diag, cudaStream_t st);

// Dynamic shared memory one CTA of the given width needs.
size_t fused_smem_bytes(int nt, int model);

// True if the fused kernel can run this lattice: LY % 4 == 0 (16-byte
// aligned row segments for the bulk copies), LY >= max(nt, 64), LX >= 1.
bool fused_supported(int LX, int LY, int nt);

} // namespace mlb
