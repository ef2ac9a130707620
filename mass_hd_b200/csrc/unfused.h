// Host entry points of the unfused step kernels (unfused.cu).
#pragma once

#include "lb_common.cuh"

namespace mlb {

// scalar ghost kinds (src/fields.hpp:705-778)
enum { BC_NEUMANN = 0, BC_DIRICHLET0 = 1, BC_COPYDERIV = 2 };
// scalar ghost layouts: channel (pbc left/right), box, full pbc
enum { BCM_CHANNEL = 0, BCM_BOX = 1, BCM_PBC = 2 };
// blocks of the FP32 countphi sum; the conservation scalar needs
// 1 + PHI_PARTS doubles
constexpr int PHI_PARTS = 512;
// population ghost layouts (src/fields.hpp:792-930)
enum { LBK_PBC = 0, LBK_FREESLIP_CHANNEL = 1, LBK_NOSLIP_CHANNEL = 2,
       LBK_FREESLIP_BOX = 3, LBK_NOSLIP_BOX = 4 };

template<typename T>
struct ScalarBC
{
  T* f[9];
  int kind[9];
  int nf;
  int mode;
};

int lb_kind(int model, int bc);
int bc_mode(int model, int bc);
int launches_unfused(int model, int bc, unsigned npc);
// Whether a step runs one sub-step kernel per predictor and corrector
// (periodic lattice without a ghost ring, npc >= 1). Such a step called
// with diag_last = false leaves the derived fields (n, u, H, mu, dQ,
// stresses, diagnostic stresses) to replay_derived_*, which recomputes
// them from the state its last UpdateQuantities read; valid until the next
// step or change of the state.
bool substep_path(const Dims& d, const Params& P, int bc);
int replay_derived_f64(const Dims& d, const Params& P, const State<double>& s, cudaStream_t st);
int replay_derived_f32(const Dims& d, const Params& P, const State<float>& s, cudaStream_t st);

// Advance `nsteps` steps; swaps the ping-pong pointers held in `s`.
// diag_last: the last corrector UpdateQuantities also writes the seven
// diagnostic stress fields.
int step_unfused_f64(const Dims& d, const Params& P, State<double>& s, int bc,
                     unsigned nsteps, bool diag_last, cudaStream_t st);
int step_unfused_f32(const Dims& d, const Params& P, State<float>& s, int bc,
                     unsigned nsteps, bool diag_last, cudaStream_t st);

// Go-or-grow dry relaxation: `nsteps` descent steps of phi and/or Q, then
// the site-order sum of the relaxed phi into the device scalar sum_out.
int relax_unfused_f64(const Dims& d, const Params& P, State<double>& s, int bc,
                      unsigned nsteps, double dt, int relax_phi, int relax_Q,
                      double* sum_out, cudaStream_t st);
int relax_unfused_f32(const Dims& d, const Params& P, State<float>& s, int bc,
                      unsigned nsteps, double dt, int relax_phi, int relax_Q,
                      double* sum_out, cudaStream_t st);

// One corrector sub-step (UpdateQuantities and the corrector UpdateFields)
// of a periodic FP32 lattice, lyotropic or nematic: reads ff, Qxx, Qyx,
// phi, fn, QNxx, QNyx, phn (and src), writes ff_tmp, Qxx_tmp, Qyx_tmp,
// phi_tmp; with `diag`, also the derived fields of its UpdateQuantities.
int corrector_substep_f32(const Dims& d, const Params& P, const State<float>& s, bool diag,
                          cudaStream_t st);

// chi = m/phi over the domain (after an upload of m or phi)
int update_chi_f64(const Dims& d, State<double>& s, cudaStream_t st);
int update_chi_f32(const Dims& d, State<float>& s, cudaStream_t st);

} // namespace mlb
