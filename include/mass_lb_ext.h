/* mass_lb_ext.h - entry points of the sm_100a MASS step library that have
 * no counterpart in the reference (the reference is a CPU-only program with
 * no FFI): tile tuning of the fused FP32 kernel and introspection. They
 * extend the handle API of mass_lb.h and follow its conventions (0 or a
 * negative mass_lb_status, text in mass_lb_last_error()). */
#ifndef MASS_LB_EXT_H_
#define MASS_LB_EXT_H_

#include "mass_lb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Upload one primary field (MASS_LB_FF, QQXX, QQYX, PHI or, for go-or-grow,
 * M) from host memory, same layout as mass_lb_upload. Does not reset the
 * recorded totals. On a go-or-grow lattice an upload of PHI or M recomputes
 * chi = m/phi (0 where phi <= 1e-12), as UpdatePhenotypeQuantities does
 * (src/models/go-or-grow.cpp:208-216). */
int mass_lb_upload_field(mass_lb_handle* h, int field, const double* src);

/* Tile of the fused FP32 kernel: `threads` = 32 selects the warp-strip
 * kernel (64 columns per warp, 56 of them output columns); 64, 128 or 256
 * the CTA-strip kernel with that many columns per CTA strip (NT - 8 output
 * columns), which takes neither a phi source, go-or-grow nor npc > 1
 * (MASS_LB_EUNSUPPORTED). `rows`: lattice rows per chunk. set_tile(h, 0, 0) re-enables the autotuner, which
 * otherwise runs once before the first step (timing every candidate tile on
 * the live state without advancing it). The environment variable
 * MASS_LB_TILE="threads,rows" fixes the tile at handle creation.
 * EUNSUPPORTED when the handle does not use the fused kernel. */
int mass_lb_get_tile(mass_lb_handle* h, int* threads, int* rows);
int mass_lb_set_tile(mass_lb_handle* h, int threads, int rows);
int mass_lb_autotune(mass_lb_handle* h);

/* 1 if mass_lb_step runs the fused FP32 kernel, else 0. FP32 lattices with
 * LY % 4 == 0 and LY >= 64 take it: every model with npc = 1, lyotropic and
 * nematic with npc > 1 (a corrector sub-step per further corrector),
 * periodic or walled (walled: the rows next to the walls are stepped by the
 * wall sweeps beside it; LY, and for boxes LX, at least 8 + 8*npc). A
 * go-or-grow or division lattice leaves the fused kernel for the unfused
 * FP32 sweeps when conserve_phi is switched on (mass_lb_set_phi_conservation),
 * which needs a lattice-wide phi sum inside a sub-step; the dry relaxation
 * of go-or-grow runs on the sweeps and hands the state back. */
int mass_lb_uses_fused(mass_lb_handle* h);

/* Device view of the fused FP32 state (read-only for the caller): `*planes`
 * receives the base of NP float planes of LX*LY values each (g0..g8 as
 * deviations from t_v*rho, then Qxx, Qyx, then phi for the lyotropic
 * models and m for go-or-grow: 11, 12 or 13 planes), valid
 * until the next mass_lb_step / upload call. */
int mass_lb_device_state(mass_lb_handle* h, void** planes, long long* plane_stride,
                         int* nplanes);

/* Statistics of the current state with the estimators of the reference's
 * post-processing (POST/massPy, plot/python/passive_q1_alpha_regime_analysis.py):
 * <|u|^2>; enstrophy density 0.5<w^2> with w the periodic central-difference
 * vorticity, over the lattice and over phi > 0.5; the phi > 0.5 area and
 * its 4-neighbour perimeter; and the +1/2 and -1/2 nematic defects, found as
 * 4-connected same-sign clusters of sites whose director winding exceeds
 * 0.4 in magnitude. No counterpart in the reference's C++ (it is the POST
 * code's arithmetic run on the device). Synchronous. */
typedef struct {
  double mean_u2;
  double enstrophy_density;
  double enstrophy_density_phi;   /* 0 for the nematic model */
  double phi_area;                /* sites with phi > 0.5 */
  double perimeter;               /* exposed edges of the phi > 0.5 region */
  long long defects_plus;
  long long defects_minus;
  long long charged_sites;        /* sites with |charge| > 0.4 */
} mass_lb_stats;

int mass_lb_statistics(mass_lb_handle* h, mass_lb_stats* out);

/* Conservation sums of mass_lb_checks (population total, phi total,
 * non-finite flag) over an FP32 device state such as mass_lb_device_state()
 * returns, computed WITHOUT allocating device memory. This entry point has
 * no counterpart in the reference.
 *
 * For callers that cannot allocate device memory: a program whose HBM is
 * owned in full by another allocator (a framework that reserved it up
 * front, where one more cudaMalloc fails or synchronizes the device), or a
 * monitoring path that must not pay cudaMalloc/cudaFree synchronization.
 * Its scratch is a fixed 163,864-byte __device__ array inside the library,
 * held by every GPU that loads the library until the process exits.
 *
 * planes: nplanes (12 lyotropic, 11 nematic) float planes, plane_stride
 * apart, in the fused layout (g0..g8 as deviations from t_v*rho, Qxx, Qyx,
 * phi); rho: the rest density. Lattices above 67,108,864 sites (8192^2) are
 * rejected with MASS_LB_EINVAL. The device that holds `planes` must be the
 * current device and `stream` must belong to it (a handle's planes live on
 * the device it was created on); otherwise the call returns MASS_LB_EINVAL
 * without launching. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) for that device; make that first call
 * before any stream capture. The looked-up address is kept for the life of
 * the device's context: after a cudaDeviceReset the library, this call
 * included, is not to be used on that device again. The array is shared by all calls and
 * keeps the last call's contents (every call writes all it reads, so
 * nothing needs clearing); calls that overlap on the GPU race on it. Runs on
 * `stream` (a cudaStream_t, NULL = default stream) and returns after the
 * results are on the host. Errors: mass_lb_last_error(). */
int mass_lb_state_sums_noalloc(const float* planes, long long plane_stride, int nplanes,
                               unsigned LX, unsigned LY, double rho, void* stream,
                               double* fsum, double* phisum, int* nonfinite);

/* ---- asynchronous transfers -------------------------------------------------
 * The state's transfers without a wait on the host, for pipelines that keep
 * several lattices busy: one lattice's input goes up and another's result
 * comes down while a third steps. Both take pinned host buffers only
 * (MASS_LB_EINVAL otherwise) and are ordered on the handle's stream with
 * its steps. The host buffers must stay untouched, and `out` unread, until
 * mass_lb_synchronize returns. The copies and their FP64<->FP32 conversion
 * kernels run on a transfer stream of the device's highest priority that
 * is forked from the handle's stream and joined back to it, so that they
 * take the SMs ahead of other handles' queued steps; the order seen on the
 * handle's stream is unchanged.
 *
 * mass_lb_upload_async: mass_lb_upload's work. The totals of the new state
 * (mass_lb_initial_totals) are computed on the stream too and read when
 * first asked for.
 *
 * mass_lb_download_async: mass_lb_download of ff, QQxx, QQyx or phi.
 *
 * End every asynchronous pipeline with mass_lb_synchronize, not with a wait
 * on the stream of one's own: it is the call that reads the fused kernel's
 * device error word (a copy wait that timed out inside a step) and turns it
 * into MASS_LB_ECUDA. A pipeline that only synchronizes the stream could
 * read a result that such a step left incomplete. */
int mass_lb_upload_async(mass_lb_handle* h, const double* ff, const double* QQxx,
                         const double* QQyx, const double* phi);
int mass_lb_download_async(mass_lb_handle* h, int field, double* out);

/* Device-side order between two handles, without a wait on the host: the
 * work queued on `h` after this call starts only when the work queued on
 * `before` up to this call has finished. A pipeline over several lattices
 * uses it to keep their steps one after another (each run of steps then has
 * the whole GPU) while the other lattices' transfers run beside them. The
 * handles may be on different devices; h == before is a no-op. */
int mass_lb_stream_wait(mass_lb_handle* h, mass_lb_handle* before);

/* ---- rows of the primary state: domain decomposition ------------------------
 * The reference runs one lattice in one process (its only mention of MPI is
 * a comment, src/models.hpp:15); these calls have no counterpart there.
 * They let a caller split one periodic lattice into x-slabs, one per GPU:
 * each GPU holds its rows plus 4 halo rows on each side as an ordinary
 * periodic lattice of (rows + 8) x LY sites, and before every step the
 * halo rows are refreshed from the neighbouring slabs. One Step() reaches
 * 4 rows in x (predictor UpdateQuantities, predictor UpdateFields with
 * Move, corrector UpdateQuantities, corrector UpdateFields), so the owned
 * rows then advance exactly as in the whole lattice, bit for bit.
 *
 * mass_lb_rows_layout: planes per site (12 lyotropic: 9 populations, Qxx,
 *   Qyx, phi; 11 nematic) and bytes per value (4 in FP32, where the
 *   populations are stored as deviations from t_v*rho; 8 in FP64).
 * mass_lb_get_rows / mass_lb_put_rows: rows [x0, x0 + nrows) of every
 *   primary plane to / from a DEVICE buffer of the handle's device laid out
 *   [plane][row][y] in that storage format (nplanes * nrows * LY values),
 *   ordered on the handle's stream, no host wait. put_rows replaces state:
 *   it first settles the derived fields the last step left pending.
 *   Lyotropic and nematic periodic lattices (MASS_LB_EUNSUPPORTED
 *   otherwise).
 * mass_lb_checks_rows: mass_lb_checks over rows [x0, x0 + nrows) only (the
 *   owned rows of a slab), for a sum over slabs. Synchronous.
 * mass_lb_set_step_rows: from now on each step writes rows [x0, x0 + nrows)
 *   only (a slab's owned rows; the halo rows' new values would be thrown
 *   away by the next exchange), so the step costs what the owned rows cost.
 *   The rows read still wrap periodically over the lattice. Rows outside
 *   the range are left as they were two steps before. nrows = 0 restores
 *   whole-lattice steps. FP32 fused periodic lattices with npc = 1
 *   (MASS_LB_EUNSUPPORTED otherwise). */
int mass_lb_rows_layout(mass_lb_handle* h, int* nplanes, int* elem_bytes);
int mass_lb_set_step_rows(mass_lb_handle* h, unsigned x0, unsigned nrows);
int mass_lb_get_rows(mass_lb_handle* h, unsigned x0, unsigned nrows, void* dst);
int mass_lb_put_rows(mass_lb_handle* h, unsigned x0, unsigned nrows, const void* src);
int mass_lb_checks_rows(mass_lb_handle* h, unsigned x0, unsigned nrows, double* fsum,
                        double* phisum, int* nonfinite);

/* ---- checkpoints ------------------------------------------------------------
 *
 * Full-precision binary checkpoint of a lattice, filling the role of the
 * reference's unimplemented input archive (src/serialization.hpp:276-286).
 * The file holds a header (model, precision, LX, LY, bc, npc, step count,
 * the conservation totals of the runtime checks, the parameters) and the
 * primary state - ff, QQxx, QQyx, phi and, for go-or-grow, m - as IEEE
 * doubles in the reference's
 * site order, guarded by an FNV-1a checksum. Everything else a step uses is
 * recomputed from these, so a loaded lattice continues bit for bit as if it
 * had never stopped (FP32 values are stored exactly as doubles; an FP32
 * handle writes its populations as the deviations from t_v*rho it holds,
 * format version 2, so that sites near rest keep every bit; version 1
 * files still load). A
 * checkpoint loads into a handle of the same model and lattice size; the
 * precision and boundary may differ. Errors (MASS_LB_EINVAL): unreadable
 * file, wrong magic or version, other model or size, short or corrupted
 * payload. Division-model masks, counters and the RNG state belong to the
 * host model and are not part of the file. */
int mass_lb_save(mass_lb_handle* h, const char* path);
int mass_lb_load(mass_lb_handle* h, const char* path);

/* ---- division models ------------------------------------------------------
 *
 * Hooks for the reference's LyotropicWithDivision (src/models/
 * lyotropic-with-division.cpp), lyotropic and go-or-grow (whose source is
 * chi*phi*r, see below).
 *
 * mass_lb_set_phi_source: per-site phi source rate r (LX*LY host doubles,
 * site order k = y + LY*x). After every UpdateFields (predictor and
 * corrector) phi_tmp += phi*r, which is LyotropicWithDivision::UpdateFields
 * (:111-124) with r = alpha*division_mask - beta*death_mask. The masks
 * themselves are drawn on the host by the caller (SetMasks, :35-106), which
 * uploads the new r whenever they change. NULL removes the source. On FP32
 * fused lattices the source runs in the warp-strip kernel (the tile is
 * re-tuned among those). Ensembles reject runs that carry a source.
 *
 * mass_lb_set_phi_conservation: the conserve_phi correction the division
 * models switch on when division and death are off (:29-30):
 * Dp -= (sum phi - totalphi)/(LX*LY) (src/models/lyotropic.cpp:299), with
 * sum phi taken before each UpdateFields in site order (serially, so FP64
 * results match the serial reference bit for bit; this costs one pass over
 * phi by a single thread per sub-step). totalphi is the sum of phi at
 * Configure() (:152). FP64 and FP32-with-walls only: the fused FP32 kernel
 * has no lattice-wide sum between the halves of a sub-step
 * (MASS_LB_EUNSUPPORTED). */
int mass_lb_set_phi_source(mass_lb_handle* h, const double* rate);
int mass_lb_set_phi_conservation(mass_lb_handle* h, int on, double totalphi);

/* The masks themselves on the device, with the caller's random numbers
 * (SetMasks, :35-106), so that the reference's generator stream stays with
 * the caller while the per-site work and the transfers of phi and of the
 * rate plane disappear.
 *
 * mass_lb_mask_candidates: *count = the number of domain sites with
 * phi >= 0.5. These are the sites that draw one random_real() each, in
 * site order k = y + LY*x. Synchronous.
 *
 * mass_lb_draw_mask: kind 0 (division) or 1 (death). `draws` holds one
 * uniform per candidate site in site order (ndraws must equal the count of
 * the last mass_lb_mask_candidates). A candidate becomes a centre when its
 * draw is below coef*phi*(1 - phi/phi_critical) (division) or coef*phi
 * (death). The mask of that kind becomes the set of sites whose periodic
 * distance (dx, dy) to some centre has dx^2 + dy^2 <= ceil(radius^2).
 * Then the phi source becomes alpha*division_mask - beta*death_mask, as
 * mass_lb_set_phi_source(alpha*dm - beta*de) would set it. Both masks start
 * empty. Asynchronous on the handle's stream; `draws` may be reused as
 * soon as the call returns (it is copied to an internal pinned buffer).
 *
 * mass_lb_get_mask: the current mask of a kind as LX*LY bytes (0/1), site
 * order. */
int mass_lb_mask_candidates(mass_lb_handle* h, long long* count);
int mass_lb_draw_mask(mass_lb_handle* h, int kind, const double* draws, long long ndraws,
                      double coef, double phi_critical, double radius, double alpha, double beta);
int mass_lb_get_mask(mass_lb_handle* h, int kind, unsigned char* out);

/* The same masks without a round trip to the host: the caller supplies
 * uniforms ahead of need, in stream order, and the device takes exactly one
 * per candidate site and mask drawn.
 *
 * mass_lb_mask_supply: append n uniforms to the lattice's queue (a ring of
 * 6*LX*LY + 65536 draws; MASS_LB_EINVAL if the unconsumed draws would not
 * fit). Asynchronous; `u` may be reused on return.
 *
 * mass_lb_mask_staging: a pinned host buffer of at least n doubles that the
 * caller may fill and then pass as `u` to mass_lb_mask_supply, which sends
 * it up without copying it first. It is free to write when this call
 * returns (the previous supply's copy from it has been read); ask again
 * before each fill.
 *
 * mass_lb_draw_masks_queued: `kinds` bit 0 draws the division mask, bit 1
 * the death mask. The candidates are counted on the device. The division
 * mask takes the next `count` queued draws, then the death mask the `count`
 * after those, as the reference draws them. Then the source becomes
 * alpha*division_mask - beta*death_mask, as mass_lb_draw_mask sets it.
 * Asynchronous: one cooperative kernel launch does the whole draw. A
 * caller that keeps at least 2*LX*LY draws unconsumed never
 * runs the queue dry. When it does run dry, the next
 * mass_lb_mask_consumed fails with MASS_LB_EINVAL.
 *
 * mass_lb_mask_consumed: the number of queued draws taken so far, up to and
 * including the last mass_lb_draw_masks_queued (waits for that draw only).
 *
 * mass_lb_mask_progress: the same count as far as the device has got,
 * without waiting: `consumed` after the last queued draw that has finished,
 * and `pending` queued draws issued after it. A caller that keeps
 * 2*LX*LY*(pending + 1) draws beyond `consumed` supplied never runs the
 * queue dry and, with pending <= 2, stays within the ring. */
int mass_lb_mask_supply(mass_lb_handle* h, const double* u, long long n);
int mass_lb_mask_staging(mass_lb_handle* h, long long n, double** buf);
int mass_lb_draw_masks_queued(mass_lb_handle* h, int kinds, double division_coef,
                              double division_radius, double death_coef, double death_radius,
                              double phi_critical, double alpha, double beta);
int mass_lb_mask_consumed(mass_lb_handle* h, long long* consumed);
int mass_lb_mask_progress(mass_lb_handle* h, long long* consumed, int* pending);

/* ---- go-or-grow -----------------------------------------------------------
 *
 * Parameters of the reference's GoOrGrow (src/models/go-or-grow.hpp:9-20,
 * runcard names B, Snem, Dchi, Achi, Ochi, phiswitch, growTogether) and the
 * phi-critical of LyotropicWithDivision. A go-or-grow handle starts with
 * B = Dchi = Achi = Ochi = phiswitch = growTogether = 0, Snem = 1,
 * phi_critical = 1. The growth rate alpha*division_mask - beta*death_mask
 * is mass_lb_set_phi_source's rate r: after every UpdateFields
 * phi += chi*phi*r and m grows by chi*phi*r (times chi when growTogether),
 * src/models/go-or-grow.cpp:329-391. EUNSUPPORTED on other models. */
typedef struct {
  double B, Snem, Dchi, Achi, Ochi, phiswitch, phi_critical;
  int growTogether;
} mass_lb_go_or_grow_params;

int mass_lb_set_go_or_grow_params(mass_lb_handle* h, const mass_lb_go_or_grow_params* p);

/* GoOrGrow::RelaxFreeEnergy (src/models/go-or-grow.cpp:42-119) on the
 * device: `steps` explicit descent steps of phi (relax_phi != 0) and Q
 * (relax_Q != 0) with time step dt, walls as the reference applies them;
 * then *phisum (may be NULL) receives the relaxed total of phi summed in
 * site order, which the reference stores as totalphi, countphi and ptot.
 * Also resets the recorded ptot to that sum. Populations are untouched
 * (the reference's ResetHydrodynamics, :121-141, is an upload of the rest
 * equilibrium). FP64 results equal the reference's bit for bit.
 * Synchronous. EUNSUPPORTED on other models. */
int mass_lb_relax_free_energy(mass_lb_handle* h, unsigned steps, double dt, int relax_phi,
                              int relax_Q, double* phisum);

/* ---- batched ensembles --------------------------------------------------
 *
 * Many independent FP32 periodic lattices, of uneven sizes and parameters,
 * advanced together: one step of every run is ONE persistent kernel launch
 * whose warps pull (run, strip, chunk) work items from a packed list, largest
 * run first, through a device counter; per-run parameters sit in constant
 * memory. Two steps are replayed as one CUDA graph. The reference has no
 * such call: a parameter sweep there is one `mass` process per runcard, each
 * calling Model::Step() from Algorithm() (src/main.cpp:132-197) on its own
 * lattice.
 *
 * Each run is an ordinary FP32 handle (mass_lb_ensemble_run), so the
 * single-lattice calls upload, download, check and measure it; its state
 * after k ensemble steps is bit-identical to k mass_lb_step calls on the
 * fused single-lattice path. All runs share one model and use npc = 1; every
 * LY must be a multiple of 4 and at least 64. At most 192 runs are active on
 * a device at a time, across all ensembles. */
typedef struct mass_lb_ensemble mass_lb_ensemble;

int mass_lb_ensemble_create(int nruns, const mass_lb_params* params, const unsigned* LX,
                            const unsigned* LY, mass_lb_ensemble** out);
void mass_lb_ensemble_destroy(mass_lb_ensemble* e);
int mass_lb_ensemble_size(mass_lb_ensemble* e);
/* the handle of run i (owned by the ensemble; NULL if i is out of range) */
mass_lb_handle* mass_lb_ensemble_run(mass_lb_ensemble* e, int i);
/* nsteps steps of every run; returns after they are done. The first call
 * picks the chunk height by timing (MASS_LB_ENSEMBLE_ROWS=<n> fixes it). */
int mass_lb_ensemble_step(mass_lb_ensemble* e, unsigned nsteps);
/* chunk height in rows (0 before the first step) */
int mass_lb_ensemble_get_rows(mass_lb_ensemble* e);

#ifdef __cplusplus
}
#endif
#endif
