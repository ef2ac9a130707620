/* mass_lb.h - C ABI of the Blackwell (sm_100a) implementation of the MASS
 * lyotropic / nematic time step.
 *
 * This is the drop-in boundary beneath the reference's model plugin API:
 * a Model subclass registered with declare_model<T>(name, desc)
 * (src/models.hpp:197-205 of the reference) owns one handle and forwards
 *   Model::Initialize()      -> mass_lb_create       (src/models.hpp:60)
 *   Model::Configure()       -> mass_lb_upload       (src/models.hpp:67)
 *   Model::Step()            -> mass_lb_step         (src/models.hpp:86)
 *   Model::RuntimeChecks()   -> mass_lb_checks       (src/models.hpp:101)
 *   serialize_frame()        -> mass_lb_download     (src/models/lyotropic.hpp:121-138,
 *                                                     src/models/nematic.hpp:103-108)
 * The reference itself is CPU-only and has no FFI; these entry points are
 * the calls that its Lyotropic / Nematic members would make
 * (src/models/lyotropic.cpp:500-549, src/models/nematic.cpp:370-407).
 *
 * Conventions
 *  - Every function returns 0 (MASS_LB_OK) or a negative mass_lb_status.
 *    Nothing throws across this boundary. mass_lb_last_error() gives text.
 *  - The caller owns host buffers; the library owns device buffers.
 *  - Host arrays use the reference's layout: site index k = y + LY*x
 *    (src/geometry.hpp:430), populations site-major ff[9*k + v] with the D2Q9
 *    order of src/geometry.hpp:17-27.
 *  - One CUDA stream per handle. A handle is not thread-safe; distinct
 *    handles may be used from distinct threads.
 */
#ifndef MASS_LB_H_
#define MASS_LB_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MASS_LB_ABI_VERSION 1

typedef struct mass_lb_handle mass_lb_handle;

/* MASS_LB_GO_OR_GROW: the reference's GoOrGrow (src/models/go-or-grow.cpp),
 * the lyotropic model with a crowding penalty, a preferred nematic order and
 * a phenotype density m = phi*chi (chi = 1 grow, 0 go). Its extra parameters
 * are set by mass_lb_set_go_or_grow_params (mass_lb_ext.h). */
enum mass_lb_model { MASS_LB_LYOTROPIC = 0, MASS_LB_NEMATIC = 1, MASS_LB_GO_OR_GROW = 2 };

/* MASS_LB_FP64: the oracle mode. Unfused sweeps in the reference's own
 *   evaluation order, no FMA contraction, IEEE division: agrees with the
 *   reference's double-precision build bit for bit on identical inputs.
 * MASS_LB_FP32: the production mode. Populations stored as deviations from
 *   the rest state t_v*rho, one fused sm_100a kernel per time step
 *   (periodic lattices), FP32 arithmetic, FP64 conservation sums. */
enum mass_lb_precision { MASS_LB_FP64 = 0, MASS_LB_FP32 = 1 };

enum mass_lb_status {
  MASS_LB_OK = 0,
  MASS_LB_EINVAL = -1,        /* bad argument */
  MASS_LB_ECUDA = -2,         /* CUDA runtime error (see last_error) */
  MASS_LB_ENOMEM = -3,        /* device allocation failed */
  MASS_LB_EUNSUPPORTED = -4,  /* option/field not available in this mode */
  MASS_LB_ENOTFINITE = -5,    /* NaN/Inf found in the state */
  MASS_LB_ENODEV = -6         /* no CUDA device / not sm_100 */
};

/* Model parameters, named as the reference's runcard options.
 * Lyotropic: src/models/lyotropic.cpp:556-599 (conc is the "conc" config
 *   option, used by the zetaI term at :236-240).
 * Nematic: src/models/nematic.cpp:414-435; pass Gamma in GammaQ and tau in
 *   tauNem (tauIso, GammaP, AA, KK, zetaI, conc are ignored). Thermal noise
 *   (Q_kBT, u_kBT) is not supported: those must be 0 in the caller. */
typedef struct {
  int model;
  double GammaQ, GammaP, xi, tauNem, tauIso, rho, friction;
  double AA, CC, LL, KK, zeta, zetaI, conc;
  unsigned npc;
} mass_lb_params;

/* Field identifiers for mass_lb_download / mass_lb_upload_field. */
enum mass_lb_field {
  /* primary state (also accepted by mass_lb_upload_field) */
  MASS_LB_FF = 0,        /* LX*LY*9 */
  MASS_LB_QQXX = 1,
  MASS_LB_QQYX = 2,
  MASS_LB_PHI = 3,       /* lyotropic only */
  /* values computed by the last UpdateQuantities() of the last step (the
   * corrector), exactly what the reference holds in these members when
   * WriteFrame() runs */
  MASS_LB_N = 4, MASS_LB_UX = 5, MASS_LB_UY = 6,
  MASS_LB_UX_PHI = 7, MASS_LB_UY_PHI = 8,
  MASS_LB_HHXX = 9, MASS_LB_HHYX = 10, MASS_LB_MU = 11,
  MASS_LB_DXQQXX = 12, MASS_LB_DYQQXX = 13, MASS_LB_DXQQYX = 14, MASS_LB_DYQQYX = 15,
  MASS_LB_SIGMAXX = 16, MASS_LB_SIGMAYY = 17, MASS_LB_SIGMAYX = 18, MASS_LB_SIGMAXY = 19,
  MASS_LB_SIGMA_BULK = 20, MASS_LB_SIGMA_ELASTIC_XX = 21, MASS_LB_SIGMA_ELASTIC_YX = 22,
  MASS_LB_SIGMA_PHASE_FIELD_XX = 23, MASS_LB_SIGMA_PHASE_FIELD_YX = 24,
  MASS_LB_SIGMA_ACTIVE_XX = 25, MASS_LB_SIGMA_ACTIVE_YX = 26,
  /* step-internal predictor values (FP64 mode only) */
  MASS_LB_FN = 27,       /* LX*LY*9 */
  MASS_LB_QNXX = 28, MASS_LB_QNYX = 29, MASS_LB_PHN = 30,
  /* go-or-grow only: the phenotype density m (primary state, uploadable),
   * chi = m/phi (derived from m and phi), and m's predictor (FP64 only) */
  MASS_LB_M = 31, MASS_LB_CHI = 32, MASS_LB_MN = 33,
  MASS_LB_NUM_FIELDS = 34
};

/* ABI version compiled into the library (== MASS_LB_ABI_VERSION). */
int mass_lb_abi_version(void);

/* Text of the last error on the calling thread ("" if none). */
const char* mass_lb_last_error(void);

/* Name of a field as it appears in the reference's frame JSON / members
 * ("ff", "QQxx", "sigma_bulk", ...), or NULL for an invalid id. */
const char* mass_lb_field_name(int field);

/* Create a handle on the current CUDA device: allocate the device state for
 * an LX x LY lattice with boundary flag `bc` (0 = periodic; 1..4 = the
 * reference's channel/box walls; >= 5 = periodic with a ghost layer, which
 * computes the same values as 0). The state is zero until uploaded.
 * Replaces Model::Initialize() (src/models/lyotropic.cpp:23-67). */
int mass_lb_create(const mass_lb_params* params, unsigned LX, unsigned LY,
                   unsigned bc, int precision, mass_lb_handle** out);

/* Free every device resource of the handle. NULL is accepted. */
void mass_lb_destroy(mass_lb_handle* h);

/* Upload the primary state from host memory: ff (LX*LY*9, site-major),
 * QQxx, QQyx (LX*LY) and, for lyotropic and go-or-grow, phi (LX*LY; may be
 * NULL for the nematic model). Replaces the state written by
 * Model::Configure() (src/models/lyotropic.cpp:149-156). Synchronous. Also
 * records the reference totals used by mass_lb_checks (ftot, ptot). A
 * go-or-grow lattice keeps its m (zero until uploaded with
 * mass_lb_upload_field) and recomputes chi = m/phi. */
int mass_lb_upload(mass_lb_handle* h, const double* ff, const double* QQxx,
                   const double* QQyx, const double* phi);

/* Advance `nsteps` calls of Model::Step() (src/models/lyotropic.cpp:500-525,
 * src/models/nematic.cpp:370-395). Asynchronous on the handle's stream. */
int mass_lb_step(mass_lb_handle* h, unsigned nsteps);

/* Copy one field to host memory (LX*LY doubles, or LX*LY*9 for FF / FN).
 * Synchronous. In FP32 mode the derived fields (N .. SIGMA_ACTIVE_YX) are
 * produced by re-running the last step from the retained previous state
 * with the diagnostic outputs enabled (the state itself is unchanged).
 * Returns MASS_LB_EUNSUPPORTED for FN, QNXX, QNYX, PHN, MN in FP32 mode, for PHI and the
 * phase-field fields in the nematic model, for M, CHI, MN outside go-or-grow,
 * or when no step has run yet for a derived field in FP32 mode. */
int mass_lb_download(mass_lb_handle* h, int field, double* out);

/* FP64 sums used by Model::RuntimeChecks() (src/models/lyotropic.cpp:527-549):
 * total of all populations and of phi over the domain, Kahan-compensated on
 * the device, and a flag that is 1 if any state value is NaN or Inf.
 * Any pointer may be NULL. Synchronous. */
int mass_lb_checks(mass_lb_handle* h, double* fsum, double* phisum, int* nonfinite);

/* Totals recorded at upload time (ftot, ptot of the reference). */
int mass_lb_initial_totals(mass_lb_handle* h, double* ftot, double* ptot);

/* Block until all work queued on the handle's stream is done. */
int mass_lb_synchronize(mass_lb_handle* h);

/* The handle's cudaStream_t (as void*), for callers that time or order
 * work around mass_lb_step. */
void* mass_lb_stream(mass_lb_handle* h);

/* Number of kernel launches one mass_lb_step(h, 1) issues. */
int mass_lb_launches_per_step(mass_lb_handle* h);

#ifdef __cplusplus
}
#endif
#endif
