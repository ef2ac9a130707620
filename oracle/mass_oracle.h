/* CPU oracle for the MASS lyotropic / nematic Model::Step() hot path.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C, FP64, single-threaded restatement of
 * the reference algorithm, used by the tests and by bench.py's CPU-baseline
 * leg as the checker. The product (mass_hd_b200/, include/mass_lb.h) never
 * links or calls it.
 *
 * Parity: pinned against the reference's own model sources compiled in
 * oracle/_ref (golden fixtures in tests/golden/, generated by
 * tests/golden/gen_golden.py). Every arithmetic expression keeps the
 * reference's evaluation order so that results agree bit for bit.
 */
#ifndef MASS_ORACLE_H_
#define MASS_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

enum { MO_LYOTROPIC = 0, MO_NEMATIC = 1 };

/* Runcard parameters. Lyotropic names follow src/models/lyotropic.cpp:556-583.
 * The nematic model uses Gamma -> GammaQ and tau -> tauNem (tauIso unused). */
typedef struct {
  int model;
  double GammaQ, GammaP, xi, tauNem, tauIso, rho, friction;
  double AA, CC, LL, KK, zeta, zetaI, conc;
  unsigned npc;
} mo_params;

typedef struct mo_state mo_state;

mo_state* mo_new(const mo_params* p, unsigned LX, unsigned LY, unsigned BC);
void mo_free(mo_state* s);
/* Domain values; "ff"/"fn" are LX*LY*9 site-major, other fields LX*LY. */
int mo_set_field(mo_state* s, const char* name, const double* src);
int mo_get_field(mo_state* s, const char* name, double* dst);
void mo_step(mo_state* s, unsigned nsteps);
/* Sum of all populations / of phi over the domain (RuntimeChecks sums). */
void mo_totals(mo_state* s, double* fsum, double* phisum);

#ifdef __cplusplus
}
#endif
#endif
