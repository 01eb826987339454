/* accel_oracle.h — TEST INFRASTRUCTURE ONLY: the CPU oracle for the tracking path.
 *
 * A plain-C restatement of the reference's per-particle integrators and element passes, working
 * on the same accel_elem_desc descriptors as the engine's C-ABI.  Its arithmetic keeps the
 * reference's operation order so that, built without FMA contraction, it is bit-identical to the
 * reference library (checked against oracle/_ref and the committed golden fixtures).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the product never does.
 */
#ifndef ACCEL_ORACLE_H
#define ACCEL_ORACLE_H
#include <stdint.h>
#include "accel_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Gaussian source for quantum excitation (statistical parity only): state is a 64-bit seed. */
typedef struct orc_rng { uint64_t s[2]; int have; double spare; } orc_rng;
void   orc_rng_seed(orc_rng* g, uint64_t seed);
double orc_gauss(orc_rng* g);

/* Element pass over N AoS particles; lost particles (x NaN) are skipped. */
int  orc_pass_element(const accel_elem_desc* e, double* r, int N, orc_rng* g);
/* Elements [st, ed) over N particles; OpenMP blocks over particles like ALine::pass when
 * nthreads > 1 (wake elements always see the whole beam). */
int  orc_pass_line(const accel_elem_desc* el, int n, double* r, int N, int st, int ed,
                   int nthreads, orc_rng* g);
/* nturn turns with the per-turn NaN scan; loss_turn may be NULL. */
int  orc_track(const accel_elem_desc* el, int n, double* r, int N, int nturn, int32_t* loss_turn,
               int nthreads, uint64_t seed);
/* Central-difference 6x6 matrix over [st, ed) around (0,0,0,0,0,dpp) (ALine::getm66). */
void orc_m66(const accel_elem_desc* el, int n, int st, int ed, double dpp, double delta,
             double* m36);
/* Same around an arbitrary point r0. */
void orc_m66_at(const accel_elem_desc* el, int n, int st, int ed, const double* r0, double delta,
                double* m36);
/* Beam moments (calc_beam_stat). */
int  orc_beam_stat(const double* r, int N, double* mean, double* sigma, double* cross);
/* Apply one-turn radiation/cavity/wake flags as ALine::set_*_onoff do. */
void orc_set_flags(accel_elem_desc* el, int n, int rad_flag, int cavity_on, int wake_on);

#ifdef __cplusplus
}
#endif
#endif
