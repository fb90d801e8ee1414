/*
 * TEST INFRASTRUCTURE ONLY.  Plain-C restatement of the reference's
 * Cahn-Hilliard step and its seeded initial condition, used by the tests,
 * the smoke check and the CPU-baseline leg of the benchmark as the oracle.
 * Nothing in the product path links or calls it.
 *
 * Layout: dense, x fastest, no ghost nodes: index x + nx*(y + ny*z).
 * Parity is pinned against the reference CPU build (oracle/_ref, built from
 * the reference's own SfieldFD/Rand sources) by tests/test_oracle.py and by
 * the golden fixtures in tests/golden/.
 */
#ifndef MB_CH_ORACLE_H
#define MB_CH_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mersenne twister MT19937 as in the reference's Rand class (rand.cpp). */
typedef struct {
    uint32_t mt[624];
    uint32_t index;
} cho_rand;

void cho_rand_init(cho_rand* r, uint32_t seed);
uint32_t cho_rand_u32(cho_rand* r);
double cho_rand_uniform(cho_rand* r);
double cho_rand_normal(cho_rand* r);

/* Seeded initial condition (reference loop order x, y, z; see ch_oracle.c). */
void cho_ic(const int dims[3], double co, double amp, int gaussian, uint32_t seed, double* out);

/* One explicit step; bc[d] = 1 periodic, 0 no-flux.  `mu` is scratch of the
 * field's size.  c_out may not alias c_in. */
void cho_step(const int dims[3], const double spacing[3], double dt, double M, double kap,
              const int bc[3], const double* c_in, double* c_out, double* mu);

/* nsteps steps; c holds the initial field and receives the result. */
int cho_run(const int dims[3], const double spacing[3], double dt, double M, double kap,
            const int bc[3], double* c, int nsteps);

/* Diagnostics of a field:
 *  out[0] mass        sum(c)*dV, Neumaier-compensated, x-fastest order
 *  out[1] mass_plain  sum(c)*dV, plain left-to-right sum
 *  out[2] energy      sum[(c^2-1)^2/4 + kap/2 |grad+ c|^2]*dV, compensated,
 *                     forward differences with the boundary flags bc
 *  out[3] abs_mass    sum|c|*dV, compensated
 *  out[4] max_abs     max|c|
 *  out[5] nonfinite   number of NaN/Inf sites */
void cho_reduce(const int dims[3], const double spacing[3], double kap, const int bc[3],
                const double* c, double out[6]);

/* Same diagnostics for a float32 field (values widened to double). */
void cho_reduce_f32(const int dims[3], const double spacing[3], double kap, const int bc[3],
                    const float* c, double out[6]);

#ifdef __cplusplus
}
#endif

#endif
