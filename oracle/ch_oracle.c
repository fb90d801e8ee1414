/*
 * TEST INFRASTRUCTURE ONLY: the oracle for the GPU path (see ch_oracle.h).
 * Compiled with -ffp-contract=off so that every product and sum is rounded
 * separately, in the order written, as in the reference's x86-64 build.
 */
#include "ch_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- Mersenne twister: rand.cpp:24-36 (init), :38-55 (twist),
 *      :58-78 (tempering), :81-84 (uniform), :87-94 (normal).
 *      The constants are MT19937's published parameters (rand.hpp:29-52). */

void cho_rand_init(cho_rand* r, uint32_t seed)
{
    r->mt[0] = seed;
    for (uint32_t i = 1; i < 624; i++)
        r->mt[i] = 1812433253u * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + i;
    r->index = 624;
}

static void cho_rand_twist(cho_rand* r)
{
    for (uint32_t i = 0; i < 624; i++) {
        uint32_t x = (r->mt[i] & 0x80000000u) + (r->mt[(i + 1) % 624] & 0x7fffffffu);
        uint32_t xa = x >> 1;
        if (x & 1u) xa ^= 0x9908B0DFu;
        r->mt[i] = r->mt[(i + 397) % 624] ^ xa;
    }
    r->index = 0;
}

uint32_t cho_rand_u32(cho_rand* r)
{
    if (r->index >= 624) cho_rand_twist(r);
    uint32_t y = r->mt[r->index++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9D2C5680u;
    y ^= (y << 15) & 0xEFC60000u;
    y ^= (y >> 18);
    return y;
}

double cho_rand_uniform(cho_rand* r) { return (double)cho_rand_u32(r) / (double)4294967295u; }

double cho_rand_normal(cho_rand* r)
{
    double u1 = cho_rand_uniform(r);
    double u2 = cho_rand_uniform(r);
    /* the reference's Box-Muller uses this literal for pi (rand.cpp:92) */
    return sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265359 * u2);
}

/* ---- initial condition: TIPSphil::initPhaseField loop order
 *      (TIPSphil.cpp:86-96: i outer, j, k inner) with the seeded generator.
 *      uniform: co + amp*(u - 0.5); gaussian: co + amp*normal(). */
void cho_ic(const int dims[3], double co, double amp, int gaussian, uint32_t seed, double* out)
{
    cho_rand r;
    cho_rand_init(&r, seed);
    const size_t nx = (size_t)dims[0], ny = (size_t)dims[1], nz = (size_t)dims[2];
    for (size_t i = 0; i < nx; i++)
        for (size_t j = 0; j < ny; j++)
            for (size_t k = 0; k < nz; k++) {
                double v = gaussian ? co + amp * cho_rand_normal(&r)
                                    : co + amp * (cho_rand_uniform(&r) - 0.5);
                out[i + nx * (j + ny * k)] = v;
            }
}

/* ---- neighbours.  Ghost values of SfieldFD::updateBoundaries
 *      (SfieldFD.cpp:187-251; x via mpiBorderExchange :260-288 with np == 1):
 *      periodic: ghost 0 = n-1, ghost n+1 = 0;  no-flux: ghost 0 = 0,
 *      ghost n+1 = n-1 (in 0-based interior indices). */
static inline size_t nb_minus(size_t i, size_t n, int periodic)
{
    if (i > 0) return i - 1;
    return periodic ? n - 1 : 0;
}
static inline size_t nb_plus(size_t i, size_t n, int periodic)
{
    if (i + 1 < n) return i + 1;
    return periodic ? 0 : n - 1;
}

/* 7-point Laplacian in the reference's operation order
 * (SfieldFD.cpp:296-302 and :310-325):
 *   ((a[+x] + a[-x] - 2*a)/dx2 + (a[+y] + a[-y] - 2*a)/dy2) + (a[+z] + a[-z] - 2*a)/dz2 */
static inline double lap7(const double* a, size_t x, size_t y, size_t z, const size_t n[3],
                          const int bc[3], double dx2, double dy2, double dz2)
{
    const size_t sy = n[0], sz = n[0] * n[1];
    const size_t c = x + sy * y + sz * z;
    const double a0 = a[c];
    const double xp = a[nb_plus(x, n[0], bc[0]) + sy * y + sz * z];
    const double xm = a[nb_minus(x, n[0], bc[0]) + sy * y + sz * z];
    const double yp = a[x + sy * nb_plus(y, n[1], bc[1]) + sz * z];
    const double ym = a[x + sy * nb_minus(y, n[1], bc[1]) + sz * z];
    const double zp = a[x + sy * y + sz * nb_plus(z, n[2], bc[2])];
    const double zm = a[x + sy * y + sz * nb_minus(z, n[2], bc[2])];
    const double lapx = (xp + xm - 2 * a0) / (dx2);
    const double lapy = (yp + ym - 2 * a0) / (dy2);
    const double lapz = (zp + zm - 2 * a0) / (dz2);
    return lapx + lapy + lapz;
}

/* One step of the CHBasic model (oracle/refmodel/CHBasic.cpp, after
 * TIPSphil::updatePhaseField, TIPSphil.cpp:113-211):
 *   mu    = (c*c*c - c) - kap*lap(c)
 *   c_out = c + lap(mu)*(dt*M)         (operator*(double) :544-550, then += :438-442) */
void cho_step(const int dims[3], const double spacing[3], double dt, double M, double kap,
              const int bc[3], const double* c_in, double* c_out, double* mu)
{
    const size_t n[3] = {(size_t)dims[0], (size_t)dims[1], (size_t)dims[2]};
    const double dx2 = spacing[0] * spacing[0];
    const double dy2 = spacing[1] * spacing[1];
    const double dz2 = spacing[2] * spacing[2];
    const double dtM = dt * M;
    for (size_t z = 0; z < n[2]; z++)
        for (size_t y = 0; y < n[1]; y++)
            for (size_t x = 0; x < n[0]; x++) {
                const size_t i = x + n[0] * (y + n[1] * z);
                const double cc = c_in[i];
                const double df = cc * cc * cc - cc;
                const double lapc = lap7(c_in, x, y, z, n, bc, dx2, dy2, dz2);
                mu[i] = df - kap * lapc;
            }
    for (size_t z = 0; z < n[2]; z++)
        for (size_t y = 0; y < n[1]; y++)
            for (size_t x = 0; x < n[0]; x++) {
                const size_t i = x + n[0] * (y + n[1] * z);
                const double lapmu = lap7(mu, x, y, z, n, bc, dx2, dy2, dz2);
                c_out[i] = c_in[i] + lapmu * dtM;
            }
}

int cho_run(const int dims[3], const double spacing[3], double dt, double M, double kap,
            const int bc[3], double* c, int nsteps)
{
    const size_t count = (size_t)dims[0] * dims[1] * dims[2];
    double* tmp = (double*)malloc(count * sizeof(double));
    double* mu = (double*)malloc(count * sizeof(double));
    if (!tmp || !mu) {
        free(tmp);
        free(mu);
        return -1;
    }
    for (int s = 0; s < nsteps; s++) {
        cho_step(dims, spacing, dt, M, kap, bc, c, tmp, mu);
        memcpy(c, tmp, count * sizeof(double));
    }
    free(tmp);
    free(mu);
    return 0;
}

/* ---- diagnostics (no reference counterpart: the reference logs neither
 *      mass nor energy).  Neumaier's compensated sum. */
typedef struct {
    double s, c;
} cho_ksum;

static inline void ks_add(cho_ksum* k, double v)
{
    double t = k->s + v;
    if (fabs(k->s) >= fabs(v))
        k->c += (k->s - t) + v;
    else
        k->c += (v - t) + k->s;
    k->s = t;
}

#define CHO_REDUCE_BODY(T)                                                                \
    const size_t n[3] = {(size_t)dims[0], (size_t)dims[1], (size_t)dims[2]};              \
    const double dv = spacing[0] * spacing[1] * spacing[2];                               \
    cho_ksum mass = {0, 0}, energy = {0, 0}, absm = {0, 0};                               \
    double plain = 0.0, maxabs = 0.0, nonfinite = 0.0;                                    \
    for (size_t z = 0; z < n[2]; z++)                                                     \
        for (size_t y = 0; y < n[1]; y++)                                                 \
            for (size_t x = 0; x < n[0]; x++) {                                           \
                const size_t i = x + n[0] * (y + n[1] * z);                               \
                const double v = (double)c[i];                                            \
                if (!isfinite(v)) {                                                       \
                    nonfinite += 1.0;                                                     \
                    continue;                                                             \
                }                                                                         \
                const double gx = ((double)c[nb_plus(x, n[0], bc[0]) + n[0] * (y + n[1] * z)] - v) / spacing[0]; \
                const double gy = ((double)c[x + n[0] * (nb_plus(y, n[1], bc[1]) + n[1] * z)] - v) / spacing[1]; \
                const double gz = ((double)c[x + n[0] * (y + n[1] * nb_plus(z, n[2], bc[2]))] - v) / spacing[2]; \
                const double w = v * v - 1.0;                                             \
                const double f = 0.25 * w * w + 0.5 * kap * (gx * gx + gy * gy + gz * gz); \
                ks_add(&mass, v);                                                         \
                ks_add(&absm, fabs(v));                                                   \
                ks_add(&energy, f);                                                       \
                plain += v;                                                               \
                if (fabs(v) > maxabs) maxabs = fabs(v);                                   \
            }                                                                             \
    out[0] = (mass.s + mass.c) * dv;                                                      \
    out[1] = plain * dv;                                                                  \
    out[2] = (energy.s + energy.c) * dv;                                                  \
    out[3] = (absm.s + absm.c) * dv;                                                      \
    out[4] = maxabs;                                                                      \
    out[5] = nonfinite;

void cho_reduce(const int dims[3], const double spacing[3], double kap, const int bc[3],
                const double* c, double out[6])
{
    CHO_REDUCE_BODY(double)
}

void cho_reduce_f32(const int dims[3], const double spacing[3], double kap, const int bc[3],
                    const float* c, double out[6])
{
    CHO_REDUCE_BODY(float)
}
