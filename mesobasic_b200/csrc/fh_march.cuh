// Fused variable-mobility step (TIPSphil, TIPSbathPHIL, SIPS and a field of
// SIPSternary) on the z-marching skeleton of the Cahn-Hilliard kernels: one
// launch per step, one pass over HBM (read c, write c_new), FP64 with every
// operation rounded on its own in the reference's order.
//
// Reference step (TIPSphil::updatePhaseField, TIPSphil.cpp:113-211):
//     c.updateBoundaries;  mu, mob per site (Flory-Huggins, Phillies)
//     mu.updateBoundaries; mob.updateBoundaries
//     c += dt * mu.Laplacian(mob)          SfieldFD.cpp:333-355
//     c += dt * noise * (r - 0.5)          TIPSphil.cpp:200-209
//
// A work item is a y-tile of ty rows x a z-chunk; the CTA marches through
// the chunk's planes.  Per plane i:
//   stage A: mu and 1/mob on the ty+2 rows y0-1..y0+ty of plane i (c rows
//            y0-2..y0+ty+1 come through a TMA ring, halo 2); mu and 1/mob
//            go to 3-slot shared-memory rings, never to HBM;
//   stage B: div(mob grad mu) on plane i-1 with the harmonic-mean face
//            mobilities 2/(1/mob_a + 1/mob_b) -- the reciprocals are formed
//            once per site in stage A and reused by all six faces that touch
//            the site, where the reference divides again for each face (the
//            same operands in the same order, so the same values) -- then
//            c_new = c + dt*lap and the noise term, stored to HBM.
// A thread owns 4 consecutive x of one row (32 bytes), so its sites form one
// group of the noise generator's counter (site/4).
// Boundaries as updateBoundaries (SfieldFD.cpp:187-251): periodic axes wrap;
// on a no-flux axis the ghost equals the adjacent interior node, for c (the
// ring loads clamped rows and planes) and for mu and mob (the centre value
// is substituted for an out-of-domain neighbour).
// The per-x constants of the step (temperature, chi, the SIPS mobility
// scale) are computed once per item into a shared-memory table (fh_column).
#pragma once

#include "ch_device.cuh"

namespace mg {

constexpr int kFhBlock = 512;  // threads of the fused variable-mobility kernel
constexpr int kFhMaxNx = 256;  // one TMA box per row

__device__ __forceinline__ void lds4d(uint32_t a, double (&v)[4])
{
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "r"(a) : "memory");
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v[2]), "=d"(v[3]) : "r"(a + 16u) : "memory");
}
__device__ __forceinline__ void sts4d(uint32_t a, const double (&v)[4])
{
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v[0]), "d"(v[1]) : "memory");
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a + 16u), "d"(v[2]), "d"(v[3]) : "memory");
}
__device__ __forceinline__ double lds1d(uint32_t a)
{
    double x;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(x) : "r"(a) : "memory");
    return x;
}

// Shared memory: head | c ring NBUF x cplane | mu ring 3 x mplane |
// 1/mob ring 3 x mplane | column table kFhMaxNx x FhCol (doubles throughout).
template <int NBUF, bool FLAT>
__global__ void __launch_bounds__(kFhBlock, 1) fh_march_kernel(StepArgs a)
{
    step_counts(a);
    using A = Arith<double>;
    constexpr int U = (NBUF % 3 == 0) ? NBUF : 3 * NBUF;

    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* smem_raw = smem_dyn + ((128u - (smem_addr(smem_dyn) & 127u)) & 127u);
    SmemHead* head = reinterpret_cast<SmemHead*>(smem_raw);
    const uint32_t cbase = smem_addr(smem_raw) + (uint32_t)(((sizeof(SmemHead) + 127) / 128) * 128);
    const uint32_t cplaneB = (uint32_t)a.cplane * 8u, mplaneB = (uint32_t)a.mplane * 8u;
    const uint32_t mubase = cbase + NBUF * cplaneB;
    const uint32_t rmbase = mubase + 3u * mplaneB;
    FhCol* coltab = reinterpret_cast<FhCol*>(smem_raw + (rmbase + 3u * mplaneB - smem_addr(smem_raw)));
    const uint32_t bar0 = smem_addr(&head->bar[0]);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&head->bar[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t ph = 0;

    for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
        const int j = find_job(a.item_begin, a.njobs, item);
        JobDev* J = a.jobs + __ldg(a.job_slot + j);
        const int local = item - __ldg(a.item_begin + j);
        if (tid == 0) head->step = *((volatile long long*)&J->step);
        __syncthreads();
        const long long step = head->step;
        if (step >= J->target) {
            __syncthreads();
            continue;
        }
        const FhDev& F = *J->fh;
        const int nx = J->nx, ny = J->ny, nz = J->nz;
        const int flags = J->flags;
        const bool perX = flags & JF_PER_X, perY = flags & JF_PER_Y, perZ = flags & JF_PER_Z;
        const bool divX = flags & JF_DIV_X, divY = flags & JF_DIV_Y, divZ = flags & JF_DIV_Z;
        const double cx = J->cx, cy = J->cy, cz = J->cz, kap = J->kap, dt = J->dtM_dt;
        const double cs = (double)(step + 1);  // the step being taken (PFApp's current_step)
        const int par = (int)(step & 1);
        const double* __restrict__ src = static_cast<const double*>(J->buf[par]);
        double* __restrict__ dst = static_cast<double*>(J->buf[par ^ 1]);
        (void)src;
        const CUtensorMap* tm_body = J->tmap + 2 * par;
        const CUtensorMap* tm_row = J->tmap + 2 * par + 1;

        // per-x constants of this step
        for (int x = tid; x < nx; x += blockDim.x) coltab[x] = fh_column(F, x, cs, dt);

        // ---- tile geometry
        const int ty = FLAT ? 1 : J->ty;
        const int CY = FLAT ? 1 : ty + 4, MY = FLAT ? 1 : ty + 2;
        const uint32_t rowB = (uint32_t)nx * 8u;
        const uint32_t plane_bytes = (uint32_t)CY * rowB;
        const long long pstride = (long long)nx * ny;
        const int tile = local % J->ntile, chunk = local / J->ntile;
        const int own_lo = FLAT ? 0 : tile * ty;
        const int own_hi = FLAT ? 1 : min(ny, own_lo + ty);
        const int y0 = FLAT ? 0 : min(own_lo, ny - ty);
        const int zs = (int)((long long)chunk * nz / J->nchunk);
        const int ze = (int)((long long)(chunk + 1) * nz / J->nchunk);
        const int L = ze - zs;
        const int dir = (chunk & 1) ? -1 : 1;
        const int zfirst = dir > 0 ? zs - 2 : ze + 1;
        const int yh0 = FLAT ? 0 : wrap_or_clamp(y0 - 2, ny, perY);
        const int yh1 = FLAT ? 0 : wrap_or_clamp(y0 - 1, ny, perY);
        const int yh2 = FLAT ? 0 : wrap_or_clamp(y0 + ty, ny, perY);
        const int yh3 = FLAT ? 0 : wrap_or_clamp(y0 + ty + 1, ny, perY);

        // ---- thread geometry: strip q (x0 = 4q) of mu row m
        const int nq = nx >> 2;
        const bool active = tid < nq * MY;
        const int m = active ? tid / nq : 0;
        const int x0 = 4 * (tid % nq);
        const int y = FLAT ? 0 : y0 - 1 + m;
        const bool outrow = active && (FLAT || (m >= 1 && m <= ty && y >= own_lo && y < own_hi));
        // no-flux y: the neighbour row lies outside the domain
        const bool subUp = !FLAT && !perY && y - 1 < 0;
        const bool subDn = !FLAT && !perY && y + 1 >= ny;
        const int xl = wrap_or_clamp(x0 - 1, nx, perX), xr = wrap_or_clamp(x0 + 4, nx, perX);
        const int crow = FLAT ? 0 : m + 1;  // c row of the strip in a ring plane
        const uint32_t cOwn = (uint32_t)(crow * nx + x0) * 8u;
        const uint32_t cRow = (uint32_t)(crow * nx) * 8u;
        const uint32_t mOwn = (uint32_t)(m * nx + x0) * 8u, mRow = (uint32_t)(m * nx) * 8u;
        const long long site_row = (long long)max(y, 0) * nx + x0;
        double* g = dst + (long long)zfirst * pstride + site_row;
        const long long gstep = (long long)dir * pstride;
        const bool noisy = J->noise != 0.0;
        const bool linear = F.model == kFhLinear;
        const double noise = J->noise, cutoff = J->noise_cutoff;
        const uint2 key = make_uint2((uint32_t)J->noise_seed, (uint32_t)(J->noise_seed >> 32));
        const long long st = step + 1;  // the noise counter's step (the step just taken)

        const int producer = (MY - 1) * nq;
        const int nplanes = L + 4;
        auto issue = [&](int p, int slot) {
            const uint32_t dp = cbase + (uint32_t)slot * cplaneB;
            const uint32_t bar = bar0 + 8u * (uint32_t)slot;
            const int zc = wrap_or_clamp(zfirst + dir * p, nz, perZ);
            mbar_arrive_expect_tx(&head->bar[slot], plane_bytes + a.tx_extra);
            if (FLAT) {
                tma_load_3d_s(dp, tm_row, bar, 0, 0, zc);
            } else {
                tma_load_3d_s(dp, tm_row, bar, 0, yh0, zc);
                tma_load_3d_s(dp + rowB, tm_row, bar, 0, yh1, zc);
                tma_load_3d_s(dp + 2 * rowB, tm_body, bar, 0, y0, zc);
                tma_load_3d_s(dp + (uint32_t)(ty + 2) * rowB, tm_row, bar, 0, yh2, zc);
                tma_load_3d_s(dp + (uint32_t)(ty + 3) * rowB, tm_row, bar, 0, yh3, zc);
            }
        };
        __syncthreads();  // column table ready
        if (tid == producer) {
#pragma unroll
            for (int s = 0; s < NBUF; ++s)
                if (s < nplanes) issue(s, s);
        }
        bool failed = false;
        int nw = 0;
        auto wait_slot = [&](int s) {
            if (!mbar_wait_bounded(&head->bar[s], (ph >> s) & 1u, a.spin_limit)) {
                failed = true;
                return;
            }
            ph ^= 1u << s;
            ++nw;
        };
        auto zout = [&](int p) { return !perZ && (zfirst + dir * p < 0 || zfirst + dir * p >= nz); };

        double R[3][4];  // c of planes i-1, i, i+1 at the strip (rotating roles)
        wait_slot(0);
        lds4d(cbase + cOwn, R[0]);
        wait_slot(1);
        lds4d(cbase + cplaneB + cOwn, R[1]);
        const int ilast = L + 2;
        int ifail = 0;
        for (int b = 0; ifail == 0; ++b) {
            bool done = false;
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const int i = b * U + k + 1;
                if (i > ilast) {
                    done = true;
                    break;
                }
                const int sI = (k + 1) % NBUF, sN = (k + 2) % NBUF;
                double(&cp)[4] = R[k % 3];
                double(&cc)[4] = R[(k + 1) % 3];
                double(&cn)[4] = R[(k + 2) % 3];
                const uint32_t msl = (uint32_t)((k + 1) % 3), mslp = (uint32_t)(k % 3), mslpp = (uint32_t)((k + 2) % 3);
                wait_slot(sN);
                lds4d(cbase + sN * cplaneB + cOwn, cn);
                // ---- stage A: mu and 1/mob on plane i
                if (active) {
                    const uint32_t pl = cbase + sI * cplaneB;
                    double up[4], dn[4];
                    if (!FLAT) {
                        lds4d(pl + cOwn - rowB, up);
                        lds4d(pl + cOwn + rowB, dn);
                    }
                    const double xm0 = lds1d(pl + cRow + (uint32_t)xl * 8u);
                    const double xp3 = lds1d(pl + cRow + (uint32_t)xr * 8u);
                    double mu[4], rm[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const double c0 = cc[e];
                        const double xm = e > 0 ? cc[e - 1] : xm0;
                        const double xp = e < 3 ? cc[e + 1] : xp3;
                        const double ym = FLAT ? c0 : up[e], yp = FLAT ? c0 : dn[e];
                        const double lapc =
                            lap7<double, FLAT, false>(c0, xp, xm, yp, ym, cn[e], cp[e], cx, cy, cz, divX, divY, divZ);
                        fh_site_r(F, coltab[x0 + e], c0, lapc, kap, &mu[e], &rm[e]);
                    }
                    sts4d(mubase + msl * mplaneB + mOwn, mu);
                    sts4d(rmbase + msl * mplaneB + mOwn, rm);
                }
                // ---- stage B: c_new on plane i-1 (its mu rows were published
                // by the previous plane's barrier; planes i-2 and i at the
                // strip are this thread's own)
                if (i >= 3 && outrow) {
                    const uint32_t q = mslp * mplaneB;
                    double a0[4], r0[4], az_m[4], rz_m[4], az_p[4], rz_p[4];
                    lds4d(mubase + q + mOwn, a0);
                    lds4d(rmbase + q + mOwn, r0);
                    lds4d(mubase + mslpp * mplaneB + mOwn, az_m);
                    lds4d(rmbase + mslpp * mplaneB + mOwn, rz_m);
                    lds4d(mubase + msl * mplaneB + mOwn, az_p);
                    lds4d(rmbase + msl * mplaneB + mOwn, rz_p);
                    const bool sLo = zout(i - 2), sHi = zout(i);
                    double ay_m[4], ry_m[4], ay_p[4], ry_p[4];
                    if (!FLAT) {
                        lds4d(mubase + q + mOwn - rowB, ay_m);
                        lds4d(rmbase + q + mOwn - rowB, ry_m);
                        lds4d(mubase + q + mOwn + rowB, ay_p);
                        lds4d(rmbase + q + mOwn + rowB, ry_p);
                    }
                    const double axm0 = lds1d(mubase + q + mRow + (uint32_t)xl * 8u);
                    const double rxm0 = lds1d(rmbase + q + mRow + (uint32_t)xl * 8u);
                    const double axp3 = lds1d(mubase + q + mRow + (uint32_t)xr * 8u);
                    const double rxp3 = lds1d(rmbase + q + mRow + (uint32_t)xr * 8u);
                    uint32_t word[4] = {0u, 0u, 0u, 0u};
                    if (noisy) {
                        const long long gsite = ((long long)(zfirst + dir * (i - 1)) * pstride + site_row) >> 2;
                        const uint4 w = philox4x32_10(
                            make_uint4((uint32_t)gsite, (uint32_t)(gsite >> 32), (uint32_t)st, (uint32_t)(st >> 32)), key);
                        word[0] = w.x, word[1] = w.y, word[2] = w.z, word[3] = w.w;
                    }
                    double o[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const double am = e > 0 ? a0[e - 1] : axm0, rmm = e > 0 ? r0[e - 1] : rxm0;
                        const double ap = e < 3 ? a0[e + 1] : axp3, rpp = e < 3 ? r0[e + 1] : rxp3;
                        const double zm = sLo ? a0[e] : az_m[e], rzm = sLo ? r0[e] : rz_m[e];
                        const double zp = sHi ? a0[e] : az_p[e], rzp = sHi ? r0[e] : rz_p[e];
                        double ym = a0[e], rym = r0[e], yp = a0[e], ryp = r0[e];
                        if (!FLAT) {
                            ym = subUp ? a0[e] : ay_m[e], rym = subUp ? r0[e] : ry_m[e];
                            yp = subDn ? a0[e] : ay_p[e], ryp = subDn ? r0[e] : ry_p[e];
                        }
                        double lap;
                        if (linear) {
                            const double lx = fh_axis_r(am, ap, a0[e], rmm, rpp, r0[e], cx, divX);
                            const double lz = fh_axis_r(zm, zp, a0[e], rzm, rzp, r0[e], cz, divZ);
                            lap = FLAT ? A::add(lx, lz)
                                       : A::add(A::add(lx, fh_axis_r(ym, yp, a0[e], rym, ryp, r0[e], cy, divY)), lz);
                        } else {
                            const FhFrac fx = fh_axis_frac(am, ap, a0[e], rmm, rpp, r0[e], cx, divX);
                            const FhFrac fz = fh_axis_frac(zm, zp, a0[e], rzm, rzp, r0[e], cz, divZ);
                            const FhFrac fy = FLAT ? FhFrac{0.0, 1.0} : fh_axis_frac(ym, yp, a0[e], rym, ryp, r0[e], cy, divY);
                            lap = fh_div_frac(fx, fy, fz, FLAT);
                        }
                        double v = A::add(cp[e], A::mul(dt, lap));  // c += dt * lap (TIPSphil.cpp:194)
                        if (noisy) {
                            // TIPSphil.cpp:200-209 (SIPS.cpp:239-240: none at or above the cutoff)
                            const double r = A::add(A::mul((double)word[e], 2.3283064365386963e-10), 1.1641532182693481e-10);
                            const double val = v >= cutoff ? 0.0 : A::mul(noise, A::sub(r, 0.5));
                            v = A::add(v, A::mul(dt, val));
                        }
                        o[e] = v;
                    }
                    *reinterpret_cast<double2*>(g) = make_double2(o[0], o[1]);
                    *reinterpret_cast<double2*>(g + 2) = make_double2(o[2], o[3]);
                }
                if (__syncthreads_or(failed)) {
                    ifail = i;
                    done = true;
                    break;
                }
                // planes <= i were last read above: slot i takes plane i+NBUF,
                // and after the first plane slot 0 (plane 0, read only as a
                // z-queue register in the prologue) takes plane NBUF
                if (tid == producer) {
                    if (i == 1 && NBUF < nplanes) issue(NBUF, 0);
                    if (i + NBUF < nplanes) issue(i + NBUF, sI);
                }
                g += gstep;
            }
            if (done) break;
        }
        if (ifail) {
            if (tid == 0) {
                // planes issued before the barrier of plane ifail: NBUF at the start,
                // then NBUF + 1 after plane 1 and one more after each later plane
                const int nissued = min(nplanes, ifail >= 2 ? NBUF + ifail : NBUF);
                for (int p = nw; p < nissued; ++p) {
                    const int s = p % NBUF;
                    mbar_wait_bounded(&head->bar[s], (ph >> s) & 1u, a.spin_limit);
                    ph ^= 1u << s;
                }
                atomicMax(&J->err, DEV_TMA_TIMEOUT);
                atomicMax(a.err, DEV_TMA_TIMEOUT);
            }
            return;
        }
        // ---- completion count; the CTA of the job's last item advances it
        const int nitems_job = J->ntile * J->nchunk;
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            const unsigned prev = atomicAdd(&J->done, 1u);
            if (prev == (unsigned)nitems_job - 1u) {
                __threadfence();
                J->done = 0;
                if (noisy) J->noise_step = st;
                J->step = step + 1;
            }
        }
        __syncthreads();
    }
}

// Mobility of every site for the step that produced the current field (the
// input of that step is still in the other ping-pong buffer): the field of
// mg_fh_mobility.  Before any step, the mobility of the first step.
__global__ void fh_mobility_kernel(const JobDev* job, double* out)
{
    using A = Arith<double>;
    const JobDev& J = *job;
    const FhDev& F = *J.fh;
    const int nx = J.nx, ny = J.ny, nz = J.nz;
    const size_t n = (size_t)nx * ny * nz;
    const long long taken = J.step;
    const long long s_in = taken > 0 ? taken - 1 : 0;  // the step whose input is wanted
    const double* __restrict__ c = static_cast<const double*>(J.buf[s_in & 1]);
    const double cs = (double)(s_in + 1);
    const bool pX = J.flags & JF_PER_X, pY = J.flags & JF_PER_Y, pZ = J.flags & JF_PER_Z;
    for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(s % nx), y = (int)((s / nx) % ny), z = (int)(s / ((size_t)nx * ny));
        auto at = [&](int xx, int yy, int zz) { return c[((size_t)zz * ny + yy) * nx + xx]; };
        const double cc = c[s];
        const double xp = at(wrap_or_clamp(x + 1, nx, pX), y, z), xm = at(wrap_or_clamp(x - 1, nx, pX), y, z);
        const double zp = at(x, y, wrap_or_clamp(z + 1, nz, pZ)), zm = at(x, y, wrap_or_clamp(z - 1, nz, pZ));
        double lapc;
        if (J.flags & JF_FLAT) {
            lapc = A::add(axis_term(xp, xm, cc, J.cx, J.flags & JF_DIV_X), axis_term(zp, zm, cc, J.cz, J.flags & JF_DIV_Z));
        } else {
            const double yp = at(x, wrap_or_clamp(y + 1, ny, pY), z), ym = at(x, wrap_or_clamp(y - 1, ny, pY), z);
            lapc = A::add(A::add(axis_term(xp, xm, cc, J.cx, J.flags & JF_DIV_X), axis_term(yp, ym, cc, J.cy, J.flags & JF_DIV_Y)),
                          axis_term(zp, zm, cc, J.cz, J.flags & JF_DIV_Z));
        }
        double mu, mob;
        fh_site(F, cc, lapc, J.kap, x, cs, J.dtM_dt, &mu, &mob);
        out[s] = mob;
    }
}

}  // namespace mg
