// Fused Cahn-Hilliard step for sm_100a.
//
// One launch advances every job of a work list by one explicit step
//     mu    = (c^3 - c) - kappa * lap(c)
//     c_new = c + lap(mu) * (dt*M)
// in a single pass over HBM: c is read once (plus halo re-reads that hit L2)
// and c_new is written once.  mu never leaves shared memory.
//
// Work decomposition.  A job's field is dense and x-fastest.  A work item is
// (y-tile, z-chunk): the CTA owns full x-rows y0..y0+TY-1 and marches through
// the planes of its z-chunk.  Per plane it
//   1. TMA-loads the c plane rows y0-2..y0+TY+1 (halo 2, periodic rows
//      wrapped by coordinate) into a ring of NBUF shared-memory planes;
//   2. computes mu on the halo-1 rows y0-1..y0+TY for that plane;
//   3. computes lap(mu) and c_new for the plane behind it and stores it.
// Each thread owns VEC consecutive x (one 16-byte vector) in two rows and
// keeps c and mu of the previous/current/next plane of those sites in
// registers, so the z-direction taps never touch shared memory; x-taps come
// from warp shuffles, y-taps from shared memory.  Neighbouring z-chunks march
// in opposite directions so that the z-halo planes two chunks share are read
// at the same time (start or end of the kernel) and hit L2.
//
// Two-dimensional jobs (nz == 1) are run as (nx, 1, ny): the y axis is flat
// (its Laplacian term is exactly zero in the reference) and the CTA marches
// along the original y.  Flat jobs use the FLAT instantiation (one row per
// plane, no y taps).
//
// Boundary conditions follow SfieldFD::updateBoundaries (SfieldFD.cpp:187-251):
// periodic axes wrap; on no-flux axes a ghost node equals the adjacent
// interior node, for c and for mu alike, which the kernel realises by
// substituting the centre value for an out-of-domain neighbour.
#pragma once

#include "ch_types.h"
#include "mg_device.cuh"

namespace mg {

template <typename T>
struct alignas(16) Vec {
    static constexpr int N = 16 / sizeof(T);
    T v[N];
};

template <typename T>
__device__ __forceinline__ Vec<T> ld_vec(const T* p)
{
    return *reinterpret_cast<const Vec<T>*>(p);
}
template <typename T>
__device__ __forceinline__ void st_vec(T* p, const Vec<T>& q)
{
    *reinterpret_cast<Vec<T>*>(p) = q;
}

// (a[+] + a[-] - 2*a) scaled by c: multiply (power-of-two spacing, exact) or
// divide (otherwise), as SfieldFD::Laplacian writes it (SfieldFD.cpp:296-302).
template <typename T>
__device__ __forceinline__ T axis_term(T plus, T minus, T centre, double c, bool divide)
{
    using A = Arith<T>;
    T num = A::sub(A::add(plus, minus), A::mul(T(2), centre));
    return divide ? A::div(num, T(c)) : A::mul(num, T(c));
}

__device__ __forceinline__ int wrap_or_clamp(int i, int n, bool periodic)
{
    if (periodic) {
        i %= n;
        return i < 0 ? i + n : i;
    }
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// Locate job for a flat item index (item_begin is ascending).
__device__ __forceinline__ int find_job(const int* item_begin, int njobs, int item)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(item_begin + mid) <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename T, int NBUF, bool FLAT>
__global__ void __launch_bounds__(512, 1) ch_step_kernel(StepArgs a)
{
    constexpr int VEC = Vec<T>::N;
    constexpr int R = FLAT ? 1 : 2;  // rows per thread
    using A = Arith<T>;

    extern __shared__ __align__(128) unsigned char smem_dyn[];
    // TMA destinations must be 128-byte aligned: align the base explicitly
    // (the host sizes the allocation with 128 bytes of slack)
    unsigned char* smem_raw = smem_dyn + ((128u - (smem_addr(smem_dyn) & 127u)) & 127u);
    SmemHead* head = reinterpret_cast<SmemHead*>(smem_raw);
    T* cbase = reinterpret_cast<T*>(smem_raw + ((sizeof(SmemHead) + 127) / 128) * 128);
    T* mbase = cbase + (size_t)NBUF * a.cplane;

    const int tid = threadIdx.x;
    const int lane = tid & 31;

    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&head->bar[b], 1);
        fence_mbar_init();
        head->abort = 0;
    }
    __syncthreads();

    long long gseq = 0;  // c planes issued by this CTA (ring slot = gseq % NBUF)

    for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
        const int j = find_job(a.item_begin, a.njobs, item);
        JobDev* J = a.jobs + __ldg(a.job_slot + j);
        const int local = item - __ldg(a.item_begin + j);

        if (tid == 0) {
            head->step = *((volatile long long*)&J->step);
            head->delta = *((volatile double*)&J->delta);
        }
        __syncthreads();
        const long long step = head->step;
        const double delta = head->delta;
        if (step >= J->target) {  // uniform: read once by thread 0
            __syncthreads();        // head->step is rewritten for the next item
            continue;
        }

        const int nx = J->nx, ny = J->ny, nz = J->nz;
        const int ty = J->ty, flags = J->flags, bw = J->bw;
        const bool perX = flags & JF_PER_X, perY = flags & JF_PER_Y, perZ = flags & JF_PER_Z;
        const bool divX = flags & JF_DIV_X, divY = flags & JF_DIV_Y, divZ = flags & JF_DIV_Z;
        const bool massfb = flags & JF_MASS;
        const double cx = J->cx, cy = J->cy, cz = J->cz;
        const T kap = T(J->kap), dtM = T(J->dtM);
        const int par = (int)(step & 1);
        T* __restrict__ dst = static_cast<T*>(J->buf[par ^ 1]);
        const CUtensorMap* tm_body = J->tmap + 2 * par;
        const CUtensorMap* tm_row = J->tmap + 2 * par + 1;

        const int CY = FLAT ? 1 : ty + 4;  // c rows in a plane
        const int MY = FLAT ? 1 : ty + 2;  // mu rows in a plane
        const int npiece = nx / bw;
        const uint32_t plane_bytes = (uint32_t)(CY * nx * sizeof(T));

        // ---- tile geometry
        const int tile = local % J->ntile;
        const int chunk = local / J->ntile;
        const int own_lo = FLAT ? 0 : tile * ty;
        const int own_hi = FLAT ? 1 : min(ny, own_lo + ty);
        const int y0 = FLAT ? 0 : min(own_lo, ny - ty);
        const int zs = (int)((long long)chunk * nz / J->nchunk);
        const int ze = (int)((long long)(chunk + 1) * nz / J->nchunk);
        const int L = ze - zs;
        const int dir = (chunk & 1) ? -1 : 1;
        auto zseq = [&](int i) { return dir > 0 ? zs - 2 + i : ze + 1 - i; };  // c plane i, i = 0..L+3

        // ---- thread geometry (fixed for the item)
        const int nq = nx / VEC;
        const int ntr = FLAT ? 1 : MY / 2;
        const int tjob = nq * ntr;
        const bool active = tid < tjob;
        const int t = active ? tid : 0;
        const int tx = t % nq, tr = t / nq;
        const int x0 = tx * VEC;
        auto col = [&](int x, int rows) { return (x / bw) * rows * bw + (x % bw); };
        const int xl = x0 == 0 ? (perX ? nx - 1 : 0) : x0 - 1;
        const int xr = x0 + VEC >= nx ? (perX ? 0 : nx - 1) : x0 + VEC;
        const int cOwn = col(x0, CY), cL = col(xl, CY), cR = col(xr, CY);
        const int mOwn = col(x0, MY), mL = col(xl, MY), mR = col(xr, MY);
        const bool leftSm = (lane == 0) || (tx == 0);
        const bool rightSm = (lane == 31) || (tx == nq - 1);

        // own mu rows m0 = 2*tr, m1 = m0+1 (region row m <-> y = y0 - 1 + m)
        const int m0 = FLAT ? 0 : 2 * tr;
        int yrow[2], outrow[2];
        bool subUp[2], subDn[2];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int m = m0 + r;
            const int y = FLAT ? 0 : y0 - 1 + m;
            yrow[r] = y;
            outrow[r] = active && (r < R) && (FLAT || (m >= 1 && m <= ty && y >= own_lo && y < own_hi));
            subUp[r] = !FLAT && !perY && (y - 1 < 0 || y - 1 >= ny);
            subDn[r] = !FLAT && !perY && (y + 1 < 0 || y + 1 >= ny);
        }

        auto cplane = [&](long long g) { return cbase + (size_t)(g % NBUF) * a.cplane; };
        auto mplane = [&](int i) { return mbase + (size_t)(i % 3) * a.mplane; };

        // ---- producer: TMA of c plane i into ring slot g
        auto issue = [&](int i, long long g) {
            if (tid != 0) return;
            T* p = cplane(g);
            uint64_t* bar = &head->bar[g % NBUF];
            const int zc = wrap_or_clamp(zseq(i), nz, perZ);
            mbar_arrive_expect_tx(bar, plane_bytes + a.tx_extra);
            for (int pc = 0; pc < npiece; ++pc) {
                T* pp = p + (size_t)pc * CY * bw;
                const int xc = pc * bw;
                if (FLAT) {
                    tma_load_3d(pp, tm_row, bar, xc, 0, zc);
                } else {
                    tma_load_3d(pp, tm_row, bar, xc, wrap_or_clamp(y0 - 2, ny, perY), zc);
                    tma_load_3d(pp + bw, tm_row, bar, xc, wrap_or_clamp(y0 - 1, ny, perY), zc);
                    tma_load_3d(pp + 2 * bw, tm_body, bar, xc, y0, zc);
                    tma_load_3d(pp + (size_t)(ty + 2) * bw, tm_row, bar, xc, wrap_or_clamp(y0 + ty, ny, perY), zc);
                    tma_load_3d(pp + (size_t)(ty + 3) * bw, tm_row, bar, xc,
                                wrap_or_clamp(y0 + ty + 1, ny, perY), zc);
                }
            }
        };
        auto wait = [&](long long g) {
            if (!mbar_wait_bounded(&head->bar[g % NBUF], (uint32_t)((g / NBUF) & 1), a.spin_limit)) {
                head->abort = 1;
                atomicMax(&J->err, DEV_TMA_TIMEOUT);
                atomicMax(a.err, DEV_TMA_TIMEOUT);
            }
        };

        // own values of a c plane: rows m0+1 .. m0+R in c-plane rows
        auto load_own = [&](const T* p, Vec<T> (&o)[2]) {
#pragma unroll
            for (int r = 0; r < R; ++r) o[r] = ld_vec(p + cOwn + (m0 + 1 + r - (FLAT ? 1 : 0)) * bw);
        };

        const long long g0 = gseq;
        const int nplanes = L + 4;
        const int npro = min(NBUF, nplanes);
        for (int i = 0; i < npro; ++i) issue(i, g0 + i);
        int issued = npro;  // planes issued so far (uniform)
        int waited = 2;     // planes waited so far (uniform)

        Vec<T> cP[2], cC[2], cN[2], mP[2], mC[2], mN[2];
        double macc = 0.0;

        wait(g0);
        load_own(cplane(g0), cP);
        wait(g0 + 1);
        load_own(cplane(g0 + 1), cC);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
#pragma unroll
            for (int e = 0; e < VEC; ++e) mP[r].v[e] = mC[r].v[e] = T(0);
        }

        for (int i = 1; i <= L + 2; ++i) {
            // c plane i+1 (own values): z neighbour of mu(i)
            wait(g0 + i + 1);
            waited = i + 2;
            load_own(cplane(g0 + i + 1), cN);

            // ---- stage A: mu on plane i
            {
                const T* p = cplane(g0 + i);
                const int zi = zseq(i);
                const bool sLo = !perZ && (zseq(i - 1) < 0 || zseq(i - 1) >= nz);
                const bool sHi = !perZ && (zseq(i + 1) < 0 || zseq(i + 1) >= nz);
                (void)zi;
                Vec<T> up, dn;
                if (!FLAT) {
                    up = ld_vec(p + cOwn + m0 * bw);
                    dn = ld_vec(p + cOwn + (m0 + 3) * bw);
                }
                T* mp = mplane(i);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int crow = FLAT ? 0 : m0 + 1 + r;
                    T lft = __shfl_up_sync(0xffffffffu, cC[r].v[VEC - 1], 1);
                    T rgt = __shfl_down_sync(0xffffffffu, cC[r].v[0], 1);
                    if (leftSm) lft = p[cL + crow * bw];
                    if (rightSm) rgt = p[cR + crow * bw];
                    Vec<T> mu;
#pragma unroll
                    for (int e = 0; e < VEC; ++e) {
                        const T c0 = cC[r].v[e];
                        const T xm = e > 0 ? cC[r].v[e - 1] : lft;
                        const T xp = e < VEC - 1 ? cC[r].v[e + 1] : rgt;
                        const T zm = sLo ? c0 : cP[r].v[e];
                        const T zp = sHi ? c0 : cN[r].v[e];
                        T lap;
                        if (FLAT) {
                            lap = A::add(axis_term(xp, xm, c0, cx, divX), axis_term(zp, zm, c0, cz, divZ));
                        } else {
                            T ym = r == 0 ? up.v[e] : cC[0].v[e];
                            T yp = r == R - 1 ? dn.v[e] : cC[1].v[e];
                            if (subUp[r]) ym = c0;
                            if (subDn[r]) yp = c0;
                            lap = A::add(A::add(axis_term(xp, xm, c0, cx, divX), axis_term(yp, ym, c0, cy, divY)),
                                         axis_term(zp, zm, c0, cz, divZ));
                        }
                        const T df = A::sub(A::mul(A::mul(c0, c0), c0), c0);
                        mu.v[e] = A::sub(df, A::mul(kap, lap));
                    }
                    mN[r] = mu;
                    if (active) st_vec(mp + mOwn + (m0 + r) * bw, mu);
                }
            }
            __syncthreads();
            if (head->abort) break;
            // ring slot of plane i-1 is free: refill it with plane i-1+NBUF
            if (i - 1 + NBUF < nplanes) {
                issue(i - 1 + NBUF, g0 + i - 1 + NBUF);
                issued = i + NBUF;
            }

            // ---- stage B: output plane i-1
            if (i >= 3) {
                const T* mp = mplane(i - 1);
                const int zo = zseq(i - 1);
                const bool sLo = !perZ && (zseq(i - 2) < 0 || zseq(i - 2) >= nz);
                const bool sHi = !perZ && (zseq(i) < 0 || zseq(i) >= nz);
                Vec<T> up, dn;
                if (!FLAT) {
                    up = ld_vec(mp + mOwn + (m0 > 0 ? m0 - 1 : 0) * bw);
                    dn = ld_vec(mp + mOwn + (m0 + 2 < MY ? m0 + 2 : MY - 1) * bw);
                }
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int mrow = FLAT ? 0 : m0 + r;
                    T lft = __shfl_up_sync(0xffffffffu, mC[r].v[VEC - 1], 1);
                    T rgt = __shfl_down_sync(0xffffffffu, mC[r].v[0], 1);
                    if (leftSm) lft = mp[mL + mrow * bw];
                    if (rightSm) rgt = mp[mR + mrow * bw];
                    if (!outrow[r]) continue;
                    Vec<T> out;
#pragma unroll
                    for (int e = 0; e < VEC; ++e) {
                        const T m = mC[r].v[e];
                        const T xm = e > 0 ? mC[r].v[e - 1] : lft;
                        const T xp = e < VEC - 1 ? mC[r].v[e + 1] : rgt;
                        const T zm = sLo ? m : mP[r].v[e];
                        const T zp = sHi ? m : mN[r].v[e];
                        T lap;
                        if (FLAT) {
                            lap = A::add(axis_term(xp, xm, m, cx, divX), axis_term(zp, zm, m, cz, divZ));
                        } else {
                            T ym = r == 0 ? up.v[e] : mC[0].v[e];
                            T yp = r == R - 1 ? dn.v[e] : mC[1].v[e];
                            if (subUp[r]) ym = m;
                            if (subDn[r]) yp = m;
                            lap = A::add(A::add(axis_term(xp, xm, m, cx, divX), axis_term(yp, ym, m, cy, divY)),
                                         axis_term(zp, zm, m, cz, divZ));
                        }
                        const T c0 = cP[r].v[e];
                        T cn;
                        if constexpr (sizeof(T) == 4) {
                            if (massfb) {
                                const T u = lap * dtM;
                                cn = (T)(((double)c0 + (double)u) + delta);
                            } else {
                                cn = fmaf(lap, dtM, c0);
                            }
                            if (massfb) macc += (double)cn;
                        } else {
                            cn = A::add(c0, A::mul(lap, dtM));
                        }
                        out.v[e] = cn;
                    }
                    const int y = yrow[r];
                    st_vec(dst + ((size_t)zo * ny + y) * nx + x0, out);
                }
            }
            // rotate the register planes
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                cP[r] = cC[r];
                cC[r] = cN[r];
                mP[r] = mC[r];
                mC[r] = mN[r];
            }
        }
        gseq = g0 + nplanes;

        if (head->abort) {
            // drain: wait (bounded) for the planes issued but not yet
            // consumed, so no copy lands after the CTA has exited
            for (int i = waited; i < issued; ++i) {
                const long long g = g0 + i;
                mbar_wait_bounded(&head->bar[g % NBUF], (uint32_t)((g / NBUF) & 1), a.spin_limit);
            }
            return;
        }

        // ---- item epilogue: partial mass, completion count, last-item work
        const int nitems_job = J->ntile * J->nchunk;
        if (massfb) {
            const int nw = (tjob + 31) >> 5;
            double2 v = make_double2(active ? macc : 0.0, 0.0);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                double2 o = shfl_down_pair(v, off);
                if (lane + off < 32) v = pair_add(v, o);
            }
            if (lane == 0 && (tid >> 5) < nw) head->red[tid >> 5] = v;
            __syncthreads();
            if (tid < 32) {
                double2 r = lane < nw ? head->red[lane] : make_double2(0.0, 0.0);
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    double2 o = shfl_down_pair(r, off);
                    if (lane + off < 32) r = pair_add(r, o);
                }
                if (lane == 0) J->partial[local] = r;
            }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            const unsigned prev = atomicAdd(&J->done, 1u);
            head->flag = (prev == (unsigned)nitems_job - 1u);
            if (head->flag) __threadfence();
        }
        __syncthreads();
        if (head->flag) {
            if (massfb && tid < 32) {
                double2 r = make_double2(0.0, 0.0);
                for (int k = lane; k < nitems_job; k += 32) {
                    double2 pv = __ldcg(J->partial + k);
                    r = pair_add(r, pv);
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    double2 o = shfl_down_pair(r, off);
                    if (lane + off < 32) r = pair_add(r, o);
                }
                if (lane == 0) {
                    const double m = r.x + r.y;
                    J->mass_last = m;
                    J->delta = (J->mass_target - m) * J->inv_nsites;
                }
            }
            if (tid == 0) {
                J->done = 0;
                J->step = step + 1;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Generic path for shapes the tiled kernel does not take (nx not a multiple
// of the 16-byte vector, or nx > 256 and not a multiple of 256): one thread
// per site, mu evaluated at each of the seven taps.  Same arithmetic, same
// boundary semantics; used for small or odd grids.
template <typename T>
__device__ __forceinline__ T mu_at(const T* __restrict__ c, int x, int y, int z, const JobDev& J)
{
    using A = Arith<T>;
    const int nx = J.nx, ny = J.ny, nz = J.nz;
    const bool pX = J.flags & JF_PER_X, pY = J.flags & JF_PER_Y, pZ = J.flags & JF_PER_Z;
    auto at = [&](int xx, int yy, int zz) { return c[((size_t)zz * ny + yy) * nx + xx]; };
    const T c0 = at(x, y, z);
    const T xp = at(wrap_or_clamp(x + 1, nx, pX), y, z), xm = at(wrap_or_clamp(x - 1, nx, pX), y, z);
    const T zp = at(x, y, wrap_or_clamp(z + 1, nz, pZ)), zm = at(x, y, wrap_or_clamp(z - 1, nz, pZ));
    T lap;
    if (J.flags & JF_FLAT) {
        lap = A::add(axis_term(xp, xm, c0, J.cx, J.flags & JF_DIV_X), axis_term(zp, zm, c0, J.cz, J.flags & JF_DIV_Z));
    } else {
        const T yp = at(x, wrap_or_clamp(y + 1, ny, pY), z), ym = at(x, wrap_or_clamp(y - 1, ny, pY), z);
        lap = A::add(A::add(axis_term(xp, xm, c0, J.cx, J.flags & JF_DIV_X), axis_term(yp, ym, c0, J.cy, J.flags & JF_DIV_Y)),
                     axis_term(zp, zm, c0, J.cz, J.flags & JF_DIV_Z));
    }
    return A::sub(A::sub(A::mul(A::mul(c0, c0), c0), c0), A::mul(T(J.kap), lap));
}

template <typename T>
__global__ void ch_step_generic_kernel(JobDev* job)
{
    using A = Arith<T>;
    const JobDev& J = *job;
    const int nx = J.nx, ny = J.ny, nz = J.nz;
    const size_t n = (size_t)nx * ny * nz;
    const size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (J.step >= J.target || s >= n) return;
    const int par = (int)(J.step & 1);
    const T* __restrict__ c = static_cast<const T*>(J.buf[par]);
    T* __restrict__ out = static_cast<T*>(J.buf[par ^ 1]);
    const int x = (int)(s % nx), y = (int)((s / nx) % ny), z = (int)(s / ((size_t)nx * ny));
    const bool pX = J.flags & JF_PER_X, pY = J.flags & JF_PER_Y, pZ = J.flags & JF_PER_Z;
    const T m = mu_at(c, x, y, z, J);
    // ghost mu on a no-flux side equals the centre value
    auto mnb = [&](int xx, int yy, int zz) { return (xx == x && yy == y && zz == z) ? m : mu_at(c, xx, yy, zz, J); };
    const T xp = mnb(wrap_or_clamp(x + 1, nx, pX), y, z), xm = mnb(wrap_or_clamp(x - 1, nx, pX), y, z);
    const T zp = mnb(x, y, wrap_or_clamp(z + 1, nz, pZ)), zm = mnb(x, y, wrap_or_clamp(z - 1, nz, pZ));
    T lap;
    if (J.flags & JF_FLAT) {
        lap = A::add(axis_term(xp, xm, m, J.cx, J.flags & JF_DIV_X), axis_term(zp, zm, m, J.cz, J.flags & JF_DIV_Z));
    } else {
        const T yp = mnb(x, wrap_or_clamp(y + 1, ny, pY), z), ym = mnb(x, wrap_or_clamp(y - 1, ny, pY), z);
        lap = A::add(A::add(axis_term(xp, xm, m, J.cx, J.flags & JF_DIV_X), axis_term(yp, ym, m, J.cy, J.flags & JF_DIV_Y)),
                     axis_term(zp, zm, m, J.cz, J.flags & JF_DIV_Z));
    }
    out[s] = A::add(c[s], A::mul(lap, T(J.dtM)));
}

// advances the step counter after a generic-path step
__global__ void ch_step_generic_finish(JobDev* job)
{
    if (threadIdx.x == 0 && blockIdx.x == 0 && job->step < job->target) job->step += 1;
}

// resets the mutable state of a job slot
__global__ void ch_job_reset(JobDev* job, long long target)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        job->step = 0;
        job->target = target;
        job->done = 0;
        job->err = 0;
        job->delta = 0.0;
    }
}

template <typename S, typename D>
__global__ void ch_convert(const S* __restrict__ src, D* __restrict__ dst, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (D)src[i];
}

// ---------------------------------------------------------------------------
// Diagnostics of the current field of one job: compensated FP64 sums of
// mass, |c| and free energy, max|c| and the count of non-finite sites, in a
// fixed reduction order (fixed grid, fixed trees).
//   F = sum[(c^2-1)^2/4 + kap/2 |grad+ c|^2] dV, forward differences.
template <typename T>
__global__ void __launch_bounds__(kDiagThreads) ch_diag_partial(const JobDev* job, double spx, double spy, double spz,
                                                                double2* part /* [kDiagBlocks][3] */,
                                                                double* pmax, double* pbad)
{
    __shared__ double2 scratch[32];
    __shared__ double smax[32], sbad[32];
    const JobDev& J = *job;
    const int nx = J.nx, ny = J.ny, nz = J.nz;
    const size_t n = (size_t)nx * ny * nz;
    const T* c = static_cast<const T*>(J.buf[J.step & 1]);
    const bool pX = J.flags & JF_PER_X, pY = J.flags & JF_PER_Y, pZ = J.flags & JF_PER_Z;
    const bool flat = J.flags & JF_FLAT;
    double2 sm = make_double2(0, 0), sa = make_double2(0, 0), se = make_double2(0, 0);
    double mx = 0.0, bad = 0.0;
    for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (size_t)gridDim.x * blockDim.x) {
        const double v = (double)c[s];
        if (!isfinite(v)) {
            bad += 1.0;
            continue;
        }
        const int x = (int)(s % nx), y = (int)((s / nx) % ny), z = (int)(s / ((size_t)nx * ny));
        auto at = [&](int xx, int yy, int zz) { return (double)c[((size_t)zz * ny + yy) * nx + xx]; };
        const double gx = (at(wrap_or_clamp(x + 1, nx, pX), y, z) - v) / spx;
        const double gy = flat ? 0.0 : (at(x, wrap_or_clamp(y + 1, ny, pY), z) - v) / spy;
        const double gz = (at(x, y, wrap_or_clamp(z + 1, nz, pZ)) - v) / spz;
        const double w = v * v - 1.0;
        const double f = 0.25 * w * w + 0.5 * J.kap * (gx * gx + gy * gy + gz * gz);
        sm = pair_add(sm, make_double2(v, 0.0));
        sa = pair_add(sa, make_double2(fabs(v), 0.0));
        se = pair_add(se, make_double2(f, 0.0));
        mx = fmax(mx, fabs(v));
    }
    double2 r0 = block_pair_sum(sm, scratch);
    double2 r1 = block_pair_sum(sa, scratch);
    double2 r2 = block_pair_sum(se, scratch);
    // max and count
    for (int off = 16; off > 0; off >>= 1) {
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
        bad += __shfl_down_sync(0xffffffffu, bad, off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        smax[warp] = mx;
        sbad[warp] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            m = fmax(m, smax[w]);
            b += sbad[w];
        }
        part[blockIdx.x * 3 + 0] = r0;
        part[blockIdx.x * 3 + 1] = r1;
        part[blockIdx.x * 3 + 2] = r2;
        pmax[blockIdx.x] = m;
        pbad[blockIdx.x] = b;
    }
}

__global__ void ch_diag_final(const double2* part, const double* pmax, const double* pbad, int nblocks, double dv,
                              Diag* out)
{
    __shared__ double2 scratch[32];
    double2 a0 = make_double2(0, 0), a1 = make_double2(0, 0), a2 = make_double2(0, 0);
    double mx = 0.0, bad = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        a0 = pair_add(a0, part[b * 3 + 0]);
        a1 = pair_add(a1, part[b * 3 + 1]);
        a2 = pair_add(a2, part[b * 3 + 2]);
        mx = fmax(mx, pmax[b]);
        bad += pbad[b];
    }
    a0 = block_pair_sum(a0, scratch);
    a1 = block_pair_sum(a1, scratch);
    a2 = block_pair_sum(a2, scratch);
    __shared__ double smax[32], sbad[32];
    for (int off = 16; off > 0; off >>= 1) {
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
        bad += __shfl_down_sync(0xffffffffu, bad, off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        smax[warp] = mx;
        sbad[warp] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            m = fmax(m, smax[w]);
            b += sbad[w];
        }
        out->mass = (a0.x + a0.y) * dv;
        out->abs_mass = (a1.x + a1.y) * dv;
        out->energy = (a2.x + a2.y) * dv;
        out->max_abs = m;
        out->nonfinite = b;
    }
}

// Sum of the stored field (no dV), for the FP32 mass target.
template <typename T>
__global__ void ch_mass_partial(const JobDev* job, double2* part)
{
    __shared__ double2 scratch[32];
    const JobDev& J = *job;
    const size_t n = (size_t)J.nx * J.ny * J.nz;
    const T* c = static_cast<const T*>(J.buf[J.step & 1]);
    double2 s = make_double2(0, 0);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s = pair_add(s, make_double2((double)c[i], 0.0));
    s = block_pair_sum(s, scratch);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void ch_mass_final(const double2* part, int nblocks, JobDev* job)
{
    __shared__ double2 scratch[32];
    double2 s = make_double2(0, 0);
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s = pair_add(s, part[b]);
    s = block_pair_sum(s, scratch);
    if (threadIdx.x == 0) {
        job->mass_target = s.x + s.y;
        job->mass_last = s.x + s.y;
        job->delta = 0.0;
    }
}

}  // namespace mg
