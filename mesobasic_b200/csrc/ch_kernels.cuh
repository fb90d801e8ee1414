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

#include "ch_device.cuh"

namespace mg {

// NXC: row width fixed at compile time (0: read from the job), so that row,
// half and piece offsets fold into instruction immediates.
template <typename T, int NBUF, bool FLAT, bool SIMPLE, bool MASS, int NXC = 0>
__global__ void __launch_bounds__(NXC ? kMaxBlock : kMaxBlockGeneric, 1) ch_step_kernel(StepArgs a)
{
    step_counts(a);
    constexpr int W = Strip<T>::W;  // elements per thread strip
    constexpr bool PAIRS = (sizeof(T) == 4) && SIMPLE;
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
    }
    __syncthreads();

    long long gseq = 0;  // c planes issued by this CTA before the current item

    for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
        const int j = find_job(a.item_begin, a.njobs, item);
        JobDev* J = a.jobs + __ldg(a.job_slot + j);
        const int local = item - __ldg(a.item_begin + j);

        if (tid == 0) {
            head->step = *((volatile long long*)&J->step);
            head->nudge_begin = *((volatile long long*)&J->nudge_begin);
            head->nudge_count = *((volatile long long*)&J->nudge_count);
        }
        __syncthreads();
        const long long step = head->step;
        // this step's stored field is summed (mass feedback) on every
        // mass_every-th step; the nudges it yields go into the next step
        const bool measure = MASS && (step + 1) % J->mass_every == 0;
        if (step >= J->target) {  // uniform: read once by thread 0
            __syncthreads();        // head->step is rewritten for the next item
            continue;
        }

        const int nx = NXC ? NXC : J->nx, ny = J->ny, nz = J->nz;
        const int ty = J->ty, flags = J->flags, bw = NXC ? (NXC < 256 ? NXC : 256) : J->bw;
        const bool perX = flags & JF_PER_X, perY = flags & JF_PER_Y, perZ = flags & JF_PER_Z;
        const bool divX = flags & JF_DIV_X, divY = flags & JF_DIV_Y, divZ = flags & JF_DIV_Z;
        const double cx = J->cx, cy = J->cy, cz = J->cz;
        const T kap = T(J->kap), dtM = T(J->dtM);
        // paired FP32 path: 1/dx^2 folded into kappa and dt*M
        const float kapc = (float)(J->kap * cx), dtMc = (float)(J->dtM * cx);
        const int par = (int)(step & 1);
        T* __restrict__ dst = static_cast<T*>(J->buf[par ^ 1]);
        const CUtensorMap* tm_body = J->tmap + 2 * par;
        const CUtensorMap* tm_row = J->tmap + 2 * par + 1;

        const int CY = FLAT ? 1 : ty + 4;  // c rows in a plane
        const int MY = FLAT ? 1 : ty + 2;  // mu rows in a plane (one thread row each)
        const int npiece = nx / bw;
        const uint32_t plane_bytes = (uint32_t)(CY * nx * sizeof(T));
        const size_t pstride = (size_t)nx * ny;
        // planes the mass-nudge window reaches: [wz0, wz1], and [0, wz2] for
        // the part that wraps past the last site
        int wz0 = 1 << 30, wz1 = -1, wz2 = -1;
        if constexpr (MASS) {
            const long long nsites = (long long)pstride * nz, na = llabs(head->nudge_count);
            if (na > 0) {
                const long long w0 = head->nudge_begin, w1 = w0 + na;
                wz0 = (int)(w0 / (long long)pstride);
                wz1 = (int)((min(w1, nsites) - 1) / (long long)pstride);
                if (w1 > nsites) wz2 = (int)((w1 - nsites - 1) / (long long)pstride);
            }
        }

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
        const int zfirst = dir > 0 ? zs - 2 : ze + 1;  // c plane i lies at z = zfirst + dir*i
        const int yh0 = FLAT ? 0 : wrap_or_clamp(y0 - 2, ny, perY);
        const int yh1 = FLAT ? 0 : wrap_or_clamp(y0 - 1, ny, perY);
        const int yh2 = FLAT ? 0 : wrap_or_clamp(y0 + ty, ny, perY);
        const int yh3 = FLAT ? 0 : wrap_or_clamp(y0 + ty + 1, ny, perY);

        // ---- thread geometry (fixed for the item): thread tx of mu row m owns
        // the 16-byte halves at x = HW*tx (A) and x = HW*tx + nx/2 (B)
        constexpr int HW = W / 2;
        const int nq = nx / W;
        const int tjob = nq * MY;
        const bool active = tid < tjob;
        const int t = active ? tid : 0;
        const int tx = t % nq, m = FLAT ? 0 : t / nq;
        const int xA = tx * HW, xB = xA + nx / 2;
        auto col = [&](int x, int rows) { return (x / bw) * rows * bw + (x % bw); };
        auto wrapx = [&](int x) { return x < 0 ? (perX ? x + nx : 0) : (x >= nx ? (perX ? x - nx : nx - 1) : x); };
        const int cOwn = col(xA, CY), cOffB = col(xB, CY) - cOwn;
        const int mOwn = col(xA, MY), mOffB = col(xB, MY) - mOwn;
        // row-relative shared-memory columns of the four x neighbours
        const int cLA = col(wrapx(xA - 1), CY), cRA = col(xA + HW, CY);
        const int cLB = col(xB - 1, CY), cRB = col(wrapx(xB + HW), CY);
        const int mLA = col(wrapx(xA - 1), MY), mRA = col(xA + HW, MY);
        const int mLB = col(xB - 1, MY), mRB = col(wrapx(xB + HW), MY);
        // a row of nq threads is a segment of the warp when nq is a power of
        // two <= 32 (neighbours by lane index, with wrap); otherwise shuffle by
        // one lane and read the ends of warps and rows from shared memory
        const bool seg = nq <= 32 && (nq & (nq - 1)) == 0;
        const int segbase = lane & ~(nq - 1);
        const int lsrc = seg ? (segbase | ((lane - 1) & (nq - 1))) : ((lane + 31) & 31);
        const int rsrc = seg ? (segbase | ((lane + 1) & (nq - 1))) : ((lane + 1) & 31);
        const bool leftSm = !seg && ((lane == 0) || (tx == 0));
        const bool rightSm = !seg && ((lane == 31) || (tx == nq - 1));
        const bool first = tx == 0, last = tx == nq - 1;

        const int y = FLAT ? 0 : y0 - 1 + m;
        const size_t rowoff = (size_t)max(y, 0) * nx + xA;
        const int gOffB = nx / 2;
        const bool outrow = active && (FLAT || (m >= 1 && m <= ty && y >= own_lo && y < own_hi));
        const bool subUp = !FLAT && !perY && (y - 1 < 0 || y - 1 >= ny);
        const bool subDn = !FLAT && !perY && (y + 1 < 0 || y + 1 >= ny);
        const int cRowOwn = FLAT ? 0 : m + 1;
        const int mUpRow = FLAT ? 0 : max(m - 1, 0), mDnRow = FLAT ? 0 : min(m + 1, MY - 1);

        // c ring: plane i sits in slot (s0 + i) mod NBUF; its barrier phase
        // flips every time the slot index wraps
        const int s0 = (int)(gseq % NBUF);
        const uint32_t ph0 = (uint32_t)((gseq / NBUF) & 1);
        auto cslot = [&](int i) { return (s0 + i) % NBUF; };
        auto cphase = [&](int i) { return ph0 ^ (uint32_t)(((s0 + i) / NBUF) & 1); };
        auto cplane = [&](int i) { return cbase + (size_t)cslot(i) * a.cplane; };
        auto mplane = [&](int slot) { return mbase + (size_t)slot * a.mplane; };
        auto zout = [&](int i) { return !perZ && (zfirst + dir * i < 0 || zfirst + dir * i >= nz); };

        // ---- producer: TMA of c plane i into its ring slot.  The producer is
        // the first thread of the last mu row, which has no outputs and so no
        // stage-B work (thread 0 when flat)
        const int producer = FLAT ? 0 : (MY - 1) * nq;
        auto issue = [&](int i) {
            if (tid != producer) return;
            T* p = cplane(i);
            uint64_t* bar = &head->bar[cslot(i)];
            const int zc = wrap_or_clamp(zfirst + dir * i, nz, perZ);
            mbar_arrive_expect_tx(bar, plane_bytes + a.tx_extra);
            for (int pc = 0; pc < npiece; ++pc) {
                T* pp = p + (size_t)pc * CY * bw;
                const int xc = pc * bw;
                if (FLAT) {
                    tma_load_3d(pp, tm_row, bar, xc, 0, zc);
                } else {
                    tma_load_3d(pp, tm_row, bar, xc, yh0, zc);
                    tma_load_3d(pp + bw, tm_row, bar, xc, yh1, zc);
                    tma_load_3d(pp + 2 * bw, tm_body, bar, xc, y0, zc);
                    tma_load_3d(pp + (size_t)(ty + 2) * bw, tm_row, bar, xc, yh2, zc);
                    tma_load_3d(pp + (size_t)(ty + 3) * bw, tm_row, bar, xc, yh3, zc);
                }
            }
        };
        bool failed = false;  // a bounded wait of this thread ran out
        auto wait = [&](int i) {
            if (!mbar_wait_bounded(&head->bar[cslot(i)], cphase(i), a.spin_limit)) {
                failed = true;
                atomicMax(&J->err, DEV_TMA_TIMEOUT);
                atomicMax(a.err, DEV_TMA_TIMEOUT);
            }
        };
        // x neighbours of the two halves of a strip: lA/rA left/right of half
        // A, lB/rB of half B (row-relative shared-memory columns cl*, cr*)
        auto edges = [&](const Strip<T>& v, const T* rowp, int clA, int crA, int clB, int crB, T& lA, T& rA, T& lB,
                         T& rB) {
            if constexpr (sizeof(T) == 8) {
                // FP64: from the row in shared memory (a 64-bit value costs two
                // shuffles and two selects per use)
                lA = rowp[clA];
                rA = rowp[crA];
                lB = rowp[clB];
                rB = rowp[crB];
                return;
            }
            const T aF = v.get(0), aL = v.get(HW - 1), bF = v.get(HW), bL = v.get(W - 1);
            const T sAL = __shfl_sync(0xffffffffu, aL, lsrc), sBL = __shfl_sync(0xffffffffu, bL, lsrc);
            const T sAF = __shfl_sync(0xffffffffu, aF, rsrc), sBF = __shfl_sync(0xffffffffu, bF, rsrc);
            if (seg) {
                // thread 0's left is the last thread's B (A) half; the last
                // thread's right is thread 0's B (A) half
                lA = first ? sBL : sAL;
                lB = first ? sAL : sBL;
                rA = last ? sBF : sAF;
                rB = last ? sAF : sBF;
                if (!perX && first) lA = aF;
                if (!perX && last) rB = bL;
            } else {
                lA = sAL, lB = sBL, rA = sAF, rB = sBF;
                if (leftSm) {
                    lA = rowp[clA];
                    lB = rowp[clB];
                }
                if (rightSm) {
                    rA = rowp[crA];
                    rB = rowp[crB];
                }
            }
        };

        const int nplanes = L + 4;
        const int npro = min(NBUF, nplanes);
        for (int i = 0; i < npro; ++i) issue(i);
        int issued = npro;  // planes issued so far (uniform)
        int waited = 0;     // planes waited so far (uniform)
        long long macc = 0;  // stored mass of this thread's strips, 2^-32 units

        // One plane of the march: mu on plane i (stage A), then c_new on
        // plane i-1 (stage B).  Register roles rotate between the three call
        // sites so the z-queue never moves: cp/cc/cn = c(i-1), c(i), c(i+1);
        // mp/mc/mn = mu(i-2), mu(i-1), mu(i).  mslot/mslot_prev are the mu
        // ring slots of planes i and i-1 (fixed per call site).
        auto plane = [&](int i, int mslot, int mslot_prev, Strip<T>& cp, Strip<T>& cc, Strip<T>& cn, Strip<T>& mp,
                         Strip<T>& mc, Strip<T>& mn) -> bool {
            wait(i + 1);
            waited = i + 2;
            cn = ld_strip(cplane(i + 1) + cOwn + cRowOwn * bw, cOffB);
            // ---- stage A: mu on plane i
            {
                const T* p = cplane(i);
                Strip<T> up, dn;
                if constexpr (!FLAT) {
                    up = ld_strip(p + cOwn + m * bw, cOffB);
                    dn = ld_strip(p + cOwn + (m + 2) * bw, cOffB);
                }
                T lA, rA, lB, rB;
                const T* rowp = p + cRowOwn * bw;
                edges(cc, rowp, cLA, cRA, cLB, cRB, lA, rA, lB, rB);
                if constexpr (PAIRS) {
                    unsigned long long lp[4];
                    lap_pairs<FLAT>(cc, lA, rA, lB, rB, up, dn, cp, cn, lp);
                    const unsigned long long m1 = splat2(-1.f), mk = splat2(-kapc);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const unsigned long long df = mul2(cc.p[k], fma2(cc.p[k], cc.p[k], m1));
                        mn.p[k] = fma2(lp[k], mk, df);
                    }
                } else {
                    const bool sLo = zout(i - 1), sHi = zout(i + 1);
                    T mu[W];
#pragma unroll
                    for (int e = 0; e < W; ++e) {
                        const T c0 = cc.get(e);
                        const int h = e / HW, k = e % HW;
                        const T xm = k > 0 ? cc.get(e - 1) : (h == 0 ? lA : lB);
                        const T xp = k < HW - 1 ? cc.get(e + 1) : (h == 0 ? rA : rB);
                        T zm = cp.get(e), zp = cn.get(e), ym = c0, yp = c0;
                        if constexpr (!FLAT) {
                            ym = up.get(e);
                            yp = dn.get(e);
                        }
                        if constexpr (!SIMPLE) {
                            if (sLo) zm = c0;
                            if (sHi) zp = c0;
                            if (subUp) ym = c0;
                            if (subDn) yp = c0;
                        }
                        const T lap = lap7<T, FLAT, SIMPLE>(c0, xp, xm, yp, ym, zp, zm, cx, cy, cz, divX, divY, divZ);
                        mu[e] = chem_pot(c0, lap, kap);
                    }
                    if constexpr (sizeof(T) == 4) {
#pragma unroll
                        for (int k = 0; k < 4; ++k) mn.p[k] = pk2(mu[2 * k], mu[2 * k + 1]);
                    } else {
#pragma unroll
                        for (int e = 0; e < W; ++e) mn.v[e] = mu[e];
                    }
                }
                if (active) st_strip(mplane(mslot) + mOwn + m * bw, mOffB, mn);
            }
            if (__syncthreads_or(failed)) return false;  // the plane's barrier, and a uniform abort
            // planes <= i were last read by stage A of this plane (and as `cn`
            // before it): their ring slots take the planes up to i+NBUF
            for (; issued <= i + NBUF && issued < nplanes; ++issued) issue(issued);
            // ---- stage B: output plane i-1
            if (i >= 3) {
                const T* q = mplane(mslot_prev);
                const int zo = zfirst + dir * (i - 1);
                const size_t zoff = (size_t)zo * pstride;
                Strip<T> up, dn;
                if constexpr (!FLAT) {
                    up = ld_strip(q + mOwn + mUpRow * bw, mOffB);
                    dn = ld_strip(q + mOwn + mDnRow * bw, mOffB);
                }
                T lA, rA, lB, rB;
                const int mrow = FLAT ? 0 : m;
                edges(mc, q + mrow * bw, mLA, mRA, mLB, mRB, lA, rA, lB, rB);
                // does the mass-nudge window reach into this plane?  (uniform)
                const bool hit = MASS && ((zo >= wz0 && zo <= wz1) || zo <= wz2);
                if (outrow) {
                    Strip<T> out;
                    if constexpr (PAIRS) {
                        unsigned long long lp[4];
                        lap_pairs<FLAT>(mc, lA, rA, lB, rB, up, dn, mp, mn, lp);
                        const unsigned long long dt2 = splat2(dtMc);
#pragma unroll
                        for (int k = 0; k < 4; ++k) out.p[k] = fma2(lp[k], dt2, cp.p[k]);
                        if constexpr (MASS) {
                            if (hit && window_reaches((long long)(zoff + rowoff - xA), nx, head->nudge_begin,
                                                      head->nudge_count, (long long)pstride * nz)) {
                                float o[8];
#pragma unroll
                                for (int e = 0; e < 8; ++e) o[e] = out.get(e);
                                nudge_strip(o, (long long)(zoff + rowoff), gOffB, head->nudge_begin, head->nudge_count,
                                            (long long)pstride * nz);
#pragma unroll
                                for (int k = 0; k < 4; ++k) out.p[k] = pk2(o[2 * k], o[2 * k + 1]);
                            }
                            if (measure) macc += strip_mass(out.get(0), out.get(1), out.get(2), out.get(3), out.get(4), out.get(5),
                                               out.get(6), out.get(7));
                        }
                    } else {
                        const bool sLo = zout(i - 2), sHi = zout(i);
                        T o[W];
#pragma unroll
                        for (int e = 0; e < W; ++e) {
                            const T mu = mc.get(e);
                            const int h = e / HW, k = e % HW;
                            const T xm = k > 0 ? mc.get(e - 1) : (h == 0 ? lA : lB);
                            const T xp = k < HW - 1 ? mc.get(e + 1) : (h == 0 ? rA : rB);
                            T zm = mp.get(e), zp = mn.get(e), ym = mu, yp = mu;
                            if constexpr (!FLAT) {
                                ym = up.get(e);
                                yp = dn.get(e);
                            }
                            if constexpr (!SIMPLE) {
                                if (sLo) zm = mu;
                                if (sHi) zp = mu;
                                if (subUp) ym = mu;
                                if (subDn) yp = mu;
                            }
                            const T lap = lap7<T, FLAT, SIMPLE>(mu, xp, xm, yp, ym, zp, zm, cx, cy, cz, divX, divY, divZ);
                            const T c0 = cp.get(e);
                            if constexpr (sizeof(T) == 4) {
                                o[e] = fmaf(lap, dtM, c0);
                            } else {
                                o[e] = A::add(c0, A::mul(lap, dtM));
                            }
                        }
                        if constexpr (sizeof(T) == 4) {
                            if constexpr (MASS) {
                                if (hit && window_reaches((long long)(zoff + rowoff - xA), nx, head->nudge_begin,
                                                          head->nudge_count, (long long)pstride * nz)) {
                                    float t[8];
#pragma unroll
                                    for (int e = 0; e < 8; ++e) t[e] = o[e];
                                    nudge_strip(t, (long long)(zoff + rowoff), gOffB, head->nudge_begin,
                                                head->nudge_count, (long long)pstride * nz);
#pragma unroll
                                    for (int e = 0; e < 8; ++e) o[e] = t[e];
                                }
                                if (measure) macc += strip_mass(o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7]);
                            }
#pragma unroll
                            for (int k = 0; k < 4; ++k) out.p[k] = pk2(o[2 * k], o[2 * k + 1]);
                        } else {
#pragma unroll
                            for (int e = 0; e < W; ++e) out.v[e] = o[e];
                        }
                    }
                    st_strip(dst + zoff + rowoff, gOffB, out);
                }
            }
            return true;
        };

        Strip<T> c0r, c1r, c2r, m0r, m1r, m2r;
        zero_strip(m0r);
        zero_strip(m1r);
        wait(0);
        c0r = ld_strip(cplane(0) + cOwn + cRowOwn * bw, cOffB);
        wait(1);
        c1r = ld_strip(cplane(1) + cOwn + cRowOwn * bw, cOffB);
        waited = 2;

        // planes i = 1, 4, 7, ... have i mod 3 == 1: mu slots 1, 2, 0 in turn
        bool ok = true;
        int i = 1;
        for (; ok && i + 2 <= L + 2; i += 3) {
            ok = plane(i, 1, 0, c0r, c1r, c2r, m0r, m1r, m2r);
            if (ok) ok = plane(i + 1, 2, 1, c1r, c2r, c0r, m1r, m2r, m0r);
            if (ok) ok = plane(i + 2, 0, 2, c2r, c0r, c1r, m2r, m0r, m1r);
        }
        if (ok && i <= L + 2) {
            ok = plane(i, 1, 0, c0r, c1r, c2r, m0r, m1r, m2r);
            ++i;
        }
        if (ok && i <= L + 2) ok = plane(i, 2, 1, c1r, c2r, c0r, m1r, m2r, m0r);
        gseq += nplanes;

        if (!ok) {
            // drain: wait (bounded) for the planes issued but not yet
            // consumed, so no copy lands after the CTA has exited
            for (int k = waited; k < issued; ++k)
                mbar_wait_bounded(&head->bar[cslot(k)], cphase(k), a.spin_limit);
            return;
        }

        // ---- item epilogue: partial mass, completion count, last-item work
        const int nitems_job = J->ntile * J->nchunk;
        if (measure) {
            // |strip| < 2^36 units, a thread holds at most nz strips, a CTA
            // at most 640 threads: the item sum fits 64 bits
            long long* red = reinterpret_cast<long long*>(head->red);
            const int nw = (tjob + 31) >> 5;
            long long v = active ? macc : 0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0 && (tid >> 5) < nw) red[tid >> 5] = v;
            __syncthreads();
            if (tid < 32) {
                long long r = lane < nw ? red[lane] : 0;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) r += __shfl_down_sync(0xffffffffu, r, off);
                if (lane == 0) J->partial[local] = r;
            }
        }
        if (measure) __threadfence();  // this item's part of the new field, before the completion count
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            const unsigned prev = atomicAdd(&J->done, 1u);
            head->flag = (prev == (unsigned)nitems_job - 1u);
            if (head->flag) __threadfence();
        }
        __syncthreads();
        if (head->flag) {
            if constexpr (MASS)
                mass_feedback_step_end(J, measure, (long long)pstride * nz, nitems_job, reinterpret_cast<float*>(dst),
                                       head);
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

// ---------------------------------------------------------------------------
// Per-step noise, the random fluctuation term of TIPSphil::updatePhaseField
// (TIPSphil.cpp:200-209): after a step every site gets c += dt*(noise*(r -
// 0.5)), each product rounded on its own as there.  SIPS skips sites at or
// above phiCutoff (SIPS.cpp:226-248); SIPSternary adds the negated increment
// to its second field (SIPSternary.cpp:256-277), which a negative strength
// with the same seed gives exactly.  The reference draws r
// from rand(); here r comes from Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011), keyed by the
// job's seed, with counter (site / 4, step): four sites per draw, r =
// (word + 0.5) * 2^-32, so r depends on (seed, site, step) only.

// Adds the noise of the step just taken (the job's step counter) once: a
// replayed graph step that skipped the job leaves noise_step == step, and
// the blocks return.  The last block to finish records the step.
template <typename T>
__global__ void ch_noise_kernel(JobDev* job)
{
    __shared__ long long st;
    __shared__ int go;
    JobDev* J = job;
    if (threadIdx.x == 0) {
        st = *((volatile long long*)&J->step);
        go = st > *((volatile long long*)&J->noise_step);
    }
    __syncthreads();
    if (!go) return;
    T* c = static_cast<T*>(J->buf[st & 1]);
    const long long n = (long long)J->nx * J->ny * J->nz;
    const double noise = J->noise, dt = J->dtM_dt, cutoff = J->noise_cutoff;
    const uint2 key = make_uint2((uint32_t)J->noise_seed, (uint32_t)(J->noise_seed >> 32));
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; 4 * g < n; g += (long long)gridDim.x * blockDim.x) {
        const uint4 w = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)(g >> 32), (uint32_t)st, (uint32_t)(st >> 32)), key);
        const uint32_t word[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const long long s = 4 * g + e;
            if (s >= n) break;
            const double r = __dadd_rn(__dmul_rn((double)word[e], 2.3283064365386963e-10), 1.1641532182693481e-10);
            const T cs = c[s];
            // SIPS.cpp:239-240: no noise where c >= phiCutoff (the cutoff is +inf elsewhere)
            const double val = (double)cs >= cutoff ? 0.0 : __dmul_rn(noise, __dsub_rn(r, 0.5));
            const double inc = __dmul_rn(dt, val);
            if constexpr (sizeof(T) == 8) c[s] = __dadd_rn(cs, inc);
            else c[s] = cs + (float)inc;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&J->noise_done, 1u) == gridDim.x - 1) {
            J->noise_step = st;
            J->noise_done = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Variable-mobility steps, FP64, every operation rounded on its own in the
// reference's order; log, exp, pow, erf and sqrt are CUDA's (within an ulp or
// two of the host's libm).  Pass 1 stores mu and the mobility of every site;
// pass 2 forms the harmonic-mean Laplacian of SfieldFD::Laplacian(const
// SfieldFD&) (SfieldFD.cpp:333-355) and updates c.  Boundaries as the
// reference's updateBoundaries: periodic axes wrap, a no-flux neighbour is the
// site itself.  The models (FhModel):
//  - TIPSphil::updatePhaseField (TIPSphil.cpp:113-211) and TIPSbathPHIL's
//    (TIPSbathPHIL.cpp:114-208): Flory-Huggins mu scaled by kT, Phillies
//    mobility over the second derivative, crystallisation factor;
//  - SIPS::updatePhaseField (SIPS.cpp:130-249): chi(x, step) from an erf
//    front, mu from the clamped concentration, Phillies mobility scaled by
//    0.95 + 0.25*log(1.0225 - chi fraction);
//  - one field of SIPSternary::updatePhaseField (SIPSternary.cpp:132-278).
//    There the Flory-Huggins derivatives are assigned to variables declared
//    inside the branches (SIPSternary.cpp:175-216), which shadow the df_c and
//    df_n that mu is formed from, so mu = 0.0 - K*lap(c) and the mobility is
//    the constant Mpp (Mnn): the fields step independently.  The GPU takes
//    the same arithmetic.

// The scalars of a job the variable-mobility passes use at every site,
// copied out of JobDev once per thread.
struct FhView {
    int nx, ny, nz, flags;
    double cx, cy, cz, kap, dt, noise, cutoff;
};
__device__ __forceinline__ FhView fh_view(const JobDev& J)
{
    return {J.nx, J.ny, J.nz, J.flags, J.cx, J.cy, J.cz, J.kap, J.dtM_dt, J.noise, J.noise_cutoff};
}

// The neighbours of site s one step down / up an axis of length n and
// stride st, from its coordinate i: the periodic wrap, or on a no-flux axis
// the site itself (the ghost copy): the site at coordinate
// wrap_or_clamp(i -/+ 1, n) on that axis, without its modulo and without
// forming the index from (x, y, z).
// I is the index type: 32-bit for fields of fewer than 2^31 sites (one
// integer instruction per step where 64-bit indices take two), else size_t.
template <typename I>
__device__ __forceinline__ I fh_down(I s, int i, I st, I span, bool per)
{
    return i > 0 ? s - st : (per ? s + span : s);
}
template <typename I>
__device__ __forceinline__ I fh_up(I s, int i, int n, I st, I span, bool per)
{
    return i < n - 1 ? s + st : (per ? s - span : s);
}

// Pass 1: mu and the reciprocal mobility 1/mob of every site (F.mu, F.mob).
// A thread keeps one x for all its sites (the grid's stride is a multiple
// of nx), so the per-x constants of the step (fh_column) are formed once.
template <typename I>
__device__ __forceinline__ void fh_mu_mob_sites(const JobDev& J, const FhDev& F, const FhView& V)
{
    using A = Arith<double>;
    const int nx = V.nx, ny = V.ny, nz = V.nz;
    const I n = (I)nx * ny * nz;
    const double* __restrict__ c = static_cast<const double*>(J.buf[J.step & 1]);
    // the step being taken (PFApp passes it as current_step)
    const double cs = (double)(J.step + 1);
    const bool pX = V.flags & JF_PER_X, pY = V.flags & JF_PER_Y, pZ = V.flags & JF_PER_Z;
    const I first = (I)blockIdx.x * blockDim.x + threadIdx.x;
    const I stride = (I)gridDim.x * blockDim.x;  // a multiple of nx (the host's launch)
    const int x = (int)(first % nx);
    const FhCol col = fh_column(F, x, cs, V.dt);
    // the row (y, z) of site s, advanced by the stride's whole rows without
    // a division per site
    const I r0 = first / nx, dr = stride / nx;
    int y = (int)(r0 % ny), z = (int)(r0 / ny);
    const int dy = (int)(dr % ny), dz = (int)(dr / ny);
    // strides and wrap spans of the three axes
    const I sy = (I)nx, sz = (I)nx * ny;
    const I wx = (I)(nx - 1), wy = (I)(ny - 1) * sy, wz = (I)(nz - 1) * sz;
    for (I s = first; s < n; s += stride) {
        const double cc = c[s];
        const double xp = c[fh_up(s, x, nx, (I)1, wx, pX)], xm = c[fh_down(s, x, (I)1, wx, pX)];
        const double zp = c[fh_up(s, z, nz, sz, wz, pZ)], zm = c[fh_down(s, z, sz, wz, pZ)];
        double lapc;
        if (V.flags & JF_FLAT) {
            lapc = A::add(axis_term(xp, xm, cc, V.cx, V.flags & JF_DIV_X), axis_term(zp, zm, cc, V.cz, V.flags & JF_DIV_Z));
        } else {
            const double yp = c[fh_up(s, y, ny, sy, wy, pY)], ym = c[fh_down(s, y, sy, wy, pY)];
            lapc = A::add(A::add(axis_term(xp, xm, cc, V.cx, V.flags & JF_DIV_X), axis_term(yp, ym, cc, V.cy, V.flags & JF_DIV_Y)),
                          axis_term(zp, zm, cc, V.cz, V.flags & JF_DIV_Z));
        }
        double mu, rmob;
        fh_site_r(F, col, cc, lapc, V.kap, &mu, &rmob);
        F.mu[s] = mu;
        F.mob[s] = rmob;  // the reciprocal every face of the site uses
        y += dy;
        z += dz;
        if (y >= ny) {
            y -= ny;
            z += 1;
        }
    }
}

__global__ void __launch_bounds__(256, 4) fh_mu_mob_kernel(JobDev* job)
{
    const JobDev& J = *job;
    if (J.step >= J.target) return;
    // the job's scalars, read once (the field stores may alias *job as far
    // as the compiler knows); the model's fields stay in memory, which
    // measured faster here than a copy that spills
    const FhView V = fh_view(J);
    if ((long long)V.nx * V.ny * V.nz < (1LL << 31)) fh_mu_mob_sites<uint32_t>(J, *J.fh, V);
    else fh_mu_mob_sites<size_t>(J, *J.fh, V);
}

// Pass 2: c += dt * div(mob grad mu) (SfieldFD::Laplacian(const SfieldFD&),
// SfieldFD.cpp:333-355) from mu and the reciprocal mobilities of pass 1:
// each face's harmonic mean 2/(1/mob_a + 1/mob_b) from the two stored
// reciprocals.  A constant-mobility field (SIPSternary) takes the
// reference's per-axis form with its operands in its order, so the same
// value; the Flory-Huggins models take the three axes over one common
// denominator (fh_div_frac), one division per site instead of six.
// Then the per-step noise (TIPSphil.cpp:200-209) with the word
// ch_noise_kernel gives the site: one draw of the counter-based generator
// per four consecutive sites (site/4, step).
template <typename I>
__device__ __forceinline__ double fh_update_site(const FhView& J, const double* __restrict__ c,
                                                 const double* __restrict__ mu, const double* __restrict__ rmob,
                                                 I s, int x, int y, int z, bool linear)
{
    using A = Arith<double>;
    const int nx = J.nx, ny = J.ny, nz = J.nz;
    const bool pX = J.flags & JF_PER_X, pY = J.flags & JF_PER_Y, pZ = J.flags & JF_PER_Z;
    const double a0 = mu[s], ro = rmob[s];
    const I sy = (I)nx, sz = (I)nx * ny;
    const I wx = (I)(nx - 1), wy = (I)(ny - 1) * sy, wz = (I)(nz - 1) * sz;
    const I ixm = fh_down(s, x, (I)1, wx, pX), ixp = fh_up(s, x, nx, (I)1, wx, pX);
    const I izm = fh_down(s, z, sz, wz, pZ), izp = fh_up(s, z, nz, sz, wz, pZ);
    const bool flat = J.flags & JF_FLAT;
    I iym = s, iyp = s;
    if (!flat) iym = fh_down(s, y, sy, wy, pY), iyp = fh_up(s, y, ny, sy, wy, pY);
    double lap;
    if (linear) {
        // constant mobility (SIPSternary): the reference's per-axis form, bit for bit
        const double lx = fh_axis_r(mu[ixm], mu[ixp], a0, rmob[ixm], rmob[ixp], ro, J.cx, J.flags & JF_DIV_X);
        const double lz = fh_axis_r(mu[izm], mu[izp], a0, rmob[izm], rmob[izp], ro, J.cz, J.flags & JF_DIV_Z);
        if (flat) {
            lap = A::add(lx, lz);
        } else {
            const double ly = fh_axis_r(mu[iym], mu[iyp], a0, rmob[iym], rmob[iyp], ro, J.cy, J.flags & JF_DIV_Y);
            lap = A::add(A::add(lx, ly), lz);
        }
    } else {
        const FhFrac fx = fh_axis_frac(mu[ixm], mu[ixp], a0, rmob[ixm], rmob[ixp], ro, J.cx, J.flags & JF_DIV_X);
        const FhFrac fz = fh_axis_frac(mu[izm], mu[izp], a0, rmob[izm], rmob[izp], ro, J.cz, J.flags & JF_DIV_Z);
        FhFrac fy{0.0, 1.0};
        if (!flat) fy = fh_axis_frac(mu[iym], mu[iyp], a0, rmob[iym], rmob[iyp], ro, J.cy, J.flags & JF_DIV_Y);
        lap = fh_div_frac(fx, fy, fz, flat);
    }
    return A::add(c[s], A::mul(J.dt, lap));  // c += dt * lap (TIPSphil.cpp:194)
}

// A warp takes 128 consecutive sites, lane l the sites base + 32e + l
// (e = 0..3), so every gather of mu and 1/mob is one coalesced run per warp.
// The noise counter keeps its grouping (site/4, step): lane l draws the
// words of group base/4 + l, and the lane of a site takes its word from the
// group's lane by shuffles, the same word the site gets in ch_noise_kernel.
__global__ void __launch_bounds__(256, 4) fh_update_kernel(JobDev* job)
{
    using A = Arith<double>;
    const JobDev& J = *job;
    // the model's and the job's fields, read once: as far as the compiler
    // knows the field stores below may alias them, so it would read them
    // again for every site
    const FhDev F = *J.fh;
    const FhView V = fh_view(J);
    const long long n = (long long)J.nx * J.ny * J.nz;
    const int lane = threadIdx.x & 31;
    const long long base = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 128;  // the warp's sites
    if (J.step >= J.target || base >= n) return;  // uniform over the warp
    const int par = (int)(J.step & 1);
    const double* __restrict__ c = static_cast<const double*>(J.buf[par]);
    double* __restrict__ out = static_cast<double*>(J.buf[par ^ 1]);
    const bool linear = F.model == kFhLinear;
    const bool small = n < (1LL << 31);  // 32-bit site indices
    uint32_t word[4] = {0u, 0u, 0u, 0u};
    const bool noisy = J.noise != 0.0;
    if (noisy) {
        const long long st = J.step + 1;  // the step being taken
        const long long g = base / 4 + lane;  // sites 4g .. 4g+3
        const uint2 key = make_uint2((uint32_t)J.noise_seed, (uint32_t)(J.noise_seed >> 32));
        const uint4 w = philox4x32_10(make_uint4((uint32_t)g, (uint32_t)(g >> 32), (uint32_t)st, (uint32_t)(st >> 32)), key);
        word[0] = w.x, word[1] = w.y, word[2] = w.z, word[3] = w.w;
    }
    // coordinates of the lane's first site; each next one lies 32 sites on
    long long s = base + lane;
    const long long r0 = s / J.nx;
    int x = (int)(s - r0 * J.nx), y = (int)(r0 % J.ny), z = (int)(r0 / J.ny);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if (e > 0) {
            s += 32;
            x += 32;
            while (x >= V.nx) {
                x -= V.nx;
                if (++y == V.ny) {
                    y = 0;
                    ++z;
                }
            }
        }
        // the word of site s: group s/4 is lane 8e + l/4's, component s & 3 = l & 3
        uint32_t wd = 0u;
        if (noisy) {
            const int src = 8 * e + (lane >> 2), k = lane & 3;
            const uint32_t w0 = __shfl_sync(0xffffffffu, word[0], src), w1 = __shfl_sync(0xffffffffu, word[1], src);
            const uint32_t w2 = __shfl_sync(0xffffffffu, word[2], src), w3 = __shfl_sync(0xffffffffu, word[3], src);
            wd = k == 0 ? w0 : (k == 1 ? w1 : (k == 2 ? w2 : w3));
        }
        if (s >= n) continue;
        double v = small ? fh_update_site(V, c, F.mu, F.mob, (uint32_t)s, x, y, z, linear)
                         : fh_update_site(V, c, F.mu, F.mob, (size_t)s, x, y, z, linear);
        if (noisy) {
            // SIPS.cpp:239-240: no noise at or above the cutoff (+inf elsewhere)
            const double r = A::add(A::mul((double)wd, 2.3283064365386963e-10), 1.1641532182693481e-10);
            const double val = v >= V.cutoff ? 0.0 : A::mul(V.noise, A::sub(r, 0.5));
            v = A::add(v, A::mul(V.dt, val));
        }
        out[s] = v;
    }
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
        job->nudge_begin = 0;
        job->nudge_count = 0;
        job->nudge_applied = 0;
        job->nudge_rest = 0;
        job->noise_step = 0;
        job->noise_done = 0;
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

// Stored mass of an uploaded FP32 field, measured as the step kernel
// measures it (strip_mass, 2^-32 units): the FP32 mass target.
__global__ void ch_mass_partial(const JobDev* job, long long* part)
{
    __shared__ long long red[32];
    const JobDev& J = *job;
    const int nx = J.nx, nq = nx / 8;
    const long long nstrips = (long long)J.ny * J.nz * nq;
    const float* c = static_cast<const float*>(J.buf[J.step & 1]);
    long long s = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nstrips;
         t += (long long)gridDim.x * blockDim.x) {
        const float* row = c + (t / nq) * nx;
        const int xa = 4 * (int)(t % nq), xb = xa + nx / 2;
        s += strip_mass(row[xa], row[xa + 1], row[xa + 2], row[xa + 3], row[xb], row[xb + 1], row[xb + 2], row[xb + 3]);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long b = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += red[w];
        part[blockIdx.x] = b;
    }
}

__global__ void ch_mass_final(const long long* part, int nblocks, JobDev* job)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    __int128 s = 0;
    for (int b = 0; b < nblocks; ++b) s += part[b];
    const double m = (double)s / (double)kMassScale;
    job->mass_target = m;
    job->mass_last = m;
    job->nudge_begin = 0;
    job->nudge_count = 0;
    job->nudge_applied = 0;
    job->nudge_rest = 0;
}

}  // namespace mg
