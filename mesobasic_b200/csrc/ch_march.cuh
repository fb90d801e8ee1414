// The fused Cahn-Hilliard step for the common case -- every axis periodic
// with equal spacing, 3-D, a row width NXC <= 256 fixed at compile time --
// in FP32 (paired f32x2 arithmetic, optional FP64 mass feedback) and FP64
// (every operation rounded on its own, in the reference's order).
//
// Same decomposition, tile, TMA ring, register z-queues, arithmetic and
// epilogue as ch_step_kernel (ch_kernels.cuh), so the results are
// bit-identical to it; what changes is the per-plane overhead of the march:
//  - the plane loop is unrolled by lcm(NBUF, 3), so the ring slot of every
//    plane, the mu-ring slot and the register roles of the z-queues are
//    compile-time constants; each item starts its planes at ring slot 0,
//    and the mbarrier parity of a slot is one bit of a mask that flips on
//    every completed wait;
//  - a plane is "wait for c(i+1); mu on plane i; barrier; refill; c_new on
//    plane i-1".  (Running stage B before the barrier, so that both stages
//    share one stretch, measured 1-7 % slower.)
//  - x-neighbours: FP32 rows whose threads form a power-of-two segment of
//    a warp take them from warp shuffles; other rows (FP64, FP32 widths 96,
//    160, 192, 224) from the row in shared memory.
#pragma once

#include "ch_device.cuh"

namespace mg {

template <typename T>
struct MarchIO;

template <>
struct MarchIO<float> {
    static __device__ __forceinline__ Strip<float> lds(uint32_t a, uint32_t offB) { return lds_strip(a, offB); }
    static __device__ __forceinline__ void sts(uint32_t a, uint32_t offB, const Strip<float>& s)
    {
        sts_v2(a, s.p[0], s.p[1]);
        sts_v2(a + offB, s.p[2], s.p[3]);
    }
    static __device__ __forceinline__ void stg(float* g, int offB, const Strip<float>& s)
    {
        stg_v2(g, s.p[0], s.p[1]);
        stg_v2(g + offB, s.p[2], s.p[3]);
    }
    static __device__ __forceinline__ float ld1(uint32_t a)
    {
        float x;
        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(x) : "r"(a) : "memory");
        return x;
    }
};

template <>
struct MarchIO<double> {
    static __device__ __forceinline__ Strip<double> lds(uint32_t a, uint32_t offB)
    {
        Strip<double> s;
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(s.v[0]), "=d"(s.v[1]) : "r"(a) : "memory");
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(s.v[2]), "=d"(s.v[3]) : "r"(a + offB) : "memory");
        return s;
    }
    static __device__ __forceinline__ void sts(uint32_t a, uint32_t offB, const Strip<double>& s)
    {
        asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(s.v[0]), "d"(s.v[1]) : "memory");
        asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a + offB), "d"(s.v[2]), "d"(s.v[3]) : "memory");
    }
    static __device__ __forceinline__ void stg(double* g, int offB, const Strip<double>& s)
    {
        *reinterpret_cast<double2*>(g) = make_double2(s.v[0], s.v[1]);
        *reinterpret_cast<double2*>(g + offB) = make_double2(s.v[2], s.v[3]);
    }
    static __device__ __forceinline__ double ld1(uint32_t a)
    {
        double x;
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(x) : "r"(a) : "memory");
        return x;
    }
};

// mu of one strip (stage A) from the strip c, its x-neighbours, the rows
// above/below (up/dn) and the planes before/after (zl/zh)
template <typename T>
__device__ __forceinline__ void march_mu(const Strip<T>& c, T lA, T rA, T lB, T rB, const Strip<T>& up,
                                         const Strip<T>& dn, const Strip<T>& zl, const Strip<T>& zh, double kap,
                                         float kapc, Strip<T>& mu)
{
    if constexpr (sizeof(T) == 4) {
        unsigned long long lp[4];
        lap_pairs<false>(c, lA, rA, lB, rB, up, dn, zl, zh, lp);
        const unsigned long long m1 = splat2(-1.f), mk = splat2(-kapc);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const unsigned long long df = mul2(c.p[k], fma2(c.p[k], c.p[k], m1));
            mu.p[k] = fma2(lp[k], mk, df);
        }
    } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const double xm = (e & 1) ? c.v[e - 1] : (e == 0 ? lA : lB);
            const double xp = (e & 1) ? (e == 1 ? rA : rB) : c.v[e + 1];
            const double lap = lap7<double, false, true>(c.v[e], xp, xm, dn.v[e], up.v[e], zh.v[e], zl.v[e], 1.0, 1.0,
                                                         1.0, false, false, false);
            mu.v[e] = chem_pot(c.v[e], lap, kap);
        }
    }
}

// c_new of one strip (stage B): c + lap(mu) * dt*M
template <typename T>
__device__ __forceinline__ void march_update(const Strip<T>& mu, T lA, T rA, T lB, T rB, const Strip<T>& up,
                                             const Strip<T>& dn, const Strip<T>& zl, const Strip<T>& zh,
                                             const Strip<T>& c, double dtM, float dtMc, Strip<T>& out)
{
    if constexpr (sizeof(T) == 4) {
        unsigned long long lp[4];
        lap_pairs<false>(mu, lA, rA, lB, rB, up, dn, zl, zh, lp);
        const unsigned long long dt2 = splat2(dtMc);
#pragma unroll
        for (int k = 0; k < 4; ++k) out.p[k] = fma2(lp[k], dt2, c.p[k]);
    } else {
        using A = Arith<double>;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const double xm = (e & 1) ? mu.v[e - 1] : (e == 0 ? lA : lB);
            const double xp = (e & 1) ? (e == 1 ? rA : rB) : mu.v[e + 1];
            const double lap = lap7<double, false, true>(mu.v[e], xp, xm, dn.v[e], up.v[e], zh.v[e], zl.v[e], 1.0, 1.0,
                                                         1.0, false, false, false);
            out.v[e] = A::add(c.v[e], A::mul(lap, dtM));
        }
    }
}

// Ring and shared-memory state of a CTA running march items.
struct MarchCta {
    SmemHead* head;
    uint32_t cbase, mbase, bar0;
    uint32_t ph;  // parity of the next completion of each ring slot (bit s)
};

// shared-memory elements of a c plane and a mu plane: compile-time when the
// tile height TY is (every job of the launch has it; NXC is a multiple of 32,
// so the rounded plane of the host equals the product)
template <int NXC, int TY>
__device__ __forceinline__ uint32_t march_cplane(const StepArgs& a)
{
    return TY ? (uint32_t)((TY + 4) * NXC) : (uint32_t)a.cplane;
}
template <int NXC, int TY>
__device__ __forceinline__ uint32_t march_mplane(const StepArgs& a)
{
    return TY ? (uint32_t)((TY + 2) * NXC) : (uint32_t)a.mplane;
}

template <int NBUF>
__device__ __forceinline__ MarchCta march_setup(const StepArgs& a, uint32_t es, uint32_t cplane)
{
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* smem_raw = smem_dyn + ((128u - (smem_addr(smem_dyn) & 127u)) & 127u);
    MarchCta m;
    m.head = reinterpret_cast<SmemHead*>(smem_raw);
    m.cbase = smem_addr(smem_raw) + (uint32_t)(((sizeof(SmemHead) + 127) / 128) * 128);
    m.mbase = m.cbase + NBUF * cplane * es;
    m.bar0 = smem_addr(&m.head->bar[0]);
    m.ph = 0;
    if (threadIdx.x == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&m.head->bar[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    return m;
}

// One work item (y-tile x z-chunk) of job J, slot `local` among its items.
// Returns false when a bounded wait ran out (the CTA must exit; the job and
// the launch are flagged and the copies in flight drained).
template <typename T, int NXC, int NBUF, bool MASS, int TY>
__device__ __forceinline__ bool march_item(const StepArgs& a, JobDev* J, int local, MarchCta& cta)
{
    constexpr int W = Strip<T>::W, HW = W / 2;
    constexpr int NQ = NXC / W;  // threads per row
    constexpr bool SEG = sizeof(T) == 4 && NQ <= 32 && (NQ & (NQ - 1)) == 0;
    constexpr uint32_t ES = sizeof(T);
    constexpr uint32_t ROWB = NXC * ES;        // bytes of a shared-memory row (one TMA box)
    constexpr uint32_t HALFB = NXC / 2 * ES;   // half B of a strip sits nx/2 elements after half A
    constexpr int U = (NBUF % 3 == 0) ? NBUF : 3 * NBUF;  // planes per unrolled block
    static_assert(NXC % W == 0 && NXC <= 256 && !(MASS && sizeof(T) == 8), "unsupported march variant");
    static_assert(NBUF >= 3 && NBUF <= 8, "ring depth");
    using IO = MarchIO<T>;

    SmemHead* head = cta.head;
    const uint32_t cbase = cta.cbase, mbase = cta.mbase, bar0 = cta.bar0;
    const uint32_t cplaneB = march_cplane<NXC, TY>(a) * ES, mplaneB = march_mplane<NXC, TY>(a) * ES;
    const int spin = (int)min(a.spin_limit, (long long)0x7fffffff);
    uint32_t& ph = cta.ph;
    const int tid = threadIdx.x;
    const int lane = tid & 31;

    // lane segment of a row (SEG) and the row-relative x of the strip halves
    const int tx = tid % NQ;
    const int segbase = lane & ~(NQ - 1);
    const int lsrc = segbase | ((lane - 1) & (NQ - 1));
    const int rsrc = segbase | ((lane + 1) & (NQ - 1));
    const bool first = tx == 0, last = tx == NQ - 1;
    const int xA = tx * HW;
    // row-relative byte offsets of the four x-neighbours (shared-memory edges)
    const uint32_t oLA = (uint32_t)((xA + NXC - 1) % NXC) * ES, oRA = (uint32_t)(xA + HW) * ES;
    const uint32_t oLB = (uint32_t)(xA + NXC / 2 - 1) * ES, oRB = (uint32_t)((xA + NXC / 2 + HW) % NXC) * ES;

    {
        if (tid == 0) {
            head->step = *((volatile long long*)&J->step);
            head->nudge_begin = *((volatile long long*)&J->nudge_begin);
            head->nudge_count = *((volatile long long*)&J->nudge_count);
        }
        __syncthreads();
        const long long step = head->step;
        const bool measure = MASS && (step + 1) % J->mass_every == 0;
        if (step >= J->target) {
            __syncthreads();
            return true;
        }

        const int ny = J->ny, nz = J->nz;
        const int ty = TY ? TY : J->ty;
        const double kap = J->kap, dtM = J->dtM;
        const float kapc = (float)(J->kap * J->cx), dtMc = (float)(J->dtM * J->cx);
        const int par = (int)(step & 1);
        T* __restrict__ dst = static_cast<T*>(J->buf[par ^ 1]);
        const CUtensorMap* tm_body = J->tmap + 2 * par;
        const CUtensorMap* tm_row = J->tmap + 2 * par + 1;

        const int CY = ty + 4, MY = ty + 2;
        const uint32_t plane_bytes = (uint32_t)CY * ROWB;
        const long long pstride = (long long)NXC * ny;
        int wz0 = 1 << 30, wz1 = -1, wz2 = -1;
        if constexpr (MASS) {
            const long long nsites = pstride * nz, na = llabs(head->nudge_count);
            if (na > 0) {
                const long long w0 = head->nudge_begin, w1 = w0 + na;
                wz0 = (int)(w0 / pstride);
                wz1 = (int)((min(w1, nsites) - 1) / pstride);
                if (w1 > nsites) wz2 = (int)((w1 - nsites - 1) / pstride);
            }
        }

        // ---- tile geometry
        const int tile = local % J->ntile;
        const int chunk = local / J->ntile;
        const int own_lo = tile * ty;
        const int own_hi = min(ny, own_lo + ty);
        const int y0 = min(own_lo, ny - ty);
        const int zs = (int)((long long)chunk * nz / J->nchunk);
        const int ze = (int)((long long)(chunk + 1) * nz / J->nchunk);
        const int L = ze - zs;
        const int dir = (chunk & 1) ? -1 : 1;
        const int zfirst = dir > 0 ? zs - 2 : ze + 1;  // c plane p lies at z = zfirst + dir*p
        const int yh0 = wrap_or_clamp(y0 - 2, ny, true);
        const int yh1 = wrap_or_clamp(y0 - 1, ny, true);
        const int yh2 = wrap_or_clamp(y0 + ty, ny, true);
        const int yh3 = wrap_or_clamp(y0 + ty + 1, ny, true);

        // ---- thread geometry: row m of the mu rows
        const int tjob = NQ * MY;
        const bool active = tid < tjob;
        const int m = active ? tid / NQ : 0;
        const uint32_t cOwn = (uint32_t)((m + 1) * NXC + xA) * ES;  // c row m+1 of a plane
        const uint32_t cUp = cOwn - ROWB, cDn = cOwn + ROWB;
        const uint32_t cRow = (uint32_t)((m + 1) * NXC) * ES;
        const uint32_t mOwn = (uint32_t)(m * NXC + xA) * ES;
        const uint32_t mUp = (uint32_t)(max(m - 1, 0) * NXC + xA) * ES;
        const uint32_t mDn = (uint32_t)(min(m + 1, MY - 1) * NXC + xA) * ES;
        const uint32_t mRow = (uint32_t)(m * NXC) * ES;
        const int y = y0 - 1 + m;
        const bool outrow = active && m >= 1 && m <= ty && y >= own_lo && y < own_hi;
        const long long site_row = (long long)max(y, 0) * NXC + xA;
        T* g = dst + (long long)zfirst * pstride + site_row;  // output pointer of plane 0
        const long long gstep = (long long)dir * pstride;

        const int producer = (MY - 1) * NQ;
        const int nplanes = L + 4;
        auto issue = [&](int p, int slot) {
            const uint32_t dstp = cbase + (uint32_t)slot * cplaneB;
            const uint32_t bar = bar0 + 8u * (uint32_t)slot;
            const int zc = wrap_or_clamp(zfirst + dir * p, nz, true);
            mbar_arrive_expect_tx(&head->bar[slot], plane_bytes + a.tx_extra);
            tma_load_3d_s(dstp, tm_row, bar, 0, yh0, zc);
            tma_load_3d_s(dstp + ROWB, tm_row, bar, 0, yh1, zc);
            tma_load_3d_s(dstp + 2 * ROWB, tm_body, bar, 0, y0, zc);
            tma_load_3d_s(dstp + (uint32_t)(ty + 2) * ROWB, tm_row, bar, 0, yh2, zc);
            tma_load_3d_s(dstp + (uint32_t)(ty + 3) * ROWB, tm_row, bar, 0, yh3, zc);
        };
        if (tid == producer) {
#pragma unroll
            for (int s = 0; s < NBUF; ++s)
                if (s < nplanes) issue(s, s);
        }

        bool failed = false;
        int nw = 0;  // planes this thread has waited for
        auto wait_slot = [&](int s) {
            if (!mbar_wait_bounded32(&head->bar[s], (ph >> s) & 1u, spin)) {
                failed = true;
                return;
            }
            ph ^= 1u << s;
            ++nw;
        };

        auto edges = [&](const Strip<T>& v, uint32_t rowaddr, T& lA, T& rA, T& lB, T& rB) {
            if constexpr (SEG) {
                const float aF = v.get(0), aL = v.get(HW - 1), bF = v.get(HW), bL = v.get(W - 1);
                const float sAL = __shfl_sync(0xffffffffu, aL, lsrc), sBL = __shfl_sync(0xffffffffu, bL, lsrc);
                const float sAF = __shfl_sync(0xffffffffu, aF, rsrc), sBF = __shfl_sync(0xffffffffu, bF, rsrc);
                lA = first ? sBL : sAL;
                lB = first ? sAL : sBL;
                rA = last ? sBF : sAF;
                rB = last ? sAF : sBF;
            } else {
                lA = IO::ld1(rowaddr + oLA);
                rA = IO::ld1(rowaddr + oRA);
                lB = IO::ld1(rowaddr + oLB);
                rB = IO::ld1(rowaddr + oRB);
            }
        };

        Strip<T> R[3], Mq[3];
        zero_strip(Mq[0]);
        zero_strip(Mq[2]);
        wait_slot(0);
        R[0] = IO::lds(cbase + cOwn, HALFB);
        wait_slot(1);
        R[1] = IO::lds(cbase + cplaneB + cOwn, HALFB);
        long long macc = 0;
        const int ilast = L + 2;
        int ifail = 0;  // the plane whose barrier saw a failed wait (0: none)

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
                Strip<T>& cp = R[k % 3];
                Strip<T>& cc = R[(k + 1) % 3];
                Strip<T>& cn = R[(k + 2) % 3];
                Strip<T>& mp = Mq[(k + 2) % 3];
                Strip<T>& mc = Mq[k % 3];
                Strip<T>& mn = Mq[(k + 1) % 3];
                const uint32_t msl = (uint32_t)((k + 1) % 3), mslp = (uint32_t)(k % 3);
                wait_slot(sN);
                cn = IO::lds(cbase + sN * cplaneB + cOwn, HALFB);
                // ---- stage A: mu on plane i
                {
                    const uint32_t pl = cbase + sI * cplaneB;
                    const Strip<T> up = IO::lds(pl + cUp, HALFB);
                    const Strip<T> dn = IO::lds(pl + cDn, HALFB);
                    T lA, rA, lB, rB;
                    edges(cc, pl + cRow, lA, rA, lB, rB);
                    march_mu<T>(cc, lA, rA, lB, rB, up, dn, cp, cn, kap, kapc, mn);
                    if (active) IO::sts(mbase + msl * mplaneB + mOwn, HALFB, mn);
                }
                // ---- stage B: c_new on plane i-1
                auto stage_b = [&]() {
                    if (i < 3) return;
                    const uint32_t q = mbase + mslp * mplaneB;
                    const Strip<T> up = IO::lds(q + mUp, HALFB);
                    const Strip<T> dn = IO::lds(q + mDn, HALFB);
                    T lA, rA, lB, rB;
                    edges(mc, q + mRow, lA, rA, lB, rB);
                    if (!outrow) return;
                    Strip<T> out;
                    march_update<T>(mc, lA, rA, lB, rB, up, dn, mp, mn, cp, dtM, dtMc, out);
                    if constexpr (MASS) {
                        const int zo = zfirst + dir * (i - 1);
                        const bool hit = (zo >= wz0 && zo <= wz1) || zo <= wz2;
                        if (hit) {
                            const long long s0 = (long long)zo * pstride + site_row;
                            if (window_reaches(s0 - xA, NXC, head->nudge_begin, head->nudge_count, pstride * nz)) {
                                float o[8];
#pragma unroll
                                for (int e = 0; e < 8; ++e) o[e] = out.get(e);
                                nudge_strip(o, s0, NXC / 2, head->nudge_begin, head->nudge_count, pstride * nz);
#pragma unroll
                                for (int kk = 0; kk < 4; ++kk) out.p[kk] = pk2(o[2 * kk], o[2 * kk + 1]);
                            }
                        }
                        if (measure)
                            macc += strip_mass(out);
                    }
                    IO::stg(g, NXC / 2, out);
                };
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
                stage_b();
                g += gstep;
            }
            if (done) break;
        }

        if (ifail) {
            // drain: wait (bounded) for the planes issued but not consumed, so
            // no copy lands after the CTA has exited; the job and the launch
            // are flagged
            if (tid == 0) {
                // planes issued before the barrier of plane ifail: NBUF at the start,
                // then NBUF + 1 after plane 1 and one more after each later plane
                const int nissued = min(nplanes, ifail >= 2 ? NBUF + ifail : NBUF);
                for (int p = nw; p < nissued; ++p) {
                    const int s = p % NBUF;
                    mbar_wait_bounded32(&head->bar[s], (ph >> s) & 1u, spin);
                    ph ^= 1u << s;
                }
                atomicMax(&J->err, DEV_TMA_TIMEOUT);
                atomicMax(a.err, DEV_TMA_TIMEOUT);
            }
            return false;
        }

        // ---- item epilogue (as ch_step_kernel): partial mass, completion
        // count, last-item work
        const int nitems_job = J->ntile * J->nchunk;
        if constexpr (MASS) {
            if (measure) {
                long long* red = reinterpret_cast<long long*>(head->red);
                const int nwarp = (tjob + 31) >> 5;
                long long v = active ? macc : 0;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
                if (lane == 0 && (tid >> 5) < nwarp) red[tid >> 5] = v;
                __syncthreads();
                if (tid < 32) {
                    long long r = lane < nwarp ? red[lane] : 0;
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) r += __shfl_down_sync(0xffffffffu, r, off);
                    if (lane == 0) J->partial[local] = r;
                }
                __threadfence();  // this item's part of the new field, before the completion count
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
            if constexpr (MASS)
                mass_feedback_step_end(J, measure, pstride * nz, nitems_job, reinterpret_cast<float*>(dst), head);
            if (tid == 0) {
                J->done = 0;
                J->step = step + 1;
            }
        }
        __syncthreads();
    }
    return true;
}

// One job class: every job of the launch has row width NXC.
// TY > 0: every job of the launch has tile height TY (its plane sizes and
// tile geometry are compile-time constants); 0: read from the job.
template <typename T, int NXC, int NBUF, bool MASS, int TY = 0>
__global__ void __launch_bounds__(kMaxBlock, 1) ch_march_kernel(StepArgs a)
{
    step_counts(a);
    MarchCta cta = march_setup<NBUF>(a, sizeof(T), march_cplane<NXC, TY>(a));
    for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
        const int j = find_job(a.item_begin, a.njobs, item);
        JobDev* J = a.jobs + __ldg(a.job_slot + j);
        const int local = item - __ldg(a.item_begin + j);
        if (!march_item<T, NXC, NBUF, MASS, TY>(a, J, local, cta)) return;
    }
}

}  // namespace mg
