// The FP32 march step (periodic 3-D, equal spacing, row width NXC a multiple
// of 32 up to 256) written for the compiler's scheduler:
//  - shared memory is read and written through C++ float4 accesses, which
//    the compiler may order freely between the ring waits and the barriers
//    (the TMA ring and its mbarriers stay in PTX);
//  - the paired arithmetic uses the float2 f32x2 builtins of sm_100, so
//    pairs live in register pairs the allocator sees, with no 64-bit
//    pack/unpack in between;
//  - the per-plane bookkeeping is constant-folded: tile height, plane
//    sizes, ring slots and z-queue roles are compile-time, the z index of
//    a plane is advanced without a modulo.
// Decomposition, tile, ring, epilogue and every per-site operation (and
// its order) are those of ch_march_kernel<float> (ch_march.cuh), so the two
// give the same bits.
#pragma once

#include "ch_march.cuh"

namespace mg {

// a thread's 8 sites of one row: half A at x .. x+3, half B at x+NXC/2 ..
struct S8 {
    float4 a, b;
};

template <int NXC>
__device__ __forceinline__ S8 lds8(const float* p)
{
    S8 s;
    s.a = *reinterpret_cast<const float4*>(p);
    s.b = *reinterpret_cast<const float4*>(p + NXC / 2);
    return s;
}
template <int NXC>
__device__ __forceinline__ void sts8(float* p, const S8& s)
{
    *reinterpret_cast<float4*>(p) = s.a;
    *reinterpret_cast<float4*>(p + NXC / 2) = s.b;
}

__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float4 cat2(float2 l, float2 h) { return make_float4(l.x, l.y, h.x, h.y); }

// per site fma(c, -6, ((left + right) + (zlo + zhi)) + (up + dn)): the
// operations of lap_pairs<false> in its order.  Pairs: (a.x, a.y),
// (a.z, a.w), (b.x, b.y), (b.z, b.w).
__device__ __forceinline__ void lap8(const S8& c, float lA, float rA, float lB, float rB, const S8& up,
                                     const S8& dn, const S8& zl, const S8& zh, float2 (&o)[4])
{
    const float2 m6 = make_float2(-6.f, -6.f);
    const float2 sx[4] = {make_float2(__fadd_rn(lA, c.a.y), __fadd_rn(c.a.x, c.a.z)),
                          make_float2(__fadd_rn(c.a.y, c.a.w), __fadd_rn(c.a.z, rA)),
                          make_float2(__fadd_rn(lB, c.b.y), __fadd_rn(c.b.x, c.b.z)),
                          make_float2(__fadd_rn(c.b.y, c.b.w), __fadd_rn(c.b.z, rB))};
    const float2 cc[4] = {lo2(c.a), hi2(c.a), lo2(c.b), hi2(c.b)};
    const float2 zs[4] = {__fadd2_rn(lo2(zl.a), lo2(zh.a)), __fadd2_rn(hi2(zl.a), hi2(zh.a)),
                          __fadd2_rn(lo2(zl.b), lo2(zh.b)), __fadd2_rn(hi2(zl.b), hi2(zh.b))};
    const float2 ys[4] = {__fadd2_rn(lo2(up.a), lo2(dn.a)), __fadd2_rn(hi2(up.a), hi2(dn.a)),
                          __fadd2_rn(lo2(up.b), lo2(dn.b)), __fadd2_rn(hi2(up.b), hi2(dn.b))};
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = __ffma2_rn(cc[k], m6, __fadd2_rn(__fadd2_rn(sx[k], zs[k]), ys[k]));
}

// the stored mass of 8 sites in 2^-32 units, as strip_mass computes it
__device__ __forceinline__ long long mass8(const float2 (&v)[4])
{
    constexpr float kM1 = 24576.0f;     // 1.5 * 2^14
    constexpr float kM2 = 12582912.0f;  // 1.5 * 2^23
    const float2 m1 = make_float2(kM1, kM1), m2 = make_float2(kM2, kM2), sc = make_float2(kMassScale, kMassScale);
    uint32_t ht = 0u, ly = 0u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        // t rounds x to the 2^-9 grid; lo = x - (t - M1) is exact
        const float2 t = __fadd2_rn(v[k], m1);
        const float2 lo = __ffma2_rn(__fadd2_rn(t, make_float2(-kM1, -kM1)), make_float2(-1.f, -1.f), v[k]);
        const float2 y = __ffma2_rn(lo, sc, m2);
        ht += __float_as_uint(t.x) + __float_as_uint(t.y);
        ly += __float_as_uint(y.x) + __float_as_uint(y.y);
    }
    const int32_t h = (int32_t)(ht - 8u * __float_as_uint(kM1));
    const int32_t l = (int32_t)(ly - 8u * __float_as_uint(kM2));
    return (long long)h * 8388608LL + (long long)l;
}

template <int NXC, int NBUF, bool MASS, int TY>
__device__ __forceinline__ bool march2_item(const StepArgs& a, JobDev* J, int local, MarchCta& cta)
{
    constexpr int NQ = NXC / 8;  // threads per row
    // rows whose threads form a power-of-two segment of a warp take their
    // x-neighbours from shuffles, other rows from the row in shared memory
    constexpr bool SEG = NQ <= 32 && (NQ & (NQ - 1)) == 0;
    static_assert(NXC >= 64 && NXC <= 256 && NXC % 32 == 0, "rows of 64..256 sites, a multiple of 32");
    static_assert(TY >= 0 && NBUF >= 3 && NBUF <= 8, "tile height, ring depth");
    constexpr uint32_t ROWB = NXC * 4;
    constexpr int U = (NBUF % 3 == 0) ? NBUF : 3 * NBUF;  // planes per unrolled block

    SmemHead* head = cta.head;
    const uint32_t cbase = cta.cbase, bar0 = cta.bar0;
    float* const cring = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(head) +
                                                   (((sizeof(SmemHead) + 127) / 128) * 128));
    const int spin = (int)min(a.spin_limit, (long long)0x7fffffff);
    uint32_t& ph = cta.ph;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int tx = tid % NQ;
    const int segbase = lane & ~(NQ - 1);
    const int lsrc = segbase | ((lane - 1) & (NQ - 1));
    const int rsrc = segbase | ((lane + 1) & (NQ - 1));
    const bool first = tx == 0, last = tx == NQ - 1;
    const int xA = tx * 4;
    // row-relative offsets of the four x-neighbours (shared-memory edges)
    const int oLA = (xA + NXC - 1) % NXC, oRA = xA + 4, oLB = xA + NXC / 2 - 1, oRB = (xA + NXC / 2 + 4) % NXC;

    // the per-item scalars that need 64-bit divisions are formed once, by
    // thread 0, and broadcast (head->red is free until the item epilogue)
    const int ny = J->ny, nz = J->nz;
    // tile height: compile-time (TY > 0), else the job's; ring slots are
    // spaced by the launch's largest plane (StepArgs cplane / mplane)
    const int ty = TY > 0 ? TY : J->ty;
    const int MY = ty + 2;
    const int CPL = TY > 0 ? (TY + 4) * NXC : a.cplane, MPL = TY > 0 ? (TY + 2) * NXC : a.mplane;
    const uint32_t PLANEB = (uint32_t)(ty + 4) * ROWB;
    float* const mring = cring + NBUF * CPL;
    const long long pstride = (long long)NXC * ny;
    int* const hw = reinterpret_cast<int*>(head->red);
    if (tid == 0) {
        const long long st = *((volatile long long*)&J->step);
        const long long nb = *((volatile long long*)&J->nudge_begin);
        const long long nc = *((volatile long long*)&J->nudge_count);
        head->step = st;
        head->nudge_begin = nb;
        head->nudge_count = nc;
        int wz0 = 1 << 30, wz1 = -1, wz2 = -1;
        if (MASS) {
            const long long nsites = pstride * nz, na = nc < 0 ? -nc : nc;
            if (na > 0) {
                const long long w1 = nb + na;
                wz0 = (int)(nb / pstride);
                wz1 = (int)((min(w1, nsites) - 1) / pstride);
                if (w1 > nsites) wz2 = (int)((w1 - nsites - 1) / pstride);
            }
        }
        hw[0] = MASS && (st + 1) % J->mass_every == 0;
        hw[1] = wz0;
        hw[2] = wz1;
        hw[3] = wz2;
    }
    __syncthreads();
    const long long step = head->step;
    if (step >= J->target) {
        __syncthreads();
        return true;
    }
    const bool measure = MASS && hw[0] != 0;
    const int wz0 = hw[1], wz1 = hw[2], wz2 = hw[3];

    const float kapc = (float)(J->kap * J->cx), dtMc = (float)(J->dtM * J->cx);
    const float2 mk = make_float2(-kapc, -kapc), dt2 = make_float2(dtMc, dtMc), m1 = make_float2(-1.f, -1.f);
    const int par = (int)(step & 1);
    float* __restrict__ dst = static_cast<float*>(J->buf[par ^ 1]);
    const CUtensorMap* tm_body = J->tmap + 2 * par;
    const CUtensorMap* tm_row = J->tmap + 2 * par + 1;

    // ---- tile geometry (32-bit: chunk * nz and the row indices fit)
    const int ntile = J->ntile, nchunk = J->nchunk;
    const int chunk = local / ntile;
    const int tile = local - chunk * ntile;
    const int own_lo = tile * ty;
    const int own_hi = min(ny, own_lo + ty);
    const int y0 = min(own_lo, ny - ty);
    const int zs = chunk * nz / nchunk;
    const int ze = (chunk + 1) * nz / nchunk;
    const int L = ze - zs;
    const int dir = (chunk & 1) ? -1 : 1;
    const int zfirst = dir > 0 ? zs - 2 : ze + 1;
    // rows y0-2 .. y0+ty+1 wrap by at most one period
    auto wrap = [ny](int v) { return v < 0 ? v + ny : (v >= ny ? v - ny : v); };
    const int yh0 = wrap(y0 - 2), yh1 = wrap(y0 - 1), yh2 = wrap(y0 + ty), yh3 = wrap(y0 + ty + 1);

    // ---- thread geometry: row m of the mu rows
    const bool active = tid < NQ * MY;
    const int m = active ? tid / NQ : 0;
    const float* const cOwn = cring + (m + 1) * NXC + xA;
    const float* const cRow = cring + (m + 1) * NXC;
    float* const mOwn = mring + m * NXC + xA;
    const float* const mRow = mring + m * NXC;
    const float* const mUp = mring + max(m - 1, 0) * NXC + xA;
    const float* const mDn = mring + min(m + 1, MY - 1) * NXC + xA;
    const int y = y0 - 1 + m;
    const bool outrow = active && m >= 1 && m <= ty && y >= own_lo && y < own_hi;
    const long long site_row = (long long)max(y, 0) * NXC + xA;
    float* g = dst + (long long)zfirst * pstride + site_row;
    const long long gstep = (long long)dir * pstride;

    const int producer = (MY - 1) * NQ;
    const int nplanes = L + 4;
    // z of the next plane the producer issues, wrapped incrementally
    int zissue = zfirst < 0 ? zfirst + nz : (zfirst >= nz ? zfirst - nz : zfirst);
    auto issue = [&](int slot) {
        const uint32_t dstp = cbase + (uint32_t)(slot * CPL * 4);
        const uint32_t bar = bar0 + 8u * (uint32_t)slot;
        const int zc = zissue;
        zissue += dir;
        if (zissue < 0) zissue += nz;
        if (zissue >= nz) zissue -= nz;
        mbar_arrive_expect_tx(&head->bar[slot], PLANEB + a.tx_extra);
        tma_load_3d_s(dstp, tm_row, bar, 0, yh0, zc);
        tma_load_3d_s(dstp + ROWB, tm_row, bar, 0, yh1, zc);
        tma_load_3d_s(dstp + 2 * ROWB, tm_body, bar, 0, y0, zc);
        tma_load_3d_s(dstp + (uint32_t)(ty + 2) * ROWB, tm_row, bar, 0, yh2, zc);
        tma_load_3d_s(dstp + (uint32_t)(ty + 3) * ROWB, tm_row, bar, 0, yh3, zc);
    };
    if (tid == producer) {
#pragma unroll
        for (int s = 0; s < NBUF; ++s)
            if (s < nplanes) issue(s);
    }

    bool failed = false;
    int nw = 0;
    auto wait_slot = [&](int s) {
        if (!mbar_wait_bounded32(&head->bar[s], (ph >> s) & 1u, spin)) {
            failed = true;
            return;
        }
        ph ^= 1u << s;
        ++nw;
    };
    // x-neighbours of a strip's two halves: from the lanes of its row
    // segment, or from its row in shared memory
    auto edges = [&](const S8& v, const float* row, float& lA, float& rA, float& lB, float& rB) {
        if constexpr (SEG) {
            const float sAL = __shfl_sync(0xffffffffu, v.a.w, lsrc), sBL = __shfl_sync(0xffffffffu, v.b.w, lsrc);
            const float sAF = __shfl_sync(0xffffffffu, v.a.x, rsrc), sBF = __shfl_sync(0xffffffffu, v.b.x, rsrc);
            lA = first ? sBL : sAL;
            lB = first ? sAL : sBL;
            rA = last ? sBF : sAF;
            rB = last ? sAF : sBF;
        } else {
            lA = row[oLA];
            rA = row[oRA];
            lB = row[oLB];
            rB = row[oRB];
        }
    };

    S8 R[3], Mq[3];
    Mq[0].a = Mq[0].b = Mq[2].a = Mq[2].b = make_float4(0.f, 0.f, 0.f, 0.f);
    wait_slot(0);
    R[0] = lds8<NXC>(cOwn);
    wait_slot(1);
    R[1] = lds8<NXC>(cOwn + CPL);
    long long macc = 0;
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
            S8& cp = R[k % 3];
            S8& cc = R[(k + 1) % 3];
            S8& cn = R[(k + 2) % 3];
            S8& mp = Mq[(k + 2) % 3];
            S8& mc = Mq[k % 3];
            S8& mn = Mq[(k + 1) % 3];
            const int msl = (k + 1) % 3, mslp = k % 3;
            wait_slot(sN);
            cn = lds8<NXC>(cOwn + sN * CPL);
            // ---- stage A: mu on plane i
            {
                const float* pl = cOwn + sI * CPL;
                const S8 up = lds8<NXC>(pl - NXC);
                const S8 dn = lds8<NXC>(pl + NXC);
                float lA, rA, lB, rB;
                edges(cc, cRow + sI * CPL, lA, rA, lB, rB);
                float2 lp[4];
                lap8(cc, lA, rA, lB, rB, up, dn, cp, cn, lp);
                const float2 c2[4] = {lo2(cc.a), hi2(cc.a), lo2(cc.b), hi2(cc.b)};
                float2 mu[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) mu[q] = __ffma2_rn(lp[q], mk, __fmul2_rn(c2[q], __ffma2_rn(c2[q], c2[q], m1)));
                mn.a = cat2(mu[0], mu[1]);
                mn.b = cat2(mu[2], mu[3]);
                if (active) sts8<NXC>(mOwn + msl * MPL, mn);
            }
            if (__syncthreads_or(failed)) {
                ifail = i;
                done = true;
                break;
            }
            if (tid == producer) {
                if (i == 1 && NBUF < nplanes) issue(0);
                if (i + NBUF < nplanes) issue(sI);
            }
            // ---- stage B: c_new on plane i-1
            if (i >= 3) {
                const S8 up = lds8<NXC>(mUp + mslp * MPL);
                const S8 dn = lds8<NXC>(mDn + mslp * MPL);
                float lA, rA, lB, rB;
                edges(mc, mRow + mslp * MPL, lA, rA, lB, rB);
                if (outrow) {
                    float2 lp[4];
                    lap8(mc, lA, rA, lB, rB, up, dn, mp, mn, lp);
                    const float2 c2[4] = {lo2(cp.a), hi2(cp.a), lo2(cp.b), hi2(cp.b)};
                    float2 o[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) o[q] = __ffma2_rn(lp[q], dt2, c2[q]);
                    if constexpr (MASS) {
                        const int zo = zfirst + dir * (i - 1);
                        const bool hit = (zo >= wz0 && zo <= wz1) || zo <= wz2;
                        if (hit) {
                            const long long s0 = (long long)zo * pstride + site_row;
                            if (window_reaches(s0 - xA, NXC, head->nudge_begin, head->nudge_count, pstride * nz)) {
                                float v[8] = {o[0].x, o[0].y, o[1].x, o[1].y, o[2].x, o[2].y, o[3].x, o[3].y};
                                nudge_strip(v, s0, NXC / 2, head->nudge_begin, head->nudge_count, pstride * nz);
#pragma unroll
                                for (int q = 0; q < 4; ++q) o[q] = make_float2(v[2 * q], v[2 * q + 1]);
                            }
                        }
                        if (measure) macc += mass8(o);
                    }
                    *reinterpret_cast<float4*>(g) = cat2(o[0], o[1]);
                    *reinterpret_cast<float4*>(g + NXC / 2) = cat2(o[2], o[3]);
                }
            }
            g += gstep;
        }
        if (done) break;
    }

    if (ifail) {
        if (tid == 0) {
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

    // ---- item epilogue (as march_item)
    const int nitems_job = J->ntile * J->nchunk;
    if constexpr (MASS) {
        if (measure) {
            long long* red = reinterpret_cast<long long*>(head->red);
            const int nwarp = (NQ * MY + 31) >> 5;
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
            __threadfence();
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
            mass_feedback_step_end(J, measure, pstride * nz, nitems_job, dst, head);
        if (tid == 0) {
            J->done = 0;
            J->step = step + 1;
        }
    }
    __syncthreads();
    return true;
}

// Every job of the launch: FP32, row width NXC, tile height TY (0: each job's own).
// A fixed tile height bounds the registers for two CTAs per SM (of the
// block the host launches: the tile's threads rounded up to whole warps).
template <int NXC, int NBUF, bool MASS, int TY>
__global__ void __launch_bounds__(TY > 0 ? ((TY + 2) * (NXC / 8) + 31) / 32 * 32 : kMaxBlock, TY > 0 ? 2 : 1)
    ch_march2_kernel(StepArgs a)
{
    step_counts(a);
    MarchCta cta = march_setup<NBUF>(a, 4u, TY > 0 ? (uint32_t)((TY + 4) * NXC) : (uint32_t)a.cplane);
    for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
        const int j = find_job(a.item_begin, a.njobs, item);
        JobDev* J = a.jobs + __ldg(a.job_slot + j);
        const int local = item - __ldg(a.item_begin + j);
        if (!march2_item<NXC, NBUF, MASS, TY>(a, J, local, cta)) return;
    }
}

}  // namespace mg
