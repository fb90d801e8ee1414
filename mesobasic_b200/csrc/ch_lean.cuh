// Lean FP32 variant of the fused Cahn-Hilliard step for the common case:
// every axis periodic with equal spacing (SIMPLE), 3-D, row width NXC fixed
// at compile time with a row of threads that is a power-of-two segment of a
// warp (NXC = 64, 128, 256).  Same work decomposition, ring, register
// z-queues, arithmetic and epilogue as ch_step_kernel<float, NBUF, false,
// true, MASS, NXC> -- the results are bit-identical -- with less per-plane
// overhead:
//  - every shared-memory access is one 32-bit-addressed ld/st.shared.v2.u64
//    whose address is fixed per item (the plane's ring slot adds a uniform
//    offset);
//  - ring slots and barrier parities roll forward in registers instead of
//    being recomputed from the plane index;
//  - a thread's row, lane segment and neighbours are compile-time shapes.
#pragma once

#include "ch_kernels.cuh"

namespace mg {

template <int NXC, int NBUF, bool MASS>
__global__ void __launch_bounds__(kMaxBlock, 1) ch_lean_kernel(StepArgs a)
{
    step_counts(a);
    constexpr int W = 8, HW = 4;
    constexpr int NQ = NXC / W;  // threads per row
    static_assert(NXC % W == 0 && NXC <= 256 && NQ <= 32 && (NQ & (NQ - 1)) == 0,
                  "a row of threads must be a power-of-two segment of a warp");
    constexpr uint32_t ROWB = NXC * 4;         // bytes of a shared-memory row (one TMA box wide)
    constexpr uint32_t HALFB = NXC / 2 * 4;    // half B of a strip sits nx/2 floats after half A

    extern __shared__ __align__(128) unsigned char smem_dyn[];
    unsigned char* smem_raw = smem_dyn + ((128u - (smem_addr(smem_dyn) & 127u)) & 127u);
    SmemHead* head = reinterpret_cast<SmemHead*>(smem_raw);
    const uint32_t cbase = smem_addr(smem_raw) + (uint32_t)(((sizeof(SmemHead) + 127) / 128) * 128);
    const uint32_t cplaneB = (uint32_t)a.cplane * 4u, mplaneB = (uint32_t)a.mplane * 4u;
    const uint32_t mbase = cbase + NBUF * cplaneB;
    const uint32_t bar0 = smem_addr(&head->bar[0]);

    const int tid = threadIdx.x;
    const int lane = tid & 31;

    if (tid == 0) {
        for (int b = 0; b < NBUF; ++b) mbar_init(&head->bar[b], 1);
        fence_mbar_init();
    }
    __syncthreads();

    // ring state carried across items: the slot the next issued plane goes
    // to and the parity of each slot's next completion
    int ring = 0;
    uint32_t parity = 0;

    // lane segment of a row (fixed for the kernel)
    const int tx = tid & (NQ - 1);
    const int segbase = lane & ~(NQ - 1);
    const int lsrc = segbase | ((lane - 1) & (NQ - 1));
    const int rsrc = segbase | ((lane + 1) & (NQ - 1));
    const bool first = tx == 0, last = tx == NQ - 1;
    const int xA = tx * HW;

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
        if (step >= J->target) {
            __syncthreads();
            continue;
        }

        const int ny = J->ny, nz = J->nz;
        const int ty = J->ty;
        const float kapc = (float)(J->kap * J->cx), dtMc = (float)(J->dtM * J->cx);
        const int par = (int)(step & 1);
        float* __restrict__ dst = static_cast<float*>(J->buf[par ^ 1]);
        const CUtensorMap* tm_body = J->tmap + 2 * par;
        const CUtensorMap* tm_row = J->tmap + 2 * par + 1;

        const int CY = ty + 4, MY = ty + 2;
        const uint32_t plane_bytes = (uint32_t)CY * ROWB;
        const size_t pstride = (size_t)NXC * ny;
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
        const int own_lo = tile * ty;
        const int own_hi = min(ny, own_lo + ty);
        const int y0 = min(own_lo, ny - ty);
        const int zs = (int)((long long)chunk * nz / J->nchunk);
        const int ze = (int)((long long)(chunk + 1) * nz / J->nchunk);
        const int L = ze - zs;
        const int dir = (chunk & 1) ? -1 : 1;
        const int zfirst = dir > 0 ? zs - 2 : ze + 1;
        const int yh0 = wrap_or_clamp(y0 - 2, ny, true);
        const int yh1 = wrap_or_clamp(y0 - 1, ny, true);
        const int yh2 = wrap_or_clamp(y0 + ty, ny, true);
        const int yh3 = wrap_or_clamp(y0 + ty + 1, ny, true);

        // ---- thread geometry: row m of the mu rows, half A at x = 4*tx
        const int tjob = NQ * MY;
        const bool active = tid < tjob;
        const int m = active ? tid / NQ : 0;
        const uint32_t cOwn = (uint32_t)((m + 1) * NXC + xA) * 4u;  // c row m+1 of a plane
        const uint32_t cUp = cOwn - ROWB, cDn = cOwn + ROWB;
        const uint32_t mOwn = (uint32_t)(m * NXC + xA) * 4u;
        const uint32_t mUp = (uint32_t)(max(m - 1, 0) * NXC + xA) * 4u;
        const uint32_t mDn = (uint32_t)(min(m + 1, MY - 1) * NXC + xA) * 4u;
        const int y = y0 - 1 + m;
        const bool outrow = active && m >= 1 && m <= ty && y >= own_lo && y < own_hi;
        float* __restrict__ grow = dst + (size_t)max(y, 0) * NXC + xA;
        const long long site_row = (long long)max(y, 0) * NXC + xA;

        const int producer = (MY - 1) * NQ;
        const int s0 = ring;
        auto issue = [&](int i) {
            if (tid != producer) return;
            const int slot = (s0 + i) % NBUF;
            const uint32_t p = cbase + (uint32_t)slot * cplaneB;
            const uint32_t bar = bar0 + 8u * (uint32_t)slot;
            const int zc = wrap_or_clamp(zfirst + dir * i, nz, true);
            mbar_arrive_expect_tx(&head->bar[slot], plane_bytes + a.tx_extra);
            tma_load_3d_s(p, tm_row, bar, 0, yh0, zc);
            tma_load_3d_s(p + ROWB, tm_row, bar, 0, yh1, zc);
            tma_load_3d_s(p + 2 * ROWB, tm_body, bar, 0, y0, zc);
            tma_load_3d_s(p + (uint32_t)(ty + 2) * ROWB, tm_row, bar, 0, yh2, zc);
            tma_load_3d_s(p + (uint32_t)(ty + 3) * ROWB, tm_row, bar, 0, yh3, zc);
        };
        bool failed = false;
        // waits on the slot of the next plane in order; the parity bit of
        // that slot flips with every completed wait
        int wslot = s0;
        auto wait_next = [&]() {
            const uint32_t ph = (parity >> wslot) & 1u;
            if (!mbar_wait_bounded(&head->bar[wslot], ph, a.spin_limit)) {
                failed = true;
                atomicMax(&J->err, DEV_TMA_TIMEOUT);
                atomicMax(a.err, DEV_TMA_TIMEOUT);
            }
            parity ^= 1u << wslot;
            wslot = wslot + 1 == NBUF ? 0 : wslot + 1;
        };

        const int nplanes = L + 4;
        const int npro = min(NBUF, nplanes);
        for (int i = 0; i < npro; ++i) issue(i);
        int issued = npro;
        int waited = 0;
        long long macc = 0;
        // shared-memory address of c plane i (slot (s0 + i) mod NBUF), rolled forward
        uint32_t cpl_i = cbase + (uint32_t)s0 * cplaneB;  // plane 0
        auto next_plane = [&](uint32_t p) { return p + cplaneB == cbase + NBUF * cplaneB ? cbase : p + cplaneB; };

        auto edges = [&](const Strip<float>& v, float& lA, float& rA, float& lB, float& rB) {
            const float aF = v.get(0), aL = v.get(HW - 1), bF = v.get(HW), bL = v.get(W - 1);
            const float sAL = __shfl_sync(0xffffffffu, aL, lsrc), sBL = __shfl_sync(0xffffffffu, bL, lsrc);
            const float sAF = __shfl_sync(0xffffffffu, aF, rsrc), sBF = __shfl_sync(0xffffffffu, bF, rsrc);
            lA = first ? sBL : sAL;
            lB = first ? sAL : sBL;
            rA = last ? sBF : sAF;
            rB = last ? sAF : sBF;
        };

        // One plane of the march (see ch_step_kernel): mu on plane i (stage
        // A), then c_new on plane i-1 (stage B).  cp/cc/cn = c(i-1), c(i),
        // c(i+1); mp/mc/mn = mu(i-2), mu(i-1), mu(i); MS/MSP = mu ring slots
        // of planes i and i-1.
        auto plane = [&](int i, uint32_t msl, uint32_t mslp, Strip<float>& cp, Strip<float>& cc, Strip<float>& cn,
                         Strip<float>& mp, Strip<float>& mc, Strip<float>& mn) -> bool {
            const uint32_t pi = cpl_i;           // plane i
            const uint32_t pn = next_plane(pi);  // plane i+1
            wait_next();
            waited = i + 2;
            cn = lds_strip(pn + cOwn, HALFB);
            {
                const Strip<float> up = lds_strip(pi + cUp, HALFB);
                const Strip<float> dn = lds_strip(pi + cDn, HALFB);
                float lA, rA, lB, rB;
                edges(cc, lA, rA, lB, rB);
                unsigned long long lp[4];
                lap_pairs<false>(cc, lA, rA, lB, rB, up, dn, cp, cn, lp);
                const unsigned long long m1 = splat2(-1.f), mk = splat2(-kapc);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const unsigned long long df = mul2(cc.p[k], fma2(cc.p[k], cc.p[k], m1));
                    mn.p[k] = fma2(lp[k], mk, df);
                }
                if (active) {
                    const uint32_t ma = mbase + msl * mplaneB + mOwn;
                    sts_v2(ma, mn.p[0], mn.p[1]);
                    sts_v2(ma + HALFB, mn.p[2], mn.p[3]);
                }
            }
            if (__syncthreads_or(failed)) return false;
            for (; issued <= i + NBUF && issued < nplanes; ++issued) issue(issued);
            cpl_i = pn;
            if (i >= 3) {
                const uint32_t q = mbase + mslp * mplaneB;
                const Strip<float> up = lds_strip(q + mUp, HALFB);
                const Strip<float> dn = lds_strip(q + mDn, HALFB);
                float lA, rA, lB, rB;
                edges(mc, lA, rA, lB, rB);
                const int zo = zfirst + dir * (i - 1);
                const bool hit = MASS && ((zo >= wz0 && zo <= wz1) || zo <= wz2);
                if (outrow) {
                    Strip<float> out;
                    unsigned long long lp[4];
                    lap_pairs<false>(mc, lA, rA, lB, rB, up, dn, mp, mn, lp);
                    const unsigned long long dt2 = splat2(dtMc);
#pragma unroll
                    for (int k = 0; k < 4; ++k) out.p[k] = fma2(lp[k], dt2, cp.p[k]);
                    const size_t zoff = (size_t)zo * pstride;
                    if constexpr (MASS) {
                        if (hit && window_reaches((long long)zoff + site_row - xA, NXC, head->nudge_begin,
                                                  head->nudge_count, (long long)pstride * nz)) {
                            float o[8];
#pragma unroll
                            for (int e = 0; e < 8; ++e) o[e] = out.get(e);
                            nudge_strip(o, (long long)zoff + site_row, NXC / 2, head->nudge_begin,
                                        head->nudge_count, (long long)pstride * nz);
#pragma unroll
                            for (int k = 0; k < 4; ++k) out.p[k] = pk2(o[2 * k], o[2 * k + 1]);
                        }
                        if (measure) macc += strip_mass(out);
                    }
                    float* g = grow + zoff;
                    stg_v2(g, out.p[0], out.p[1]);
                    stg_v2(g + NXC / 2, out.p[2], out.p[3]);
                }
            }
            return true;
        };

        Strip<float> c0r, c1r, c2r, m0r, m1r, m2r;
        zero_strip(m0r);
        zero_strip(m1r);
        wait_next();
        c0r = lds_strip(cpl_i + cOwn, HALFB);
        cpl_i = next_plane(cpl_i);
        wait_next();
        c1r = lds_strip(cpl_i + cOwn, HALFB);
        waited = 2;

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
        ring = (s0 + nplanes) % NBUF;

        if (!ok) {
            for (int k = waited; k < issued; ++k) {
                const int sl = (s0 + k) % NBUF;
                mbar_wait_bounded(&head->bar[sl], (parity >> sl) & 1u, a.spin_limit);
                parity ^= 1u << sl;
            }
            return;
        }

        // ---- item epilogue (as ch_step_kernel)
        const int nitems_job = J->ntile * J->nchunk;
        if (measure) {
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
            if constexpr (MASS) mass_feedback_step_end(J, measure, (long long)pstride * nz, nitems_job, dst, head);
            if (tid == 0) {
                J->done = 0;
                J->step = step + 1;
            }
        }
        __syncthreads();
    }
}

}  // namespace mg
