// Device helpers shared by the Cahn-Hilliard step kernels (ch_kernels.cuh,
// ch_lean.cuh, ch_march.cuh): thread strips and their paired FP32
// arithmetic, the 7-point Laplacian and chemical potential in the
// reference's operation order, shared-memory and TMA access in 32-bit
// shared addresses, work-item lookup and the FP32 mass feedback.
#pragma once

#include "ch_types.h"
#include "mg_device.cuh"

namespace mg {

// ---------------------------------------------------------------- strips
// A thread owns a 32-byte strip of one row: 8 floats or 4 doubles.  FP32
// strips are held as four 64-bit pairs so the arithmetic can use the paired
// f32x2 instructions of sm_100.

template <typename T>
struct Strip;

template <>
struct Strip<float> {
    static constexpr int W = 8;
    unsigned long long p[4];
    __device__ __forceinline__ float get(int e) const
    {
        float a, b;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(p[e >> 1]));
        return (e & 1) ? b : a;
    }
};

template <>
struct Strip<double> {
    static constexpr int W = 4;
    double v[4];
    __device__ __forceinline__ double get(int e) const { return v[e]; }
};

__device__ __forceinline__ unsigned long long pk2(float a, float b)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r)
{
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c)
{
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ unsigned long long splat2(float a) { return pk2(a, a); }

// A strip is two 16-byte halves: half A at p, half B at p + off (the
// halves of neighbouring threads are adjacent, so every warp-wide access is
// one contiguous run and free of bank conflicts).
template <typename T>
__device__ __forceinline__ Strip<T> ld_strip(const T* p, int off)
{
    Strip<T> s;
    if constexpr (sizeof(T) == 4) {
        const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(p);
        const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(p + off);
        s.p[0] = a.x, s.p[1] = a.y, s.p[2] = b.x, s.p[3] = b.y;
    } else {
        const double2 a = *reinterpret_cast<const double2*>(p);
        const double2 b = *reinterpret_cast<const double2*>(p + off);
        s.v[0] = a.x, s.v[1] = a.y, s.v[2] = b.x, s.v[3] = b.y;
    }
    return s;
}

template <typename T>
__device__ __forceinline__ void st_strip(T* p, int off, const Strip<T>& s)
{
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(s.p[0], s.p[1]);
        *reinterpret_cast<ulonglong2*>(p + off) = make_ulonglong2(s.p[2], s.p[3]);
    } else {
        *reinterpret_cast<double2*>(p) = make_double2(s.v[0], s.v[1]);
        *reinterpret_cast<double2*>(p + off) = make_double2(s.v[2], s.v[3]);
    }
}

template <typename T>
__device__ __forceinline__ void zero_strip(Strip<T>& s)
{
    if constexpr (sizeof(T) == 4) {
        s.p[0] = s.p[1] = s.p[2] = s.p[3] = 0ull;
    } else {
        s.v[0] = s.v[1] = s.v[2] = s.v[3] = 0.0;
    }
}

// Laplacian numerator sums of a strip with paired FP32 arithmetic, SIMPLE
// geometry (all periodic, equal spacing): per pair
// (x sum) + (y sum) + (z sum) - 2*dims*centre.  Half A is pairs 0-1 with x
// neighbours lA/rA, half B pairs 2-3 with lB/rB.
template <bool FLAT>
__device__ __forceinline__ void lap_pairs(const Strip<float>& c, float lA, float rA, float lB, float rB,
                                          const Strip<float>& up, const Strip<float>& dn, const Strip<float>& zlo,
                                          const Strip<float>& zhi, unsigned long long (&out)[4])
{
    const unsigned long long m6 = splat2(FLAT ? -4.f : -6.f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int h = k >> 1;  // half
        const float xm0 = (k & 1) == 0 ? (h == 0 ? lA : lB) : c.get(2 * k - 1);
        const float xp1 = (k & 1) == 1 ? (h == 0 ? rA : rB) : c.get(2 * k + 2);
        const unsigned long long sx = pk2(xm0 + c.get(2 * k + 1), c.get(2 * k) + xp1);
        unsigned long long sacc = add2(sx, add2(zlo.p[k], zhi.p[k]));
        if constexpr (!FLAT) sacc = add2(sacc, add2(up.p[k], dn.p[k]));
        out[k] = fma2(c.p[k], m6, sacc);
    }
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

// The 7-point Laplacian of one site in the reference's order
// ((lapx + lapy) + lapz), SfieldFD.cpp:296-302.  FLAT drops the y term,
// which is exactly zero in the reference for a flat axis.  SIMPLE (every
// axis periodic, equal spacing): FP64 skips the multiplications by
// 1/d^2 = 1, which are exact identities; FP32 uses the algebraically equal
// ((sum of six neighbours) - 6c) / d^2.
template <typename T, bool FLAT, bool SIMPLE>
__device__ __forceinline__ T lap7(T c0, T xp, T xm, T yp, T ym, T zp, T zm, double cx, double cy, double cz,
                                  bool divX, bool divY, bool divZ)
{
    using A = Arith<T>;
    if constexpr (SIMPLE) {
        if constexpr (sizeof(T) == 8) {
            const T c2 = A::mul(T(2), c0);
            const T lx = A::sub(A::add(xp, xm), c2);
            const T lz = A::sub(A::add(zp, zm), c2);
            if constexpr (FLAT) {
                return A::add(lx, lz);
            } else {
                const T ly = A::sub(A::add(yp, ym), c2);
                return A::add(A::add(lx, ly), lz);
            }
        } else {
            T s = (xp + xm) + (zp + zm);
            if constexpr (!FLAT) s += (yp + ym);
            return fmaf(FLAT ? -4.f : -6.f, c0, s) * (float)cx;
        }
    } else {
        if constexpr (FLAT) {
            return A::add(axis_term(xp, xm, c0, cx, divX), axis_term(zp, zm, c0, cz, divZ));
        } else {
            return A::add(A::add(axis_term(xp, xm, c0, cx, divX), axis_term(yp, ym, c0, cy, divY)),
                          axis_term(zp, zm, c0, cz, divZ));
        }
    }
}

// mu = (c*c*c - c) - kappa*lap (FP64 in that order; FP32 contracted)
template <typename T>
__device__ __forceinline__ T chem_pot(T c0, T lap, T kap)
{
    if constexpr (sizeof(T) == 8) {
        using A = Arith<T>;
        return A::sub(A::sub(A::mul(A::mul(c0, c0), c0), c0), A::mul(kap, lap));
    } else {
        return fmaf(-kap, lap, fmaf(c0 * c0, c0, -c0));
    }
}

// MurmurHash3's 32-bit finaliser (public domain): a bijective mixer.
__device__ __forceinline__ uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
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

// The stored mass of one thread strip in 2^-32 units: each of its 8 values
// rounded to the nearest multiple of 2^-32 (ties to even), the integers
// added.  The rounding uses FP32 arithmetic and bit patterns only, no
// conversion instructions: t = x + 1.5*2^14 rounds x to the 2^-9 grid
// (hi = t - 1.5*2^14, exact), lo = x - hi is exact with |lo| <= 2^-10, and
// y = lo*2^32 + 1.5*2^23 rounds lo*2^32 to an integer; on [2^14, 2^15) and
// [2^23, 2^24) consecutive floats have consecutive bit patterns, so
// bits(t) - bits(1.5*2^14) = hi/2^-9 and bits(y) - bits(1.5*2^23) = the
// rounded lo*2^32.  Exact for |x| < 2^12.  The same function measures the
// field at upload and after every measured step, so the measure does not
// depend on the decomposition.
__device__ __forceinline__ long long strip_mass(const Strip<float>& s)
{
    constexpr float kM1 = 24576.0f;     // 1.5 * 2^14
    constexpr float kM2 = 12582912.0f;  // 1.5 * 2^23
    const unsigned long long m1 = splat2(kM1), m2 = splat2(kM2), sc = splat2(kMassScale);
    uint32_t ht = 0u, ly = 0u;  // sums of bit patterns, modulo 2^32
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const unsigned long long t = add2(s.p[k], m1);
        const unsigned long long lo = sub2(s.p[k], sub2(t, m1));
        const unsigned long long y = fma2(lo, sc, m2);
        ht += (uint32_t)t + (uint32_t)(t >> 32);
        ly += (uint32_t)y + (uint32_t)(y >> 32);
    }
    const int32_t h = (int32_t)(ht - 8u * __float_as_uint(kM1));  // in units of 2^-9
    const int32_t l = (int32_t)(ly - 8u * __float_as_uint(kM2));  // in units of 2^-32
    return (long long)h * 8388608LL + (long long)l;
}

__device__ __forceinline__ long long strip_mass(float o0, float o1, float o2, float o3, float o4, float o5, float o6,
                                                float o7)
{
    Strip<float> s;
    s.p[0] = pk2(o0, o1);
    s.p[1] = pk2(o2, o3);
    s.p[2] = pk2(o4, o5);
    s.p[3] = pk2(o6, o7);
    return strip_mass(s);
}

// Does the nudge window [w0, w0 + |cnt|) (wrapping at nsites) reach the row
// of sites [rs, rs + len)?  Asked only in planes the window reaches, so that
// only the threads of the rows it covers take the out-of-line nudge.
__device__ __forceinline__ bool window_reaches(long long rs, long long len, long long w0, long long cnt,
                                               long long nsites)
{
    const long long w1 = w0 + (cnt < 0 ? -cnt : cnt);
    if (rs < w1 && rs + len > w0) return true;
    return w1 > nsites && rs < w1 - nsites;
}

// Adds the mass nudge to the elements of a thread's 8-float strip whose sites
// lie in the nudge window (sites of element e: site0 + e for e < 4, site0 +
// offB + e - 4 for the second half).  Called only for planes the window
// reaches, so it stays out of line.
static __device__ __noinline__ void nudge_strip(float* o, long long site0, long long offB, long long w0, long long cnt,
                                         long long nsites)
{
    const long long na = cnt < 0 ? -cnt : cnt;
    const float nudge = cnt < 0 ? -kNudge : kNudge;
    for (int e = 0; e < 8; ++e) {
        long long r = site0 + (e < 4 ? e : offB + e - 4) - w0;
        if (r < 0) r += nsites;
        if (r < na) o[e] += nudge;
    }
}

// FP32 mass feedback at the end of a step, run by the whole CTA that
// finished the job's last item of the step (every item has stored its part
// of the new field and fenced it).  The nudges this step added inside the
// stencil are booked.  On a measured step the stored mass M (the items'
// partial sums in item order) gives:
//  - the correction: round((target - M) / kNudge) nudges, added here to
//    consecutive sites of the new field, so the stored mass leaves every
//    measured step on target;
//  - the rounding defect of the interval since the last measure (the change
//    of stored mass the nudges did not make), d per step: each step of the
//    coming interval adds round(-d / kNudge) nudges inside the stencil, so
//    the mass stays on target between measures while rounding losses are
//    systematic (they are while the field evolves slowly).
// kNudge is a multiple of the unit in the last place of every float below 2
// in magnitude, so each nudge moves the stored sum by exactly its size.  The
// window of nudged sites moves on by a golden-ratio fraction of the field
// every step.
__device__ __forceinline__ void mass_feedback_step_end(JobDev* J, bool measure, long long nsites, int nitems_job,
                                                       float* field, SmemHead* head)
{
    const int tid = threadIdx.x, lane = tid & 31;
    const long long stride = (long long)(0.6180339887498949 * (double)nsites) | 1;
    if (tid < 32) {
        __int128 r = 0;
        if (measure) {
            for (int k = lane; k < nitems_job; k += 32) r += __ldcg(J->partial + k);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const unsigned long long lo = __shfl_down_sync(0xffffffffu, (unsigned long long)r, off);
                const long long hi = __shfl_down_sync(0xffffffffu, (long long)(r >> 64), off);
                r += ((__int128)hi << 64) | (__int128)lo;
            }
        }
        if (lane == 0) {
            J->nudge_applied += J->nudge_count;
            long long now = 0;
            if (measure) {
                const double mm = (double)r / (double)kMassScale;
                const double d =
                    ((mm - J->mass_last) - (double)J->nudge_applied * (double)kNudge) / (double)J->mass_every;
                double k = rint((J->mass_target - mm) / (double)kNudge);
                double kr = rint(-d / (double)kNudge);
                k = fmin(fmax(k, -(double)nsites), (double)nsites);
                kr = fmin(fmax(kr, -(double)nsites), (double)nsites);
                now = (long long)k;
                J->mass_last = mm + k * (double)kNudge;
                J->nudge_applied = 0;
                J->nudge_rest = (long long)kr;
            }
            head->nudge_begin = J->nudge_begin;
            head->nudge_count = now;
            const long long w = now != 0 ? (J->nudge_begin + stride) % nsites : J->nudge_begin;
            J->nudge_count = J->nudge_rest;
            J->nudge_begin = (w + stride) % nsites;
        }
    }
    __syncthreads();
    const long long cnt = head->nudge_count, w0 = head->nudge_begin;
    const long long na = cnt < 0 ? -cnt : cnt;
    const float nudge = cnt < 0 ? -kNudge : kNudge;
    for (long long q = tid; q < na; q += blockDim.x) {
        long long site = w0 + q;
        if (site >= nsites) site -= nsites;
        field[site] = __ldcg(field + site) + nudge;
    }
}

// ---------------------------------------------------- shared-memory access
__device__ __forceinline__ void lds_v2(uint32_t addr, unsigned long long& x, unsigned long long& y)
{
    asm volatile("ld.shared.v2.u64 {%0, %1}, [%2];" : "=l"(x), "=l"(y) : "r"(addr) : "memory");
}
__device__ __forceinline__ void sts_v2(uint32_t addr, unsigned long long x, unsigned long long y)
{
    asm volatile("st.shared.v2.u64 [%0], {%1, %2};" ::"r"(addr), "l"(x), "l"(y) : "memory");
}
__device__ __forceinline__ void stg_v2(void* p, unsigned long long x, unsigned long long y)
{
    asm volatile("st.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(x), "l"(y) : "memory");
}
// strip of 8 floats: half A at addr, half B at addr + offB
__device__ __forceinline__ Strip<float> lds_strip(uint32_t addr, uint32_t offB)
{
    Strip<float> s;
    lds_v2(addr, s.p[0], s.p[1]);
    lds_v2(addr + offB, s.p[2], s.p[3]);
    return s;
}
__device__ __forceinline__ void tma_load_3d_s(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// ------------------------------------------------- per-step noise generator
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011): counter of four 32-bit words, key of two.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

// ----------------------------------------- variable-mobility site models
// Per-x constants of one step of a variable-mobility model (FhModel): the
// parts of the site formulas that depend only on the step and on x, formed
// with the same operations as in the per-site form.
struct FhCol {
    double T, kT, chi, D;  // TIPSphil / TIPSbathPHIL: temperature, kT, chi, clamped D
    double scale;          // SIPS: mobility scale 0.95 + 0.25*log(1.0225 - chi fraction)
    // The reciprocal mobility of fh_site_r as a quotient q = f''/Dp:
    // q > qlo -> rlo and q < qhi -> rhi (the reference's clamps, their
    // reciprocals formed as the reference forms them), else q * fac.
    double Dm, invN, conv, qlo, qhi, rlo, rhi, fac;  // conv: Mweight/Mvolume (phi to g/L)
};

__device__ __forceinline__ FhCol fh_column(const FhDev& F, int x, double cs, double dt)
{
    using A = Arith<double>;
    FhCol k{};
    if (F.model == kFhLinear) return k;
    if (F.model == kFhSips) {
        // SIPS.cpp:160-170: chi from chiPN (the bath, x < NSdepth) toward
        // chiPS behind an erf front; kT at the initial temperature
        k.kT = A::div(F.Tinit, 273.0);
        if (x >= F.NSdepth)
            k.chi = A::add(A::mul(A::sub(F.chiPS, F.chiPN),
                                  erf(A::div((double)(x + 1), A::mul(2.0, sqrt(A::mul(A::mul(F.chiCond, cs), dt)))))),
                           F.chiPN);
        else
            k.chi = F.chiPN;
        const double frac = A::div(A::sub(k.chi, F.chiPS), A::sub(F.chiPN, F.chiPS));
        k.scale = A::add(0.95, A::mul(0.25, log(A::sub(1.0225, frac))));
        // SIPS.cpp:203-206: Mc in [0.00001, 1], then mob = Mc * scale
        k.Dm = F.D0;
        k.invN = A::div(1.0, F.N);
        k.conv = A::div(F.Mweight, F.Mvolume);
        k.qlo = 100000.0;
        k.qhi = 1.0;
        k.rlo = A::div(1.0, A::mul(0.00001, k.scale));
        k.rhi = A::div(1.0, A::mul(1.0, k.scale));
        k.fac = A::div(1.0, k.scale);
        return k;
    }
    // temperature of the step: a uniform ramp, or the bath profile along x
    // (TIPSbathPHIL.cpp:118-121)
    if (F.model == kFhBath)
        k.T = A::add(A::mul(A::sub(F.Tinit, F.Tbath),
                            erf(A::div((double)(x + 1), A::mul(2.0, sqrt(A::mul(A::mul(F.thermCond, cs), dt)))))),
                     F.Tbath);
    else
        k.T = A::sub(F.Tinit, A::mul(A::sub(F.Tinit, F.Tbath), A::div(cs, (double)F.nstep)));
    k.kT = A::div(k.T, 273.0);
    k.chi = A::add(A::div(F.alpha, k.T), F.beta);
    k.D = A::mul(F.D0, A::div(k.T, F.Tinit));
    if (k.D > F.D0) k.D = F.D0;
    // TIPSphil.cpp:172-175: Mc < 0.000001 -> 0.000001, then Mc > D0 -> D0,
    // then the crystallisation factor 0.001
    const bool cryst = k.T <= F.Tcrystal;
    const double mlo = 0.000001 > F.D0 ? F.D0 : 0.000001;
    k.Dm = k.D;
    k.invN = A::div(1.0, F.N);
    k.conv = A::div(F.Mweight, F.Mvolume);
    k.qlo = 1000000.0;
    k.qhi = A::div(1.0, F.D0);
    k.rlo = A::div(1.0, cryst ? A::mul(mlo, 0.001) : mlo);
    k.rhi = A::div(1.0, cryst ? A::mul(F.D0, 0.001) : F.D0);
    k.fac = cryst ? 1000.0 : 1.0;
    return k;
}

// x^nu of the Phillies mobility.  x^1 is x exactly (the reference's
// default nu = 1), which spares the general pow.
__device__ __forceinline__ double fh_pow(double x, double nu)
{
    return nu == 1.0 ? x : pow(x, nu);
}

// mu and mobility of one site from its concentration cc, its Laplacian
// lapc and the column constants k, every operation rounded on its own in
// the reference's order: TIPSphil.cpp:135-177 (and TIPSbathPHIL's),
// SIPS.cpp:160-208 with getFHcc, philliesDiffusion and secondDerFH of
// SIPS.cpp:254-285, and one field of SIPSternary.cpp:175-216, whose
// branch-local derivatives leave mu = 0.0 - K*lap(c) and a constant
// mobility.
__device__ __forceinline__ void fh_site_col(const FhDev& F, const FhCol& k, double cc, double lapc, double kap,
                                            double* mu, double* mob)
{
    using A = Arith<double>;
    if (F.model == kFhLinear) {
        *mu = A::sub(0.0, A::mul(kap, lapc));
        *mob = F.Mconst;
        return;
    }
    if (F.model == kFhSips) {
        const double cfh = cc < 0.0 ? 0.001 : (cc > 1.0 ? 0.999 : cc);
        double df = A::add(A::sub(A::sub(A::div(A::add(log(cfh), 1.0), F.N), log(A::sub(1.0, cfh))), 1.0),
                           A::mul(k.chi, A::sub(1.0, A::mul(2.0, cfh))));
        if (cc <= 0.0) df = A::mul(A::mul(-1.5, F.A), sqrt(-cc));
        *mu = A::sub(df, A::mul(kap, lapc));
        double cphil;
        if (cc >= 1.0) cphil = A::div(A::mul(1.0, F.Mweight), F.Mvolume);
        else if (cc < 0.0) cphil = A::div(A::mul(0.000001, F.Mweight), F.Mvolume);
        else cphil = A::div(A::mul(cc, F.Mweight), F.Mvolume);
        double ddf = A::mul(0.5, A::add(A::div(1.0, A::mul(F.N, cc)), A::div(1.0, A::sub(1.0, cc))));
        ddf = A::mul(ddf, k.kT);
        const double Dp = A::mul(F.D0, exp(A::mul(-F.gamma, fh_pow(cphil, F.nu))));
        double Mc = A::div(Dp, ddf);
        if (Mc > 1.0) Mc = 1.0;
        else if (Mc < 0.00001) Mc = 0.00001;
        *mob = A::mul(Mc, k.scale);
        return;
    }
    // chemical potential: df = ((log(cc)+1)/N - log(1-cc) - 1 + chi*(1-2cc)) * kT
    double df = A::add(A::sub(A::sub(A::div(A::add(log(cc), 1.0), F.N), log(A::sub(1.0, cc))), 1.0),
                       A::mul(k.chi, A::sub(1.0, A::mul(2.0, cc))));
    df = A::mul(df, k.kT);
    if (cc <= 0.0) df = A::mul(A::mul(-1.5, F.A), sqrt(-cc));
    *mu = A::sub(df, A::mul(kap, lapc));
    // Phillies self-diffusion over the second derivative of the free energy
    double cc_phil, ddf;
    if (cc >= 1.0) {
        cc_phil = A::div(A::mul(1.0, F.Mweight), F.Mvolume);
        ddf = A::mul(0.5, A::add(A::div(1.0, A::mul(F.N, 0.999)), A::div(1.0, A::sub(1.0, 0.999))));
    } else if (cc < 0.0) {
        const double cm = 0.0001;
        cc_phil = A::div(A::mul(cm, F.Mweight), F.Mvolume);
        ddf = A::mul(0.5, A::add(A::div(1.0, A::mul(F.N, cm)), A::div(1.0, A::sub(1.0, cm))));
    } else {
        cc_phil = A::div(A::mul(cc, F.Mweight), F.Mvolume);
        ddf = A::mul(0.5, A::add(A::div(1.0, A::mul(F.N, cc)), A::div(1.0, A::sub(1.0, cc))));
    }
    ddf = A::mul(ddf, k.kT);
    const double Dp = A::mul(k.D, exp(A::mul(-F.gamma, fh_pow(cc_phil, F.nu))));
    double Mc = A::div(Dp, ddf);
    if (Mc < 0.000001) Mc = 0.000001;
    if (Mc > F.D0) Mc = F.D0;
    if (k.T <= F.Tcrystal) Mc = A::mul(Mc, 0.001);
    *mob = Mc;
}

// the same for a site at x in step cs (the step being taken, as PFApp
// passes it) with time step dt
__device__ __forceinline__ void fh_site(const FhDev& F, double cc, double lapc, double kap, int x, double cs, double dt,
                                        double* mu, double* mob)
{
    fh_site_col(F, fh_column(F, x, cs, dt), cc, lapc, kap, mu, mob);
}

// mu and the reciprocal mobility 1/mob of one site, as the update passes
// use them.  For TIPSphil, TIPSbathPHIL and SIPS at 0 < cc < 1 (the sites of
// a field inside the Flory-Huggins range) the mobility is taken as one
// quotient: with u = 1 - cc the second derivative is
// f'' = kT (u + N cc) / (2 N cc u), so
//   1/mob = f'' / Dp = kT (u + N cc) / (2 N cc u Dm e),   e = exp(-gamma phi^nu),
// and the reference's clamps on Mc become bounds on that quotient, the
// clamped values' reciprocals formed per column as the reference forms them
// (FhCol).  That is one division where the reference takes six
// (1/(N cc), 1/(1 - cc), the conversion to g/L, Dp/f'', 1/Mc, and the
// 1/N of mu, here a product with 1/N); the result agrees with the
// reference's to a few ulp.  Everywhere else (cc <= 0, cc >= 1, NaN) and
// for kFhLinear: fh_site_col's reference-order arithmetic and 1/mob.
// Explicit fma and rounded operations, so every kernel that inlines this
// forms the same bits.
__device__ __forceinline__ void fh_site_r(const FhDev& F, const FhCol& k, double cc, double lapc, double kap,
                                          double* mu, double* rmob)
{
    using A = Arith<double>;
    if (F.model == kFhLinear || !(cc > 0.0 && cc < 1.0)) {
        double mob;
        fh_site_col(F, k, cc, lapc, kap, mu, &mob);
        *rmob = A::div(1.0, mob);
        return;
    }
    const double u = A::sub(1.0, cc);
    const double lc = log(cc), lu = log(u);
    // ((log(cc) + 1)/N - log(1 - cc) - 1 + chi (1 - 2 cc)), times kT for TIPSphil
    double df = A::add(A::sub(A::sub(A::mul(A::add(lc, 1.0), k.invN), lu), 1.0), A::mul(k.chi, fma(-2.0, cc, 1.0)));
    if (F.model != kFhSips) df = A::mul(df, k.kT);
    *mu = fma(-kap, lapc, df);
    const double phi = A::mul(cc, k.conv);
    const double e = exp(A::mul(-F.gamma, fh_pow(phi, F.nu)));
    const double num = A::mul(k.kT, fma(F.N, cc, u));
    const double den = A::mul(A::mul(A::mul(2.0, A::mul(F.N, cc)), u), A::mul(k.Dm, e));
    const double q = A::div(num, den);
    *rmob = q > k.qlo ? k.rlo : (q < k.qhi ? k.rhi : A::mul(q, k.fac));
}

// One axis of SfieldFD::Laplacian(const SfieldFD& mob) (SfieldFD.cpp:333-355)
// from the reciprocal mobilities rm, rp, ro of the minus, plus and centre
// sites: b1 = 2/(1/mob- + 1/mob0), b2 = 2/(1/mob+ + 1/mob0),
// (a-*b1 + a+*b2 - (b1+b2)*a0) / d^2 (divide, or multiply by 1/d^2).
__device__ __forceinline__ double fh_axis_r(double am, double ap, double a0, double rm, double rp, double ro,
                                            double coef, bool divide)
{
    using A = Arith<double>;
    const double b1 = A::div(2.0, A::add(rm, ro));
    const double b2 = A::div(2.0, A::add(rp, ro));
    const double num = A::sub(A::add(A::mul(am, b1), A::mul(ap, b2)), A::mul(A::add(b1, b2), a0));
    return divide ? A::div(num, coef) : A::mul(num, coef);
}

// One axis of the same divergence as a fraction n/q: with the face sums
// s1 = 1/mob- + 1/mob0 and s2 = 1/mob+ + 1/mob0 the faces are 2/s1 and
// 2/s2, and (a- b1 + a+ b2 - (b1 + b2) a0)/d^2 = 2 n/q with
// n = (a- - a0) s2 + (a+ - a0) s1 and q = s1 s2 d^2 (or n times the
// multiplier 1/d^2).
struct FhFrac {
    double n, q;
};
__device__ __forceinline__ FhFrac fh_axis_frac(double am, double ap, double a0, double rm, double rp, double ro,
                                               double coef, bool divide)
{
    using A = Arith<double>;
    const double s1 = A::add(rm, ro), s2 = A::add(rp, ro);
    double n = fma(A::sub(am, a0), s2, A::mul(A::sub(ap, a0), s1));
    double q = A::mul(s1, s2);
    if (divide) q = A::mul(q, coef);
    else n = A::mul(n, coef);
    return {n, q};
}

// The divergence of a site of a TIPSphil, TIPSbathPHIL or SIPS field from
// its axes' fractions over one common denominator, one division where the
// reference's form takes six (nine with unequal spacing):
// 2 (nx qy qz + ny qx qz + nz qx qy) / (qx qy qz), without y when flat.
// The face sums are at most twice the largest reciprocal mobility the
// models' clamps allow (about 2e9), so the products stay far inside the
// double range.  Agrees with the per-axis form to a few ulp of its terms.
__device__ __forceinline__ double fh_div_frac(FhFrac x, FhFrac y, FhFrac z, bool flat)
{
    using A = Arith<double>;
    if (flat) return A::div(A::mul(2.0, fma(x.n, z.q, A::mul(z.n, x.q))), A::mul(x.q, z.q));
    const double qxy = A::mul(x.q, y.q);
    const double nxy = fma(x.n, y.q, A::mul(y.n, x.q));
    return A::div(A::mul(2.0, fma(nxy, z.q, A::mul(z.n, qxy))), A::mul(qxy, z.q));
}

}  // namespace mg
