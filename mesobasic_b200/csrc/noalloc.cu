// mg_field_stats_noalloc: the diagnostics of mg_ch_reduce (mass, |c|,
// free energy, max|c|, non-finite count) for a field the caller holds in
// device memory, computed without allocating anything.
//
// Who needs it: a caller that must not allocate while it runs --
//   - a host thread that shares the device with running simulations, where a
//     cudaMalloc/cudaFree may synchronise the device and stall them;
//   - a service whose HBM is fully committed to resident fields by its
//     admission budget, so that even a small allocation can fail;
//   - code that only borrows a device pointer (a field owned by another
//     library) and has no handle of this library to hang scratch on.
// mg_ch_reduce allocates its partial-sum buffers with the handle; this entry
// point keeps them in one file-scope device array instead.
//
// Scratch: g_noalloc_scratch below, kNoAllocScratchBytes bytes (about
// 256 KB): a completion counter, the result, and one partial per plane.  A
// plane is one z-slice (nz > 1) or one x-row (two-dimensional fields,
// nz == 1), so fields with more than kNoAllocMaxPlanes planes are rejected
// with MG_EINVAL.
//
// Set-up: every call looks up the array's device address
// (cudaGetSymbolAddress, with that device current), so a device reset
// between calls cannot leave a stale address behind.  The first lookup on a
// device loads this library's device code there: make that first call
// before any stream capture on the device.  Every call clears the
// completion counter (cudaMemsetAsync on the caller's stream) before its
// launch.
//
// Concurrency: all calls on one device share the one scratch array, so calls
// that overlap in time -- from several host threads, or on several streams
// -- race and may return wrong numbers.  Issue them one at a time.  A call
// that returns MG_ETIMEOUT leaves its kernel queued or running on the
// caller's stream: synchronise that stream before the next call on the
// device, or the next call races it.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <mutex>
#include <thread>

#include "engine.h"
#include "mg_device.cuh"

namespace mg {
namespace {

constexpr int kNoAllocMaxPlanes = 4096;
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxDevices = 64;

struct PlanePartial {
    double2 mass, abs_mass, energy;  // compensated (sum, error) pairs
    double max_abs, bad;
};

// scratch layout: [0, 256) counter + result; then the plane partials
constexpr size_t kCounterOff = 0;
constexpr size_t kResultOff = 64;
constexpr size_t kPlaneOff = 256;
static_assert(kResultOff + sizeof(Diag) <= kPlaneOff, "result does not fit the scratch head");
constexpr size_t kNoAllocScratchBytes = kPlaneOff + (size_t)kNoAllocMaxPlanes * sizeof(PlanePartial);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

__device__ __forceinline__ int wrap_clamp(int i, int n, bool periodic)
{
    if (periodic) return i >= n ? i - n : i;  // i in [0, n]
    return i >= n ? n - 1 : i;
}

// One block per plane.  The last block to finish sums the plane partials in
// plane order with a fixed tree, so the result does not depend on timing.
template <typename T>
__global__ void __launch_bounds__(kNoAllocThreads)
    plane_stats_kernel(const T* __restrict__ c, int nx, int ny, int nz, int perX, int perY, int perZ, double spx,
                       double spy, double spz, double kap, double dv, long long plane_sites, unsigned char* scratch)
{
    __shared__ double2 red[32];
    __shared__ double smax[32], sbad[32];
    __shared__ int last;
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kCounterOff);
    Diag* result = reinterpret_cast<Diag*>(scratch + kResultOff);
    PlanePartial* part = reinterpret_cast<PlanePartial*>(scratch + kPlaneOff);

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const long long s0 = (long long)blockIdx.x * plane_sites;
    double2 sm = make_double2(0, 0), sa = make_double2(0, 0), se = make_double2(0, 0);
    double mx = 0.0, bad = 0.0;
    for (long long s = s0 + threadIdx.x; s < s0 + plane_sites; s += blockDim.x) {
        const double v = (double)c[s];
        if (!isfinite(v)) {
            bad += 1.0;
            continue;
        }
        const int x = (int)(s % nx), y = (int)((s / nx) % ny), z = (int)(s / ((long long)nx * ny));
        auto at = [&](int xx, int yy, int zz) { return (double)c[((long long)zz * ny + yy) * nx + xx]; };
        const double gx = (at(wrap_clamp(x + 1, nx, perX), y, z) - v) / spx;
        const double gy = (at(x, wrap_clamp(y + 1, ny, perY), z) - v) / spy;
        const double gz = (at(x, y, wrap_clamp(z + 1, nz, perZ)) - v) / spz;
        const double w = v * v - 1.0;
        const double f = 0.25 * w * w + 0.5 * kap * (gx * gx + gy * gy + gz * gz);
        sm = pair_add(sm, make_double2(v, 0.0));
        sa = pair_add(sa, make_double2(fabs(v), 0.0));
        se = pair_add(se, make_double2(f, 0.0));
        mx = fmax(mx, fabs(v));
    }
    sm = block_pair_sum(sm, red);
    sa = block_pair_sum(sa, red);
    se = block_pair_sum(se, red);
    for (int off = 16; off > 0; off >>= 1) {
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
        bad += __shfl_down_sync(0xffffffffu, bad, off);
    }
    if (lane == 0) smax[warp] = mx, sbad[warp] = bad;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0, b = 0.0;
        for (int w = 0; w < nwarps; ++w) m = fmax(m, smax[w]), b += sbad[w];
        PlanePartial p;
        p.mass = sm, p.abs_mass = sa, p.energy = se, p.max_abs = m, p.bad = b;
        part[blockIdx.x] = p;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();

    // ---- last block: fixed-order sum over the planes
    double2 a0 = make_double2(0, 0), a1 = make_double2(0, 0), a2 = make_double2(0, 0);
    mx = 0.0, bad = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        const double* q = reinterpret_cast<const double*>(part + b);
        a0 = pair_add(a0, make_double2(__ldcg(q + 0), __ldcg(q + 1)));
        a1 = pair_add(a1, make_double2(__ldcg(q + 2), __ldcg(q + 3)));
        a2 = pair_add(a2, make_double2(__ldcg(q + 4), __ldcg(q + 5)));
        mx = fmax(mx, __ldcg(q + 6));
        bad += __ldcg(q + 7);
    }
    a0 = block_pair_sum(a0, red);
    a1 = block_pair_sum(a1, red);
    a2 = block_pair_sum(a2, red);
    for (int off = 16; off > 0; off >>= 1) {
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
        bad += __shfl_down_sync(0xffffffffu, bad, off);
    }
    __syncthreads();  // smax/sbad are reused
    if (lane == 0) smax[warp] = mx, sbad[warp] = bad;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0, b = 0.0;
        for (int w = 0; w < nwarps; ++w) m = fmax(m, smax[w]), b += sbad[w];
        result->mass = (a0.x + a0.y) * dv;
        result->abs_mass = (a1.x + a1.y) * dv;
        result->energy = (a2.x + a2.y) * dv;
        result->max_abs = m;
        result->nonfinite = b;
    }
}

// device address of g_noalloc_scratch on the current device, looked up on
// every call (cheap once the module is loaded)
unsigned char* scratch_address(int device, int* rc)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        *rc = fail(MG_ECUDA, "cudaGetSymbolAddress of the no-allocation scratch failed on device %d: %s", device,
                   cudaGetErrorString(e));
        return nullptr;
    }
    *rc = MG_OK;
    return static_cast<unsigned char*>(p);
}

int field_stats_noalloc(const void* field, const mg_ch_params* p, int device, cudaStream_t stream,
                        long long timeout_us, mg_ch_stats* out)
{
    if (!field || !p || !out) return fail(MG_EINVAL, "null argument");
    if (p->nx < 1 || p->ny < 1 || p->nz < 1) return fail(MG_EINVAL, "grid %dx%dx%d is empty", p->nx, p->ny, p->nz);
    if (!(p->dx > 0.0) || !(p->dy > 0.0) || !(p->dz > 0.0)) return fail(MG_EINVAL, "spacings must be positive");
    if (p->precision != MG_FP64 && p->precision != MG_FP32) return fail(MG_EINVAL, "precision must be MG_FP64 or MG_FP32");
    if (device < 0 || device >= kNoAllocMaxDevices)
        return fail(MG_EINVAL, "device %d is outside 0..%d", device, kNoAllocMaxDevices - 1);
    const int planes = p->nz > 1 ? p->nz : p->ny;
    const long long plane_sites = p->nz > 1 ? (long long)p->nx * p->ny : (long long)p->nx;
    if (planes > kNoAllocMaxPlanes)
        return fail(MG_EINVAL,
                    "field has %d planes (%s); the no-allocation reduction takes at most %d -- use mg_ch_reduce",
                    planes, p->nz > 1 ? "nz" : "ny of a 2-D field", kNoAllocMaxPlanes);

    int prev = 0;
    MG_CUDA(cudaGetDevice(&prev));
    struct Restore {
        int d;
        ~Restore() { cudaSetDevice(d); }
    } restore{prev};
    MG_CUDA(cudaSetDevice(device));
    int rc = MG_OK;
    unsigned char* scratch = scratch_address(device, &rc);
    if (!scratch) return rc;

    MG_CUDA(cudaMemsetAsync(scratch + kCounterOff, 0, sizeof(unsigned int), stream));
    const double dv = p->dx * p->dy * p->dz;
    if (p->precision == MG_FP64)
        plane_stats_kernel<double><<<planes, kNoAllocThreads, 0, stream>>>(
            static_cast<const double*>(field), p->nx, p->ny, p->nz, p->bx != 0, p->by != 0, p->bz != 0, p->dx, p->dy,
            p->dz, p->kappa, dv, plane_sites, scratch);
    else
        plane_stats_kernel<float><<<planes, kNoAllocThreads, 0, stream>>>(
            static_cast<const float*>(field), p->nx, p->ny, p->nz, p->bx != 0, p->by != 0, p->bz != 0, p->dx, p->dy,
            p->dz, p->kappa, dv, plane_sites, scratch);
    MG_CUDA(cudaGetLastError());

    // bounded wait for the stream, then read the result back
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t e = cudaStreamQuery(stream);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) MG_CUDA(e);
        if (timeout_us >= 0) {
            const auto us =
                std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
            if (us > timeout_us)
                return fail(MG_ETIMEOUT,
                            "reduction not finished after %lld us; its kernel is still on the stream: synchronise "
                            "the stream before the next call",
                            timeout_us);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    Diag d;
    MG_CUDA(cudaMemcpyAsync(&d, scratch + kResultOff, sizeof(Diag), cudaMemcpyDeviceToHost, stream));
    MG_CUDA(cudaStreamSynchronize(stream));
    out->mass = d.mass;
    out->energy = d.energy;
    out->abs_mass = d.abs_mass;
    out->max_abs = d.max_abs;
    out->nonfinite = (long long)d.nonfinite;
    out->step = -1;
    if (out->nonfinite > 0) return fail(MG_ENONFINITE, "%lld sites are NaN or Inf", out->nonfinite);
    return MG_OK;
}

}  // namespace
}  // namespace mg

extern "C" int mg_field_stats_noalloc(const void* field_dev, const mg_ch_params* params, int device, void* stream,
                                      long long timeout_us, mg_ch_stats* out)
{
    mg::clear_error();
    return mg::field_stats_noalloc(field_dev, params, device, static_cast<cudaStream_t>(stream), timeout_us, out);
}
