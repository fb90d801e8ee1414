// Host engine of libmesogpu: job setup, tensor maps, launch groups, CUDA
// graphs, transfers, diagnostics.  See engine.h.
#include "engine.h"
#include "ch_kernels.cuh"
#include "ch_lean.cuh"
#include "ch_march.cuh"
#include "fh_march.cuh"

#include <cufft.h>
#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <thread>

namespace mg {

static bool march_enabled();

// ------------------------------------------------------------------ errors
static thread_local std::string t_err;

int fail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
    return code;
}
void clear_error() { t_err.clear(); }
const char* last_error() { return t_err.c_str(); }

// ------------------------------------------------------------ device info
int device_info(int device, DevInfo* out)
{
    static std::mutex mu;
    static std::map<int, DevInfo> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(device);
    if (it != cache.end()) {
        *out = it->second;
        return MG_OK;
    }
    int count = 0;
    MG_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(MG_EINVAL, "device %d not present (%d devices)", device, count);
    cudaDeviceProp prop;
    MG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(MG_EINVAL, "device %d is sm_%d%d; this library is built for sm_100a", device,
                                     prop.major, prop.minor);
    DevInfo d;
    d.sms = prop.multiProcessorCount;
    d.smem_optin = prop.sharedMemPerBlockOptin;
    d.total_mem = prop.totalGlobalMem;
    d.major = prop.major;
    d.minor = prop.minor;
    cache[device] = d;
    *out = d;
    return MG_OK;
}

// ------------------------------------------------------------ tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int get_encode(EncodeTiledFn* fn)
{
    static EncodeTiledFn cached = nullptr;
    static std::once_flag once;
    static cudaError_t status = cudaSuccess;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        status = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (status == cudaSuccess && q == cudaDriverEntryPointSuccess) cached = reinterpret_cast<EncodeTiledFn>(p);
    });
    if (!cached) return fail(MG_ECUDA, "cuTensorMapEncodeTiled unavailable (%s)", cudaGetErrorString(status));
    *fn = cached;
    return MG_OK;
}

// body map: box (bw, ty, 1); row map: box (bw, 1, 1)
static int encode_maps(const Job& j, CUtensorMap host_maps[4])
{
    EncodeTiledFn enc;
    MG_TRY(get_encode(&enc));
    const Geometry& g = j.g;
    const int bw = std::min(g.lnx, 256);
    for (int b = 0; b < 2; ++b) {
        cuuint64_t dims[3] = {(cuuint64_t)g.lnx, (cuuint64_t)g.lny, (cuuint64_t)g.lnz};
        cuuint64_t strides[2] = {(cuuint64_t)g.lnx * g.es, (cuuint64_t)g.lnx * g.lny * g.es};
        cuuint32_t estr[3] = {1, 1, 1};
        const CUtensorMapDataType dt = g.es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        for (int m = 0; m < 2; ++m) {
            cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)(m == 0 ? (g.flat ? 1 : j.tiling.ty) : 1), 1};
            CUresult r = enc(&host_maps[2 * b + m], dt, 3, j.buf[b], dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return fail(MG_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
        }
    }
    return MG_OK;
}

// ------------------------------------------------------------ geometry
int validate_params(const mg_ch_params& p)
{
    if (p.nx < 1 || p.ny < 1 || p.nz < 1) return fail(MG_EINVAL, "grid %dx%dx%d: every dimension must be >= 1", p.nx, p.ny, p.nz);
    const double n = (double)p.nx * p.ny * p.nz;
    if (n > 4.0e10) return fail(MG_EINVAL, "grid of %.3g sites is too large", n);
    if (!(p.dx > 0) || !(p.dy > 0) || !(p.dz > 0) || !std::isfinite(p.dx) || !std::isfinite(p.dy) || !std::isfinite(p.dz))
        return fail(MG_EINVAL, "grid spacing must be positive and finite");
    if (!std::isfinite(p.dt) || !std::isfinite(p.M) || !std::isfinite(p.kappa))
        return fail(MG_EINVAL, "dt, M and kappa must be finite");
    if ((p.bx != 0 && p.bx != 1) || (p.by != 0 && p.by != 1) || (p.bz != 0 && p.bz != 1))
        return fail(MG_EINVAL, "bx, by, bz must be 0 (no-flux) or 1 (periodic)");
    if (p.precision != MG_FP64 && p.precision != MG_FP32) return fail(MG_EINVAL, "precision must be MG_FP64 or MG_FP32");
    if (p.mass_correct && p.precision != MG_FP32) return fail(MG_EINVAL, "mass_correct applies to MG_FP32 only");
    if (!(p.noise >= 0) || !std::isfinite(p.noise)) return fail(MG_EINVAL, "noise must be finite and >= 0");
    return MG_OK;
}

int make_geometry(const mg_ch_params& p, Geometry* out)
{
    MG_TRY(validate_params(p));
    Geometry g;
    g.es = p.precision == MG_FP32 ? 4 : 8;
    if (p.nz == 1 && p.ny > 1) {
        // 2-D: run as (nx, 1, ny); the reference's z Laplacian term is 0
        g.lnx = p.nx, g.lny = 1, g.lnz = p.ny;
        g.lsx = p.dx, g.lsy = p.dz, g.lsz = p.dy;
        g.perx = p.bx, g.pery = 1, g.perz = p.by;
        g.flat = true;
    } else {
        g.lnx = p.nx, g.lny = p.ny, g.lnz = p.nz;
        g.lsx = p.dx, g.lsy = p.dy, g.lsz = p.dz;
        g.perx = p.bx, g.pery = p.by, g.perz = p.bz;
        g.flat = (p.ny == 1);
    }
    g.n = (size_t)p.nx * p.ny * p.nz;
    *out = g;
    return MG_OK;
}

bool tma_shape_ok(const Geometry& g)
{
    const int w = kStripBytes / g.es;  // elements per thread strip
    if (g.lnx % w != 0) return false;
    // rows wider than one 256-element TMA box: both strip halves (x and
    // x + nx/2) must sit at the same position of their boxes
    if (g.lnx > 256 && g.lnx % 512 != 0) return false;
    const int bw = std::min(g.lnx, 256);
    if ((bw * g.es) % 128 != 0) return false;  // 128-byte aligned TMA destinations
    if (g.lnx / w > 512) return false;
    if (!g.flat && g.lny < 2) return false;
    return true;
}

static int round_up(int v, int m) { return (v + m - 1) / m * m; }

// the step kernel has a compile-time row-width variant for this job
// row widths with compile-time variants of the step kernel: 256 with ring
// depths 4 and 8; the widths of batched and large jobs with depth 4
static const int kFixedWidths[] = {64, 96, 128, 160, 192, 224, 256, 512};

static bool fixed_width(int nx, int nbuf)
{
    if (nx == 256) return nbuf == 4 || nbuf == 8;
    if (nbuf != 4) return false;
    for (int w : kFixedWidths)
        if (w == nx) return true;
    return false;
}

bool fixed_width_kernel(const Geometry& g, int nbuf)
{
    if (!geometry_simple(g) || g.flat) return false;
    if (fixed_width(g.lnx, nbuf)) return true;
    // a march variant (launch bound kMaxBlock) for this width and ring depth
    return march_enabled() &&
           (g.es == 4 ? march_kernel_f32(g.lnx, nbuf, false) : march_kernel_f64(g.lnx, nbuf)) != nullptr;
}

int plan_tiling(const Geometry& g, const mg_tiling& t, const DevInfo& d, TilePlan* out)
{
    TilePlan pl;
    if (t.path == 1) {
        pl.tma_ok = false;
        pl.block = 256;
        pl.nitems = 1;
        *out = pl;
        return MG_OK;
    }
    if (t.path != 0) return fail(MG_EINVAL, "tiling path must be 0 or 1");
    if (!tma_shape_ok(g)) return fail(MG_EINVAL, "shape %dx%dx%d (%s) is not taken by the tiled kernel", g.lnx, g.lny,
                                      g.lnz, g.es == 4 ? "fp32" : "fp64");
    if (!nbuf_ok(t.nbuf)) return fail(MG_EINVAL, "nbuf must be 3, 4, 6 or 8");
    if (t.nchunk < 1 || t.nchunk > g.lnz) return fail(MG_EINVAL, "nchunk %d outside [1, %d]", t.nchunk, g.lnz);
    const int nq = g.lnx / (kStripBytes / g.es);
    int CY, MY, ntr;
    if (g.flat) {
        if (t.ty != 1) return fail(MG_EINVAL, "2-D jobs use ty = 1");
        CY = MY = 1;
        ntr = 1;
        pl.ntile = 1;
    } else {
        if (t.ty < 1 || t.ty > g.lny || t.ty > 252)
            return fail(MG_EINVAL, "ty %d must be in [1, ny] (ny = %d)", t.ty, g.lny);
        CY = t.ty + 4;
        MY = t.ty + 2;
        ntr = MY;  // one mu row per thread row
        pl.ntile = (g.lny + t.ty - 1) / t.ty;
    }
    pl.block = round_up(nq * ntr, 32);
    const int maxb = fixed_width_kernel(g, t.nbuf) ? kMaxBlock : kMaxBlockGeneric;
    if (pl.block > maxb) return fail(MG_EINVAL, "tile needs %d threads (> %d); lower ty", nq * ntr, maxb);
    pl.cplane = round_up(CY * g.lnx, 32);
    pl.mplane = round_up(MY * g.lnx, 32);
    const size_t head = (sizeof(SmemHead) + 127) / 128 * 128 + 128;  // + alignment slack
    pl.smem = head + (size_t)t.nbuf * pl.cplane * g.es + (size_t)3 * pl.mplane * g.es;
    if (pl.smem > d.smem_optin)
        return fail(MG_EINVAL, "tile needs %zu bytes of shared memory (> %zu); lower ty", pl.smem, d.smem_optin);
    pl.nitems = pl.ntile * t.nchunk;
    pl.tma_ok = true;
    *out = pl;
    return MG_OK;
}

// The fused variable-mobility kernel (fh_march.cuh) takes FP64 rows of at
// most 256 elements whose width is a multiple of 16 (128-byte aligned
// shared-memory rows for the TMA), 3-D with ny >= 2 or flat.
bool fh_shape_ok(const Geometry& g)
{
    return g.es == 8 && g.lnx % 16 == 0 && g.lnx <= kFhMaxNx && (g.flat || g.lny >= 2);
}

static size_t fh_smem(int nbuf, int cplane, int mplane)
{
    const size_t head = (sizeof(SmemHead) + 127) / 128 * 128 + 128;  // + alignment slack
    return head + (size_t)nbuf * cplane * 8 + (size_t)6 * mplane * 8 + (size_t)kFhMaxNx * sizeof(FhCol);
}

int plan_fh_tiling(const Geometry& g, const mg_tiling& t, const DevInfo& d, TilePlan* out)
{
    TilePlan pl;
    if (t.path == 1) {
        pl.tma_ok = false;
        pl.block = 256;
        pl.nitems = 1;
        *out = pl;
        return MG_OK;
    }
    if (t.path != 0) return fail(MG_EINVAL, "tiling path must be 0 or 1");
    if (!fh_shape_ok(g)) return fail(MG_EINVAL, "shape %dx%dx%d is not taken by the fused variable-mobility kernel",
                                     g.lnx, g.lny, g.lnz);
    if (t.nbuf != 3) return fail(MG_EINVAL, "the fused variable-mobility kernel uses nbuf 3");
    if (t.nchunk < 1 || t.nchunk > g.lnz) return fail(MG_EINVAL, "nchunk %d outside [1, %d]", t.nchunk, g.lnz);
    int CY = 1, MY = 1;
    if (g.flat) {
        if (t.ty != 1) return fail(MG_EINVAL, "2-D jobs use ty = 1");
        pl.ntile = 1;
    } else {
        if (t.ty < 1 || t.ty > g.lny) return fail(MG_EINVAL, "ty %d must be in [1, ny] (ny = %d)", t.ty, g.lny);
        CY = t.ty + 4;
        MY = t.ty + 2;
        pl.ntile = (g.lny + t.ty - 1) / t.ty;
    }
    if ((g.lnx / 4) * MY > kFhBlock) return fail(MG_EINVAL, "tile needs %d threads (> %d); lower ty", (g.lnx / 4) * MY, kFhBlock);
    pl.block = kFhBlock;
    pl.cplane = round_up(CY * g.lnx, 32);
    pl.mplane = round_up(MY * g.lnx, 32);
    pl.smem = fh_smem(t.nbuf, pl.cplane, pl.mplane);
    if (pl.smem > d.smem_optin)
        return fail(MG_EINVAL, "tile needs %zu bytes of shared memory (> %zu); lower ty", pl.smem, d.smem_optin);
    pl.nitems = pl.ntile * t.nchunk;
    pl.tma_ok = true;
    *out = pl;
    return MG_OK;
}

// deepest tile that fits the block and shared memory; z chunks to give
// every SM about one item (one CTA per SM)
static mg_tiling fh_default_tiling(const Geometry& g, const DevInfo& d)
{
    if (!fh_shape_ok(g)) return mg_tiling{1, 1, 4, 1};
    int ty = 1;
    if (!g.flat)
        for (int t = std::min(g.lny, kFhBlock / (g.lnx / 4) - 2); t >= 1; --t) {
            TilePlan pl;
            if (plan_fh_tiling(g, mg_tiling{t, 1, 3, 0}, d, &pl) == MG_OK) {
                ty = t;
                break;
            }
            clear_error();
        }
    const int ntile = g.flat ? 1 : (g.lny + ty - 1) / ty;
    int nchunk = std::max(1, (3 * d.sms + ntile - 1) / ntile);  // about three waves of items
    nchunk = std::min(nchunk, std::max(1, g.lnz / 8));
    if (nchunk > 1 && (nchunk & 1)) nchunk += 1;
    nchunk = std::min(nchunk, g.lnz);
    return mg_tiling{ty, nchunk, 3, 0};
}

template <typename T, bool FLAT, bool SIMPLE, bool MASS>
static StepKernel pick_nbuf(int nbuf)
{
    switch (nbuf) {
        case 3: return ch_step_kernel<T, 3, FLAT, SIMPLE, MASS>;
        case 4: return ch_step_kernel<T, 4, FLAT, SIMPLE, MASS>;
        case 6: return ch_step_kernel<T, 6, FLAT, SIMPLE, MASS>;
        default: return ch_step_kernel<T, 8, FLAT, SIMPLE, MASS>;
    }
}

template <typename T, bool FLAT, bool SIMPLE, bool MASS>
static StepKernel pick_maxt(int nbuf, int /*block*/)
{
    return pick_nbuf<T, FLAT, SIMPLE, MASS>(nbuf);
}

// row widths with a compile-time specialisation of the step kernel
// FP32 rows whose threads form a power-of-two segment of a warp take the
// lean variant (bit-identical results, less per-plane overhead)
template <bool MASS>
static StepKernel pick_lean(int nx, int nbuf)
{
    switch (nx) {
    case 64: return nbuf == 4 ? ch_lean_kernel<64, 4, MASS> : nullptr;
    case 128: return nbuf == 4 ? ch_lean_kernel<128, 4, MASS> : nullptr;
    case 256:
        switch (nbuf) {
        case 3: return ch_lean_kernel<256, 3, MASS>;
        case 4: return ch_lean_kernel<256, 4, MASS>;
        case 6: return ch_lean_kernel<256, 6, MASS>;
        default: return ch_lean_kernel<256, 8, MASS>;
        }
    default: return nullptr;
    }
}

template <typename T, bool FLAT, bool MASS>
static StepKernel pick_fixed(int nx, int nbuf)
{
    if (nx == 256) return nbuf == 8 ? ch_step_kernel<T, 8, FLAT, true, MASS, 256> : ch_step_kernel<T, 4, FLAT, true, MASS, 256>;
    if (nbuf != 4) return nullptr;
    switch (nx) {
    case 64: return ch_step_kernel<T, 4, FLAT, true, MASS, 64>;
    case 96: return ch_step_kernel<T, 4, FLAT, true, MASS, 96>;
    case 128: return ch_step_kernel<T, 4, FLAT, true, MASS, 128>;
    case 160: return ch_step_kernel<T, 4, FLAT, true, MASS, 160>;
    case 192: return ch_step_kernel<T, 4, FLAT, true, MASS, 192>;
    case 224: return ch_step_kernel<T, 4, FLAT, true, MASS, 224>;
    case 512: return ch_step_kernel<T, 4, FLAT, true, MASS, 512>;
    default: return nullptr;
    }
}

template <typename T, bool MASS>
static StepKernel pick_shape(bool flat, bool simple, int nbuf, int block)
{
    if (flat) return simple ? pick_maxt<T, true, true, MASS>(nbuf, block) : pick_maxt<T, true, false, MASS>(nbuf, block);
    return simple ? pick_maxt<T, false, true, MASS>(nbuf, block) : pick_maxt<T, false, false, MASS>(nbuf, block);
}

// MG_MARCH=0 selects the earlier kernels (ch_step_kernel, ch_lean_kernel)
static bool march_enabled()
{
    static const bool v = [] {
        const char* e = std::getenv("MG_MARCH");
        return !(e && e[0] == '0');
    }();
    return v;
}

StepKernel step_kernel(bool fp32, bool flat, int nbuf, bool simple, int block, bool mass, int nx)
{
    if (simple && !flat && nx > 0 && march_enabled()) {
        StepKernel k = fp32 ? march_kernel_f32(nx, nbuf, mass) : march_kernel_f64(nx, nbuf);
        if (k) return k;
    }
    if (fp32 && simple && !flat && nx > 0) {
        StepKernel k = mass ? pick_lean<true>(nx, nbuf) : pick_lean<false>(nx, nbuf);
        if (k) return k;
    }
    if (simple && !flat && (nbuf == 4 || nbuf == 8) && nx > 0) {
        StepKernel k = fp32 ? (mass ? pick_fixed<float, false, true>(nx, nbuf) : pick_fixed<float, false, false>(nx, nbuf))
                            : pick_fixed<double, false, false>(nx, nbuf);
        if (k) return k;
    }
    if (fp32) return mass ? pick_shape<float, true>(flat, simple, nbuf, block)
                          : pick_shape<float, false>(flat, simple, nbuf, block);
    return pick_shape<double, false>(flat, simple, nbuf, block);
}

bool nbuf_ok(int nbuf) { return nbuf == 3 || nbuf == 4 || nbuf == 6 || nbuf == 8; }

bool march_batch_job(const Geometry& g)
{
    if (!march_enabled() || !geometry_simple(g) || g.flat || !tma_shape_ok(g)) return false;
    return (g.es == 4 ? march_kernel_f32(g.lnx, kMarchBatchNbuf, false) : march_kernel_f64(g.lnx, kMarchBatchNbuf)) != nullptr;
}

int prepare_kernels(const DevInfo& d)
{
    static std::mutex mu;
    static bool done = false;
    std::lock_guard<std::mutex> lock(mu);
    if (done) return MG_OK;
    const int nbufs[4] = {3, 4, 6, 8};
    for (int f32 = 0; f32 < 2; ++f32)
        for (int fl = 0; fl < 2; ++fl)
            for (int sm = 0; sm < 2; ++sm)
                for (int nb : nbufs)
                    for (int bl : {256, 512})
                        for (int ms = 0; ms < 2; ++ms)
                            for (int fx : {0, 64, 96, 128, 160, 192, 224, 256, 512})
                                MG_CUDA(cudaFuncSetAttribute(step_kernel(f32, fl, nb, sm, bl, ms && f32, fx),
                                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                             (int)d.smem_optin));
    for (int ms = 0; ms < 2; ++ms)
        MG_CUDA(cudaFuncSetAttribute(march_kernel_f32(256, 3, ms, 8), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)d.smem_optin));
    for (const auto& wt : {std::pair<int, int>{64, 32}, {96, 24}, {128, 16}, {160, 14}, {192, 11}})
        MG_CUDA(cudaFuncSetAttribute(march_kernel_f32(wt.first, 3, true, wt.second),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.smem_optin));
    for (int nb : {3, 6})
        MG_CUDA(cudaFuncSetAttribute(march_kernel_f64(256, nb, 7), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)d.smem_optin));
    MG_CUDA(cudaFuncSetAttribute(fh_march_kernel<3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.smem_optin));
    MG_CUDA(cudaFuncSetAttribute(fh_march_kernel<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.smem_optin));
    done = true;
    return MG_OK;
}

// all axes that matter periodic and equal coefficients (FP64: equal to 1,
// so the multiplication can be skipped exactly)
bool geometry_simple(const Geometry& g)
{
    if (!g.perx || !g.perz || (!g.flat && !g.pery)) return false;
    const double cx = 1.0 / (g.lsx * g.lsx), cz = 1.0 / (g.lsz * g.lsz), cy = 1.0 / (g.lsy * g.lsy);
    if (cx != cz || (!g.flat && cx != cy)) return false;
    if (g.es == 8 && !(g.lsx == 1.0 && g.lsz == 1.0 && (g.flat || g.lsy == 1.0))) return false;
    return true;
}

static int occupancy(const Geometry& g, const mg_tiling& t, const TilePlan& pl, int* occ)
{
    MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, step_kernel(g.es == 4, g.flat, t.nbuf,
                                                                      geometry_simple(g), pl.block, g.es == 4, g.lnx),
                                                          pl.block, pl.smem));
    if (*occ < 1) *occ = 1;
    return MG_OK;
}

mg_tiling default_tiling(const Geometry& g, const DevInfo& d, int device)
{
    (void)device;
    mg_tiling best{1, 1, 4, 1};
    if (!tma_shape_ok(g)) return best;
    std::string key = tune_key(g);
    mg_tiling tuned;
    if (tune_lookup(key, &tuned)) {
        TilePlan pl;
        if (plan_tiling(g, tuned, d, &pl) == MG_OK) return tuned;
        clear_error();
    }
    // heuristic: the deepest tile (fewest halo rows) that keeps two CTAs per
    // SM, then enough z chunks to fill every CTA slot once, even count so
    // neighbouring chunks march towards / away from each other
    double best_score = -1.0;
    for (int nbuf : {8, 6, 4, 3}) {
        std::vector<int> tys;
        if (g.flat) tys.push_back(1);
        else
            for (int ty = 1; ty <= std::min(g.lny, 62); ++ty) tys.push_back(ty);
        for (int ty : tys) {
            mg_tiling t{ty, 1, nbuf, 0};
            TilePlan pl;
            if (plan_tiling(g, t, d, &pl) != MG_OK) {
                clear_error();
                continue;
            }
            int occ = 1;
            if (occupancy(g, t, pl, &occ) != MG_OK) {
                clear_error();
                continue;
            }
            const int slots = d.sms * occ;
            int nchunk = std::max(1, slots / pl.ntile);
            const int minplanes = g.flat ? 8 : 16;
            nchunk = std::min(nchunk, std::max(1, g.lnz / minplanes));
            if (nchunk > 1 && (nchunk & 1)) nchunk -= 1;
            const int items = pl.ntile * nchunk;
            // efficiency: filled slots x halo overheads
            const double fill = std::min(1.0, (double)items / slots);
            const double rows = g.flat ? 1.0 : (double)ty / (ty + 4);
            const double planes = (double)(g.lnz / nchunk) / (g.lnz / nchunk + 4);
            const double occw = occ >= 2 ? 1.0 : 0.85;
            // planes in flight per SM hide the load latency
            const double inflight = std::min(1.0, (double)(nbuf - 2) * occ * pl.cplane * g.es / (96.0 * 1024));
            const double score = fill * std::sqrt(rows) * planes * occw * (0.5 + 0.5 * inflight);
            if (score > best_score) {
                best_score = score;
                best = mg_tiling{ty, nchunk, nbuf, 0};
            }
        }
    }
    return best;
}

// Tiling of a job that shares its launches with other jobs (batch, server).
// Every job gets tiles of about kBatchThreads threads (ty + 2 mu rows of
// nx/W strips), so the CTAs of one launch are equally full whatever each
// job's row width; tiles are balanced to divide ny evenly; z chunks are about
// kBatchPlanes planes (16 rows for 2-D jobs; many jobs fill the grid, so no
// job is cut finer).  320 threads is the largest CTA that keeps two per SM
// at 96 registers.  A pure
// function of the shape: a job keeps its tiling for its whole life.
// environment knob: a positive integer, else `def`
int mg_env_int(const char* name, int def)
{
    const char* e = std::getenv(name);
    const int v = e ? std::atoi(e) : 0;
    return v > 0 ? v : def;
}

mg_tiling batch_tiling_for(const Geometry& g, const DevInfo& d, int device, int threads, int planes)
{
    if (!tma_shape_ok(g)) return default_tiling(g, d, device);
    const int kBatchThreads = std::max(32, threads), kBatchPlanes = std::max(1, planes);
    const int nq = g.lnx / (kStripBytes / g.es);
    const int nbuf = g.flat ? 8 : 4;
    int ty = 1;
    if (!g.flat) {
        const int maxb = fixed_width_kernel(g, nbuf) ? kMaxBlock : kMaxBlockGeneric;
        int tymax = std::max(1, kBatchThreads / nq - 2);
        tymax = std::max(tymax, std::min(8, std::max(1, maxb / nq - 2)));  // at least 8 rows where they fit
        tymax = std::min(tymax, g.lny);
        const int ntile = (g.lny + tymax - 1) / tymax;
        ty = (g.lny + ntile - 1) / ntile;
    }
    // 2-D jobs march along their rows one row per plane: shorter chunks give
    // them enough CTAs
    mg_tiling t{ty, std::max(1, g.lnz / (g.flat ? 16 : kBatchPlanes)), nbuf, 0};
    TilePlan pl;
    while (plan_tiling(g, t, d, &pl) != MG_OK) {  // shrink the tile until it fits
        clear_error();
        if (t.ty <= 1) return default_tiling(g, d, device);
        t.ty -= 1;
    }
    return t;
}

// ------------------------------------------------------------ autotune cache
static std::mutex g_tune_mu;
static std::map<std::string, std::pair<mg_tiling, double>> g_tune;
static bool g_tune_loaded = false;

std::string tune_key(const Geometry& g)
{
    char buf[128];
    std::snprintf(buf, sizeof buf, "%s:%dx%dx%d:%s", g.es == 4 ? "fp32" : "fp64", g.lnx, g.lny, g.lnz,
                  g.flat ? "flat" : "3d");
    return buf;
}

// The tuning cache: MG_TUNE_CACHE if set, else tune_cache.json next to
// this library (measured decompositions shipped with the package).
static std::string tune_path()
{
    const char* env = std::getenv("MG_TUNE_CACHE");
    if (env) return env;
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&tune_path), &info) && info.dli_fname) {
        std::string p = info.dli_fname;
        const size_t slash = p.rfind('/');
        return (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/tune_cache.json";
    }
    return "";
}

static void tune_load_file()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const std::string spath = tune_path();
    if (spath.empty()) return;
    const char* path = spath.c_str();
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    std::string s;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, k);
    std::fclose(f);
    // entries: "key": [ty, nchunk, nbuf, path, ms]
    size_t pos = 0;
    while ((pos = s.find('"', pos)) != std::string::npos) {
        size_t end = s.find('"', pos + 1);
        if (end == std::string::npos) break;
        std::string key = s.substr(pos + 1, end - pos - 1);
        size_t lb = s.find('[', end);
        if (lb == std::string::npos) break;
        mg_tiling t;
        double ms = 0;
        if (std::sscanf(s.c_str() + lb, "[%d, %d, %d, %d, %lf]", &t.ty, &t.nchunk, &t.nbuf, &t.path, &ms) == 5)
            g_tune[key] = {t, ms};
        pos = s.find(']', lb);
        if (pos == std::string::npos) break;
    }
}

bool tune_lookup(const std::string& key, mg_tiling* t)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    tune_load_file();
    auto it = g_tune.find(key);
    if (it == g_tune.end()) return false;
    *t = it->second.first;
    return true;
}

void tune_store(const std::string& key, const mg_tiling& t, double ms)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    tune_load_file();
    g_tune[key] = {t, ms};
    const char* path = std::getenv("MG_TUNE_CACHE");  // written only where the caller asks
    if (!path) return;
    FILE* f = std::fopen(path, "w");
    if (!f) return;
    std::fprintf(f, "{\n");
    size_t i = 0;
    for (auto& kv : g_tune) {
        std::fprintf(f, "  \"%s\": [%d, %d, %d, %d, %.6f]%s\n", kv.first.c_str(), kv.second.first.ty,
                     kv.second.first.nchunk, kv.second.first.nbuf, kv.second.first.path, kv.second.second,
                     ++i < g_tune.size() ? "," : "");
    }
    std::fprintf(f, "}\n");
    std::fclose(f);
}

// ------------------------------------------------------------------ Job
size_t Job::device_bytes() const
{
    return 2 * g.n * g.es + 4 * sizeof(CUtensorMap) + (size_t)std::max(plan.nitems, 1) * sizeof(long long) +
           (d_fh ? 2 * g.n * sizeof(double) + sizeof(FhDev) : 0);
}

static void fill_jobdev(const Job& j, JobDev* jd)
{
    std::memset(jd, 0, sizeof *jd);
    const Geometry& g = j.g;
    jd->buf[0] = j.buf[0];
    jd->buf[1] = j.buf[1];
    jd->tmap = j.d_tmap;
    jd->partial = j.d_partial;
    jd->fh = j.d_fh;
    jd->nx = g.lnx;
    jd->ny = g.lny;
    jd->nz = g.lnz;
    jd->ty = j.tiling.ty;
    jd->ntile = std::max(j.plan.ntile, 1);
    jd->nchunk = j.tiling.nchunk;
    jd->bw = std::min(g.lnx, 256);
    int flags = 0;
    if (g.perx) flags |= JF_PER_X;
    if (g.pery) flags |= JF_PER_Y;
    if (g.perz) flags |= JF_PER_Z;
    if (g.flat) flags |= JF_FLAT;
    if (j.p.mass_correct && g.es == 4) flags |= JF_MASS;
    jd->mass_every = std::max(j.p.mass_correct, 1);
    if (geometry_simple(g)) flags |= JF_SIMPLE;
    const double sp[3] = {g.lsx, g.lsy, g.lsz};
    double coef[3];
    for (int a = 0; a < 3; ++a) {
        const double d2 = sp[a] * sp[a];
        int e;
        const bool pow2 = std::frexp(d2, &e) == 0.5;
        if (g.es == 8 && !pow2) {
            coef[a] = d2;  // divide, as the reference does
            flags |= (JF_DIV_X << a);
        } else {
            coef[a] = 1.0 / d2;  // exact for powers of two
        }
    }
    jd->cx = coef[0];
    jd->cy = coef[1];
    jd->cz = coef[2];
    jd->flags = flags;
    jd->kap = j.p.kappa;
    jd->dtM = j.p.dt * j.p.M;
    jd->dtM_dt = j.p.dt;
    jd->noise = j.noise_negate ? -j.p.noise : j.p.noise;
    jd->noise_cutoff = j.noise_cutoff;
    jd->noise_seed = j.p.noise_seed;
    jd->inv_nsites = 1.0 / (double)g.n;
    jd->target = j.target < 0 ? LLONG_MAX : j.target;
}

// ------------------------------------------------------------------ Engine
Engine::~Engine()
{
    if (stream) cudaStreamSynchronize(stream);
    for (Job* j : jobs) {
        cudaFree(j->buf[0]);
        cudaFree(j->buf[1]);
        cudaFree(j->d_tmap);
        cudaFree(j->d_partial);
        cudaFree(j->d_fh);
        cudaFree(j->d_mu);
        cudaFree(j->d_mob);
        delete j;
    }
    jobs.clear();
    drop_graphs();
    free_groups();
    cudaFree(d_jobs_);
    cudaFree(d_err_);
    cudaFree(d_stage_);
    cudaFree(d_diag_part_);
    cudaFree(d_diag_max_);
    cudaFree(d_diag_bad_);
    cudaFree(d_diag_);
    cudaFreeHost(h_diag_);
    cudaFreeHost(h_state_);
    if (admit_) cudaStreamSynchronize(admit_);
    cudaFree(d_stage_adm_);
    cudaFree(d_part_adm_);
    free_graveyard();
    for (cudaStream_t st : aux_) cudaStreamDestroy(st);
    if (side) cudaStreamDestroy(side);
    if (admit_) cudaStreamDestroy(admit_);
    for (cudaEvent_t ev : aux_ev_) cudaEventDestroy(ev);
    if (fork_ev_) cudaEventDestroy(fork_ev_);
    if (stream) cudaStreamDestroy(stream);
}

int Engine::init(int dev, int capacity)
{
    device = dev;
    MG_TRY(device_info(dev, &info));
    MG_CUDA(cudaSetDevice(dev));
    MG_TRY(prepare_kernels(info));
    MG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    capacity_ = capacity;
    MG_CUDA(cudaMalloc(&d_jobs_, sizeof(JobDev) * capacity));
    MG_CUDA(cudaMemsetAsync(d_jobs_, 0, sizeof(JobDev) * capacity, stream));
    MG_CUDA(cudaMalloc(&d_err_, sizeof(int)));
    MG_CUDA(cudaMemsetAsync(d_err_, 0, sizeof(int), stream));
    MG_CUDA(cudaMalloc(&d_diag_part_, sizeof(double2) * 3 * kDiagBlocks));
    MG_CUDA(cudaMalloc(&d_diag_max_, sizeof(double) * kDiagBlocks));
    MG_CUDA(cudaMalloc(&d_diag_bad_, sizeof(double) * kDiagBlocks));
    MG_CUDA(cudaMalloc(&d_diag_, sizeof(Diag)));
    MG_CUDA(cudaHostAlloc(&h_diag_, sizeof(Diag), cudaHostAllocDefault));
    MG_CUDA(cudaHostAlloc(&h_state_, sizeof(JobDev), cudaHostAllocDefault));
    for (int s = capacity - 1; s >= 0; --s) free_slots_.push_back(s);
    return MG_OK;
}

int Engine::add_job(const mg_ch_params& p, long long target, Job** out, const FhDev* fh, bool noise_negate)
{
    std::unique_ptr<Job> j(new Job);
    j->p = p;
    j->noise_negate = noise_negate;
    if (fh && fh->model == kFhSips) j->noise_cutoff = fh->phiCutoff;
    MG_TRY(make_geometry(p, &j->g));
    if (free_slots_.empty() && !released_slots_.empty() && !admitting_) {
        // no launch in flight once the stream is idle: released slots are free
        MG_CUDA(cudaStreamSynchronize(stream));
        free_slots_.insert(free_slots_.end(), released_slots_.begin(), released_slots_.end());
        released_slots_.clear();
    }
    if (free_slots_.empty()) return fail(MG_ENOMEM, "no free job slot (capacity %d)", capacity_);
    const cudaStream_t wst = work_stream();
    if (fh && (p.precision != MG_FP64 || p.mass_correct))
        return fail(MG_EINVAL, "the variable-mobility model runs in FP64 without mass feedback");
    MG_CUDA(cudaSetDevice(device));
    if (fh) {
        // the fused variable-mobility kernel where the shape allows, else the
        // per-site path (path 1)
        // the two-pass kernels (path 1) by default: the step is bound by
        // FP64 arithmetic, where their occupancy beats the fused kernel's
        // (path 0, fh_march_kernel, chosen with mg_ch_set_tiling)
        j->tiling = mg_tiling{1, 1, 4, 1};
        MG_TRY(plan_fh_tiling(j->g, j->tiling, info, &j->plan));
    } else {
        j->tiling = batch_tiling ? batch_tiling_for(j->g, info, device, batch_threads, batch_planes)
                                 : default_tiling(j->g, info, device);
        MG_TRY(plan_tiling(j->g, j->tiling, info, &j->plan));
    }
    if (j->p.mass_correct && !j->plan.tma_ok)
        return fail(MG_EINVAL, "mass_correct needs a shape the tiled kernel takes (nx multiple of %d)", 32);
    j->target = target;
    const size_t bytes = j->g.n * j->g.es;
    cudaError_t e = cudaMalloc(&j->buf[0], bytes);
    if (e == cudaSuccess) e = cudaMalloc(&j->buf[1], bytes);
    if (e == cudaSuccess) e = cudaMalloc(&j->d_tmap, 4 * sizeof(CUtensorMap));
    if (e == cudaSuccess) e = cudaMalloc(&j->d_partial, sizeof(long long) * std::max(j->plan.nitems, 1));
    if (fh) {
        if (e == cudaSuccess) e = cudaMalloc(&j->d_fh, sizeof(FhDev));
        if (e == cudaSuccess) e = cudaMalloc(&j->d_mu, j->g.n * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&j->d_mob, j->g.n * sizeof(double));
        if (e == cudaSuccess) {
            FhDev f = *fh;
            f.mu = j->d_mu;
            f.mob = j->d_mob;
            e = cudaMemcpyAsync(j->d_fh, &f, sizeof f, cudaMemcpyHostToDevice, wst);
        }
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(j->buf[0]);
        cudaFree(j->buf[1]);
        cudaFree(j->d_tmap);
        cudaFree(j->d_partial);
        cudaFree(j->d_fh);
        cudaFree(j->d_mu);
        cudaFree(j->d_mob);
        return fail(e == cudaErrorMemoryAllocation ? MG_ENOMEM : MG_ECUDA, "allocating %zu bytes: %s", 2 * bytes,
                    cudaGetErrorString(e));
    }
    if (j->plan.tma_ok) {
        CUtensorMap maps[4];
        int rc = encode_maps(*j, maps);
        if (rc == MG_OK) {
            cudaError_t ce = cudaMemcpyAsync(j->d_tmap, maps, sizeof maps, cudaMemcpyHostToDevice, wst);
            if (ce != cudaSuccess) rc = fail(MG_ECUDA, "copying tensor maps: %s", cudaGetErrorString(ce));
        }
        if (rc != MG_OK) {
            cudaFree(j->buf[0]);
            cudaFree(j->buf[1]);
            cudaFree(j->d_tmap);
            cudaFree(j->d_partial);
            cudaFree(j->d_fh);
            cudaFree(j->d_mu);
            cudaFree(j->d_mob);
            return rc;
        }
    }
    j->slot = free_slots_.back();
    free_slots_.pop_back();
    JobDev jd;
    fill_jobdev(*j, &jd);
    MG_CUDA(cudaMemcpyAsync(d_jobs_ + j->slot, &jd, sizeof jd, cudaMemcpyHostToDevice, wst));
    jobs.push_back(j.get());
    dirty_ = true;
    *out = j.release();
    return MG_OK;
}

void Engine::remove_job(Job* j)
{
    auto it = std::find(jobs.begin(), jobs.end(), j);
    if (it == jobs.end()) return;
    jobs.erase(it);
    // freed at the next rebuild (which waits for the stream anyway) or at
    // destruction: cudaFree waits for the whole device, once per call
    graveyard_.insert(graveyard_.end(), {j->buf[0], j->buf[1], (void*)j->d_tmap, (void*)j->d_partial, (void*)j->d_fh,
                                         (void*)j->d_mu, (void*)j->d_mob});
    // a launch in flight may still name the slot (its items skip a finished
    // job): free again after the next rebuild, which waits for the stream
    released_slots_.push_back(j->slot);
    delete j;
    dirty_ = true;
}

int Engine::begin_admission()
{
    MG_CUDA(cudaSetDevice(device));
    if (!admit_) MG_CUDA(cudaStreamCreateWithFlags(&admit_, cudaStreamNonBlocking));
    if (!d_part_adm_) MG_CUDA(cudaMalloc(&d_part_adm_, sizeof(long long) * kDiagBlocks));
    admitting_ = true;
    return MG_OK;
}

int Engine::end_admission()
{
    admitting_ = false;
    if (admit_) MG_CUDA(cudaStreamSynchronize(admit_));
    return MG_OK;
}

int Engine::set_tiling(Job* j, const mg_tiling& t)
{
    TilePlan pl;
    mg_tiling t_in = t;
    // variable mobility: path 0 with ty 0 asks for the fused kernel's own tiling
    if (j->d_fh && t.path == 0 && t.ty == 0) t_in = fh_default_tiling(j->g, info);
    const mg_tiling& tt = t_in;
    if (j->d_fh) MG_TRY(plan_fh_tiling(j->g, tt, info, &pl));
    else MG_TRY(plan_tiling(j->g, tt, info, &pl));
    if (j->p.mass_correct && !pl.tma_ok) return fail(MG_EINVAL, "mass_correct needs the tiled kernel");
    MG_CUDA(cudaStreamSynchronize(stream));
    long long* part = nullptr;
    MG_CUDA(cudaMalloc(&part, sizeof(long long) * std::max(pl.nitems, 1)));
    const mg_tiling old = j->tiling;
    const TilePlan old_plan = j->plan;
    j->tiling = tt;
    j->plan = pl;
    if (pl.tma_ok) {
        // new maps at a new address: a launch never sees a map rewritten in place
        CUtensorMap maps[4];
        CUtensorMap* d_new = nullptr;
        int rc = encode_maps(*j, maps);
        if (rc == MG_OK) {
            cudaError_t e = cudaMalloc(&d_new, sizeof maps);
            if (e == cudaSuccess) e = cudaMemcpyAsync(d_new, maps, sizeof maps, cudaMemcpyHostToDevice, stream);
            if (e != cudaSuccess) rc = fail(MG_ECUDA, "tensor maps: %s", cudaGetErrorString(e));
        }
        if (rc != MG_OK) {
            j->tiling = old;
            j->plan = old_plan;
            cudaFree(d_new);
            cudaFree(part);
            return rc;
        }
        cudaFree(j->d_tmap);
        j->d_tmap = d_new;
    }
    cudaFree(j->d_partial);
    j->d_partial = part;
    // rewrite the static part of the slot, keep the mutable state
    MG_TRY(read_state(j, h_state_));
    JobDev jd;
    fill_jobdev(*j, &jd);
    jd.nudge_begin = h_state_->nudge_begin;
    jd.nudge_count = h_state_->nudge_count;
    jd.mass_target = h_state_->mass_target;
    jd.mass_last = h_state_->mass_last;
    jd.step = h_state_->step;
    jd.target = h_state_->target;
    jd.err = h_state_->err;
    MG_CUDA(cudaMemcpyAsync(d_jobs_ + j->slot, &jd, sizeof jd, cudaMemcpyHostToDevice, stream));
    dirty_ = true;
    return MG_OK;
}

void Engine::free_groups()
{
    for (Group& g : groups_) {
        cudaFree(g.d_item_begin);
        cudaFree(g.d_slot);
        cudaFree(g.d_counts);
    }
    groups_.clear();
}

void Engine::drop_graphs()
{
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
}

void Engine::free_graveyard()
{
    for (void* p : graveyard_) cudaFree(p);
    graveyard_.clear();
}

StepKernel Engine::group_kernel(const Group& g) const
{
    if (g.fhm) return g.flat ? fh_march_kernel<3, true> : fh_march_kernel<3, false>;
    if (g.simple && !g.flat && g.fixed_nx > 0 && g.fixed_ty > 0 && march_enabled()) {
        // every job of the group has the same width and tile height: the
        // variant with both fixed at compile time, where one exists
        StepKernel k = g.fp32 ? march_kernel_f32(g.fixed_nx, g.nbuf, g.mass, g.fixed_ty)
                              : march_kernel_f64(g.fixed_nx, g.nbuf, g.fixed_ty);
        if (k) return k;
    }
    return step_kernel(g.fp32, g.flat, g.nbuf, g.simple, g.block, g.mass, g.fixed_nx);
}

// The job list, item offsets and (stable lanes) counts of a group, written
// to its device tables.  Every host-to-device write of engine metadata (job
// slots, launch tables, tensor maps) is ordered on the engine's stream: a
// synchronous cudaMemcpy from pageable memory may return before its DMA has
// landed, and the engine's non-blocking stream is not ordered after the
// legacy stream, so the next kernel could read the old contents (a recycled
// slot's buffers, a tensor map not yet written).
int Engine::write_tables(const Group& g)
{
    std::vector<int> begin, slot;
    int items = 0;
    for (Job* j : g.jobs) {
        begin.push_back(items);
        slot.push_back(j->slot);
        items += j->plan.nitems;
    }
    begin.push_back(items);
    if ((int)slot.size() > g.table_cap) return fail(MG_EINVAL, "launch table holds %d jobs, not %zu", g.table_cap, slot.size());
    MG_CUDA(cudaMemcpyAsync(g.d_item_begin, begin.data(), sizeof(int) * begin.size(), cudaMemcpyHostToDevice, stream));
    if (!slot.empty())
        MG_CUDA(cudaMemcpyAsync(g.d_slot, slot.data(), sizeof(int) * slot.size(), cudaMemcpyHostToDevice, stream));
    if (g.d_counts) {
        const int counts[2] = {(int)g.jobs.size(), items};
        MG_CUDA(cudaMemcpyAsync(g.d_counts, counts, sizeof counts, cudaMemcpyHostToDevice, stream));
    }
    return MG_OK;
}

// Maps the new groups onto the current stable lanes: every new group needs a
// lane of the same kernel whose block and planes hold its tiles; lanes left
// without a group run empty (their CTAs find no item).  Lanes that bake a
// job into the graph (per-site jobs, noise launches) rule the refresh out.
bool Engine::refresh_tables(std::vector<Group>& ng)
{
    if (groups_.empty()) return false;
    auto bakes_jobs = [](const Group& g) {
        if (g.generic) return true;
        for (Job* j : g.jobs)
            if (j->p.noise > 0 && !g.fhm) return true;
        return false;
    };
    for (const Group& l : groups_)
        if (bakes_jobs(l) || !l.d_counts) return false;
    std::vector<int> lane_of(ng.size(), -1);
    std::vector<bool> used(groups_.size(), false);
    for (size_t i = 0; i < ng.size(); ++i) {
        const Group& g = ng[i];
        if (bakes_jobs(g)) return false;
        for (size_t l = 0; l < groups_.size(); ++l) {
            const Group& L = groups_[l];
            if (used[l] || L.key != g.key || L.sub != g.sub || group_kernel(L) != group_kernel(g)) continue;
            if (g.block > L.block || g.cplane > L.cplane || g.mplane > L.mplane) return false;
            // more items than CTAs, while the lane could keep more resident
            if (g.nitems > L.grid && L.grid < L.grid_max) return false;
            lane_of[i] = (int)l;
            used[l] = true;
            break;
        }
        if (lane_of[i] < 0) return false;
    }
    for (size_t l = 0; l < groups_.size(); ++l) {
        groups_[l].jobs.clear();
        groups_[l].nitems = 0;
    }
    for (size_t i = 0; i < ng.size(); ++i) {
        Group& L = groups_[lane_of[i]];
        L.jobs = ng[i].jobs;
        L.nitems = ng[i].nitems;
    }
    for (const Group& L : groups_)
        if (write_tables(L) != MG_OK) {
            clear_error();
            return false;
        }
    return true;
}

int Engine::rebuild()
{
    MG_CUDA(cudaStreamSynchronize(stream));
    if (admit_) MG_CUDA(cudaStreamSynchronize(admit_));
    free_graveyard();
    free_slots_.insert(free_slots_.end(), released_slots_.begin(), released_slots_.end());
    released_slots_.clear();
    // Several jobs: one ring depth per class (3 planes for 3-D jobs of a
    // march width, 4 for other 3-D jobs, 8 for 2-D) so that each class steps
    // in one launch.  Only nbuf changes; the tile rows and z chunks, which
    // fix a job's reduction order and so its results, stay as chosen.
    const bool shared = jobs.size() > 1 || stable_lanes;  // launches shared by several jobs
    if (shared)
        for (Job* j : jobs) {
            if (!j->plan.tma_ok || j->d_fh) continue;
            const int nb = j->g.flat ? 8 : (march_batch_job(j->g) ? kMarchBatchNbuf : 4);
            if (j->tiling.nbuf == nb) continue;
            mg_tiling t = j->tiling;
            t.nbuf = nb;
            TilePlan pl;
            if (plan_tiling(j->g, t, info, &pl) == MG_OK && pl.nitems == j->plan.nitems && pl.ntile == j->plan.ntile) {
                j->tiling = t;
                j->plan = pl;
            } else {
                clear_error();
            }
        }
    const size_t head = (sizeof(SmemHead) + 127) / 128 * 128 + 128;  // + alignment slack
    auto group_smem = [&](int nbuf, int cplane, int mplane, int es) {
        return head + (size_t)nbuf * cplane * es + (size_t)3 * mplane * es;
    };
    // one launch per (precision, flat, simple, mass, nbuf, row-width kernel)
    // class; a class whose planes together outgrow shared memory is split;
    // generic jobs run on their own
    std::vector<Group> ng;  // the new launch groups
    std::map<long long, std::vector<Group>> by_key;
    std::map<int, Group> fh_groups;  // fused variable-mobility jobs by flatness
    for (Job* j : jobs) {
        if (j->d_fh && j->plan.tma_ok) {
            Group& g = fh_groups[j->g.flat ? 1 : 0];
            g.key = -1 - (j->g.flat ? 1 : 0);
            g.fhm = true;
            g.flat = j->g.flat;
            g.nbuf = j->tiling.nbuf;
            g.jobs.push_back(j);
            continue;
        }
        if (!j->plan.tma_ok) {
            Group g;
            g.generic = true;
            g.fp32 = j->g.es == 4;
            g.jobs.push_back(j);
            ng.push_back(g);
            continue;
        }
        const bool simple = geometry_simple(j->g);
        const bool mass = j->p.mass_correct && j->g.es == 4;
        const int fixed = fixed_width_kernel(j->g, j->tiling.nbuf) ? j->g.lnx : 0;
        const long long key = (long long)((j->g.es == 4 ? 1 : 0) | (j->g.flat ? 2 : 0) | (simple ? 4 : 0) |
                                          (mass ? 8 : 0) | (j->tiling.nbuf << 4)) |
                              ((long long)fixed << 12);
        std::vector<Group>& gs = by_key[key];
        const int es = j->g.es;
        if (gs.empty() || group_smem(j->tiling.nbuf, std::max(gs.back().cplane, j->plan.cplane),
                                     std::max(gs.back().mplane, j->plan.mplane), es) > info.smem_optin)
            gs.emplace_back();
        Group& g = gs.back();
        g.key = key;
        g.sub = (int)gs.size() - 1;
        g.fp32 = j->g.es == 4;
        g.flat = j->g.flat;
        g.simple = simple;
        g.mass = mass;
        g.nbuf = j->tiling.nbuf;
        g.cplane = std::max(g.cplane, j->plan.cplane);
        g.mplane = std::max(g.mplane, j->plan.mplane);
        g.jobs.push_back(j);
    }
    for (auto& kv : by_key)
        for (Group& g : kv.second) {
            g.cplane = 0;
            g.mplane = 0;
            ng.push_back(g);
        }
    for (auto& kv : fh_groups) ng.push_back(kv.second);
    for (Group& g : ng) {
        if (g.generic) continue;
        int items = 0;
        for (Job* j : g.jobs) {
            items += j->plan.nitems;
            g.block = std::max(g.block, j->plan.block);
            g.cplane = std::max(g.cplane, j->plan.cplane);
            g.mplane = std::max(g.mplane, j->plan.mplane);
        }
        g.nitems = items;
        g.fixed_nx = g.jobs.front()->g.lnx;
        g.fixed_ty = g.jobs.front()->tiling.ty;
        for (Job* j : g.jobs) {
            if (j->g.lnx != g.fixed_nx) g.fixed_nx = 0;
            if (j->tiling.ty != g.fixed_ty) g.fixed_ty = 0;
        }
    }
    // a job-set change that fits the stable lanes: rewrite their tables,
    // keep the graphs
    if (stable_lanes && refresh_tables(ng)) {
        ++refreshes_;
        dirty_ = false;
        return MG_OK;
    }
    ++rebuilds_;
    drop_graphs();
    free_groups();
    groups_ = ng;
    for (Group& g : groups_) {
        if (g.generic) continue;
        if (stable_lanes) {
            // the largest tile this class has seen sizes the lane, so that
            // later jobs fit it without a new capture
            HighWater& h = hw_[{g.key, g.sub}];
            h.block = std::max(h.block, g.block);
            h.cplane = std::max(h.cplane, g.cplane);
            h.mplane = std::max(h.mplane, g.mplane);
            h.items = std::max(h.items, g.nitems);
            g.block = h.block;
            g.cplane = h.cplane;
            g.mplane = h.mplane;
        }
        g.smem = g.fhm ? fh_smem(g.nbuf, g.cplane, g.mplane) : group_smem(g.nbuf, g.cplane, g.mplane, g.fp32 ? 4 : 8);
        if (g.smem > info.smem_optin) return fail(MG_EINVAL, "batch group needs %zu bytes of shared memory", g.smem);
        int occ = 1;
        MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, group_kernel(g), g.block, g.smem));
        occ = std::max(occ, 1);
        // a stable lane keeps its grid whatever the item count: persistent
        // CTAs, as many as the most items the lane has held (up to what the
        // GPU keeps resident), so that a lane of a few small jobs does not
        // launch a full grid of CTAs that find no item every step; a job set
        // with more items than the grid rebuilds the lane (refresh_tables)
        g.grid_max = info.sms * occ;
        g.grid = stable_lanes ? std::min(g.grid_max, std::max(1, hw_[{g.key, g.sub}].items))
                              : std::min(g.nitems, g.grid_max);
        g.table_cap = stable_lanes ? std::max(capacity_, 1) : (int)g.jobs.size();
        MG_CUDA(cudaMalloc(&g.d_item_begin, sizeof(int) * (g.table_cap + 1)));
        MG_CUDA(cudaMalloc(&g.d_slot, sizeof(int) * g.table_cap));
        if (stable_lanes) MG_CUDA(cudaMalloc(&g.d_counts, sizeof(int) * 2));
        MG_TRY(write_tables(g));
    }
    // streams and events of the lanes (created here, never inside a capture)
    size_t lanes = 0;
    for (const Group& g : groups_) lanes += g.generic ? g.jobs.size() : 1;
    while (lanes > 1 && aux_.size() < lanes) {
        cudaStream_t st;
        cudaEvent_t ev;
        MG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaStreamDestroy(st);
            return fail(MG_ECUDA, "creating a lane event failed");
        }
        aux_.push_back(st);
        aux_ev_.push_back(ev);
    }
    if (lanes > 1 && !fork_ev_) MG_CUDA(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
    dirty_ = false;
    return MG_OK;
}

// Polls of a TMA completion barrier before the kernel gives up (reads the
// environment on every call so tests can shorten it).
static long long spin_limit()
{
    const char* e = std::getenv("MG_SPIN_LIMIT");
    const long long v = e ? std::atoll(e) : 0;
    return v > 0 ? v : (1LL << 22);
}

// Test hook for the bounded device waits: MG_FAULT_TX_EXTRA=<bytes> makes
// every plane's barrier expect more bytes than its copies deliver, so each
// wait runs out of polls and the kernel reports DEV_TMA_TIMEOUT.
static uint32_t fault_tx_extra()
{
    const char* e = std::getenv("MG_FAULT_TX_EXTRA");
    const long long v = e ? std::atoll(e) : 0;
    return v > 0 && v < 4096 ? (uint32_t)v : 0u;
}

// One step of one lane on stream `st`: a launch group, or one generic job.
int Engine::launch_lane(const Group& g, Job* generic_job, cudaStream_t st)
{
    if (g.generic) {
        Job* j = generic_job;
        const unsigned blocks = (unsigned)((j->g.n + 255) / 256);
        if (j->d_fh) {  // variable mobility: mu and 1/mob, then the update
            // pass 1's grid stride is a multiple of nx, so each thread keeps one x
            const long long l = std::lcm((long long)j->g.lnx, 256LL);
            long long q = std::max(1LL, 8LL * info.sms * 256 / l);
            q = std::min(q, std::max(1LL, (long long)((j->g.n + l - 1) / l)));
            fh_mu_mob_kernel<<<(unsigned)(l * q / 256), 256, 0, st>>>(d_jobs_ + j->slot);
            fh_update_kernel<<<(unsigned)((j->g.n / 4 + 256) / 256), 256, 0, st>>>(d_jobs_ + j->slot);
        } else if (g.fp32) {
            ch_step_generic_kernel<float><<<blocks, 256, 0, st>>>(d_jobs_ + j->slot);
        } else {
            ch_step_generic_kernel<double><<<blocks, 256, 0, st>>>(d_jobs_ + j->slot);
        }
        ch_step_generic_finish<<<1, 32, 0, st>>>(d_jobs_ + j->slot);
    } else {
        StepArgs a{};
        a.jobs = d_jobs_;
        a.job_slot = g.d_slot;
        a.item_begin = g.d_item_begin;
        a.njobs = (int)g.jobs.size();
        a.nitems = g.nitems;
        a.counts = g.d_counts;
        a.cplane = g.cplane;
        a.mplane = g.mplane;
        a.spin_limit = spin_limit();
        a.err = d_err_;
        a.tx_extra = fault_tx_extra();
        group_kernel(g)<<<g.grid, g.block, g.smem, st>>>(a);
    }
    // the noise term, per job that has one, after the step
    auto noise = [&](Job* j) {
        if (!(j->p.noise > 0)) return;
        const unsigned blocks = (unsigned)std::min<long long>((j->g.n / 4 + 256) / 256, 8LL * info.sms);
        if (g.fp32) ch_noise_kernel<float><<<blocks, 256, 0, st>>>(d_jobs_ + j->slot);
        else ch_noise_kernel<double><<<blocks, 256, 0, st>>>(d_jobs_ + j->slot);
    };
    // variable-mobility steps add their noise themselves (fh_update_kernel,
    // fh_march_kernel)
    if (g.generic) {
        if (!generic_job->d_fh) noise(generic_job);
    } else if (!g.fhm) {
        for (Job* j : g.jobs) noise(j);
    }
    MG_CUDA(cudaGetLastError());
    return MG_OK;
}

// k steps of every job.  Lanes (launch groups; generic jobs one by one) hold
// disjoint jobs, so with several lanes each runs its k steps on its own
// stream, forked from and joined back into `stream`: small classes fill the
// GPU beside large ones instead of after them.
int Engine::launch_steps(int k)
{
    std::vector<std::pair<const Group*, Job*>> lanes;
    for (const Group& g : groups_) {
        if (g.generic)
            for (Job* j : g.jobs) lanes.emplace_back(&g, j);
        else
            lanes.emplace_back(&g, nullptr);
    }
    if (lanes.size() <= 1) {
        for (int i = 0; i < k; ++i)
            for (auto& l : lanes) MG_TRY(launch_lane(*l.first, l.second, stream));
        return MG_OK;
    }
    if (aux_.size() < lanes.size() || !fork_ev_) return fail(MG_ECUDA, "lane streams missing (engine not rebuilt)");
    MG_CUDA(cudaEventRecord(fork_ev_, stream));
    for (size_t i = 0; i < lanes.size(); ++i) {
        MG_CUDA(cudaStreamWaitEvent(aux_[i], fork_ev_, 0));
        for (int s = 0; s < k; ++s) MG_TRY(launch_lane(*lanes[i].first, lanes[i].second, aux_[i]));
        MG_CUDA(cudaEventRecord(aux_ev_[i], aux_[i]));
        MG_CUDA(cudaStreamWaitEvent(stream, aux_ev_[i], 0));
    }
    return MG_OK;
}

int Engine::graph_for(int k, cudaGraphExec_t* out)
{
    auto it = graphs_.find(k);
    if (it != graphs_.end()) {
        *out = it->second;
        return MG_OK;
    }
    cudaGraph_t graph;
    MG_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int rc = MG_OK;
    rc = launch_steps(k);
    cudaError_t e = cudaStreamEndCapture(stream, &graph);
    if (rc != MG_OK) {
        if (e == cudaSuccess) cudaGraphDestroy(graph);
        return rc;
    }
    MG_CUDA(e);
    cudaGraphExec_t exec;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    MG_CUDA(e);
    graphs_[k] = exec;
    *out = exec;
    return MG_OK;
}

static int graph_steps()
{
    static int v = [] {
        const char* e = std::getenv("MG_GRAPH_STEPS");
        return e ? std::max(0, std::atoi(e)) : 50;
    }();
    return v;
}

int Engine::enqueue_steps(int nsteps)
{
    if (nsteps < 0) return fail(MG_EINVAL, "nsteps must be >= 0");
    if (poisoned_)
        return fail(MG_EDEVICE, "an earlier step reported a device error; this handle takes no further steps");
    MG_CUDA(cudaSetDevice(device));
    if (dirty_) MG_TRY(rebuild());
    if (jobs.empty()) return MG_OK;
    const int gk = graph_max_steps > 0 ? std::min(graph_max_steps, graph_steps()) : graph_steps();
    while (nsteps > 0) {
        if (gk >= 2 && nsteps >= 2) {
            const int k = std::min(nsteps, gk);
            cudaGraphExec_t ex;
            MG_TRY(graph_for(k, &ex));
            MG_CUDA(cudaGraphLaunch(ex, stream));
            nsteps -= k;
        } else {
            MG_TRY(launch_steps(1));
            nsteps -= 1;
        }
    }
    return MG_OK;
}

int Engine::sync(long long timeout_us)
{
    MG_CUDA(cudaSetDevice(device));
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(stream);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) MG_CUDA(e);
        if (timeout_us >= 0) {
            const auto us =
                std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
            if (us > timeout_us) return fail(MG_ETIMEOUT, "GPU work not finished after %lld us", timeout_us);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    int err = 0;
    MG_CUDA(cudaMemcpy(&err, d_err_, sizeof err, cudaMemcpyDeviceToHost));
    if (err != DEV_OK) {
        // a bounded wait ran out: copies may still have been in flight when
        // the CTA gave up, so the fields and the ring state are not trusted
        poisoned_ = true;
        return fail(MG_EDEVICE, "a step kernel reported device error %d (TMA wait ran out)", err);
    }
    return MG_OK;
}

int Engine::read_state(Job* j, JobDev* out)
{
    MG_CUDA(cudaSetDevice(device));
    return read_state_on(j, out, stream);
}

int Engine::read_state_on(Job* j, JobDev* out, cudaStream_t st)
{
    MG_CUDA(cudaMemcpyAsync(h_state_, d_jobs_ + j->slot, sizeof(JobDev), cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaStreamSynchronize(st));
    *out = *h_state_;
    return MG_OK;
}

int Engine::ensure_stage(size_t n)
{
    if (stage_n_ >= n) return MG_OK;
    cudaFree(d_stage_);
    d_stage_ = nullptr;
    stage_n_ = 0;
    cudaError_t e = cudaMalloc(&d_stage_, n * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(MG_ENOMEM, "staging buffer of %zu doubles: %s", n, cudaGetErrorString(e));
    }
    stage_n_ = n;
    return MG_OK;
}

int Engine::upload(Job* j, const double* host, long long target)
{
    if (!host) return fail(MG_EINVAL, "null field");
    MG_CUDA(cudaSetDevice(device));
    const cudaStream_t wst = work_stream();
    if (j->g.es == 8) {
        MG_CUDA(cudaMemcpyAsync(j->buf[0], host, j->g.n * 8, cudaMemcpyHostToDevice, wst));
    } else {
        double* stage;
        if (admitting_) {
            // the admission's own staging: the engine's is in use by the
            // downloads of finished jobs on the side stream
            if (stage_adm_n_ < j->g.n) {
                if (d_stage_adm_) graveyard_.push_back(d_stage_adm_);  // a copy may still read it
                d_stage_adm_ = nullptr;
                stage_adm_n_ = 0;
                MG_CUDA(cudaMalloc(&d_stage_adm_, j->g.n * sizeof(double)));
                stage_adm_n_ = j->g.n;
            }
            stage = d_stage_adm_;
        } else {
            MG_TRY(ensure_stage(j->g.n));
            stage = d_stage_;
        }
        MG_CUDA(cudaMemcpyAsync(stage, host, j->g.n * 8, cudaMemcpyHostToDevice, wst));
        ch_convert<double, float><<<4 * info.sms, 256, 0, wst>>>(stage, static_cast<float*>(j->buf[0]), j->g.n);
    }
    j->target = target;
    ch_job_reset<<<1, 32, 0, wst>>>(d_jobs_ + j->slot, target < 0 ? LLONG_MAX : target);
    if (j->g.es == 4) {
        // scratch for the block sums: d_diag_part_ (3 x kDiagBlocks double2),
        // or the admission's own
        long long* part = admitting_ ? d_part_adm_ : reinterpret_cast<long long*>(d_diag_part_);
        ch_mass_partial<<<kDiagBlocks, kDiagThreads, 0, wst>>>(d_jobs_ + j->slot, part);
        ch_mass_final<<<1, 32, 0, wst>>>(part, kDiagBlocks, d_jobs_ + j->slot);
    }
    MG_CUDA(cudaGetLastError());
    return MG_OK;
}

int Engine::to_double(Job* j, double* d_dst)
{
    MG_TRY(read_state(j, h_state_));
    const void* cur = j->buf[h_state_->step & 1];
    if (j->g.es == 8) {
        MG_CUDA(cudaMemcpyAsync(d_dst, cur, j->g.n * 8, cudaMemcpyDeviceToDevice, stream));
    } else {
        ch_convert<float, double><<<4 * info.sms, 256, 0, stream>>>(static_cast<const float*>(cur), d_dst, j->g.n);
        MG_CUDA(cudaGetLastError());
    }
    return MG_OK;
}

int Engine::download(Job* j, double* host)
{
    if (!host) return fail(MG_EINVAL, "null field");
    MG_TRY(sync(-1));
    return download_on(j, host, stream);
}

int Engine::ensure_side()
{
    if (!side) MG_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    return MG_OK;
}

int Engine::download_finished(Job* j, double* host)
{
    if (!host) return fail(MG_EINVAL, "null field");
    MG_CUDA(cudaSetDevice(device));
    MG_TRY(ensure_side());
    return download_on(j, host, side);
}

// copies the job's current field to the host through stream `st` and waits
// for that stream only
int Engine::download_on(Job* j, double* host, cudaStream_t st)
{
    MG_TRY(read_state_on(j, h_state_, st));
    const void* cur = j->buf[h_state_->step & 1];
    if (j->g.es == 8) {
        MG_CUDA(cudaMemcpyAsync(host, cur, j->g.n * 8, cudaMemcpyDeviceToHost, st));
    } else {
        MG_TRY(ensure_stage(j->g.n));
        ch_convert<float, double><<<4 * info.sms, 256, 0, st>>>(static_cast<const float*>(cur), d_stage_, j->g.n);
        MG_CUDA(cudaMemcpyAsync(host, d_stage_, j->g.n * 8, cudaMemcpyDeviceToHost, st));
    }
    MG_CUDA(cudaStreamSynchronize(st));
    return MG_OK;
}

int Engine::mobility(Job* j, double* host)
{
    if (!host) return fail(MG_EINVAL, "null field");
    if (!j->d_fh) return fail(MG_EINVAL, "not a variable-mobility job");
    MG_TRY(sync(-1));
    // recomputed from the input of the last step, which the other ping-pong
    // buffer still holds (the fused kernel keeps the mobility on chip)
    fh_mobility_kernel<<<4 * info.sms, 256, 0, stream>>>(d_jobs_ + j->slot, j->d_mob);
    MG_CUDA(cudaGetLastError());
    MG_CUDA(cudaMemcpyAsync(host, j->d_mob, j->g.n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    MG_CUDA(cudaStreamSynchronize(stream));
    return MG_OK;
}

int Engine::diagnostics(Job* j, mg_ch_stats* out)
{
    if (!out) return fail(MG_EINVAL, "null stats");
    MG_TRY(sync(-1));
    return diagnostics_on(j, out, stream);
}

int Engine::diagnostics_finished(Job* j, mg_ch_stats* out)
{
    if (!out) return fail(MG_EINVAL, "null stats");
    MG_CUDA(cudaSetDevice(device));
    MG_TRY(ensure_side());
    return diagnostics_on(j, out, side);
}

int Engine::diagnostics_on(Job* j, mg_ch_stats* out, cudaStream_t st)
{
    const Geometry& g = j->g;
    if (g.es == 8)
        ch_diag_partial<double><<<kDiagBlocks, kDiagThreads, 0, st>>>(d_jobs_ + j->slot, g.lsx, g.lsy, g.lsz,
                                                                       d_diag_part_, d_diag_max_, d_diag_bad_);
    else
        ch_diag_partial<float><<<kDiagBlocks, kDiagThreads, 0, st>>>(d_jobs_ + j->slot, g.lsx, g.lsy, g.lsz,
                                                                      d_diag_part_, d_diag_max_, d_diag_bad_);
    ch_diag_final<<<1, 256, 0, st>>>(d_diag_part_, d_diag_max_, d_diag_bad_, kDiagBlocks, g.lsx * g.lsy * g.lsz,
                                     d_diag_);
    MG_CUDA(cudaGetLastError());
    MG_CUDA(cudaMemcpyAsync(h_diag_, d_diag_, sizeof(Diag), cudaMemcpyDeviceToHost, st));
    MG_TRY(read_state_on(j, h_state_, st));  // syncs the stream
    out->mass = h_diag_->mass;
    out->energy = h_diag_->energy;
    out->abs_mass = h_diag_->abs_mass;
    out->max_abs = h_diag_->max_abs;
    out->nonfinite = (long long)h_diag_->nonfinite;
    out->step = h_state_->step;
    if (out->nonfinite > 0) return fail(MG_ENONFINITE, "%lld sites are NaN or Inf", out->nonfinite);
    return MG_OK;
}

int Engine::nitems_total() const
{
    int s = 0;
    for (const Group& g : groups_) s += g.generic ? (int)g.jobs.size() : g.nitems;
    return s;
}
int Engine::nctas_total() const
{
    int s = 0;
    for (const Group& g : groups_) s += g.generic ? 0 : g.grid;
    return s;
}
int Engine::nlaunch_per_step() const
{
    int s = 0;
    for (const Group& g : groups_) s += g.generic ? 2 * (int)g.jobs.size() : 1;
    return s;
}

// ------------------------------------------------------ structure factor
// Bins |F|^2/N of the half spectrum with Hermitian weights; k = 0 excluded.
__global__ void sf_bin_kernel(const cufftDoubleComplex* __restrict__ F, int nx, int ny, int nz, double rx,
                              double ry, double rz, double dk, int nbins, double inv_n, double* __restrict__ acc)
{
    // |k| / dk = sqrt(sum (m_d * L_max / L_d)^2): exact integers on equal
    // box lengths, so a mode on a bin edge lands in the same bin as in the
    // host restatement
    const int hx = nx / 2 + 1;
    const size_t total = (size_t)hx * ny * nz;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i % hx);
        const int iy = (int)((i / hx) % ny);
        const int iz = (int)(i / ((size_t)hx * ny));
        const int fy = iy <= ny / 2 ? iy : iy - ny;
        const int fz = iz <= nz / 2 ? iz : iz - nz;
        const double qx = ix * rx, qy = fy * ry, qz = fz * rz;
        const double q = sqrt(qx * qx + qy * qy + qz * qz);
        if (q <= 0.0) continue;
        const int b = (int)floor(q + 1e-9);
        if (b >= nbins) continue;
        const double kk = q * dk;
        const double w = (ix == 0 || (nx % 2 == 0 && ix == nx / 2)) ? 1.0 : 2.0;
        const double s = (F[i].x * F[i].x + F[i].y * F[i].y) * inv_n;
        atomicAdd(acc + 4 * b + 0, w);
        atomicAdd(acc + 4 * b + 1, w * kk);
        atomicAdd(acc + 4 * b + 2, w * s);
        atomicAdd(acc + 4 * b + 3, w * kk * s);
    }
}

int Engine::structure_factor(Job* j, int nbins, double* k, double* S, double* k1)
{
    if (nbins < 1 || !k || !S || !k1) return fail(MG_EINVAL, "structure_factor: bad arguments");
    MG_TRY(sync(-1));
    const mg_ch_params& p = j->p;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const size_t n = j->g.n;
    const size_t nc = (size_t)(nx / 2 + 1) * ny * nz;
    MG_TRY(ensure_stage(n));
    MG_TRY(to_double(j, d_stage_));
    cufftDoubleComplex* F = nullptr;
    double* acc = nullptr;
    MG_CUDA(cudaMalloc(&F, nc * sizeof(cufftDoubleComplex)));
    cudaError_t e = cudaMalloc(&acc, 4 * nbins * sizeof(double));
    if (e != cudaSuccess) {
        cudaFree(F);
        MG_CUDA(e);
    }
    cufftHandle plan;
    cufftResult fr;
    if (nz > 1) fr = cufftPlan3d(&plan, nz, ny, nx, CUFFT_D2Z);
    else if (ny > 1) fr = cufftPlan2d(&plan, ny, nx, CUFFT_D2Z);
    else fr = cufftPlan1d(&plan, nx, CUFFT_D2Z, 1);
    const bool planned = fr == CUFFT_SUCCESS;
    int rc = MG_OK;
    if (!planned) rc = fail(MG_ECUDA, "cufftPlan failed (%d)", (int)fr);
    if (rc == MG_OK) {
        cufftSetStream(plan, stream);
        fr = cufftExecD2Z(plan, d_stage_, F);
        if (fr != CUFFT_SUCCESS) rc = fail(MG_ECUDA, "cufftExecD2Z failed (%d)", (int)fr);
    }
    std::vector<double> h(4 * nbins);
    if (rc == MG_OK) {
        const double L = std::max({nx * p.dx, ny * p.dy, nz * p.dz});
        const double dk = 6.283185307179586476925286766559 / L;
        cudaMemsetAsync(acc, 0, 4 * nbins * sizeof(double), stream);
        sf_bin_kernel<<<8 * info.sms, 256, 0, stream>>>(F, nx, ny, nz, L / (nx * p.dx), L / (ny * p.dy),
                                                        L / (nz * p.dz), dk, nbins, 1.0 / (double)n, acc);
        cudaError_t ce = cudaMemcpyAsync(h.data(), acc, 4 * nbins * sizeof(double), cudaMemcpyDeviceToHost, stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(stream);
        if (ce != cudaSuccess) rc = fail(MG_ECUDA, "structure factor: %s", cudaGetErrorString(ce));
        double num = 0, den = 0;
        for (int b = 0; b < nbins && rc == MG_OK; ++b) {
            const double cnt = h[4 * b], ks = h[4 * b + 1], ss = h[4 * b + 2], kss = h[4 * b + 3];
            k[b] = cnt > 0 ? ks / cnt : (b + 0.5) * dk;
            S[b] = cnt > 0 ? ss / cnt : 0.0;
            num += kss;
            den += ss;
        }
        *k1 = den > 0 ? num / den : 0.0;
    }
    if (planned) cufftDestroy(plan);
    cudaFree(F);
    cudaFree(acc);
    return rc;
}

}  // namespace mg
