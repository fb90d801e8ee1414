// Legacy-VTK output formatted on the GPU (mg_ch_write_vtk): the text that
// SfieldFD::writeVTKFile (SfieldFD.cpp:363-430) writes for one rank, byte for
// byte what the host writer's "%.3f\n" lines give, without formatting every
// value on the host (a 512^3 field is 134 M lines).
//
// "%.3f" rounds the exact binary value of a double to 3 decimals, ties to
// even.  The kernel forms |x| * 1000 as p + e exactly (p rounded, e from an
// FMA), so the rounding decision uses the exact product; the sign is the sign
// bit (so -0.0004 prints "-0.000"); NaN and infinities print "nan", "-nan",
// "inf", "-inf".  Values of magnitude >= 4e12 (|x|*1000 near 2^52) are refused
// with MG_EINVAL; mg_vtk_write formats any value on the host.
//
// The selected values (x at multiples of iskip, y and z from the first plane
// in steps of jskip / kskip) are formatted in chunks: a pass computes each
// line's length, an exclusive scan gives the offsets, a second pass writes
// the characters, and the chunk is copied to pinned memory and appended.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>

#include "engine.h"

namespace mg {

void vtk_header(FILE* f, const char* tag, int nx, int ny, int nz, int iskip, int jskip, int kskip);

namespace {

constexpr long long kVtkChunk = 1ll << 23;  // values formatted per pass
constexpr int kVtkMaxLine = 24;             // "-" + 13 digits + "." + 3 digits + "\n", with room
constexpr double kVtkMaxAbs = 4.0e12;       // |x| * 1000 < 2^52: p - floor(p) is exact

struct Sel {
    int nx, ny, sx, sy, iskip, jskip, kskip;
};

// array index of the t-th selected value (x fastest)
__device__ __forceinline__ long long sel_index(const Sel& s, long long t)
{
    const long long r = t / s.sx;
    const int xi = (int)(t - r * s.sx);
    const long long kk = r / s.sy;
    const int jj = (int)(r - kk * s.sy);
    const long long x = (long long)s.iskip * (xi + 1) - 1, y = (long long)jj * s.jskip, z = kk * s.kskip;
    return (z * s.ny + y) * s.nx + x;
}

enum : int { kNum = 0, kNan = 1, kInf = 2, kRange = 3 };

// n = |x| * 1000 rounded to an integer, ties to even, on the exact product
__device__ __forceinline__ int fmt3(double x, unsigned long long& n, bool& neg)
{
    neg = signbit(x);
    if (isnan(x)) return kNan;
    if (isinf(x)) return kInf;
    const double ax = fabs(x);
    if (ax >= kVtkMaxAbs) return kRange;
    const double p = ax * 1000.0;
    const double e = fma(ax, 1000.0, -p);  // p + e == ax * 1000 exactly
    const double fl = floor(p);
    const double d = (p - fl) - 0.5;      // exact (Sterbenz) where it can be 0
    bool up;
    if (d > 0.0) up = true;
    else if (d < 0.0) up = false;
    else up = e > 0.0 || (e == 0.0 && fmod(fl, 2.0) != 0.0);
    n = (unsigned long long)fl + (up ? 1ull : 0ull);
    return kNum;
}

__device__ __forceinline__ int ndigits(unsigned long long v)
{
    int d = 1;
    while (v >= 10) {
        v /= 10;
        ++d;
    }
    return d;
}

// length of the line of x ("%.3f\n"); 0 when x is out of range
__device__ __forceinline__ unsigned int line_len(double x)
{
    unsigned long long n;
    bool neg;
    const int k = fmt3(x, n, neg);
    if (k == kRange) return 0;
    if (k != kNum) return (neg ? 1u : 0u) + 4u;  // "nan\n", "inf\n"
    return (neg ? 1u : 0u) + (unsigned)ndigits(n / 1000) + 5u;
}

__global__ void vtk_len_kernel(const double* __restrict__ f, Sel s, long long t0, long long cnt,
                               unsigned int* __restrict__ len, int* bad)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += (long long)gridDim.x * blockDim.x) {
        const unsigned int l = line_len(f[sel_index(s, t0 + t)]);
        if (l == 0) atomicExch(bad, 1);
        len[t] = l;
    }
}

__global__ void vtk_text_kernel(const double* __restrict__ f, Sel s, long long t0, long long cnt,
                                const unsigned int* __restrict__ off, char* __restrict__ out)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += (long long)gridDim.x * blockDim.x) {
        char* o = out + off[t];
        unsigned long long n;
        bool neg;
        const int k = fmt3(f[sel_index(s, t0 + t)], n, neg);
        if (k == kRange) continue;
        if (neg) *o++ = '-';
        if (k == kNan || k == kInf) {
            o[0] = k == kNan ? 'n' : 'i';
            o[1] = k == kNan ? 'a' : 'n';
            o[2] = k == kNan ? 'n' : 'f';
            o[3] = '\n';
            continue;
        }
        unsigned long long ip = n / 1000;
        unsigned int fr = (unsigned int)(n - ip * 1000);
        const int nd = ndigits(ip);
        for (int i = nd - 1; i >= 0; --i) {
            o[i] = (char)('0' + ip % 10);
            ip /= 10;
        }
        o += nd;
        o[0] = '.';
        o[1] = (char)('0' + fr / 100);
        o[2] = (char)('0' + fr / 10 % 10);
        o[3] = (char)('0' + fr % 10);
        o[4] = '\n';
    }
}

// buffers of one write, released on every path
struct VtkBuffers {
    unsigned int* len = nullptr;
    unsigned int* off = nullptr;
    char* text = nullptr;
    int* bad = nullptr;
    void* scan_tmp = nullptr;
    char* host = nullptr;
    unsigned int* host_tail = nullptr;
    FILE* f = nullptr;
    ~VtkBuffers()
    {
        cudaFree(len);
        cudaFree(off);
        cudaFree(text);
        cudaFree(bad);
        cudaFree(scan_tmp);
        cudaFreeHost(host);
        cudaFreeHost(host_tail);
        if (f) std::fclose(f);
    }
};

}  // namespace

int Engine::write_vtk(Job* j, const char* path, const char* tag, int iskip, int jskip, int kskip)
{
    if (!path || !tag) return fail(MG_EINVAL, "null argument");
    if (iskip < 1 || jskip < 1 || kskip < 1) return fail(MG_EINVAL, "skip factors must be >= 1");
    MG_TRY(sync(-1));
    MG_CUDA(cudaSetDevice(device));
    MG_TRY(ensure_stage(j->g.n));
    MG_TRY(to_double(j, d_stage_));
    const int nx = j->p.nx, ny = j->p.ny, nz = j->p.nz;
    const Sel s{nx, ny, nx / iskip, (ny - 1) / jskip + 1, iskip, jskip, kskip};
    const long long total = (long long)s.sx * s.sy * ((nz - 1) / kskip + 1);

    VtkBuffers b;
    b.f = std::fopen(path, "ab");
    if (!b.f) return fail(MG_EINVAL, "cannot open %s for appending", path);
    vtk_header(b.f, tag, nx, ny, nz, iskip, jskip, kskip);
    if (total > 0) {
        const long long ch = std::min(total, kVtkChunk);
        size_t scan_bytes = 0;
        MG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, b.len, b.off, (int)ch, stream));
        MG_CUDA(cudaMalloc(&b.len, sizeof(unsigned int) * ch));
        MG_CUDA(cudaMalloc(&b.off, sizeof(unsigned int) * ch));
        MG_CUDA(cudaMalloc(&b.text, (size_t)kVtkMaxLine * ch));
        MG_CUDA(cudaMalloc(&b.bad, sizeof(int)));
        MG_CUDA(cudaMalloc(&b.scan_tmp, std::max<size_t>(scan_bytes, 16)));
        MG_CUDA(cudaMallocHost(&b.host, (size_t)kVtkMaxLine * ch));
        MG_CUDA(cudaMallocHost(&b.host_tail, 2 * sizeof(unsigned int)));
        const int grid = 4 * info.sms, block = 256;
        for (long long t0 = 0; t0 < total; t0 += ch) {
            const long long cnt = std::min(ch, total - t0);
            MG_CUDA(cudaMemsetAsync(b.bad, 0, sizeof(int), stream));
            vtk_len_kernel<<<grid, block, 0, stream>>>(d_stage_, s, t0, cnt, b.len, b.bad);
            MG_CUDA(cudaGetLastError());
            MG_CUDA(cub::DeviceScan::ExclusiveSum(b.scan_tmp, scan_bytes, b.len, b.off, (int)cnt, stream));
            MG_CUDA(cudaMemcpyAsync(b.host_tail, b.off + cnt - 1, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream));
            MG_CUDA(cudaMemcpyAsync(b.host_tail + 1, b.len + cnt - 1, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                    stream));
            int bad = 0;
            MG_CUDA(cudaMemcpyAsync(&bad, b.bad, sizeof(int), cudaMemcpyDeviceToHost, stream));
            MG_CUDA(cudaStreamSynchronize(stream));
            if (bad) return fail(MG_EINVAL, "a value of magnitude >= %g cannot be formatted on the device (use mg_vtk_write)",
                                 kVtkMaxAbs);
            const size_t bytes = (size_t)b.host_tail[0] + b.host_tail[1];
            vtk_text_kernel<<<grid, block, 0, stream>>>(d_stage_, s, t0, cnt, b.off, b.text);
            MG_CUDA(cudaGetLastError());
            MG_CUDA(cudaMemcpyAsync(b.host, b.text, bytes, cudaMemcpyDeviceToHost, stream));
            MG_CUDA(cudaStreamSynchronize(stream));
            if (std::fwrite(b.host, 1, bytes, b.f) != bytes) return fail(MG_EINVAL, "write error on %s", path);
        }
    }
    const bool ok = std::fflush(b.f) == 0 && std::ferror(b.f) == 0;
    if (!ok) return fail(MG_EINVAL, "write error on %s", path);
    return MG_OK;
}

}  // namespace mg
