// Host side of the reference's input/output surface: the seeded initial
// condition and the legacy-VTK writer.  Compiled with -ffp-contract=off so
// the initial condition rounds exactly as the reference build does.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "mesogpu.h"

namespace mg {
int fail(int code, const char* fmt, ...);
void clear_error();

// The header block of SfieldFD::writeVTKFile (SfieldFD.cpp:383-399) for a
// single rank; shared by the host and device writers.
void vtk_header(FILE* f, const char* tag, int nx, int ny, int nz, int iskip, int jskip, int kskip)
{
    const char* d = "   ";
    std::fprintf(f, "# vtk DataFile Version 3.1\n");
    std::fprintf(f, "VTK file containing grid data\n");
    std::fprintf(f, "ASCII\n");
    std::fprintf(f, " \n");
    std::fprintf(f, "DATASET STRUCTURED_POINTS\n");
    std::fprintf(f, "DIMENSIONS%s%d%s%d%s%d\n", d, nx / iskip, d, ny / jskip, d, nz / kskip);
    std::fprintf(f, "ORIGIN %s0%s0%s0\n", d, d, d);
    std::fprintf(f, "SPACING%s%g%s%g%s%g\n", d, 1.0 * iskip, d, 1.0 * jskip, d, 1.0 * kskip);
    std::fprintf(f, " \n");
    std::fprintf(f, "POINT_DATA %d\n", (nx / iskip) * (ny / jskip) * (nz / kskip));
    std::fprintf(f, "SCALARS %s float\n", tag);
    std::fprintf(f, "LOOKUP_TABLE default\n");
}
}  // namespace mg

namespace {

// MT19937 with the reference's seeding, tempering and conversions
// (rand.cpp:24-36 init, :38-55 twist, :58-78 next, :81-84 uniform,
// :87-94 normal).  The constants are the generator's published parameters.
class Mt19937 {
   public:
    explicit Mt19937(uint32_t seed)
    {
        mt_[0] = seed;
        for (uint32_t i = 1; i < 624; ++i) mt_[i] = 1812433253u * (mt_[i - 1] ^ (mt_[i - 1] >> 30)) + i;
        idx_ = 624;
    }
    uint32_t next()
    {
        if (idx_ >= 624) twist();
        uint32_t y = mt_[idx_++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9D2C5680u;
        y ^= (y << 15) & 0xEFC60000u;
        y ^= y >> 18;
        return y;
    }
    double uniform() { return (double)next() / (double)4294967295u; }
    double normal()
    {
        const double u1 = uniform();
        const double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.14159265359 * u2);
    }

   private:
    void twist()
    {
        for (uint32_t i = 0; i < 624; ++i) {
            const uint32_t x = (mt_[i] & 0x80000000u) + (mt_[(i + 1) % 624] & 0x7fffffffu);
            uint32_t xa = x >> 1;
            if (x & 1u) xa ^= 0x9908B0DFu;
            mt_[i] = mt_[(i + 397) % 624] ^ xa;
        }
        idx_ = 0;
    }
    uint32_t mt_[624];
    uint32_t idx_;
};

}  // namespace

extern "C" {

int mg_ic_generate(const int dims[3], double co, double amp, int gaussian, unsigned seed, double* out)
{
    mg::clear_error();
    if (!dims || !out) return mg::fail(MG_EINVAL, "null argument");
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) return mg::fail(MG_EINVAL, "dimensions must be >= 1");
    Mt19937 rng(seed);
    const size_t nx = (size_t)dims[0], ny = (size_t)dims[1], nz = (size_t)dims[2];
    for (size_t i = 0; i < nx; ++i)
        for (size_t j = 0; j < ny; ++j)
            for (size_t k = 0; k < nz; ++k)
                out[i + nx * (j + ny * k)] = gaussian ? co + amp * rng.normal() : co + amp * (rng.uniform() - 0.5);
    return MG_OK;
}

// One header + data block in the layout of SfieldFD::writeVTKFile
// (SfieldFD.cpp:363-430) for a single rank: values `%.3f`, x fastest; x
// kept where the 1-based index is a multiple of iskip (:412-413), y and z
// stepping by jskip / kskip from 1 (:407-408); appended like ios::app.
int mg_vtk_write(const char* path, const char* tag, const double* field, const int dims[3], int iskip, int jskip,
                 int kskip)
{
    mg::clear_error();
    if (!path || !tag || !field || !dims) return mg::fail(MG_EINVAL, "null argument");
    if (iskip < 1 || jskip < 1 || kskip < 1) return mg::fail(MG_EINVAL, "skip factors must be >= 1");
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    FILE* f = std::fopen(path, "ab");
    if (!f) return mg::fail(MG_EINVAL, "cannot open %s for appending", path);
    std::vector<char> iobuf(1 << 20);
    std::setvbuf(f, iobuf.data(), _IOFBF, iobuf.size());
    mg::vtk_header(f, tag, nx, ny, nz, iskip, jskip, kskip);
    char line[64];
    for (int k = 1; k < nz + 1; k += kskip)
        for (int j = 1; j < ny + 1; j += jskip) {
            const double* row = field + ((size_t)(k - 1) * ny + (j - 1)) * nx;
            for (int i = 1; i < nx + 1; ++i) {
                if (i % iskip != 0) continue;
                const int len = std::snprintf(line, sizeof line, "%.3f\n", row[i - 1]);
                std::fwrite(line, 1, (size_t)len, f);
            }
        }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    if (!ok) return mg::fail(MG_EINVAL, "write error on %s", path);
    return MG_OK;
}

}  // extern "C"
