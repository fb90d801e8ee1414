// See sips_gpu.hpp.
#include "sips_gpu.hpp"

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

void check(int rc, const char* what)
{
    if (rc != MG_OK) throw std::runtime_error(std::string(what) + ": " + mg_last_error());
}

constexpr int kMaxPending = 1000;

// the grid, spacing, step and boundary keys both models share
mg_ch_params base_params(const CommonParams& p, const InputFile& in)
{
    if (p.np != 1) throw std::invalid_argument("the SIPS models run one simulation per process (np must be 1)");
    mg_ch_params gp{};
    gp.nx = p.NX;
    gp.ny = p.NY;
    gp.nz = p.NZ;
    gp.dx = p.dx;
    gp.dy = p.dy;
    gp.dz = p.dz;
    gp.dt = p.dt;
    gp.M = 1.0;
    gp.kappa = in("PFApp/kap", 1.0);
    gp.bx = in("PFApp/bx", 0);  // SIPS.cpp:35, SIPSternary.cpp:34: no-flux x by default
    gp.by = in("PFApp/by", 1);
    gp.bz = in("PFApp/bz", 1);
    gp.precision = MG_FP64;
    gp.mass_correct = 0;
    gp.noise = in("PFApp/noiseStr", 0.1);
    return gp;
}

// r - 0.5 scaled by 0.1 at every site, in the reference's draw order
std::vector<double> draws(const mg_ch_params& gp, unsigned seed)
{
    std::vector<double> d((size_t)gp.nx * gp.ny * gp.nz);
    const int dims[3] = {gp.nx, gp.ny, gp.nz};
    check(mg_ic_generate(dims, 0.0, 0.1, 0, seed, d.data()), "mg_ic_generate");  // 0.0 + 0.1*(r - 0.5)
    return d;
}

}  // namespace

// ------------------------------------------------------------------ SIPS
SIPSGPU::SIPSGPU(const CommonParams& pin, const InputFile& in) : p(pin)
{
    gp = base_params(p, in);
    seed = (unsigned)in("PFApp/seed", 42);
    gp.noise_seed = (unsigned long long)in("PFApp/noise_seed", (int)seed);
    co = in("PFApp/co", 0.1);
    sp.N = in("PFApp/N", 100.0);
    sp.A = in("PFApp/A", 1.0);
    sp.Tinit = in("PFApp/Tinit", 273.15);
    sp.chiPS = in("PFApp/chiPS", 0.034);
    sp.chiPN = in("PFApp/chiPN", 2.5);
    sp.chiCond = in("PFApp/chiCond", 1.0);
    sp.phiCutoff = in("PFApp/phiCutoff", 0.5);
    sp.nu = in("PFApp/nu", 1.0);
    sp.gamma = in("PFApp/gamma", 10.0);
    sp.D0 = in("PFApp/D0", 1.0);
    sp.Mweight = in("PFApp/Mweight", 100.0);
    sp.Mvolume = in("PFApp/Mvolume", 0.1);
    sp.NSdepth = in("PFApp/NSdepth", 0);
    check(mg_sips_create(&gp, &sp, in("PFApp/device", 0), &h), "mg_sips_create");
}

SIPSGPU::~SIPSGPU()
{
    if (!h) return;
    if (pending > 0) mg_ch_step(h, pending);
    mg_ch_sync(h, -1);
    mg_ch_destroy(h);
}

void SIPSGPU::flush()
{
    if (pending > 0) {
        const int n = pending;
        pending = 0;
        check(mg_ch_step(h, n), "mg_ch_step");
    }
}

void SIPSGPU::initPhaseField()
{
    std::vector<double> c = draws(gp, seed);
    for (size_t s = 0; s < c.size(); ++s) {
        const int x = (int)(s % gp.nx);
        c[s] = x >= sp.NSdepth ? co + c[s] : 0.0;  // the water bath below NSdepth
    }
    check(mg_ch_set_field(h, c.data()), "mg_ch_set_field");
    pending = 0;
    current_step = 0;
    outputPhaseField();
}

void SIPSGPU::updatePhaseField()
{
    if (++pending >= kMaxPending) flush();
}

void SIPSGPU::outputPhaseField()
{
    flush();
    char path[64];
    std::snprintf(path, sizeof path, "vtkoutput/c_%d.vtk", current_step);
    check(mg_ch_write_vtk(h, path, "c", p.iskip, p.jskip, p.kskip), "mg_ch_write_vtk");
}

// ----------------------------------------------------------- SIPSternary
SIPSternaryGPU::SIPSternaryGPU(const CommonParams& pin, const InputFile& in) : p(pin)
{
    gp = base_params(p, in);
    seed = (unsigned)in("PFApp/seed", 42);
    gp.noise_seed = (unsigned long long)in("PFApp/noise_seed", (int)seed);
    NSdepth = in("PFApp/NSdepth", 0);
    co = in("PFApp/co", 0.20);
    no = in("PFApp/no", 0.10);
    tp.Kpp = in("PFApp/Kpp", 1.0);
    tp.Knn = in("PFApp/Knn", 1.0);
    tp.Mpp = in("PFApp/Mpp", 1.0);
    tp.Mnn = in("PFApp/Mnn", 1.0);
    check(mg_ternary_create(&gp, &tp, in("PFApp/device", 0), &h), "mg_ternary_create");
}

SIPSternaryGPU::~SIPSternaryGPU()
{
    if (!h) return;
    if (pending > 0) mg_batch_step(h, pending);
    mg_batch_sync(h, -1);
    mg_batch_destroy(h);
}

void SIPSternaryGPU::flush()
{
    if (pending > 0) {
        const int n = pending;
        pending = 0;
        check(mg_batch_step(h, n), "mg_batch_step");
    }
}

void SIPSternaryGPU::initPhaseField()
{
    const std::vector<double> d = draws(gp, seed);
    std::vector<double> c(d.size()), n(d.size());
    for (size_t s = 0; s < d.size(); ++s) {
        const bool film = (int)(s % gp.nx) >= NSdepth;
        c[s] = film ? co + d[s] : 0.0;
        n[s] = film ? no - d[s] : 1.0;
    }
    check(mg_batch_set_field(h, 0, c.data()), "mg_batch_set_field");
    check(mg_batch_set_field(h, 1, n.data()), "mg_batch_set_field");
    pending = 0;
    current_step = 0;
    outputPhaseField();
}

void SIPSternaryGPU::updatePhaseField()
{
    if (++pending >= kMaxPending) flush();
}

void SIPSternaryGPU::outputPhaseField()
{
    flush();
    char path[64];
    std::snprintf(path, sizeof path, "vtkoutput/c_%d.vtk", current_step);
    check(mg_batch_write_vtk(h, 0, path, "c", p.iskip, p.jskip, p.kskip), "mg_batch_write_vtk");
    std::snprintf(path, sizeof path, "vtkoutput/n_%d.vtk", current_step);
    check(mg_batch_write_vtk(h, 1, path, "n", p.iskip, p.jskip, p.kskip), "mg_batch_write_vtk");
}
