// See tipsphil_gpu.hpp.
#include "tipsphil_gpu.hpp"

#include <cmath>
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

}  // namespace

TIPSphilGPU::TIPSphilGPU(const CommonParams& pin, const InputFile& in, bool bath_) : p(pin), bath(bath_)
{
    if (p.np != 1) throw std::invalid_argument("TIPSphilGPU runs one simulation per process (np must be 1)");
    gp.nx = p.NX;
    gp.ny = p.NY;
    gp.nz = p.NZ;
    gp.dx = p.dx;
    gp.dy = p.dy;
    gp.dz = p.dz;
    gp.dt = p.dt;
    gp.M = in("PFApp/M", 1.0);
    gp.kappa = in("PFApp/kap", 1.0);
    gp.bx = in("PFApp/bx", bath ? 0 : 1);  // TIPSbathPHIL.cpp:18: no-flux x by default
    gp.by = in("PFApp/by", 1);
    gp.bz = in("PFApp/bz", 1);
    gp.precision = MG_FP64;
    gp.mass_correct = 0;
    gp.noise = in("PFApp/noiseStr", 0.1);
    seed = (unsigned)in("PFApp/seed", 42);
    gp.noise_seed = (unsigned long long)in("PFApp/noise_seed", (int)seed);
    mobStep = bath ? -1 : in("PFApp/mobStep", 1);  // TIPSbathPHIL writes no mobility
    co = in("PFApp/co", 0.5);
    fp.alpha = in("PFApp/alpha", 1.0);
    fp.beta = in("PFApp/beta", 1.0);
    fp.N = in("PFApp/N", 100.0);
    fp.A = in("PFApp/A", 1.0);
    fp.Tinit = in("PFApp/Tinit", 273.0);
    fp.Tbath = in("PFApp/Tbath", 273.0);
    fp.Tcrystal = in("PFApp/Tcrystal", 273.0);
    fp.nu = in("PFApp/nu", 1.0);
    fp.gamma = in("PFApp/gamma", 10.0);
    fp.D0 = in("PFApp/D0", 0.0000001);
    fp.Mweight = in("PFApp/Mweight", 100.0);
    fp.Mvolume = in("PFApp/Mvolume", 0.1);
    fp.nstep = p.nstep;
    fp.bath = bath ? 1 : 0;
    fp.thermCond = in("PFApp/thermCond", 1.0);
    check(mg_fh_create(&gp, &fp, in("PFApp/device", 0), &h), "mg_fh_create");
}

TIPSphilGPU::~TIPSphilGPU()
{
    if (!h) return;
    if (pending > 0) mg_ch_step(h, pending);
    mg_ch_sync(h, -1);
    mg_ch_destroy(h);
}

void TIPSphilGPU::flush()
{
    if (pending > 0) {
        const int n = pending;
        pending = 0;
        check(mg_ch_step(h, n), "mg_ch_step");
    }
}

void TIPSphilGPU::initPhaseField()
{
    // TIPSphil::initPhaseField (TIPSphil.cpp:79-103): c = co + 0.1*(r - 0.5)
    std::vector<double> ic((size_t)gp.nx * gp.ny * gp.nz);
    const int dims[3] = {gp.nx, gp.ny, gp.nz};
    check(mg_ic_generate(dims, co, 0.1, 0, seed, ic.data()), "mg_ic_generate");
    check(mg_ch_set_field(h, ic.data()), "mg_ch_set_field");
    pending = 0;
    current_step = 0;
    outputPhaseField();
}

void TIPSphilGPU::updatePhaseField()
{
    ++pending;
    if (current_step == mobStep) {
        // the mobility of this step, as TIPSphil.cpp:180-185 writes it
        flush();
        std::vector<double> mob((size_t)gp.nx * gp.ny * gp.nz);
        check(mg_fh_mobility(h, mob.data()), "mg_fh_mobility");
        char path[64];
        std::snprintf(path, sizeof path, "vtkoutput/mob_%d.vtk", current_step);
        const int dims[3] = {gp.nx, gp.ny, gp.nz};
        check(mg_vtk_write(path, "mob", mob.data(), dims, p.iskip, p.jskip, p.kskip), "mg_vtk_write");
    } else if (pending >= kMaxPending) {
        flush();
    }
}

void TIPSphilGPU::outputPhaseField()
{
    flush();
    char path[64];
    std::snprintf(path, sizeof path, "vtkoutput/%s_%d.vtk", bath ? "polymer" : "c", current_step);
    check(mg_ch_write_vtk(h, path, bath ? "polymer" : "c", p.iskip, p.jskip, p.kskip), "mg_ch_write_vtk");
    if (bath) {
        // TIPSbathPHIL's TempOut: 460 from the initializer, then the bath
        // profile of the last step (TIPSbathPHIL.cpp:118-125)
        std::vector<double> T((size_t)gp.nx * gp.ny * gp.nz);
        for (size_t s = 0; s < T.size(); ++s) {
            const int i = (int)(s % gp.nx) + 1;
            T[s] = current_step == 0 ? 460.0
                                     : (fp.Tinit - fp.Tbath) * std::erf(i / (2.0 * std::sqrt(fp.thermCond * double(current_step) * gp.dt))) +
                                           fp.Tbath;
        }
        std::snprintf(path, sizeof path, "vtkoutput/temp_%d.vtk", current_step);
        const int dims[3] = {gp.nx, gp.ny, gp.nz};
        check(mg_vtk_write(path, "temp", T.data(), dims, p.iskip, p.jskip, p.kskip), "mg_vtk_write");
    }
}
