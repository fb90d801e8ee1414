// See chbasic_gpu.hpp.
#include "chbasic_gpu.hpp"

#include <cstdio>
#include <stdexcept>

namespace {

void check(int rc, const char* what)
{
    if (rc != MG_OK) throw std::runtime_error(std::string(what) + ": " + mg_last_error());
}

constexpr int kMaxPending = 1000;  // steps enqueued at once at most

}  // namespace

CHBasicGPU::CHBasicGPU(const CommonParams& pin, const InputFile& in) : p(pin)
{
    if (p.np != 1) throw std::invalid_argument("CHBasicGPU runs one simulation per process (np must be 1)");
    gp.nx = p.NX;
    gp.ny = p.NY;
    gp.nz = p.NZ;
    gp.dx = p.dx;
    gp.dy = p.dy;
    gp.dz = p.dz;
    gp.dt = p.dt;
    gp.M = in("PFApp/M", 1.0);
    gp.kappa = in("PFApp/kap", 1.0);
    gp.bx = in("PFApp/bx", 1);
    gp.by = in("PFApp/by", 1);
    gp.bz = in("PFApp/bz", 1);
    const std::string prec = in("PFApp/precision", "fp64");
    if (prec != "fp64" && prec != "fp32") throw std::invalid_argument("PFApp/precision must be fp64 or fp32");
    gp.precision = prec == "fp32" ? MG_FP32 : MG_FP64;
    gp.mass_correct = gp.precision == MG_FP32 ? in("PFApp/mass_correct", 1) : 0;
    // the reference's per-step fluctuation term (TIPSphil.cpp:200-209); off
    // by default in the plain Cahn-Hilliard model
    gp.noise = in("PFApp/noiseStr", 0.0);
    gp.noise_seed = (unsigned long long)in("PFApp/noise_seed", in("PFApp/seed", 42));
    co = in("PFApp/co", 0.0);
    noise_amp = in("PFApp/noise_amp", 0.1);
    noise_type = in("PFApp/noise_type", "uniform");
    seed = (unsigned)in("PFApp/seed", 42);
    init_output = in("PFApp/init_output", 1);
    vtk = in("PFApp/vtk", 1);
    dump_prefix = in("PFApp/dump_prefix", "");
    device = in("PFApp/device", 0);
    check(mg_ch_create(&gp, device, &h), "mg_ch_create");
}

CHBasicGPU::~CHBasicGPU()
{
    if (!h) return;
    if (pending > 0) mg_ch_step(h, pending);  // finish the run's steps
    mg_ch_sync(h, -1);
    mg_ch_destroy(h);
}

void CHBasicGPU::flush()
{
    if (pending > 0) {
        const int n = pending;
        pending = 0;
        check(mg_ch_step(h, n), "mg_ch_step");
    }
}

void CHBasicGPU::initPhaseField()
{
    // seeded version of TIPSphil::initPhaseField (TIPSphil.cpp:86-103)
    std::vector<double> ic((size_t)gp.nx * gp.ny * gp.nz);
    const int dims[3] = {gp.nx, gp.ny, gp.nz};
    check(mg_ic_generate(dims, co, noise_amp, noise_type == "gaussian", seed, ic.data()), "mg_ic_generate");
    check(mg_ch_set_field(h, ic.data()), "mg_ch_set_field");
    pending = 0;
    // the reference writes step 0 from inside the initializer too
    // (TIPSphil.cpp:102-103), so the step-0 file holds two copies
    current_step = 0;
    if (init_output) outputPhaseField();
}

void CHBasicGPU::updatePhaseField()
{
    if (++pending >= kMaxPending) flush();
}

void CHBasicGPU::getField(std::vector<double>& out)
{
    flush();
    out.resize((size_t)gp.nx * gp.ny * gp.nz);
    check(mg_ch_get_field(h, out.data()), "mg_ch_get_field");
}

void CHBasicGPU::outputPhaseField()
{
    if (vtk) {
        // SfieldFD::writeVTKFile names the file vtkoutput/<tag>_<step>.vtk
        // and appends to it (SfieldFD.cpp:363-430); the text is formatted on
        // the GPU
        flush();
        char path[64];
        std::snprintf(path, sizeof path, "vtkoutput/c_%d.vtk", current_step);
        check(mg_ch_write_vtk(h, path, "c", p.iskip, p.jskip, p.kskip), "mg_ch_write_vtk");
    }
    if (!dump_prefix.empty()) {
        std::vector<double> c;
        getField(c);
        // raw dump: int32 {xOff, nx, ny, nz, step}, then the field as
        // float64, dense x-fastest
        char name[512];
        std::snprintf(name, sizeof name, "%s_%d.rank%d", dump_prefix.c_str(), current_step, p.rank);
        FILE* f = std::fopen(name, "wb");
        if (!f) throw std::runtime_error(std::string("cannot write ") + name);
        const int hdr[5] = {p.xOff, gp.nx, gp.ny, gp.nz, current_step};
        std::fwrite(hdr, sizeof(int), 5, f);
        std::fwrite(c.data(), sizeof(double), c.size(), f);
        std::fclose(f);
    }
}
