// Test infrastructure: a C entry point that runs the reference's own
// TIPSphil::updatePhaseField (TIPSphil.cpp:113-211: Flory-Huggins chemical
// potential, Phillies mobility, harmonic-mean variable-mobility Laplacian),
// or TIPSbathPHIL's (its 1-D bath temperature), on a given field, for the
// parity tests of the GPU variable-mobility step.  The models keep their
// field private and set it only from rand(); this adapter opens the classes
// to read and write it (no reference source is changed), and runs with
// noiseStr = 0 and no mobility output.
#include <cstdio>
#include <string>
#include <vector>

#define private public
#include "PFTypes/TIPSbathPHIL.hpp"
#include "PFTypes/TIPSphil.hpp"
#undef private

namespace {

std::string kvf(const char* key, double v)
{
    char buf[96];
    std::snprintf(buf, sizeof buf, "%s=%.17g", key, v);
    return buf;
}

template <typename Model>
int run_model(const int dims[3], const double spacing[3], double dt, const int bc[3], const double* prm,
              double thermCond, int nstep_total, int first, const double* ic, int nsteps, double* out);

}  // namespace

extern "C" {

// prm: alpha, beta, N, A, Tinit, Tbath, Tcrystal, nu, gamma, D0, Mweight,
// Mvolume, kap (13 values); nstep_total is Time/nstep (the quench schedule);
// steps first..first+nsteps-1 are taken (the models read the step number).
// bath = 0 runs TIPSphil, 1 TIPSbathPHIL (thermCond: its bath diffusivity).
int fhref_run(const int dims[3], const double spacing[3], double dt, const int bc[3], const double* prm, int bath,
              double thermCond, int nstep_total, int first, const double* ic, int nsteps, double* out)
{
    if (bath) return run_model<TIPSbathPHIL>(dims, spacing, dt, bc, prm, thermCond, nstep_total, first, ic, nsteps, out);
    return run_model<TIPSphil>(dims, spacing, dt, bc, prm, thermCond, nstep_total, first, ic, nsteps, out);
}

}  // extern "C"

namespace {

template <typename Model>
int run_model(const int dims[3], const double spacing[3], double dt, const int bc[3], const double* prm,
              double thermCond, int nstep_total, int first, const double* ic, int nsteps, double* out)
{
    CommonParams p;
    p.NX = p.nx = dims[0];
    p.NY = p.ny = dims[1];
    p.NZ = p.nz = dims[2];
    p.dx = spacing[0];
    p.dy = spacing[1];
    p.dz = spacing[2];
    p.dt = dt;
    p.nstep = nstep_total;
    p.numOutputs = 0;
    p.iskip = p.jskip = p.kskip = 1;
    p.LX = p.NX * p.dx;
    p.LY = p.NY * p.dy;
    p.LZ = p.NZ * p.dz;
    p.np = 1;
    p.rank = 0;
    p.nbrL = p.nbrR = 0;
    p.xOff = 0;
    const char* names[13] = {"PFApp/alpha", "PFApp/beta", "PFApp/N", "PFApp/A", "PFApp/Tinit", "PFApp/Tbath",
                             "PFApp/Tcrystal", "PFApp/nu", "PFApp/gamma", "PFApp/D0", "PFApp/Mweight",
                             "PFApp/Mvolume", "PFApp/kap"};
    std::vector<std::string> args = {"fhref", "PFApp/noiseStr=0", "PFApp/mobStep=-1"};
    for (int k = 0; k < 13; ++k) args.push_back(kvf(names[k], prm[k]));
    args.push_back(kvf("PFApp/thermCond", thermCond));
    args.push_back(kvf("PFApp/bx", bc[0]));
    args.push_back(kvf("PFApp/by", bc[1]));
    args.push_back(kvf("PFApp/bz", bc[2]));
    std::vector<char*> argv;
    for (auto& a : args) argv.push_back(&a[0]);
    GetPot gp((int)argv.size(), argv.data());
    Model model(p, gp);
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int deli = (nz + 2) * (ny + 2), delj = nz + 2;
    auto dense = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (k - 1)); };
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j)
            for (int k = 1; k <= nz; ++k) model.c.setValue(i * deli + j * delj + k, ic[dense(i, j, k)]);
    for (int s = first; s < first + nsteps; ++s) {
        model.setTimeStep(s);
        model.updatePhaseField();
    }
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j)
            for (int k = 1; k <= nz; ++k) out[dense(i, j, k)] = model.c.getValue(i * deli + j * delj + k);
    return 0;
}

}  // namespace
