// Test infrastructure: C entry points that run the reference's own
// TIPSphil::updatePhaseField (TIPSphil.cpp:113-211: Flory-Huggins chemical
// potential, Phillies mobility, harmonic-mean variable-mobility Laplacian),
// TIPSbathPHIL's (its 1-D bath temperature), SIPS's (SIPS.cpp:130-249) or
// SIPSternary's (SIPSternary.cpp:132-278, two fields) on given fields, for
// the parity tests of the GPU variable-mobility steps.  The models keep
// their fields private and set them only from rand(); this adapter opens the
// classes to read and write them (no reference source is changed), and runs
// with noiseStr = 0 and no mobility output.
#include <cstdio>
#include <string>
#include <vector>

#define private public
#include "PFTypes/SIPS.hpp"
#include "PFTypes/SIPSternary.hpp"
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

// SIPS: prm = N, A, Tinit, chiPS, chiPN, chiCond, phiCutoff, nu, gamma, D0,
// Mweight, Mvolume, kap (13 values); steps first..first+nsteps-1.
int sipsref_run(const int dims[3], const double spacing[3], double dt, const int bc[3], const double* prm, int NSdepth,
                int first, const double* ic, int nsteps, double* out);

// SIPSternary: prm = Kpp, Knn, Mpp, Mnn; fields c and n.
int ternref_run(const int dims[3], const double spacing[3], double dt, const int bc[3], const double* prm, int first,
                const double* ic_c, const double* ic_n, int nsteps, double* out_c, double* out_n);

}  // extern "C"

namespace {

CommonParams common(const int dims[3], const double spacing[3], double dt, int nstep_total)
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
    return p;
}

// GetPot over "key=value" arguments
struct Args {
    std::vector<std::string> args{"ref"};
    void add(const char* key, double v) { args.push_back(kvf(key, v)); }
    void bc(const int b[3])
    {
        add("PFApp/bx", b[0]);
        add("PFApp/by", b[1]);
        add("PFApp/bz", b[2]);
    }
    GetPot getpot()
    {
        argv.clear();
        for (auto& a : args) argv.push_back(&a[0]);
        return GetPot((int)argv.size(), argv.data());
    }
    std::vector<char*> argv;
};

// dense x-fastest <-> SfieldFD (z fastest, one ghost layer)
void put(SfieldFD& f, const CommonParams& p, const double* src)
{
    const int deli = (p.nz + 2) * (p.ny + 2), delj = p.nz + 2;
    for (int i = 1; i <= p.nx; ++i)
        for (int j = 1; j <= p.ny; ++j)
            for (int k = 1; k <= p.nz; ++k)
                f.setValue(i * deli + j * delj + k,
                           src[(size_t)(i - 1) + (size_t)p.nx * ((size_t)(j - 1) + (size_t)p.ny * (k - 1))]);
}

void get(SfieldFD& f, const CommonParams& p, double* dst)
{
    const int deli = (p.nz + 2) * (p.ny + 2), delj = p.nz + 2;
    for (int i = 1; i <= p.nx; ++i)
        for (int j = 1; j <= p.ny; ++j)
            for (int k = 1; k <= p.nz; ++k)
                dst[(size_t)(i - 1) + (size_t)p.nx * ((size_t)(j - 1) + (size_t)p.ny * (k - 1))] =
                    f.getValue(i * deli + j * delj + k);
}

template <typename Model>
int run_model(const int dims[3], const double spacing[3], double dt, const int bc[3], const double* prm,
              double thermCond, int nstep_total, int first, const double* ic, int nsteps, double* out)
{
    const CommonParams p = common(dims, spacing, dt, nstep_total);
    const char* names[13] = {"PFApp/alpha", "PFApp/beta", "PFApp/N", "PFApp/A", "PFApp/Tinit", "PFApp/Tbath",
                             "PFApp/Tcrystal", "PFApp/nu", "PFApp/gamma", "PFApp/D0", "PFApp/Mweight",
                             "PFApp/Mvolume", "PFApp/kap"};
    Args a;
    a.add("PFApp/noiseStr", 0);
    a.add("PFApp/mobStep", -1);
    for (int k = 0; k < 13; ++k) a.add(names[k], prm[k]);
    a.add("PFApp/thermCond", thermCond);
    a.bc(bc);
    Model model(p, a.getpot());
    put(model.c, p, ic);
    for (int s = first; s < first + nsteps; ++s) {
        model.setTimeStep(s);
        model.updatePhaseField();
    }
    get(model.c, p, out);
    return 0;
}

}  // namespace

extern "C" int sipsref_run(const int dims[3], const double spacing[3], double dt, const int bc[3], const double* prm,
                           int NSdepth, int first, const double* ic, int nsteps, double* out)
{
    const CommonParams p = common(dims, spacing, dt, first + nsteps);
    const char* names[13] = {"PFApp/N",     "PFApp/A",  "PFApp/Tinit", "PFApp/chiPS",   "PFApp/chiPN",
                             "PFApp/chiCond", "PFApp/phiCutoff", "PFApp/nu", "PFApp/gamma", "PFApp/D0",
                             "PFApp/Mweight", "PFApp/Mvolume", "PFApp/kap"};
    Args a;
    a.add("PFApp/noiseStr", 0);
    a.add("PFApp/NSdepth", NSdepth);
    for (int k = 0; k < 13; ++k) a.add(names[k], prm[k]);
    a.bc(bc);
    SIPS model(p, a.getpot());
    put(model.c, p, ic);
    for (int s = first; s < first + nsteps; ++s) {
        model.setTimeStep(s);
        model.updatePhaseField();
    }
    get(model.c, p, out);
    return 0;
}

extern "C" int ternref_run(const int dims[3], const double spacing[3], double dt, const int bc[3], const double* prm,
                           int first, const double* ic_c, const double* ic_n, int nsteps, double* out_c,
                           double* out_n)
{
    const CommonParams p = common(dims, spacing, dt, first + nsteps);
    const char* names[4] = {"PFApp/Kpp", "PFApp/Knn", "PFApp/Mpp", "PFApp/Mnn"};
    Args a;
    a.add("PFApp/noiseStr", 0);
    for (int k = 0; k < 4; ++k) a.add(names[k], prm[k]);
    a.bc(bc);
    SIPSternary model(p, a.getpot());
    put(model.c, p, ic_c);
    put(model.n, p, ic_n);
    for (int s = first; s < first + nsteps; ++s) {
        model.setTimeStep(s);
        model.updatePhaseField();
    }
    get(model.c, p, out_c);
    get(model.n, p, out_n);
    return 0;
}
