// Test infrastructure: a C entry point into the reference CPU build, so the
// tests can run the reference's own SfieldFD arithmetic on seeded fields.
// Single rank; the field is dense x-fastest without ghosts.
#include <cstdio>
#include <string>
#include <vector>

#include "CHBasic.hpp"

namespace {

std::string kv(const char* key, double v)
{
    char buf[96];
    std::snprintf(buf, sizeof buf, "%s=%.17g", key, v);  // round-trips through sscanf("%lf")
    return buf;
}

CommonParams single_rank_params(const int dims[3], const double spacing[3], double dt)
{
    // the same fields PFApp fills (PFApp.cpp:18-52) for np == 1
    CommonParams p;
    p.NX = dims[0];
    p.NY = dims[1];
    p.NZ = dims[2];
    p.nx = p.NX;
    p.ny = p.NY;
    p.nz = p.NZ;
    p.dx = spacing[0];
    p.dy = spacing[1];
    p.dz = spacing[2];
    p.dt = dt;
    p.nstep = 0;
    p.numOutputs = 0;
    p.iskip = p.jskip = p.kskip = 1;
    p.LX = p.NX * p.dx;
    p.LY = p.NY * p.dy;
    p.LZ = p.NZ * p.dz;
    p.np = 1;
    p.rank = 0;
    p.nbrL = 0;
    p.nbrR = 0;
    p.xOff = 0;
    return p;
}

}  // namespace

extern "C" {

// Runs nsteps CHBasic steps of the reference build on `ic` and writes the
// final field to `out`.  bc[3] are the reference's bx,by,bz flags
// (1 periodic, 0 no-flux; SfieldFD.cpp:187-251).  Returns 0.
int chref_run(const int dims[3], const double spacing[3], double dt, double M, double kap,
              const int bc[3], const double* ic, int nsteps, double* out)
{
    CommonParams p = single_rank_params(dims, spacing, dt);
    std::vector<std::string> args = {"chref", kv("PFApp/M", M), kv("PFApp/kap", kap),
                                     kv("PFApp/bx", bc[0]), kv("PFApp/by", bc[1]),
                                     kv("PFApp/bz", bc[2]), "PFApp/init_output=0"};
    std::vector<char*> argv;
    for (auto& a : args) argv.push_back(&a[0]);
    GetPot gp((int)argv.size(), argv.data());
    CHBasic model(p, gp);
    model.setField(ic);
    for (int s = 1; s <= nsteps; ++s) {
        model.setTimeStep(s);
        model.updatePhaseField();
    }
    model.getField(out);
    return 0;
}

// Seeded initial condition from the reference's Mersenne twister.
int chref_ic(const int dims[3], double co, double amp, int gaussian, unsigned seed, double* out)
{
    CHBasic::generateIC(dims[0], dims[1], dims[2], co, amp, gaussian != 0, seed, out);
    return 0;
}

}  // extern "C"
