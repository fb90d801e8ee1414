// Test infrastructure: times the reference CPU build of the Cahn-Hilliard
// step.  The step loop is the reference's own: PFApp::stepForward ->
// PFBaseClass::updatePhaseField (PFApp.cpp:91-107) on the CHBasic type, with
// MPI ranks given by MB_SHIM_NP (see shim/mpi.h).
//
//   chref_bench Domain/nx=256 Domain/ny=256 Domain/nz=256 Time/dt=0.005 \
//               Time/nstep=10 PFApp/kap=1 [PFApp/dump_prefix=/tmp/f] ...
//
// The arguments are GetPot "section/key=value" pairs, the same keys as the
// reference's input.dat.  Rank 0 prints one JSON line with the wall time of
// the step loop only (initial condition and output excluded).
#include <chrono>
#include <cstdio>
#include <mpi.h>

#include "PFApp.hpp"

int main(int argc, char** argv)
{
    MPI::Init();
    {
        GetPot params(argc, argv);
        int nstep = params("Time/nstep", 1);
        int NX = params("Domain/nx", 1), NY = params("Domain/ny", 1), NZ = params("Domain/nz", 1);
        PFApp app(params);
        app.initSystem();
        MPI::COMM_WORLD.Barrier();
        auto t0 = std::chrono::steady_clock::now();
        for (int step = 1; step <= nstep; ++step) app.stepForward(step);
        MPI::COMM_WORLD.Barrier();
        auto t1 = std::chrono::steady_clock::now();
        double secs = std::chrono::duration<double>(t1 - t0).count();
        app.writeOutput(nstep);
        if (MPI::COMM_WORLD.Get_rank() == 0) {
            double sites = (double)NX * NY * NZ;
            std::printf(
                "{\"ranks\": %d, \"nx\": %d, \"ny\": %d, \"nz\": %d, \"steps\": %d, "
                "\"seconds\": %.6f, \"site_updates_per_s\": %.6e}\n",
                MPI::COMM_WORLD.Get_size(), NX, NY, NZ, nstep, secs,
                nstep > 0 && secs > 0 ? sites * nstep / secs : 0.0);
            std::fflush(stdout);
        }
    }
    MPI::Finalize();
    return 0;
}
