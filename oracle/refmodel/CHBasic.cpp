// Test infrastructure: see CHBasic.hpp.
#include "CHBasic.hpp"

#include <mpi.h>
#include <cstdio>
#include <vector>
#include "rand.hpp"

CHBasic::CHBasic(const CommonParams& pin, const GetPot& input_params) : p(pin), c(p)
{
    // parameter reads follow the TIPSphil constructor (TIPSphil.cpp:24-60)
    nx = p.nx;
    ny = p.ny;
    nz = p.nz;
    deli = (nz + 2) * (ny + 2);
    delj = (nz + 2);
    delk = 1;
    current_step = 0;
    bx = input_params("PFApp/bx", 1);
    by = input_params("PFApp/by", 1);
    bz = input_params("PFApp/bz", 1);
    co = input_params("PFApp/co", 0.0);
    M = input_params("PFApp/M", 1.0);
    kap = input_params("PFApp/kap", 1.0);
    noise_amp = input_params("PFApp/noise_amp", 0.1);
    noise_type = std::string(input_params("PFApp/noise_type", "uniform"));
    seed = (unsigned)input_params("PFApp/seed", 42);
    init_output = input_params("PFApp/init_output", 1);
    vtk = input_params("PFApp/vtk", 1);
    dump_prefix = std::string(input_params("PFApp/dump_prefix", ""));
}

CHBasic::~CHBasic() {}

void CHBasic::generateIC(int NX, int NY, int NZ, double co, double amp, bool gaussian,
                         unsigned seed, double* out)
{
    Rand rng(seed);
    for (int i = 0; i < NX; i++) {
        for (int j = 0; j < NY; j++) {
            for (int k = 0; k < NZ; k++) {
                double val = gaussian ? co + amp * rng.normal() : co + amp * (rng.uniform() - 0.5);
                out[(size_t)i + (size_t)NX * ((size_t)j + (size_t)NY * k)] = val;
            }
        }
    }
}

void CHBasic::initPhaseField()
{
    // Seeded version of TIPSphil::initPhaseField (TIPSphil.cpp:86-103): every
    // rank draws the global sequence in generateIC's order (x outer) and
    // keeps the draws of its own x-slab, so the field does not depend on the
    // rank count.  Draws are streamed, so a rank holds only its slab (a 512^3
    // field on 16 ranks stays at 1/16 of the grid per rank).
    Rand rng(seed);
    const bool gaussian = noise_type == "gaussian";
    for (int ig = 0; ig < p.xOff + nx; ig++) {
        const bool mine = ig >= p.xOff;
        for (int j = 0; j < p.NY; j++) {
            for (int k = 0; k < p.NZ; k++) {
                double val = gaussian ? co + noise_amp * rng.normal() : co + noise_amp * (rng.uniform() - 0.5);
                if (mine) c.setValue((ig - p.xOff + 1) * deli + (j + 1) * delj + (k + 1) * delk, val);
            }
        }
    }
    // the reference writes the step-0 file from inside the initializer as
    // well (TIPSphil.cpp:102-103), so step 0 is written twice into one file
    current_step = 0;
    if (init_output) outputPhaseField();
}

void CHBasic::updatePhaseField()
{
    c.updateBoundaries(bx, by, bz);
    MPI::COMM_WORLD.Barrier();
    SfieldFD mu(p);
    for (int i = 1; i < nx + 1; i++) {
        for (int j = 1; j < ny + 1; j++) {
            for (int k = 1; k < nz + 1; k++) {
                int ndx = i * deli + j * delj + k * delk;
                double cc = c.getValue(ndx);
                double df = cc * cc * cc - cc;
                double lapc = c.Laplacian(ndx);
                mu.setValue(ndx, df - kap * lapc);
            }
        }
    }
    mu.updateBoundaries(bx, by, bz);
    MPI::COMM_WORLD.Barrier();
    c += (p.dt * M) * mu.Laplacian();
}

void CHBasic::outputPhaseField()
{
    if (vtk) c.writeVTKFile("c", current_step, p.iskip, p.jskip, p.kskip);
    if (!dump_prefix.empty()) {
        // raw slab for the tests: int32 {xOff, nx, ny, nz, step} then
        // nx*ny*nz float64, dense x-fastest
        std::vector<double> dense((size_t)nx * ny * nz);
        getField(dense.data());
        char name[512];
        std::snprintf(name, sizeof name, "%s_%d.rank%d", dump_prefix.c_str(), current_step, p.rank);
        FILE* f = std::fopen(name, "wb");
        if (f) {
            int hdr[5] = {p.xOff, nx, ny, nz, current_step};
            std::fwrite(hdr, sizeof(int), 5, f);
            std::fwrite(dense.data(), sizeof(double), dense.size(), f);
            std::fclose(f);
        }
    }
}

void CHBasic::setField(const double* dense)
{
    for (int i = 1; i < nx + 1; i++)
        for (int j = 1; j < ny + 1; j++)
            for (int k = 1; k < nz + 1; k++)
                c.setValue(i * deli + j * delj + k * delk,
                           dense[(size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (k - 1))]);
}

void CHBasic::getField(double* dense) const
{
    for (int i = 1; i < nx + 1; i++)
        for (int j = 1; j < ny + 1; j++)
            for (int k = 1; k < nz + 1; k++)
                dense[(size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (k - 1))] =
                    c.getValue(i * deli + j * delj + k * delk);
}
