// CHBasicGPU: the Cahn-Hilliard phase-field model as a PFBaseClass plugin
// whose body is libmesogpu.so (C ABI, include/mesogpu.h).
//
//   mu    = (c^3 - c) - kap * lap(c)
//   c_new = c + (dt*M) * lap(mu)
//
// Input keys (section PFApp/), with the defaults of the reference-side
// CHBasic model and of TIPSphil's constructor (TIPSphil.cpp:24-60):
//   bx, by, bz     1 periodic / 0 no-flux        (1, 1, 1)
//   co             mean of the initial field     0.0
//   M, kap         mobility, gradient coeff.     1.0, 1.0
//   noise_amp      uniform: full width; gaussian: sigma   0.1
//   noise_type     uniform | gaussian            uniform
//   seed           MT19937 seed of the IC        42
//   init_output    write step 0 from initPhaseField as well  1
//   vtk            write vtkoutput/c_<step>.vtk  1
//   dump_prefix    also write raw dumps <prefix>_<step>.rank0   (none)
// Keys of this build only:
//   precision      fp64 (bit-identical to the reference build) | fp32   fp64
//   mass_correct   fp32: FP64 mass feedback every K-th step (0 off) 1
//   noiseStr       per-step noise c += dt*noiseStr*(u - 0.5)       0 (off)
//   noise_seed     key of the noise generator                      seed
//   device         CUDA device                                     0
//
// updatePhaseField only counts the step: pending steps are enqueued
// together (CUDA-graph replays, no host synchronisation per step) when the
// next output needs the field, every 1000 steps, and at destruction.
#pragma once

#include <string>
#include <vector>

#include "mesogpu.h"
#include "pf_model.hpp"

class CHBasicGPU : public PFBaseClass {
public:
    CHBasicGPU(const CommonParams& p, const InputFile& in);
    ~CHBasicGPU() override;

    void initPhaseField() override;
    void updatePhaseField() override;
    void outputPhaseField() override;
    void setTimeStep(int step) override { current_step = step; }

    // dense x-fastest copy of the current field
    void getField(std::vector<double>& out);
    mg_ch_t* handle() const { return h; }

private:
    void flush();

    CommonParams p;
    mg_ch_params gp{};
    mg_ch_t* h = nullptr;
    int current_step = 0;
    int pending = 0;
    double co, noise_amp;
    std::string noise_type, dump_prefix;
    unsigned seed;
    int init_output, vtk, device;
};
