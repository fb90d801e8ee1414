// TIPSphilGPU: the reference's TIPSphil model (thermally induced phase
// separation with a Flory-Huggins free energy and Phillies mobility) as a
// PFBaseClass plugin whose step is the variable-mobility update of
// libmesogpu.so (mg_fh_create).
//
// Input keys (section PFApp/) and defaults are TIPSphil's
// (TIPSphil.cpp:41-59): bx, by, bz (1), mobStep (1), co (0.5), kap (1),
// alpha (1), beta (1), N (100), A (1), Tinit, Tbath, Tcrystal (273),
// noiseStr (0.1), nu (1), gamma (10), D0 (1e-7), Mweight (100),
// Mvolume (0.1).  Differences: the initial field co + 0.1*(r - 0.5) and the
// per-step noise come from seeded generators (PFApp/seed, default 42;
// PFApp/noise_seed, default seed) where the reference seeds rand() from the
// clock.  Output: c as legacy VTK at every output step; the mobility as
// vtkoutput/mob_<mobStep>.vtk after step mobStep, as the reference writes it.
//
// With `bath` the model is TIPSbathPHIL (TIPSbathPHIL.cpp): the temperature
// is the 1-D bath profile along x (key thermCond, default 1), bx defaults to
// 0, and each output writes polymer_<step>.vtk (c) and temp_<step>.vtk (the
// temperature: 460 at step 0, the profile of the last step after it).
#pragma once

#include "mesogpu.h"
#include "pf_model.hpp"

class TIPSphilGPU : public PFBaseClass {
public:
    TIPSphilGPU(const CommonParams& p, const InputFile& in, bool bath = false);
    ~TIPSphilGPU() override;

    void initPhaseField() override;
    void updatePhaseField() override;
    void outputPhaseField() override;
    void setTimeStep(int step) override { current_step = step; }

private:
    void flush();

    CommonParams p;
    mg_ch_params gp{};
    mg_fh_params fp{};
    mg_ch_t* h = nullptr;
    int current_step = 0;
    int pending = 0;
    int mobStep;
    bool bath;
    double co;
    unsigned seed;
};
