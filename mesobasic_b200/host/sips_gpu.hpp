// SIPSGPU and SIPSternaryGPU: the reference's solvent/non-solvent induced
// phase separation models as PFBaseClass plugins stepped by libmesogpu.so.
//
// SIPSGPU (SIPS.cpp): one field c, the SIPS step of mg_sips_create.  Keys
// (section PFApp/) and defaults are SIPS's (SIPS.cpp:22-59): bx (0), by,
// bz (1), NSdepth (0), co (0.1), chiPS (0.034), chiPN (2.5), chiCond (1),
// phiCutoff (0.5), kap (1), N (100), A (1), Tinit (273.15), noiseStr (0.1),
// D0 (1), nu (1), gamma (10), Mweight (100), Mvolume (0.1).  Initial field
// (SIPS.cpp:78-122): co + 0.1*(r - 0.5) for x >= NSdepth, 0 in the bath.
// Output: c_<step>.vtk.
//
// SIPSternaryGPU (SIPSternary.cpp): fields c and n, the two-job batch of
// mg_ternary_create.  Keys: bx (0), by, bz (1), NSdepth (0), co (0.2),
// no (0.1), Kpp, Knn, Mpp, Mnn (1), noiseStr (0.1) (SIPSternary.cpp:21-63;
// the Flory-Huggins keys it reads do not reach its step).  Initial fields
// (SIPSternary.cpp:82-124): c = co + 0.1*(r - 0.5), n = no - 0.1*(r - 0.5)
// with one r per site for x >= NSdepth; c = 0, n = 1 in the bath.  Output:
// c_<step>.vtk and n_<step>.vtk.
//
// Both draw r and the per-step noise from seeded generators (PFApp/seed,
// default 42; PFApp/noise_seed, default seed) where the reference seeds
// rand() from the clock.
#pragma once

#include "mesogpu.h"
#include "pf_model.hpp"

class SIPSGPU : public PFBaseClass {
public:
    SIPSGPU(const CommonParams& p, const InputFile& in);
    ~SIPSGPU() override;

    void initPhaseField() override;
    void updatePhaseField() override;
    void outputPhaseField() override;
    void setTimeStep(int step) override { current_step = step; }

private:
    void flush();

    CommonParams p;
    mg_ch_params gp{};
    mg_sips_params sp{};
    mg_ch_t* h = nullptr;
    int current_step = 0;
    int pending = 0;
    double co;
    unsigned seed;
};

class SIPSternaryGPU : public PFBaseClass {
public:
    SIPSternaryGPU(const CommonParams& p, const InputFile& in);
    ~SIPSternaryGPU() override;

    void initPhaseField() override;
    void updatePhaseField() override;
    void outputPhaseField() override;
    void setTimeStep(int step) override { current_step = step; }

private:
    void flush();

    CommonParams p;
    mg_ch_params gp{};
    mg_ternary_params tp{};
    mg_batch_t* h = nullptr;
    int current_step = 0;
    int pending = 0;
    int NSdepth;
    double co, no;
    unsigned seed;
};
