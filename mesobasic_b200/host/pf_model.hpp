// The phase-field plugin interface of mesoBasic, mirrored for the GPU
// driver: the same CommonParams fields (src/utils/CommonParams.h), the same
// PFBaseClass virtuals and factory-by-name (PFBaseClass.hpp:14-41,
// PFBaseClass.cpp:26-55) and the same PFApp life cycle (PFApp.cpp:10-121),
// with InputFile in place of GetPot.
//
// Differences, all on error paths the reference leaves undefined:
//   - PFFactory throws std::invalid_argument for an unknown PFApp/type (the
//     reference returns NULL and the first call through it crashes);
//   - the models of this build report failures by throwing
//     std::runtime_error (the reference has no error reporting).
// One process drives one GPU; the slab split of the reference's x axis
// over MPI ranks is not used (np = 1, xOff = 0, nx = NX).
#pragma once

#include <memory>
#include <string>

#include "input_file.hpp"

struct CommonParams {
    int nx, ny, nz;  // nodes in the local domain
    int NX, NY, NZ;  // nodes in the global domain
    int rank;        // process rank
    int np;          // processes
    int nbrL;
    int nbrR;
    int xOff;
    int iskip;
    int jskip;
    int kskip;
    int nstep;
    int numOutputs;
    double dx, dy, dz;  // node spacing
    double LX, LY, LZ;  // domain size
    double dt;          // time step
};

class PFBaseClass {
public:
    // "CHBasic"/"CHBasicGPU": the GPU Cahn-Hilliard model; "TIPSphil",
    // "TIPSbathPHIL", "SIPS", "SIPSternary" (and their "...GPU" names): the
    // variable-mobility models
    static PFBaseClass* PFFactory(const CommonParams&, const InputFile&);

    virtual void initPhaseField() = 0;
    virtual void updatePhaseField() = 0;
    virtual void outputPhaseField() = 0;
    virtual void setTimeStep(int) = 0;

    virtual ~PFBaseClass() {}
};

// One phase-field application: parameters from the Domain/Time/Output
// sections, the model from PFApp/type.
class PFApp {
public:
    explicit PFApp(const InputFile& in);
    void initSystem();
    void stepForward(int step);
    void writeOutput(int step);
    const CommonParams& params() const { return p; }

private:
    CommonParams p{};
    int current_step = 0;
    std::unique_ptr<PFBaseClass> pf_object;
};
