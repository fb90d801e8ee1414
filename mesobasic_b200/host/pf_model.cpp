// See pf_model.hpp.
#include "pf_model.hpp"

#include <stdexcept>

#include "chbasic_gpu.hpp"
#include "sips_gpu.hpp"
#include "tipsphil_gpu.hpp"

PFBaseClass* PFBaseClass::PFFactory(const CommonParams& p, const InputFile& in)
{
    // PFBaseClass.cpp:33: the type defaults to "CHBasic"
    const std::string type = in("PFApp/type", "CHBasic");
    if (type == "CHBasic" || type == "CHBasicGPU") return new CHBasicGPU(p, in);
    if (type == "TIPSphil" || type == "TIPSphilGPU") return new TIPSphilGPU(p, in);
    if (type == "TIPSbathPHIL" || type == "TIPSbathPHILGPU") return new TIPSphilGPU(p, in, true);
    if (type == "SIPS" || type == "SIPSGPU") return new SIPSGPU(p, in);
    if (type == "SIPSternary" || type == "SIPSternaryGPU") return new SIPSternaryGPU(p, in);
    throw std::invalid_argument("PFApp/type '" + type +
                                "' is not provided by meso_b200 (available: CHBasic, CHBasicGPU, TIPSphil, "
                                "TIPSphilGPU, TIPSbathPHIL, TIPSbathPHILGPU, SIPS, SIPSGPU, SIPSternary, "
                                "SIPSternaryGPU)");
}

PFApp::PFApp(const InputFile& in)
{
    // the reads of PFApp.cpp:17-29, same keys and defaults
    p.NX = in("Domain/nx", 1);
    p.NY = in("Domain/ny", 1);
    p.NZ = in("Domain/nz", 1);
    p.dx = in("Domain/dx", 1.0);
    p.dy = in("Domain/dy", 1.0);
    p.dz = in("Domain/dz", 1.0);
    p.dt = in("Time/dt", 1.0);
    p.nstep = in("Time/nstep", 1);
    p.numOutputs = in("Output/numOutputs", 1);
    p.iskip = in("Output/iskip", 1);
    p.jskip = in("Output/jskip", 1);
    p.kskip = in("Output/kskip", 1);
    p.LX = p.NX * p.dx;
    p.LY = p.NY * p.dy;
    p.LZ = p.NZ * p.dz;
    // one process, whole domain (PFApp.cpp:35-52 with np = 1)
    p.np = 1;
    p.rank = 0;
    p.nbrL = 0;
    p.nbrR = 0;
    p.nx = p.NX;
    p.ny = p.NY;
    p.nz = p.NZ;
    p.xOff = 0;
    pf_object.reset(PFBaseClass::PFFactory(p, in));
}

void PFApp::initSystem() { pf_object->initPhaseField(); }

void PFApp::stepForward(int step)
{
    current_step = step;
    pf_object->setTimeStep(current_step);
    pf_object->updatePhaseField();
}

void PFApp::writeOutput(int step)
{
    pf_object->setTimeStep(step);
    pf_object->outputPhaseField();
}
