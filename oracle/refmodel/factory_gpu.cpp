// Test infrastructure: the reference's plugin factory with the drop-in GPU
// model registered, as a maintainer would add it (one line in
// PFBaseClass::PFFactory, PFBaseClass.cpp:26-55).  Linked with the
// reference's own main, MesoExecute, PFApp and model sources into
// oracle/_ref/meso_ref_gpu, so the reference driver itself steps on the GPU.
// "CHBasic" stays the CPU oracle model; every other type goes to the
// reference factory compiled under another name (see factory.cpp).
#include <string>
#include "CHBasic.hpp"
#include "CHBasicGPU.hpp"
#include "PFBaseClass.hpp"

extern PFBaseClass* mb_registered_factory(const CommonParams&, const GetPot&) __asm__(
    "_ZN11PFBaseClass20PFFactory_registeredERK12CommonParamsRK6GetPot");

PFBaseClass* PFBaseClass::PFFactory(const CommonParams& p, const GetPot& input_params)
{
    std::string pf_type = input_params("PFApp/type", "CHBasic");
    if (pf_type == "CHBasic") return new CHBasic(p, input_params);
    if (pf_type == "CHBasicGPU") return new CHBasicGPU(p, input_params);
    return mb_registered_factory(p, input_params);
}
