// Test infrastructure: registers CHBasic with the reference's plugin factory
// without editing or copying PFBaseClass.cpp.
//
// The oracle Makefile compiles the reference's PFBaseClass.cpp with
// -DPFFactory=PFFactory_registered, so its factory (PFBaseClass.cpp:26-55,
// which knows TIPSphil, TIPSbathPHIL, SIPS and SIPSternary) is emitted under
// that name.  This file defines PFBaseClass::PFFactory, the symbol PFApp
// calls (PFApp.cpp:58): it answers "CHBasic" (the reference's default type
// string, PFBaseClass.cpp:34) and hands every other type to the renamed
// reference factory.  GCC's asm label binds the renamed static member, whose
// mangled name the Makefile checks with nm.
#include <string>
#include "CHBasic.hpp"
#include "PFBaseClass.hpp"

extern PFBaseClass* mb_registered_factory(const CommonParams&, const GetPot&) __asm__(
    "_ZN11PFBaseClass20PFFactory_registeredERK12CommonParamsRK6GetPot");

PFBaseClass* PFBaseClass::PFFactory(const CommonParams& p, const GetPot& input_params)
{
    std::string pf_type = input_params("PFApp/type", "CHBasic");
    if (pf_type == "CHBasic") return new CHBasic(p, input_params);
    return mb_registered_factory(p, input_params);
}
