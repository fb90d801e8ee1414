// CHBasicGPU.hpp -- Cahn-Hilliard model whose step runs on a B200 through
// libmesogpu.so (include/mesogpu.h of mesobasic_b200).
//
// The drop-in file for the reference tree: copy it to
// src/phase_field/PFTypes/CHBasicGPU.hpp and add one line to
// PFBaseClass::PFFactory (PFBaseClass.cpp:26-55):
//     if (pf_type == "CHBasicGPU") return new CHBasicGPU(p,input_params);
// It implements the four PFBaseClass virtuals (PFBaseClass.hpp:14-41) that
// PFApp drives (PFApp.cpp:78-121): the field lives on the GPU, steps are
// counted in updatePhaseField and enqueued together (CUDA-graph replays)
// when an output needs the field, and outputPhaseField appends legacy VTK
// in the reference's format (SfieldFD.cpp:363-430).
//
// Input keys (PFApp/): M, kap, bx, by, bz, co, noise_amp, seed as the
// reference's models read them; precision (fp64 | fp32) and device are new.
# ifndef CHBASICGPU_H
# define CHBASICGPU_H

# include "../PFBaseClass.hpp"
# include "../../utils/CommonParams.h"
# include "../../utils/GetPot"
# include "mesogpu.h"
# include <cstdio>
# include <stdexcept>
# include <string>
# include <vector>

class CHBasicGPU : public PFBaseClass {
public:
   CHBasicGPU(const CommonParams& pin, const GetPot& in) : p(pin)
   {
      if (p.np != 1) throw std::runtime_error("CHBasicGPU: run with one MPI rank per simulation");
      mg_ch_params gp = {};
      gp.nx = p.NX; gp.ny = p.NY; gp.nz = p.NZ;
      gp.dx = p.dx; gp.dy = p.dy; gp.dz = p.dz; gp.dt = p.dt;
      gp.M = in("PFApp/M", 1.0);
      gp.kappa = in("PFApp/kap", 1.0);
      gp.bx = in("PFApp/bx", 1); gp.by = in("PFApp/by", 1); gp.bz = in("PFApp/bz", 1);
      gp.precision = std::string(in("PFApp/precision", "fp64")) == "fp32" ? MG_FP32 : MG_FP64;
      gp.mass_correct = gp.precision == MG_FP32 ? 1 : 0;  // FP32: mass measured and corrected every step
      co = in("PFApp/co", 0.0);
      amp = in("PFApp/noise_amp", 0.1);
      seed = (unsigned)in("PFApp/seed", 42);
      check(mg_ch_create(&gp, in("PFApp/device", 0), &h));
      dims[0] = gp.nx; dims[1] = gp.ny; dims[2] = gp.nz;
      step = 0;
      pending = 0;
   }
   ~CHBasicGPU() { mg_ch_destroy(h); }

   void initPhaseField()
   {
      std::vector<double> ic((size_t)dims[0] * dims[1] * dims[2]);
      check(mg_ic_generate(dims, co, amp, 0, seed, ic.data()));
      check(mg_ch_set_field(h, ic.data()));
      outputPhaseField();                     // step 0, as TIPSphil.cpp:102-103
   }
   void updatePhaseField() { ++pending; }      // enqueued at the next output
   void setTimeStep(int s) { step = s; }
   void outputPhaseField()
   {
      if (pending) { check(mg_ch_step(h, pending)); pending = 0; }
      std::vector<double> c((size_t)dims[0] * dims[1] * dims[2]);
      check(mg_ch_get_field(h, c.data()));
      char path[64];
      std::snprintf(path, sizeof path, "vtkoutput/c_%d.vtk", step);
      check(mg_vtk_write(path, "c", c.data(), dims, p.iskip, p.jskip, p.kskip));
   }

private:
   static void check(int rc) { if (rc != MG_OK) throw std::runtime_error(mg_last_error()); }
   CommonParams p;
   mg_ch_t* h;
   int dims[3], step, pending;
   double co, amp;
   unsigned seed;
};

# endif
