// Test infrastructure: the plain Cahn-Hilliard model for the reference CPU
// build.  It is compiled together with the reference's own sources (SfieldFD,
// Rand, PFBaseClass, PFApp, MesoExecute) into oracle/_ref/ and is the
// oracle the GPU path is compared against; nothing in the product links it.
//
// The reference factory names "CHBasic" as its default type but the class
// is absent (PFBaseClass.cpp:9,34,40).  This class fills that slot, following
// the step structure of TIPSphil::updatePhaseField (TIPSphil.cpp:113-211)
// with the Flory-Huggins terms replaced by the plain double-well
// f'(c) = c^3 - c, a constant mobility M and no per-step noise:
//
//   c.updateBoundaries(bx,by,bz)                      TIPSphil.cpp:128
//   mu = (c*c*c - c) - kap*c.Laplacian(ndx)           TIPSphil.cpp:135-147
//   mu.updateBoundaries(bx,by,bz)                     TIPSphil.cpp:190
//   c += (dt*M) * mu.Laplacian()                      TIPSphil.cpp:194
#ifndef MB_ORACLE_CHBASIC_H
#define MB_ORACLE_CHBASIC_H

#include <string>
#include "PFBaseClass.hpp"
#include "PFUtils/SfieldFD.hpp"

class CHBasic : public PFBaseClass {
   private:
    const CommonParams& p;
    int current_step;
    int nx, ny, nz;
    int deli, delj, delk;
    double co, M, kap;
    double noise_amp;
    std::string noise_type;
    unsigned seed;
    bool bx, by, bz;
    bool init_output;
    bool vtk;
    std::string dump_prefix;
    SfieldFD c;

   public:
    CHBasic(const CommonParams&, const GetPot&);
    ~CHBasic();
    void initPhaseField();
    void updatePhaseField();
    void outputPhaseField();
    void setTimeStep(int step) { current_step = step; }

    // Harness access to the local slab as a dense x-fastest array
    // (index x + nx*(y + ny*z)), without ghost nodes.
    void setField(const double* dense);
    void getField(double* dense) const;

    // Seeded initial condition over the GLOBAL grid, drawn from the
    // reference's Mersenne twister (rand.cpp) in the reference loop order
    // (x outer, then y, then z; TIPSphil.cpp:86-96):
    //   uniform:  c = co + amp*(u - 0.5),  u = Rand::uniform() in [0,1]
    //   gaussian: c = co + amp*Rand::normal()
    // Written dense x-fastest into out[NX*NY*NZ].
    static void generateIC(int NX, int NY, int NZ, double co, double amp, bool gaussian,
                           unsigned seed, double* out);
};

#endif
