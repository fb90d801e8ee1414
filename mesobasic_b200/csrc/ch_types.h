// Types shared by the step kernels and the host engine.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mg {

// a thread of the step kernel owns 32 bytes of one row: 8 floats or 4 doubles
constexpr int kStripBytes = 32;
// largest CTA of the step kernel: 640 threads for the fixed-width variants
// (at most 102 registers a thread), 512 for the generic one (128 registers)
constexpr int kMaxBlock = 640;
constexpr int kMaxBlockGeneric = 512;

enum JobFlags : int {
    JF_PER_X = 1 << 0,
    JF_PER_Y = 1 << 1,
    JF_PER_Z = 1 << 2,
    JF_DIV_X = 1 << 3,  // divide by dx^2 (dx^2 not a power of two), FP64 only
    JF_DIV_Y = 1 << 4,
    JF_DIV_Z = 1 << 5,
    JF_MASS = 1 << 6,  // FP32 mass-defect feedback (exact nudges, see kNudge)
    JF_FLAT = 1 << 7,  // logical ny == 1
    JF_SIMPLE = 1 << 8,  // all axes periodic, equal spacing (FP64: unit spacing)
};

enum DeviceError : int {
    DEV_OK = 0,
    DEV_TMA_TIMEOUT = 1,  // a TMA completion wait ran out of polls
};

// FP32 mass feedback: after every mass_every-th step the kernel sums the
// stored field in FP64 and adds round((target - sum) / kNudge) nudges of
// kNudge to consecutive sites of the new field at once.  The rounding defect
// of the interval since the last measure (the change of stored mass the
// nudges did not make) gives a per-step defect d, and each step of the next
// interval adds round(-d / kNudge) nudges inside the stencil (a window whose
// start moves by a fixed stride every step).  Rounding losses are systematic
// while the field evolves slowly, so predicting them keeps the stored mass
// on target between measurements.  kNudge = 2^-23 is a multiple
// of the unit in the last place of every float below 2 in magnitude, so each
// nudge is exact there and the stored sum meets the target to within one
// step's rounding.
constexpr float kNudge = 1.1920928955078125e-7f;  // 2^-23

// The stored mass is measured the same way by the step kernel and at upload,
// independent of the decomposition: each value is rounded to the nearest
// multiple of 2^-32 (strip_mass, exact for |c| < 2^12) and the integers are
// added (integer addition does not depend on order).
constexpr float kMassScale = 4294967296.0f;  // 2^32

// Which per-site chemical potential and mobility a variable-mobility job
// takes (the update, div(mob grad mu) with harmonic-mean face mobilities, is
// the same for all).
enum FhModel : int {
    kFhRamp = 0,    // TIPSphil::updatePhaseField (TIPSphil.cpp:113-211), uniform quench
    kFhBath = 1,    // TIPSbathPHIL (TIPSbathPHIL.cpp:114-208), 1-D bath temperature along x
    kFhSips = 2,    // SIPS::updatePhaseField (SIPS.cpp:130-249), erf non-solvent front along x
    kFhLinear = 3,  // one field of SIPSternary::updatePhaseField (SIPSternary.cpp:132-278):
                    // mu = 0.0 - K*lap(c), constant mobility
};

// Parameters and work fields of a variable-mobility job.  TIPSphil and
// TIPSbathPHIL: the Flory-Huggins chemical potential and Phillies mobility
// (constructor defaults TIPSphil.cpp:41-59); SIPS adds chiPS, chiPN, chiCond,
// phiCutoff and NSdepth (SIPS.cpp:22-59); the SIPSternary field takes kappa as
// its K and Mconst as its mobility.
struct FhDev {
    double alpha, beta, N, A, Tinit, Tbath, Tcrystal, nu, gamma, D0, Mweight, Mvolume;
    long long nstep;  // Time/nstep: length of the temperature ramp
    int model;        // FhModel
    double thermCond;
    double* mu;       // chemical potential of the step being taken
    double* mob;      // mobility of the step being taken
    double chiPS, chiPN, chiCond;  // SIPS: chi from chiPN (bath) toward chiPS behind an erf front
    int NSdepth;                   // SIPS: planes x < NSdepth are the non-solvent bath (chi = chiPN)
    double phiCutoff;              // SIPS: no noise where c >= phiCutoff after the step
    double Mconst;                 // kFhLinear: the constant mobility
};

// Per-job state in device memory.  The host fills the parameters;
// `nudge_*`, `mass_last`, `step`, `done` and `err` are updated by the kernels.
struct alignas(16) JobDev {
    void* buf[2];               // ping-pong fields; step s reads buf[s & 1]
    const CUtensorMap* tmap;    // [2 buffers][body map (bw x ty x 1), row map (bw x 1 x 1)]
    long long* partial;         // per-item stored-mass sums in 2^-32 units (JF_MASS)
    int nx, ny, nz;             // logical dims (2-D jobs: nx, 1, ny)
    int ty;                     // output rows per tile (1 when flat)
    int ntile, nchunk;          // y tiles x z chunks = items
    int flags;                  // JobFlags
    int bw;                     // TMA box width = shared-memory piece width
    double cx, cy, cz;          // 1/d^2 (multiply) or d^2 (divide when JF_DIV_*)
    double kap, dtM;            // kappa, dt*M
    double dtM_dt;              // dt (the noise term's factor)
    double inv_nsites;          // 1 / (nx*ny*nz)
    double mass_target;         // sum(c) of the uploaded field (JF_MASS)
    long long nudge_begin;      // first site of the next step's nudge window (JF_MASS)
    long long nudge_count;      // sites in the window; the sign is the nudge's
    double mass_last;           // sum(c) after the last measured step (JF_MASS)
    long long nudge_applied;    // nudges (signed count) applied since the last measured step
    long long nudge_rest;       // nudges for each unmeasured step of the interval (signed count)
    int mass_every;             // JF_MASS: the field is summed after steps s with (s + 1) % mass_every == 0
    FhDev* fh;                  // variable-mobility model (null: Cahn-Hilliard with constant M)
    double noise;               // per-step noise strength (0: none; negative: the increments negated)
    double noise_cutoff;        // sites with c >= noise_cutoff after the step get no noise (SIPS)
    unsigned long long noise_seed;
    long long noise_step;       // the last step whose noise has been added
    unsigned int noise_done;    // blocks of the running noise launch finished
    long long step;             // steps taken
    long long target;           // the job stops stepping here
    unsigned int done;          // items finished in the running launch
    int err;                    // DeviceError
};

struct StepArgs {
    JobDev* jobs;           // all job slots of the engine
    const int* job_slot;    // [njobs] slot of the launch's job j
    const int* item_begin;  // [njobs + 1], items of job j: [item_begin[j], item_begin[j+1])
    int njobs;
    int nitems;
    int cplane;             // shared-memory elements per c plane (max over jobs)
    int mplane;             // shared-memory elements per mu plane (max over jobs)
    long long spin_limit;   // polls before a TMA wait gives up
    int* err;               // launch-wide error word (max of DeviceError)
    uint32_t tx_extra;      // test hook: bytes expected beyond a plane (0 in use);
                            // nonzero makes every TMA wait run out
    const int* counts;      // non-null: device [njobs, nitems] read at kernel
                            // start in place of the two fields above (lanes
                            // whose job list is rewritten between graph replays)
};

#ifdef __CUDACC__
// the launch's job and item counts (StepArgs::counts, else the fields)
__device__ __forceinline__ void step_counts(StepArgs& a)
{
    if (a.counts) {
        a.njobs = __ldg(a.counts);
        a.nitems = __ldg(a.counts + 1);
    }
}
#endif

// Shared-memory header: NBUF mbarriers, broadcast words, reduction scratch.
struct SmemHead {
    uint64_t bar[8];
    long long step;
    int flag;
    int pad;
    long long nudge_begin, nudge_count;
    double2 red[32];
};

// Diagnostics of the current field of one job (see ch_diag_partial).
struct Diag {
    double mass, energy, abs_mass, max_abs, nonfinite;
};

constexpr int kDiagBlocks = 592;   // 4 x 148 SMs
constexpr int kDiagThreads = 256;

}  // namespace mg
