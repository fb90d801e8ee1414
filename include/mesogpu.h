/*
 * mesogpu.h -- C ABI of libmesogpu.so, the B200 (sm_100a) Cahn-Hilliard
 * phase-field step of mesoBasic's src/phase_field, re-designed for the GPU.
 *
 * Conventions
 *   - Every int-returning call returns MG_OK (0) or a negative MG_E* code;
 *     mg_last_error() gives a message for the calling thread.  No C++
 *     exception crosses this boundary.
 *   - Fields cross the boundary as dense host arrays of double, x fastest,
 *     no ghost nodes: value of node (i,j,k) (0-based) at i + nx*(j + ny*k).
 *     The reference's SfieldFD stores z fastest with one ghost layer
 *     (SfieldFD.cpp:26-64); a caller holding such an array converts it.
 *   - The library owns device memory; the caller owns host buffers.  Host
 *     buffers in pinned memory (cudaHostAlloc) transfer fastest.
 *   - A handle is driven by one host thread at a time.  Calls that enqueue
 *     GPU work return before it finishes; mg_*_sync waits (with a limit).
 *   - Two-dimensional runs are nz == 1, as in the reference (SfieldFD keeps
 *     z ghosts equal to the single plane, SfieldFD.cpp:135-140).
 */
#ifndef MESOGPU_H
#define MESOGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define MG_OK 0
#define MG_EINVAL (-1)      /* bad argument or unsupported configuration */
#define MG_ENOMEM (-2)      /* device or host allocation failed / over budget */
#define MG_ECUDA (-3)       /* a CUDA runtime or driver call failed */
#define MG_ETIMEOUT (-4)    /* a bounded wait ran out */
#define MG_ENONFINITE (-5)  /* the field holds NaN or Inf */
#define MG_EDEVICE (-6)     /* a kernel reported an error (e.g. a bounded device wait ran out) */
#define MG_ENOTFOUND (-7)   /* unknown job id */

#define MG_FP64 0
#define MG_FP32 1

/* One simulation.  Keys of the reference input file in brackets. */
typedef struct {
    int nx, ny, nz;        /* grid [Domain/nx,ny,nz] */
    double dx, dy, dz;     /* spacing [Domain/dx,dy,dz] */
    double dt;             /* time step [Time/dt] */
    double M;              /* constant mobility [PFApp/M] */
    double kappa;          /* gradient coefficient [PFApp/kap] */
    int bx, by, bz;        /* 1 periodic, 0 no-flux [PFApp/bx,by,bz] (SfieldFD.cpp:187-251) */
    int precision;         /* MG_FP64: bit-identical to the reference build;
                              MG_FP32: FP32 field, FP64 reductions */
    int mass_correct;      /* MG_FP32 only; 0: off.  K >= 1: after every K-th
                              step the kernel sums the stored field in FP64
                              and adds the defect (target - sum) back at once
                              as exact nudges of 2^-23 on a window of sites;
                              the steps in between add the rounding defect
                              per step the last interval showed, so rounding
                              errors of the field do not accumulate as a
                              drift of total mass.  The stored mass is on
                              target (to half a nudge) after every K-th step.
                              K = 1 measures every step and holds the
                              relative drift within 1e-10 at every step; the
                              Python mirror and the driver default to K = 1.
                              K = 4 costs a quarter of the measuring and is
                              on target at every 4th step only */
    double noise;          /* >0: after each step every site gets
                              c += dt * (noise * (u - 0.5)), u uniform in (0,1)
                              [PFApp/noiseStr] (TIPSphil.cpp:200-209); 0: off */
    unsigned long long noise_seed; /* key of the counter-based generator
                              (Philox4x32-10): u depends on (seed, site, step)
                              only, so it is the same alone, batched or served */
} mg_ch_params;

typedef struct {
    double mass;       /* sum(c) dV, compensated FP64 */
    double energy;     /* sum[(c^2-1)^2/4 + kappa/2 |grad+ c|^2] dV, compensated FP64 */
    double abs_mass;   /* sum|c| dV */
    double max_abs;    /* max |c| */
    long long nonfinite; /* sites holding NaN/Inf */
    long long step;    /* steps taken */
} mg_ch_stats;

/* Work decomposition of a job (see mg_autotune). */
typedef struct {
    int ty;      /* output rows per tile (3-D); 1 for 2-D jobs */
    int nchunk;  /* z chunks (2-D: row chunks) */
    int nbuf;    /* c planes in the shared-memory ring: 3, 4, 6 or 8 */
    int path;    /* 0 tiled TMA kernel, 1 generic per-site kernel */
} mg_tiling;

typedef struct mg_ch mg_ch_t;
typedef struct mg_batch mg_batch_t;
typedef struct mg_server mg_server_t;

/* Message of the last failed call on this thread ("" if none). */
const char* mg_last_error(void);

/* ----------------------------------------------------------------------
 * Single simulation: the GPU body of a PFBaseClass model.
 * -------------------------------------------------------------------- */

/* Allocates the two field buffers of one simulation on `device`.
 * Replaces: PFBaseClass::PFFactory + model constructor
 * (PFBaseClass.cpp:26-55, TIPSphil.cpp:24-60, SfieldFD.cpp:26-64). */
int mg_ch_create(const mg_ch_params* params, int device, mg_ch_t** out);

/* Uploads a field (nx*ny*nz doubles; converted to FP32 for MG_FP32 jobs)
 * and resets the step counter.  Replaces: the fill of c in
 * initPhaseField (TIPSphil.cpp:86-96). */
int mg_ch_set_field(mg_ch_t* h, const double* host);

/* Enqueues nsteps explicit steps (one fused kernel launch each, replayed
 * from a CUDA graph).  Replaces: nsteps calls of PFApp::stepForward ->
 * updatePhaseField (PFApp.cpp:91-107, TIPSphil.cpp:113-211). */
int mg_ch_step(mg_ch_t* h, int nsteps);

/* Waits for the enqueued work, at most timeout_us microseconds (<0: no
 * limit); reports kernel-side errors.  After it has returned MG_EDEVICE
 * (a bounded device wait ran out, so copies may have been in flight when
 * the kernel gave up) the handle refuses further steps with MG_EDEVICE:
 * destroy it and create a new one.  Replaces: MPI Barrier after a
 * step (TIPSphil.cpp:129,192) as the completion point. */
int mg_ch_sync(mg_ch_t* h, long long timeout_us);

/* Downloads the current field (waits for enqueued work).  Replaces: the
 * read of c in outputPhaseField -> SfieldFD::writeVTKFile (SfieldFD.cpp:363-430). */
int mg_ch_get_field(mg_ch_t* h, double* host);

/* Appends the current field to `path` as one legacy-VTK block (header +
 * "%.3f" lines, x fastest, skip rules), byte-identical to mg_vtk_write of
 * the downloaded field, but formatted on the GPU: only the text crosses to
 * the host.  Values of magnitude >= 4e12 give MG_EINVAL (mg_vtk_write takes
 * any value).  Waits for enqueued work.  Replaces: SfieldFD::writeVTKFile
 * (SfieldFD.cpp:363-430) called from outputPhaseField. */
int mg_ch_write_vtk(mg_ch_t* h, const char* path, const char* tag, int iskip, int jskip, int kskip);

/* Mass/energy diagnostics of the current field.  No reference counterpart
 * (the reference logs neither).  Returns MG_ENONFINITE if any site is not
 * finite (stats are still filled). */
int mg_ch_reduce(mg_ch_t* h, mg_ch_stats* out);

/* Radially binned structure factor S(k) = |FFT(c - <c>)|^2 / N of the
 * current field (cuFFT + binning kernel), nbins bins of width
 * dk = 2*pi/max(L); k[b] = mean |k| in bin b, S[b] = mean S in bin b;
 * *k1 = sum(|k| S)/sum(S) over every mode in the bins (k = 0 excluded).  No reference counterpart (FFTW is linked by the
 * reference but never executed, PFApp.cpp:46-48). */
int mg_ch_structure_factor(mg_ch_t* h, int nbins, double* k, double* S, double* k1);

/* The CUDA stream (cudaStream_t) the handle enqueues on, for event timing. */
void* mg_ch_stream(mg_ch_t* h);

/* Device pointer of the current field buffer (precision per params). */
void* mg_ch_field_device(mg_ch_t* h);

/* Steps taken (waits for enqueued work). */
long long mg_ch_steps(mg_ch_t* h);

int mg_ch_get_tiling(const mg_ch_t* h, mg_tiling* out);
/* Overrides the decomposition; validates it against the kernel limits.
 * Variable-mobility handles step on two per-site passes (path 1) by default;
 * path 0 selects the fused z-marching kernel (ty 0: its own tile choice),
 * which gives the same field bit for bit. */
int mg_ch_set_tiling(mg_ch_t* h, const mg_tiling* t);

/* Frees the device buffers.  Replaces: PFApp::~PFApp (PFApp.cpp:69-72). */
void mg_ch_destroy(mg_ch_t* h);

/* ----------------------------------------------------------------------
 * Variable mobility: the TIPSphil model (Flory-Huggins chemical potential,
 * Phillies mobility, div(mob grad mu) with harmonic-mean face mobilities).
 * -------------------------------------------------------------------- */

/* Keys of the reference input file in brackets, the reference defaults in
 * parentheses (TIPSphil.cpp:41-59). */
typedef struct {
    double alpha, beta;     /* chi = alpha/T + beta [PFApp/alpha (1), beta (1)] */
    double N;               /* polymer length [PFApp/N (100)] */
    double A;               /* c <= 0 branch of mu [PFApp/A (1)] */
    double Tinit, Tbath;    /* linear quench Tinit -> Tbath over nstep [PFApp/Tinit, Tbath (273)] */
    double Tcrystal;        /* mobility x 0.001 at or below it [PFApp/Tcrystal (273)] */
    double nu, gamma;       /* Phillies law D*exp(-gamma*phi^nu) [PFApp/nu (1), gamma (10)] */
    double D0;              /* diffusivity and mobility cap [PFApp/D0 (1e-7)] */
    double Mweight, Mvolume;/* phi -> g/L [PFApp/Mweight (100), Mvolume (0.1)] */
    long long nstep;        /* steps of the quench [Time/nstep] */
    int bath;               /* 0: uniform ramp (TIPSphil); 1: the 1-D bath profile of
                               TIPSbathPHIL, T = (Tinit-Tbath)*erf(i/(2*sqrt(thermCond*step*dt)))
                               + Tbath with i the 1-based x index (TIPSbathPHIL.cpp:118-121) */
    double thermCond;       /* [PFApp/thermCond (1)] */
} mg_fh_params;

/* A simulation stepped by the variable-mobility update of
 * TIPSphil::updatePhaseField (TIPSphil.cpp:113-211) instead of the constant-
 * mobility Cahn-Hilliard step: FP64 only (params->precision MG_FP64,
 * mass_correct 0); kappa is [PFApp/kap]; params->M is unused (the mobility
 * comes from the model); params->noise adds the reference's fluctuation term
 * (TIPSphil.cpp:200-209, [PFApp/noiseStr]).  Every other mg_ch_* call
 * applies.  Replaces: PFBaseClass::PFFactory returning TIPSphil or
 * TIPSbathPHIL (PFBaseClass.cpp:46-47). */
int mg_fh_create(const mg_ch_params* params, const mg_fh_params* fh, int device, mg_ch_t** out);

/* The mobility field of the last step taken (nx*ny*nz doubles, x fastest;
 * waits for enqueued work).  Replaces: the mob field TIPSphil writes at
 * PFApp/mobStep (TIPSphil.cpp:180-185). */
int mg_fh_mobility(mg_ch_t* h, double* host);

/* SIPS (SIPS.cpp): a binary polymer/solvent film in front of a non-solvent
 * bath.  Keys of the reference input file in brackets, the reference defaults
 * in parentheses (SIPS.cpp:22-59). */
typedef struct {
    double N;               /* polymer length [PFApp/N (100)] */
    double A;               /* c <= 0 branch of mu [PFApp/A (1)] */
    double Tinit;           /* kT = Tinit/273 [PFApp/Tinit (273.15)] */
    double chiPS, chiPN;    /* polymer-solvent and polymer-non-solvent chi [PFApp/chiPS (0.034), chiPN (2.5)] */
    double chiCond;         /* front diffusivity: chi = (chiPS-chiPN)*erf(i/(2*sqrt(chiCond*step*dt)))
                               + chiPN for x >= NSdepth, chiPN below (SIPS.cpp:164-170)
                               [PFApp/chiCond (1)] */
    double phiCutoff;       /* no noise where c >= phiCutoff [PFApp/phiCutoff (0.5)] */
    double nu, gamma;       /* Phillies law D0*exp(-gamma*phi^nu) [PFApp/nu (1), gamma (10)] */
    double D0;              /* [PFApp/D0 (1)] */
    double Mweight, Mvolume;/* phi -> g/L [PFApp/Mweight (100), Mvolume (0.1)] */
    int NSdepth;            /* x planes of the non-solvent bath [PFApp/NSdepth (0)] */
} mg_sips_params;

/* A simulation stepped by SIPS::updatePhaseField (SIPS.cpp:130-249): the
 * Flory-Huggins mu of the clamped concentration with chi(x, step) from the
 * erf front, Phillies mobility over the second derivative, clamped to
 * [1e-5, 1] and scaled by 0.95 + 0.25*log(1.0225 - (chi-chiPS)/(chiPN-chiPS)),
 * then div(mob grad mu) as mg_fh_create's.  FP64 only; kappa is [PFApp/kap];
 * params->M is unused; params->noise is [PFApp/noiseStr], skipped at sites
 * with c >= phiCutoff after the step.  chiPS == chiPN is refused (the
 * reference divides by their difference).  mg_fh_mobility returns the
 * mobility.  Replaces: PFBaseClass::PFFactory returning SIPS
 * (PFBaseClass.cpp:48). */
int mg_sips_create(const mg_ch_params* params, const mg_sips_params* sips, int device, mg_ch_t** out);

/* SIPSternary (SIPSternary.cpp): polymer c and non-solvent n [defaults
 * SIPSternary.cpp:21-63]. */
typedef struct {
    double Kpp, Knn;        /* gradient coefficients [PFApp/Kpp (1), Knn (1)] */
    double Mpp, Mnn;        /* mobilities [PFApp/Mpp (1), Mnn (1)] */
} mg_ternary_params;

/* The two fields of SIPSternary::updatePhaseField (SIPSternary.cpp:132-278)
 * as a batch of two jobs: job 0 is the polymer c, job 1 the non-solvent n.
 * In the reference the Flory-Huggins derivatives are assigned to variables
 * declared inside their branches (SIPSternary.cpp:175-216), so the chemical
 * potentials it uses are mu_c = 0.0 - Kpp*lap(c) and mu_n = 0.0 - Knn*lap(n),
 * with constant mobilities Mpp and Mnn; each field takes c += dt*div(M grad
 * mu) on its own, and that arithmetic is what runs here.  params->noise is
 * [PFApp/noiseStr]: c gets dt*noise*(r - 0.5), n the same increment negated
 * (SIPSternary.cpp:256-277).  FP64 only; params->kappa and M are unused.  The
 * mg_batch_* calls apply.  Replaces: PFBaseClass::PFFactory returning
 * SIPSternary (PFBaseClass.cpp:49). */
int mg_ternary_create(const mg_ch_params* params, const mg_ternary_params* t, int device, mg_batch_t** out);

/* Times candidate decompositions of `params` on `device` (scratch fields,
 * `trials` timed launches each) and returns the fastest.  Results are
 * cached per (shape, precision) in the process and, when the environment
 * variable MG_TUNE_CACHE names a file, in that JSON file, which
 * mg_ch_create consults.  No reference counterpart. */
int mg_autotune(const mg_ch_params* params, int device, int trials, mg_tiling* best, double* best_ms);

/* ----------------------------------------------------------------------
 * Host helpers over the reference's input surface.
 * -------------------------------------------------------------------- */

/* Seeded initial condition, reference loop order (x outer, then y, z):
 * uniform: co + amp*(u - 0.5), u = MT19937 u32 / 4294967295;
 * gaussian: co + amp*normal() (Box-Muller).  Replaces: the random fill of
 * TIPSphil::initPhaseField (TIPSphil.cpp:86-96) with the reference's Rand
 * (rand.cpp:24-94) seeded by `seed`. */
int mg_ic_generate(const int dims[3], double co, double amp, int gaussian, unsigned seed, double* out);

/* Appends one legacy-VTK block (header + `%.3f` values, x fastest, skip
 * rules) to `path`, byte-identical to a single-rank
 * SfieldFD::writeVTKFile(tag, step, iskip, jskip, kskip)
 * (SfieldFD.cpp:363-430). */
int mg_vtk_write(const char* path, const char* tag, const double* field, const int dims[3], int iskip, int jskip,
                 int kskip);

/* ----------------------------------------------------------------------
 * Batch: many independent simulations of uneven sizes and parameters
 * stepped by one persistent launch per precision class and step, replayed
 * from a CUDA graph.  No reference counterpart (the reference runs one
 * simulation per process).
 * -------------------------------------------------------------------- */
int mg_batch_create(const mg_ch_params* jobs, int njobs, int device, mg_batch_t** out);
int mg_batch_set_field(mg_batch_t* b, int job, const double* host);
int mg_batch_step(mg_batch_t* b, int nsteps);
int mg_batch_sync(mg_batch_t* b, long long timeout_us);
int mg_batch_get_field(mg_batch_t* b, int job, double* host);
int mg_batch_reduce(mg_batch_t* b, int job, mg_ch_stats* out);
/* mg_ch_write_vtk for one job of the batch. */
int mg_batch_write_vtk(mg_batch_t* b, int job, const char* path, const char* tag, int iskip, int jskip, int kskip);
void* mg_batch_stream(mg_batch_t* b);
/* Items (tiles) and persistent CTAs of the batch's launches. */
int mg_batch_info(const mg_batch_t* b, int* nitems, int* nctas, int* nlaunch_per_step);
/* Chooses the batch's tiles by measurement: every job is tiled for CTAs of
 * about `threads` threads and z-chunks of about `planes` planes (the same
 * targets for all jobs, so the CTAs of the shared launch are equally full);
 * each candidate pair is timed over `trials` steps of a scratch copy of the
 * batch (same shapes and parameters, zero fields, so the batch's own fields
 * and step counts are untouched).  The best pair re-tiles the batch (results
 * do not depend on the tiling) and is stored in the tuning cache under the
 * batch's composition, where mg_batch_create finds it for later batches of
 * the same mix.  No reference counterpart. */
int mg_batch_autotune(mg_batch_t* b, int trials, int* threads, int* planes, double* ms_per_step);
void mg_batch_destroy(mg_batch_t* b);

/* ----------------------------------------------------------------------
 * Server: continuous batching of simulation jobs under an HBM budget.
 * A background thread admits queued jobs as memory and slots free up,
 * steps all admitted jobs together (each to its own step count), and
 * retires finished ones.  No reference counterpart.
 * -------------------------------------------------------------------- */
typedef struct {
    long long submitted, completed, failed, running, queued;
    double p50_ms, p99_ms;       /* completion latency, arrival -> result ready */
    double mean_ms;
    double sims_per_hour;        /* completed / wall time since the first arrival */
    double site_updates_per_s;   /* sum(sites*steps) of completed jobs / wall time */
    double hbm_in_use_gb, hbm_peak_gb;
    /* where the worker thread's time went: enqueueing and waiting for step
       ticks (GPU busy), admitting jobs (allocation, upload), retiring jobs
       (download, diagnostics); ticks run, launch-set rebuilds (each
       recaptures the step graph) and job-set changes absorbed without one
       (the launch lanes' device tables rewritten, the graphs kept) */
    double step_s, admit_s, retire_s;
    long long ticks, rebuilds, refreshes;
    /* saturated rate: site-updates per second over the ticks that began
       with jobs still queued (every slot or the HBM budget taken), each
       timed from its start to the next tick's start, and how many ticks
       that was (0 when the queue never backed up) */
    double sat_site_updates_per_s;
    long long sat_ticks;
    /* device time of the ticks (CUDA events around each tick's steps on the
       engine's stream): against the wall time, how long the GPU worked */
    double gpu_s;
} mg_server_stats;

#define MG_JOB_QUEUED 0
#define MG_JOB_RUNNING 1
#define MG_JOB_DONE 2
#define MG_JOB_FAILED 3

int mg_server_create(int device, double hbm_budget_gb, int max_jobs_in_flight, int steps_per_tick,
                     mg_server_t** out);
/* Copies `ic_host` (nx*ny*nz doubles) and queues the job; returns its id. */
int mg_server_submit(mg_server_t* s, const mg_ch_params* params, const double* ic_host, long long nsteps,
                     long long* job_id);
int mg_server_poll(mg_server_t* s, long long job_id, int* state);
/* Waits (bounded) for the job, then copies its final field (may be NULL)
 * and stats and releases it. */
int mg_server_result(mg_server_t* s, long long job_id, long long timeout_us, double* field_out,
                     mg_ch_stats* stats);
int mg_server_stats_get(mg_server_t* s, mg_server_stats* out);
/* Stops accepting jobs, finishes the admitted ones, joins the thread. */
void mg_server_destroy(mg_server_t* s);

/* ----------------------------------------------------------------------
 * Diagnostics without allocation.  No reference counterpart.
 * -------------------------------------------------------------------- */

/* The statistics of mg_ch_reduce (mass, |c|, free energy, max|c|,
 * non-finite count; out->step is set to -1) of a dense x-fastest field
 * already in device memory on `device` (FP64 or FP32 per params->precision;
 * nx, ny, nz, spacings, kappa and bx/by/bz are read from params), computed
 * on `stream` (a cudaStream_t; NULL is the default stream) and waited for at
 * most timeout_us microseconds (<0: no limit).
 *
 * It allocates nothing -- no cudaMalloc/cudaFree, no allocating library
 * call -- for callers that cannot allocate: a thread that shares the device
 * with running simulations (an allocation may synchronise the device), a
 * service whose HBM is fully committed by its admission budget, or code that
 * holds only a borrowed device pointer and no handle.  Its scratch is one
 * fixed device array of about 256 KB per process, which bounds the field to
 * at most 4096 planes (nz for 3-D fields, ny for 2-D ones); larger fields
 * give MG_EINVAL (use mg_ch_reduce).  Every call looks up that array's
 * address on `device`; the first call on a device also loads the library's
 * device code there and should come before any stream capture there.
 * Calls that overlap in time on one device share the array and race: issue
 * them one at a time.  After MG_ETIMEOUT the kernel is still on `stream`:
 * synchronise that stream before calling again on the device.  Sums are
 * compensated FP64 in a fixed order; they agree with mg_ch_reduce to
 * rounding (the two sum in different orders). */
int mg_field_stats_noalloc(const void* field_dev, const mg_ch_params* params, int device, void* stream,
                           long long timeout_us, mg_ch_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* MESOGPU_H */
