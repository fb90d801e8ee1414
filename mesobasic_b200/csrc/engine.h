// Host-side engine behind the C ABI: owns device memory, job slots, the
// launch groups of the fused step kernel and their CUDA graphs.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "ch_types.h"
#include "mesogpu.h"

namespace mg {

// ---- error reporting (thread-local message, C-ABI return codes)
int fail(int code, const char* fmt, ...);
int mg_env_int(const char* name, int def);  // a positive integer from the environment, else def
void clear_error();
const char* last_error();

#define MG_CUDA(call)                                                                                    \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return ::mg::fail(MG_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                              __LINE__);                                                                 \
    } while (0)

#define MG_TRY(call)                 \
    do {                             \
        int rc_ = (call);            \
        if (rc_ != MG_OK) return rc_; \
    } while (0)

using StepKernel = void (*)(StepArgs);

struct DevInfo {
    int sms = 0;
    size_t smem_optin = 0;
    size_t total_mem = 0;
    int major = 0, minor = 0;
};
int device_info(int device, DevInfo* out);

// Geometry of one job as the kernels see it.
struct Geometry {
    int lnx = 0, lny = 0, lnz = 0;  // logical dims (2-D runs as nx, 1, ny)
    bool flat = false;
    double lsx = 1, lsy = 1, lsz = 1;  // logical spacing
    int perx = 1, pery = 1, perz = 1;  // logical periodic flags
    size_t n = 0;
    int es = 8;  // element size
};
int make_geometry(const mg_ch_params& p, Geometry* g);
int validate_params(const mg_ch_params& p);

// Resource needs of a tiling on a geometry.
struct TilePlan {
    bool tma_ok = false;  // the tiled kernel can take this shape
    int block = 0;        // threads used by a tile
    int cplane = 0, mplane = 0;
    size_t smem = 0;
    int ntile = 0, nitems = 0;
};
int plan_tiling(const Geometry& g, const mg_tiling& t, const DevInfo& d, TilePlan* out);
int plan_fh_tiling(const Geometry& g, const mg_tiling& t, const DevInfo& d, TilePlan* out);
bool fh_shape_ok(const Geometry& g);
bool tma_shape_ok(const Geometry& g);
mg_tiling default_tiling(const Geometry& g, const DevInfo& d, int device);
std::string tune_key(const Geometry& g);
// tiling of a job that shares launches: CTAs of about `threads` threads,
// z-chunks of about `planes` planes
mg_tiling batch_tiling_for(const Geometry& g, const DevInfo& d, int device, int threads, int planes);
bool tune_lookup(const std::string& key, mg_tiling* t);
void tune_store(const std::string& key, const mg_tiling& t, double ms);

struct Job {
    mg_ch_params p{};
    Geometry g;
    mg_tiling tiling{};
    TilePlan plan;
    void* buf[2] = {nullptr, nullptr};
    CUtensorMap* d_tmap = nullptr;  // 4 maps
    long long* d_partial = nullptr;
    FhDev* d_fh = nullptr;        // variable-mobility model (mg_fh_create, mg_sips_create, mg_ternary_create)
    double* d_mu = nullptr;       // its chemical potential ...
    double* d_mob = nullptr;      // ... and mobility fields
    double noise_cutoff = __builtin_huge_val();  // no noise where c >= this after a step (SIPS)
    bool noise_negate = false;    // add the negated noise increments (SIPSternary's second field)
    int slot = -1;
    long long target = -1;  // device step target (-1: unbounded)
    size_t device_bytes() const;
};

class Engine {
   public:
    Engine() = default;
    ~Engine();
    int init(int device, int capacity);

    // job lifetime: allocate buffers + maps, take a slot
    // `fh`: a variable-mobility job; its parameters (mu and mob are set here).
    // `noise_negate`: the job adds the negated noise increments.
    int add_job(const mg_ch_params& p, long long target, Job** out, const FhDev* fh = nullptr,
                bool noise_negate = false);
    int mobility(Job* j, double* host);  // last step's mobility (variable-mobility jobs)
    void remove_job(Job* j);  // releases the job; its device memory is freed at the next rebuild
    int set_tiling(Job* j, const mg_tiling& t);

    int upload(Job* j, const double* host, long long target);  // resets step
    // Admission beside running steps: between begin_admission and
    // end_admission, add_job and upload issue their device work on a stream
    // of their own with staging buffers of their own, so they overlap the
    // steps in flight on `stream` (the new jobs join the launches at the next
    // enqueue_steps).  end_admission waits for that work.  Slots of removed
    // jobs are reused only after the next rebuild, when no launch in flight
    // still names them.
    int begin_admission();
    int end_admission();
    int download(Job* j, double* host);                         // syncs
    int diagnostics(Job* j, mg_ch_stats* out);                  // syncs
    // The same for a job that has reached its step target, on a side stream
    // and without waiting for the steps in flight on the engine stream: the
    // kernels skip a finished job's items, so its field and slot stay as
    // they are.  One thread at a time (they share the staging buffers).
    int download_finished(Job* j, double* host);
    int diagnostics_finished(Job* j, mg_ch_stats* out);
    // appends the job's current field as legacy VTK, formatted on the GPU (vtk_device.cu)
    int write_vtk(Job* j, const char* path, const char* tag, int iskip, int jskip, int kskip);
    int structure_factor(Job* j, int nbins, double* k, double* S, double* k1);
    int enqueue_steps(int nsteps);  // all jobs, one launch group set per step
    int sync(long long timeout_us);
    int read_state(Job* j, JobDev* out);  // syncs; mutable state of the slot

    int nitems_total() const;
    int nctas_total() const;
    int nlaunch_per_step() const;
    long long rebuilds() const { return rebuilds_; }  // launch-set rebuilds (graphs recaptured) so far
    long long refreshes() const { return refreshes_; }  // job-set changes absorbed by rewriting lane tables

    int device = 0;
    // jobs share launches (batch, server): tile every job for equally full
    // CTAs (batch_tiling_for) instead of for the fastest standalone run
    bool batch_tiling = false;
    // threads per CTA and z-chunk length of that tiling: big tiles and long
    // chunks (fewer, longer items) suit a batch that fills the GPU by
    // itself; a server with few jobs in flight needs more, smaller items to
    // spread each job over the SMs
    int batch_threads = 320;
    int batch_planes = 128;
    // longest CUDA graph captured (0: the default of 50 steps).  An engine
    // whose job set changes often (the server) captures short graphs and
    // replays them back to back: each change costs one short capture.
    int graph_max_steps = 0;
    // stable lanes (the server): each launch class keeps one lane whose job
    // list, item offsets and counts live in device tables sized for the
    // engine's capacity, with the block and shared memory of the largest
    // tile the class has seen; a change of the job set that fits the lanes
    // rewrites the tables and keeps the captured graphs
    bool stable_lanes = false;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // created on first use (download_finished)
    DevInfo info;
    std::vector<Job*> jobs;

   private:
    struct Group {
        bool fp32 = false, flat = false, generic = false, simple = false, mass = false;
        bool fhm = false;     // fh_march_kernel: fused variable-mobility jobs
        long long key = 0;    // launch class (precision, shape class, ring, width)
        int sub = 0;          // index among the groups of one class
        int* d_counts = nullptr;  // stable lanes: device [njobs, nitems]
        int table_cap = 0;        // stable lanes: entries of d_slot (d_item_begin has one more)
        int nbuf = 4;
        std::vector<Job*> jobs;
        int nitems = 0, grid = 0, block = 0;
        int grid_max = 0;  // SMs x occupancy: the most CTAs a launch of the lane can keep resident
        int fixed_nx = 0;  // row width shared by every job of the group (0: mixed)
        int fixed_ty = 0;  // tile height shared by every job of the group (0: mixed)
        size_t smem = 0;
        int cplane = 0, mplane = 0;
        int* d_item_begin = nullptr;
        int* d_slot = nullptr;
    };
    int rebuild();
    bool refresh_tables(std::vector<Group>& ng);
    int write_tables(const Group& g);
    StepKernel group_kernel(const Group& g) const;
    struct HighWater {
        int block = 0, cplane = 0, mplane = 0;
        int items = 0;  // most work items the lane has held
    };
    std::map<std::pair<long long, int>, HighWater> hw_;  // stable lanes: largest tile seen per class
    long long refreshes_ = 0;
    void free_groups();
    int launch_lane(const Group& g, Job* generic_job, cudaStream_t st);
    int launch_steps(int k);
    long long rebuilds_ = 0;
    std::vector<void*> graveyard_;  // device buffers of removed jobs, freed by rebuild()
    void free_graveyard();
    std::vector<cudaStream_t> aux_;  // one per lane beyond the first (launch_steps)
    std::vector<cudaEvent_t> aux_ev_;
    cudaEvent_t fork_ev_ = nullptr;
    int graph_for(int k, cudaGraphExec_t* out);
    void drop_graphs();
    int to_double(Job* j, double* d_dst);   // current field -> device doubles
    int download_on(Job* j, double* host, cudaStream_t st);
    int diagnostics_on(Job* j, mg_ch_stats* out, cudaStream_t st);
    int read_state_on(Job* j, JobDev* out, cudaStream_t st);
    int ensure_side();
    int ensure_stage(size_t n);

    int capacity_ = 0;
    JobDev* d_jobs_ = nullptr;
    int* d_err_ = nullptr;
    bool poisoned_ = false;  // a kernel reported a device error: no further steps
    std::vector<int> free_slots_;
    std::vector<int> released_slots_;  // slots of removed jobs, free again after the next rebuild
    bool admitting_ = false;
    cudaStream_t admit_ = nullptr;      // admission stream (begin_admission)
    double* d_stage_adm_ = nullptr;     // admission staging (doubles) and mass partials
    size_t stage_adm_n_ = 0;
    long long* d_part_adm_ = nullptr;
    cudaStream_t work_stream() const { return admitting_ ? admit_ : stream; }
    std::vector<Group> groups_;
    bool dirty_ = true;
    std::map<int, cudaGraphExec_t> graphs_;
    double* d_stage_ = nullptr;  // conversion staging (doubles)
    size_t stage_n_ = 0;
    double2* d_diag_part_ = nullptr;
    double* d_diag_max_ = nullptr;
    double* d_diag_bad_ = nullptr;
    Diag* d_diag_ = nullptr;
    Diag* h_diag_ = nullptr;  // pinned
    JobDev* h_state_ = nullptr;  // pinned
};

// kernel table
StepKernel step_kernel(bool fp32, bool flat, int nbuf, bool simple, int block, bool mass, int nx = 0);
bool nbuf_ok(int nbuf);
// march step kernels (ch_march.cuh; march_f32.cu, march_f64.cu): periodic,
// equal spacing, 3-D, row widths up to 256, ring depths 3, 4, 6; nullptr
// where no variant exists
// ty > 0: every job of the launch has tile height ty (a specialised variant
// where one exists)
StepKernel march_kernel_f32(int nx, int nbuf, bool mass, int ty = 0);
// the march kernels of ch_march2.cuh take the widths and tiles they cover
bool march2_enabled();
StepKernel march_kernel_f64(int nx, int nbuf, int ty = 0);
// ring depth of 3-D jobs of march widths that share launches (batch, server)
constexpr int kMarchBatchNbuf = 3;
bool march_batch_job(const Geometry& g);  // a periodic 3-D job of a march width
bool geometry_simple(const Geometry& g);
bool fixed_width_kernel(const Geometry& g, int nbuf);
int prepare_kernels(const DevInfo& d);

}  // namespace mg
