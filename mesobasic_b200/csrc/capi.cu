// C ABI of libmesogpu.so (declared in include/mesogpu.h): single
// simulations, batches and the autotuner.  The server lives in server.cu,
// host I/O (initial condition, VTK) in host_io.cpp.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <new>
#include <vector>

#include "engine.h"

struct mg_ch {
    mg::Engine eng;
    mg::Job* job = nullptr;
};

struct mg_batch {
    mg::Engine eng;
    std::vector<mg::Job*> jobs;
    std::vector<mg_ch_params> params;  // as created (mg_batch_autotune builds scratch copies)
};

using mg::fail;

// a single variable-mobility simulation with model parameters f
static int create_fh(const mg_ch_params* params, const mg::FhDev& f, int device, mg_ch_t** out)
{
    mg::Geometry g;
    MG_TRY(mg::make_geometry(*params, &g));
    if (params->precision != MG_FP64 || params->mass_correct)
        return fail(MG_EINVAL, "the variable-mobility models run in FP64 without mass feedback");
    std::unique_ptr<mg_ch> h(new (std::nothrow) mg_ch);
    if (!h) return fail(MG_ENOMEM, "host allocation failed");
    MG_TRY(h->eng.init(device, 1));
    MG_TRY(h->eng.add_job(*params, -1, &h->job, &f));
    *out = h.release();
    return MG_OK;
}

extern "C" {

const char* mg_last_error(void) { return mg::last_error(); }

int mg_ch_create(const mg_ch_params* params, int device, mg_ch_t** out)
{
    mg::clear_error();
    if (!params || !out) return fail(MG_EINVAL, "null argument");
    *out = nullptr;
    mg::Geometry g;
    MG_TRY(mg::make_geometry(*params, &g));  // argument errors before any device work
    std::unique_ptr<mg_ch> h(new (std::nothrow) mg_ch);
    if (!h) return fail(MG_ENOMEM, "host allocation failed");
    MG_TRY(h->eng.init(device, 1));
    MG_TRY(h->eng.add_job(*params, -1, &h->job));
    *out = h.release();
    return MG_OK;
}

int mg_fh_create(const mg_ch_params* params, const mg_fh_params* fh, int device, mg_ch_t** out)
{
    mg::clear_error();
    if (!params || !fh || !out) return fail(MG_EINVAL, "null argument");
    *out = nullptr;
    const double v[12] = {fh->alpha, fh->beta, fh->N, fh->A, fh->Tinit, fh->Tbath, fh->Tcrystal, fh->nu, fh->gamma,
                          fh->D0, fh->Mweight, fh->Mvolume};
    for (double x : v)
        if (!std::isfinite(x)) return fail(MG_EINVAL, "variable-mobility parameters must be finite");
    if (fh->nstep < 1) return fail(MG_EINVAL, "nstep must be >= 1");
    if (fh->bath != 0 && fh->bath != 1) return fail(MG_EINVAL, "bath must be 0 or 1");
    if (!std::isfinite(fh->thermCond)) return fail(MG_EINVAL, "thermCond must be finite");
    if (fh->N == 0 || fh->Mvolume == 0 || fh->Tinit == 0) return fail(MG_EINVAL, "N, Mvolume and Tinit must be nonzero");
    mg::FhDev f{};
    f.alpha = fh->alpha;
    f.beta = fh->beta;
    f.N = fh->N;
    f.A = fh->A;
    f.Tinit = fh->Tinit;
    f.Tbath = fh->Tbath;
    f.Tcrystal = fh->Tcrystal;
    f.nu = fh->nu;
    f.gamma = fh->gamma;
    f.D0 = fh->D0;
    f.Mweight = fh->Mweight;
    f.Mvolume = fh->Mvolume;
    f.nstep = fh->nstep;
    f.model = fh->bath ? mg::kFhBath : mg::kFhRamp;
    f.thermCond = fh->thermCond;
    return create_fh(params, f, device, out);
}

int mg_sips_create(const mg_ch_params* params, const mg_sips_params* sp, int device, mg_ch_t** out)
{
    mg::clear_error();
    if (!params || !sp || !out) return fail(MG_EINVAL, "null argument");
    *out = nullptr;
    const double v[12] = {sp->N,  sp->A,     sp->Tinit, sp->chiPS, sp->chiPN,   sp->chiCond,
                          sp->phiCutoff, sp->nu, sp->gamma, sp->D0, sp->Mweight, sp->Mvolume};
    for (double x : v)
        if (!std::isfinite(x)) return fail(MG_EINVAL, "SIPS parameters must be finite");
    if (sp->chiPS == sp->chiPN) return fail(MG_EINVAL, "chiPS and chiPN must differ (the mobility scale divides by chiPN - chiPS)");
    if (sp->N == 0 || sp->Mvolume == 0) return fail(MG_EINVAL, "N and Mvolume must be nonzero");
    mg::FhDev f{};
    f.N = sp->N;
    f.A = sp->A;
    f.Tinit = sp->Tinit;
    f.nu = sp->nu;
    f.gamma = sp->gamma;
    f.D0 = sp->D0;
    f.Mweight = sp->Mweight;
    f.Mvolume = sp->Mvolume;
    f.nstep = 1;
    f.model = mg::kFhSips;
    f.chiPS = sp->chiPS;
    f.chiPN = sp->chiPN;
    f.chiCond = sp->chiCond;
    f.NSdepth = sp->NSdepth;
    f.phiCutoff = sp->phiCutoff;
    return create_fh(params, f, device, out);
}

int mg_ternary_create(const mg_ch_params* params, const mg_ternary_params* t, int device, mg_batch_t** out)
{
    mg::clear_error();
    if (!params || !t || !out) return fail(MG_EINVAL, "null argument");
    *out = nullptr;
    const double v[4] = {t->Kpp, t->Knn, t->Mpp, t->Mnn};
    for (double x : v)
        if (!std::isfinite(x)) return fail(MG_EINVAL, "SIPSternary parameters must be finite");
    if (params->precision != MG_FP64 || params->mass_correct)
        return fail(MG_EINVAL, "the SIPSternary step runs in FP64 without mass feedback");
    mg::Geometry g;
    MG_TRY(mg::make_geometry(*params, &g));
    std::unique_ptr<mg_batch> b(new (std::nothrow) mg_batch);
    if (!b) return fail(MG_ENOMEM, "host allocation failed");
    MG_TRY(b->eng.init(device, 2));
    for (int i = 0; i < 2; ++i) {
        mg_ch_params p = *params;
        p.kappa = i == 0 ? t->Kpp : t->Knn;
        mg::FhDev f{};
        f.nstep = 1;
        f.model = mg::kFhLinear;
        f.Mconst = i == 0 ? t->Mpp : t->Mnn;
        mg::Job* j = nullptr;
        MG_TRY(b->eng.add_job(p, -1, &j, &f, i == 1));
        b->jobs.push_back(j);
    }
    *out = b.release();
    return MG_OK;
}

int mg_fh_mobility(mg_ch_t* h, double* host)
{
    mg::clear_error();
    if (!h) return fail(MG_EINVAL, "null handle");
    return h->eng.mobility(h->job, host);
}

int mg_ch_set_field(mg_ch_t* h, const double* host)
{
    mg::clear_error();
    if (!h) return fail(MG_EINVAL, "null handle");
    return h->eng.upload(h->job, host, -1);
}

int mg_ch_step(mg_ch_t* h, int nsteps)
{
    mg::clear_error();
    if (!h) return fail(MG_EINVAL, "null handle");
    return h->eng.enqueue_steps(nsteps);
}

int mg_ch_sync(mg_ch_t* h, long long timeout_us)
{
    mg::clear_error();
    if (!h) return fail(MG_EINVAL, "null handle");
    return h->eng.sync(timeout_us);
}

int mg_ch_get_field(mg_ch_t* h, double* host)
{
    mg::clear_error();
    if (!h) return fail(MG_EINVAL, "null handle");
    return h->eng.download(h->job, host);
}

int mg_ch_write_vtk(mg_ch_t* h, const char* path, const char* tag, int iskip, int jskip, int kskip)
{
    mg::clear_error();
    if (!h) return fail(MG_EINVAL, "null handle");
    return h->eng.write_vtk(h->job, path, tag, iskip, jskip, kskip);
}

int mg_ch_reduce(mg_ch_t* h, mg_ch_stats* out)
{
    mg::clear_error();
    if (!h) return fail(MG_EINVAL, "null handle");
    return h->eng.diagnostics(h->job, out);
}

int mg_ch_structure_factor(mg_ch_t* h, int nbins, double* k, double* S, double* k1)
{
    mg::clear_error();
    if (!h) return fail(MG_EINVAL, "null handle");
    return h->eng.structure_factor(h->job, nbins, k, S, k1);
}

void* mg_ch_stream(mg_ch_t* h) { return h ? (void*)h->eng.stream : nullptr; }

void* mg_ch_field_device(mg_ch_t* h)
{
    if (!h) return nullptr;
    mg::JobDev st;
    if (h->eng.read_state(h->job, &st) != MG_OK) return nullptr;
    return h->job->buf[st.step & 1];
}

long long mg_ch_steps(mg_ch_t* h)
{
    if (!h) return -1;
    mg::JobDev st;
    if (h->eng.read_state(h->job, &st) != MG_OK) return -1;
    return st.step;
}

int mg_ch_get_tiling(const mg_ch_t* h, mg_tiling* out)
{
    mg::clear_error();
    if (!h || !out) return fail(MG_EINVAL, "null argument");
    *out = h->job->tiling;
    return MG_OK;
}

int mg_ch_set_tiling(mg_ch_t* h, const mg_tiling* t)
{
    mg::clear_error();
    if (!h || !t) return fail(MG_EINVAL, "null argument");
    return h->eng.set_tiling(h->job, *t);
}

void mg_ch_destroy(mg_ch_t* h) { delete h; }

// ------------------------------------------------------------- autotune
static int time_tiling(mg_ch* h, const mg_tiling& t, int trials, double* ms)
{
    MG_TRY(h->eng.set_tiling(h->job, t));
    MG_TRY(h->eng.enqueue_steps(2));  // warm-up (also captures the graph)
    cudaEvent_t e0, e1;
    MG_CUDA(cudaEventCreate(&e0));
    MG_CUDA(cudaEventCreate(&e1));
    cudaEventRecord(e0, h->eng.stream);
    int rc = h->eng.enqueue_steps(trials);
    cudaEventRecord(e1, h->eng.stream);
    cudaEventSynchronize(e1);
    float f = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MG_TRY(rc);
    MG_TRY(h->eng.sync(-1));
    *ms = f / trials;
    return MG_OK;
}

int mg_autotune(const mg_ch_params* params, int device, int trials, mg_tiling* best, double* best_ms)
{
    mg::clear_error();
    if (!params || !best) return fail(MG_EINVAL, "null argument");
    if (trials < 1) trials = 10;
    mg_ch_t* h = nullptr;
    MG_TRY(mg_ch_create(params, device, &h));
    std::unique_ptr<mg_ch> guard(h);
    const mg::Geometry& g = h->job->g;
    if (!mg::tma_shape_ok(g)) {
        *best = mg_tiling{1, 1, 4, 1};
        if (best_ms) *best_ms = -1.0;
        return MG_OK;
    }
    MG_CUDA(cudaMemsetAsync(h->job->buf[0], 0, g.n * g.es, h->eng.stream));
    MG_CUDA(cudaMemsetAsync(h->job->buf[1], 0, g.n * g.es, h->eng.stream));
    std::vector<mg_tiling> cands;
    std::vector<int> tys;
    if (g.flat) tys.push_back(1);
    else
        for (int ty = 1; ty <= std::min(g.lny, 62); ++ty) tys.push_back(ty);
    for (int nbuf : {3, 4, 6, 8})
        for (int ty : tys) {
            mg_tiling t{ty, 1, nbuf, 0};
            mg::TilePlan pl;
            if (mg::plan_tiling(g, t, h->eng.info, &pl) != MG_OK) {
                mg::clear_error();
                continue;
            }
            int occ = 1;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &occ, mg::step_kernel(g.es == 4, g.flat, nbuf, mg::geometry_simple(g), pl.block, g.es == 4, g.lnx), pl.block,
                    pl.smem) !=
                cudaSuccess)
                continue;
            occ = std::max(occ, 1);
            const int slots = h->eng.info.sms * occ;
            const int maxc = std::max(1, g.lnz / 4);
            std::vector<int> ncs;
            for (int mult = 1; mult <= 3; ++mult) {
                const int nc = std::min(maxc, std::max(1, mult * slots / pl.ntile));
                ncs.push_back(nc);
                if (nc > 1) ncs.push_back(nc & ~1);
            }
            std::sort(ncs.begin(), ncs.end());
            ncs.erase(std::unique(ncs.begin(), ncs.end()), ncs.end());
            for (int nc : ncs) {
                t.nchunk = nc;
                cands.push_back(t);
            }
        }
    double bms = 1e30;
    mg_tiling bt = h->job->tiling;
    for (const mg_tiling& t : cands) {
        double ms;
        if (time_tiling(h, t, trials, &ms) != MG_OK) {
            mg::clear_error();
            continue;
        }
        if (ms < bms) {
            bms = ms;
            bt = t;
        }
    }
    if (bms >= 1e30) return fail(MG_ECUDA, "autotune: no candidate ran");
    mg::tune_store(mg::tune_key(g), bt, bms);
    *best = bt;
    if (best_ms) *best_ms = bms;
    return MG_OK;
}

// ---------------------------------------------------------------- batch
// The composition of a batch (job shapes, precision and mass feedback, with
// their counts): the tuning-cache key of its tiles.
static std::string batch_signature(const mg_ch_params* jobs, int njobs)
{
    std::map<std::string, int> count;
    for (int i = 0; i < njobs; ++i) {
        mg::Geometry g;
        if (mg::make_geometry(jobs[i], &g) != MG_OK) {
            mg::clear_error();
            continue;
        }
        count[mg::tune_key(g) + (jobs[i].mass_correct ? ":m" : "")] += 1;
    }
    std::string s = "batch";
    for (auto& kv : count) s += "|" + kv.first + "*" + std::to_string(kv.second);
    return s;
}

int mg_batch_create(const mg_ch_params* jobs, int njobs, int device, mg_batch_t** out)
{
    mg::clear_error();
    if (!jobs || njobs < 1 || !out) return fail(MG_EINVAL, "bad arguments");
    *out = nullptr;
    for (int i = 0; i < njobs; ++i) {
        mg::Geometry g;
        if (mg::make_geometry(jobs[i], &g) != MG_OK) return fail(MG_EINVAL, "job %d: %s", i, mg::last_error());
    }
    std::unique_ptr<mg_batch> b(new (std::nothrow) mg_batch);
    if (!b) return fail(MG_ENOMEM, "host allocation failed");
    MG_TRY(b->eng.init(device, njobs));
    b->eng.batch_tiling = true;
    // tile targets: the environment, else what mg_batch_autotune measured for
    // this composition, else 320 threads and 128-plane chunks
    b->eng.batch_threads = 320;
    b->eng.batch_planes = 128;
    b->params.assign(jobs, jobs + njobs);
    mg_tiling tuned;
    if (mg::tune_lookup(batch_signature(jobs, njobs), &tuned)) {
        b->eng.batch_threads = tuned.ty;
        b->eng.batch_planes = tuned.nchunk;
    }
    b->eng.batch_threads = mg::mg_env_int("MG_BATCH_THREADS", b->eng.batch_threads);
    b->eng.batch_planes = mg::mg_env_int("MG_BATCH_PLANES", b->eng.batch_planes);
    for (int i = 0; i < njobs; ++i) {
        mg::Job* j = nullptr;
        int rc = b->eng.add_job(jobs[i], -1, &j);
        if (rc != MG_OK) return fail(rc, "job %d: %s", i, mg::last_error());
        b->jobs.push_back(j);
    }
    *out = b.release();
    return MG_OK;
}

static int batch_job(mg_batch_t* b, int job, mg::Job** j)
{
    if (!b) return fail(MG_EINVAL, "null handle");
    if (job < 0 || job >= (int)b->jobs.size()) return fail(MG_EINVAL, "job %d out of range", job);
    *j = b->jobs[job];
    return MG_OK;
}

int mg_batch_set_field(mg_batch_t* b, int job, const double* host)
{
    mg::clear_error();
    mg::Job* j;
    MG_TRY(batch_job(b, job, &j));
    return b->eng.upload(j, host, -1);
}

int mg_batch_step(mg_batch_t* b, int nsteps)
{
    mg::clear_error();
    if (!b) return fail(MG_EINVAL, "null handle");
    return b->eng.enqueue_steps(nsteps);
}

int mg_batch_sync(mg_batch_t* b, long long timeout_us)
{
    mg::clear_error();
    if (!b) return fail(MG_EINVAL, "null handle");
    return b->eng.sync(timeout_us);
}

int mg_batch_get_field(mg_batch_t* b, int job, double* host)
{
    mg::clear_error();
    mg::Job* j;
    MG_TRY(batch_job(b, job, &j));
    return b->eng.download(j, host);
}

int mg_batch_reduce(mg_batch_t* b, int job, mg_ch_stats* out)
{
    mg::clear_error();
    mg::Job* j;
    MG_TRY(batch_job(b, job, &j));
    return b->eng.diagnostics(j, out);
}

int mg_batch_write_vtk(mg_batch_t* b, int job, const char* path, const char* tag, int iskip, int jskip, int kskip)
{
    mg::clear_error();
    mg::Job* j;
    MG_TRY(batch_job(b, job, &j));
    return b->eng.write_vtk(j, path, tag, iskip, jskip, kskip);
}

void* mg_batch_stream(mg_batch_t* b) { return b ? (void*)b->eng.stream : nullptr; }

int mg_batch_info(const mg_batch_t* b, int* nitems, int* nctas, int* nlaunch)
{
    mg::clear_error();
    if (!b) return fail(MG_EINVAL, "null handle");
    if (nitems) *nitems = b->eng.nitems_total();
    if (nctas) *nctas = b->eng.nctas_total();
    if (nlaunch) *nlaunch = b->eng.nlaunch_per_step();
    return MG_OK;
}

// ms per step of a scratch batch with these tile targets (zero fields)
static int time_batch_targets(const std::vector<mg_ch_params>& params, int device, int threads, int planes,
                              int trials, double* ms, std::vector<mg_tiling>* tilings)
{
    mg::Engine e;
    MG_TRY(e.init(device, (int)params.size()));
    e.batch_tiling = true;
    e.batch_threads = threads;
    e.batch_planes = planes;
    tilings->clear();
    for (const mg_ch_params& p : params) {
        mg::Job* j = nullptr;
        MG_TRY(e.add_job(p, -1, &j));
        MG_CUDA(cudaMemsetAsync(j->buf[0], 0, j->g.n * j->g.es, e.stream));
        MG_CUDA(cudaMemsetAsync(j->buf[1], 0, j->g.n * j->g.es, e.stream));
        tilings->push_back(j->tiling);
    }
    MG_TRY(e.enqueue_steps(2));  // warm-up (also captures the graph)
    cudaEvent_t e0, e1;
    MG_CUDA(cudaEventCreate(&e0));
    MG_CUDA(cudaEventCreate(&e1));
    cudaEventRecord(e0, e.stream);
    int rc = e.enqueue_steps(trials);
    cudaEventRecord(e1, e.stream);
    cudaEventSynchronize(e1);
    float f = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MG_TRY(rc);
    MG_TRY(e.sync(-1));
    *ms = f / trials;
    return MG_OK;
}

int mg_batch_autotune(mg_batch_t* b, int trials, int* threads, int* planes, double* ms_per_step)
{
    mg::clear_error();
    if (!b) return fail(MG_EINVAL, "null handle");
    if (trials < 1) trials = 5;
    MG_TRY(b->eng.sync(-1));
    double best = 1e30;
    int bt = b->eng.batch_threads, bp = b->eng.batch_planes;
    std::vector<mg::Geometry> geo(b->params.size());
    for (size_t i = 0; i < geo.size(); ++i) MG_TRY(mg::make_geometry(b->params[i], &geo[i]));
    std::vector<std::vector<int>> seen;  // candidates that tile every job alike are timed once
    for (int t : {192, 256, 320, 384, 448, 512, 640})
        for (int p : {32, 64, 128, 256}) {
            std::vector<int> sig;
            for (const mg::Geometry& g : geo) {
                const mg_tiling tt = mg::batch_tiling_for(g, b->eng.info, b->eng.device, t, p);
                sig.insert(sig.end(), {tt.ty, tt.nchunk, tt.nbuf, tt.path});
            }
            if (std::find(seen.begin(), seen.end(), sig) != seen.end()) continue;
            seen.push_back(sig);
            double ms;
            std::vector<mg_tiling> tl;
            if (time_batch_targets(b->params, b->eng.device, t, p, trials, &ms, &tl) != MG_OK) {
                mg::clear_error();
                cudaGetLastError();
                continue;
            }
            if (ms < best) {
                best = ms;
                bt = t;
                bp = p;
            }
        }
    if (best >= 1e30) return fail(MG_ECUDA, "no tile target could be timed");
    // re-tile the batch (the fields and step counts stay)
    b->eng.batch_threads = bt;
    b->eng.batch_planes = bp;
    for (mg::Job* j : b->jobs) {
        const mg_tiling t = mg::batch_tiling_for(j->g, b->eng.info, b->eng.device, bt, bp);
        if (t.ty != j->tiling.ty || t.nchunk != j->tiling.nchunk || t.nbuf != j->tiling.nbuf || t.path != j->tiling.path)
            MG_TRY(b->eng.set_tiling(j, t));
    }
    mg::tune_store(batch_signature(b->params.data(), (int)b->params.size()), mg_tiling{bt, bp, mg::kMarchBatchNbuf, 0},
                   best);
    if (threads) *threads = bt;
    if (planes) *planes = bp;
    if (ms_per_step) *ms_per_step = best;
    return MG_OK;
}

void mg_batch_destroy(mg_batch_t* b) { delete b; }

}  // extern "C"
