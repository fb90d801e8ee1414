// Continuous-batching server over the step engine (mg_server_* in
// include/mesogpu.h).
//
// A worker thread owns one Engine.  Each tick it
//   1. admits queued jobs, oldest first, that fit the HBM budget and a free
//      slot (first fit: a large job at the head does not block small ones),
//      with their allocation and upload outside the server lock;
//   2. enqueues steps_per_tick steps for every admitted job together -- one
//      fused launch per class per step, all jobs' tiles in the same
//      persistent grid, classes side by side on their own streams; a job
//      that reaches its step count stops on the device (its tiles skip), so
//      ticks keep one length and one captured graph per job set;
//   3. retires jobs that reached their step count: downloads the field and
//      diagnostics on a side stream while the next tick runs (their tiles
//      skip, so their fields do not change), frees their memory, records
//      the latency.
// Per-job arithmetic does not depend on which other jobs share a launch:
// each job's decomposition and reduction trees depend on its own shape only.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"

using mg::fail;
using Clock = std::chrono::steady_clock;

namespace {

struct ServerJob {
    long long id = 0;
    mg_ch_params p{};
    std::vector<double> ic;
    long long nsteps = 0;
    long long done_steps = 0;
    int state = MG_JOB_QUEUED;
    mg::Job* job = nullptr;
    size_t bytes = 0;
    Clock::time_point t_submit, t_done;
    std::unique_ptr<double[]> result;  // final field (not zero-filled first)
    size_t result_n = 0;
    mg_ch_stats stats{};
    std::string error;
};

}  // namespace

struct mg_server {
    mg::Engine eng;
    double budget = 0;
    int max_inflight = 0;
    int steps_per_tick = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<ServerJob*> queue;
    std::vector<ServerJob*> running;
    std::map<long long, std::unique_ptr<ServerJob>> jobs;
    long long next_id = 1;
    bool stopping = false;
    size_t in_use = 0, peak = 0;
    long long submitted = 0, completed = 0, failed = 0;
    std::vector<double> latencies_ms;
    bool have_first = false;
    Clock::time_point t_first, t_last;
    double site_updates = 0;
    double step_s = 0, admit_s = 0, retire_s = 0;  // worker time (see mg_server_stats)
    long long ticks = 0;
    // ticks that began with jobs still queued (every slot or the budget
    // taken): their time and the site-updates they ran
    double sat_s = 0, sat_updates = 0;
    long long sat_ticks = 0;
    double gpu_s = 0;  // device time of the ticks' steps (events on the engine stream)
    cudaEvent_t ev_tick[2] = {nullptr, nullptr};

    void run();
    // jobs admitted beside a running tick, joining at the next one
    std::vector<ServerJob*> arrived;
    void admit(bool beside_tick);
    void retire(ServerJob* sj, bool ok, const char* why);
};

static size_t job_bytes(const mg_ch_params& p)
{
    const size_t n = (size_t)p.nx * p.ny * p.nz;
    return 2 * n * (p.precision == MG_FP32 ? 4 : 8) + (1 << 16);
}

// Admission.  Under the lock, the queue is scanned first fit in arrival
// order for jobs that fit the HBM budget and a free slot; they are reserved
// (their bytes counted, taken off the queue).  The device work -- buffers,
// tensor maps, upload of the initial field -- runs after the lock is
// released: only the worker thread touches the engine, so submitters never
// wait for an allocation or a copy.  beside_tick: the worker has a tick in
// flight; the device work goes on the engine's admission stream, overlapping
// it, and the jobs join the tick after (`arrived`).
void mg_server::admit(bool beside_tick)
{
    std::vector<ServerJob*> take;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (auto it = queue.begin(); it != queue.end();) {
            if ((int)(running.size() + arrived.size() + take.size()) >= max_inflight) break;
            ServerJob* sj = *it;
            if ((double)(in_use + sj->bytes) > budget) {
                ++it;
                continue;
            }
            in_use += sj->bytes;
            peak = std::max(peak, in_use);
            take.push_back(sj);
            it = queue.erase(it);
        }
    }
    if (take.empty()) return;
    std::vector<ServerJob*> ok, bad;
    std::vector<std::string> why;
    if (beside_tick && eng.begin_admission() != MG_OK) beside_tick = false;
    for (ServerJob* sj : take) {
        mg::Job* j = nullptr;
        int rc = eng.add_job(sj->p, sj->nsteps, &j);
        if (rc == MG_OK) rc = eng.upload(j, sj->ic.data(), sj->nsteps);
        if (rc != MG_OK) {
            if (j) eng.remove_job(j);
            bad.push_back(sj);
            why.push_back(mg::last_error());
            continue;
        }
        sj->job = j;
        ok.push_back(sj);
    }
    if (beside_tick && eng.end_admission() != MG_OK) {
        // the uploads did not complete: the jobs fail
        for (ServerJob* sj : ok) {
            eng.remove_job(sj->job);
            sj->job = nullptr;
            bad.push_back(sj);
            why.push_back(mg::last_error());
        }
        ok.clear();
    }
    for (ServerJob* sj : ok) std::vector<double>().swap(sj->ic);  // the uploads have read it
    std::lock_guard<std::mutex> lock(mu);
    for (ServerJob* sj : ok) {
        sj->state = MG_JOB_RUNNING;
        (beside_tick ? arrived : running).push_back(sj);
    }
    for (size_t i = 0; i < bad.size(); ++i) {
        ServerJob* sj = bad[i];
        in_use -= sj->bytes;
        sj->state = MG_JOB_FAILED;
        sj->error = why[i];
        sj->t_done = Clock::now();
        ++failed;
    }
    if (!bad.empty()) cv_done.notify_all();
}

void mg_server::retire(ServerJob* sj, bool ok, const char* why)
{
    if (ok) {
        sj->result_n = (size_t)sj->p.nx * sj->p.ny * sj->p.nz;
        sj->result.reset(new (std::nothrow) double[sj->result_n]);
        // the job has reached its step count: its field is read on the
        // engine's side stream while the next tick runs
        int rc = sj->result ? eng.download_finished(sj->job, sj->result.get())
                            : fail(MG_ENOMEM, "host allocation failed");
        if (rc == MG_OK) {
            rc = eng.diagnostics_finished(sj->job, &sj->stats);
            if (rc == MG_ENONFINITE) rc = MG_OK;  // reported in stats.nonfinite
        }
        if (rc != MG_OK) {
            ok = false;
            why = mg::last_error();
        }
    }
    eng.remove_job(sj->job);
    sj->job = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    in_use -= sj->bytes;
    sj->t_done = Clock::now();
    t_last = sj->t_done;
    if (ok) {
        sj->state = MG_JOB_DONE;
        ++completed;
        latencies_ms.push_back(std::chrono::duration<double, std::milli>(sj->t_done - sj->t_submit).count());
        site_updates += (double)sj->p.nx * sj->p.ny * sj->p.nz * (double)sj->nsteps;
    } else {
        sj->state = MG_JOB_FAILED;
        sj->error = why ? why : "failed";
        ++failed;
    }
    running.erase(std::find(running.begin(), running.end(), sj));
    cv_done.notify_all();
}

static double seconds_since(Clock::time_point t0)
{
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

void mg_server::run()
{
    cudaSetDevice(eng.device);
    // jobs that reached their step count in the last tick: retired (field
    // and diagnostics read on a side stream) while the next tick runs
    std::vector<ServerJob*> finished;
    // the saturated rate counts whole iterations, from one tick's start to
    // the next one's (the admissions and retirements between them included)
    bool prev_sat = false;
    double prev_updates = 0;
    Clock::time_point prev_t0;
    for (;;) {
        for (;;) {
            auto t0 = Clock::now();
            admit(false);
            const double as = seconds_since(t0);
            std::unique_lock<std::mutex> lock(mu);
            admit_s += as;
            if (!running.empty()) break;
            if (stopping && queue.empty()) return;
            cv_work.wait_for(lock, std::chrono::milliseconds(20));
        }
        const long long k = steps_per_tick;
        // steps only when some admitted job still has steps to take
        const bool stepping = running.size() > finished.size();
        // a tick that starts with a backlog runs at the server's saturated
        // rate; the site-updates it runs are those its jobs still owe
        bool backlog;
        double tick_updates = 0;
        {
            std::lock_guard<std::mutex> lock(mu);
            backlog = !queue.empty();
            for (ServerJob* sj : running)
                tick_updates += (double)sj->p.nx * sj->p.ny * sj->p.nz *
                                (double)std::min(k, std::max(0LL, sj->nsteps - sj->done_steps));
        }
        const auto t0 = Clock::now();
        if (prev_sat) {
            std::lock_guard<std::mutex> lock(mu);
            sat_s += std::chrono::duration<double>(t0 - prev_t0).count();
            sat_updates += prev_updates;
            ++sat_ticks;
        }
        prev_sat = false;
        if (stepping && !ev_tick[0]) {
            cudaEventCreate(&ev_tick[0]);
            cudaEventCreate(&ev_tick[1]);
        }
        if (stepping && ev_tick[0]) cudaEventRecord(ev_tick[0], eng.stream);
        int rc = stepping ? eng.enqueue_steps((int)k) : MG_OK;
        if (stepping && ev_tick[1]) cudaEventRecord(ev_tick[1], eng.stream);
        const auto t1 = Clock::now();
        for (ServerJob* sj : finished) retire(sj, true, nullptr);
        finished.clear();
        const double rs = seconds_since(t1);
        // admit the next tick's jobs while this one runs
        const auto t2 = Clock::now();
        if (stepping && rc == MG_OK) admit(true);
        const double as2 = seconds_since(t2);
        if (stepping && rc == MG_OK) rc = eng.sync(600LL * 1000 * 1000);
        {
            std::lock_guard<std::mutex> lock(mu);
            retire_s += rs;
            admit_s += as2;
            if (stepping) {
                const double ts = seconds_since(t0);
                step_s += ts;
                ++ticks;
                float ms = 0.f;
                if (rc == MG_OK && ev_tick[1] && cudaEventElapsedTime(&ms, ev_tick[0], ev_tick[1]) == cudaSuccess)
                    gpu_s += ms * 1e-3;
                else
                    cudaGetLastError();
                if (backlog && rc == MG_OK) {
                    prev_sat = true;
                    prev_updates = tick_updates;
                    prev_t0 = t0;
                }
            }
        }
        std::vector<ServerJob*> snapshot = running;  // the jobs of this tick
        {
            // the jobs admitted beside this tick join the next one
            std::lock_guard<std::mutex> lock(mu);
            running.insert(running.end(), arrived.begin(), arrived.end());
            arrived.clear();
        }
        if (rc != MG_OK) {
            const std::string why = mg::last_error();
            const std::vector<ServerJob*> all = running;
            for (ServerJob* sj : all) retire(sj, false, why.c_str());
            continue;
        }
        if (stepping)
            for (ServerJob* sj : snapshot) {
                sj->done_steps = std::min(sj->nsteps, sj->done_steps + k);
                if (sj->done_steps >= sj->nsteps) finished.push_back(sj);
            }
    }
}

extern "C" {

int mg_server_create(int device, double hbm_budget_gb, int max_jobs_in_flight, int steps_per_tick,
                     mg_server_t** out)
{
    mg::clear_error();
    if (!out || hbm_budget_gb <= 0 || max_jobs_in_flight < 1) return fail(MG_EINVAL, "bad server arguments");
    *out = nullptr;
    std::unique_ptr<mg_server> s(new (std::nothrow) mg_server);
    if (!s) return fail(MG_ENOMEM, "host allocation failed");
    // twice the slots of the jobs in flight: a retired job's slot is reused
    // only after the next rebuild, while admissions run beside a tick
    MG_TRY(s->eng.init(device, 2 * max_jobs_in_flight));
    s->eng.batch_tiling = true;
    // tile target of the served jobs: 320 threads a CTA and 64-plane z
    // chunks took 11 % less GPU time on the served stream than 256 / 16
    // (four settings measured back to back on one B200)
    s->eng.batch_threads = mg::mg_env_int("MG_SERVER_THREADS", 320);
    s->eng.batch_planes = mg::mg_env_int("MG_SERVER_PLANES", 64);
    // admissions and retirements change the job set between ticks: short
    // graphs keep the recapture after each change cheap
    s->eng.graph_max_steps = mg::mg_env_int("MG_SERVER_GRAPH_STEPS", 10);
    // job-set changes that fit the launch lanes rewrite device tables
    // instead of recapturing the graphs
    s->eng.stable_lanes = true;
    s->budget = hbm_budget_gb * 1e9;
    s->max_inflight = max_jobs_in_flight;
    s->steps_per_tick = steps_per_tick > 0 ? steps_per_tick : 100;
    mg_server* raw = s.get();
    s->worker = std::thread([raw] { raw->run(); });
    *out = s.release();
    return MG_OK;
}

int mg_server_submit(mg_server_t* s, const mg_ch_params* params, const double* ic_host, long long nsteps,
                     long long* job_id)
{
    mg::clear_error();
    if (!s || !params || !ic_host || nsteps < 1) return fail(MG_EINVAL, "bad submit arguments");
    mg::Geometry g;
    MG_TRY(mg::make_geometry(*params, &g));
    std::unique_ptr<ServerJob> sj(new (std::nothrow) ServerJob);
    if (!sj) return fail(MG_ENOMEM, "host allocation failed");
    sj->p = *params;
    sj->nsteps = nsteps;
    sj->bytes = job_bytes(*params);
    if ((double)sj->bytes > s->budget)
        return fail(MG_ENOMEM, "job needs %.3f GB, above the server budget %.3f GB", sj->bytes / 1e9, s->budget / 1e9);
    sj->ic.assign(ic_host, ic_host + g.n);
    sj->t_submit = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stopping) return fail(MG_EINVAL, "server is stopping");
    sj->id = s->next_id++;
    if (!s->have_first) {
        s->have_first = true;
        s->t_first = sj->t_submit;
    }
    if (job_id) *job_id = sj->id;
    s->queue.push_back(sj.get());
    s->jobs[sj->id] = std::move(sj);
    ++s->submitted;
    s->cv_work.notify_all();
    return MG_OK;
}

int mg_server_poll(mg_server_t* s, long long job_id, int* state)
{
    mg::clear_error();
    if (!s || !state) return fail(MG_EINVAL, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return fail(MG_ENOTFOUND, "unknown job %lld", job_id);
    *state = it->second->state;
    return MG_OK;
}

int mg_server_result(mg_server_t* s, long long job_id, long long timeout_us, double* field_out, mg_ch_stats* stats)
{
    mg::clear_error();
    if (!s) return fail(MG_EINVAL, "null handle");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return fail(MG_ENOTFOUND, "unknown job %lld", job_id);
    ServerJob* sj = it->second.get();
    auto finished = [&] { return sj->state == MG_JOB_DONE || sj->state == MG_JOB_FAILED; };
    if (timeout_us < 0) s->cv_done.wait(lock, finished);
    else if (!s->cv_done.wait_for(lock, std::chrono::microseconds(timeout_us), finished))
        return fail(MG_ETIMEOUT, "job %lld not finished after %lld us", job_id, timeout_us);
    if (sj->state == MG_JOB_FAILED) {
        std::string why = sj->error;
        s->jobs.erase(it);
        return fail(MG_EDEVICE, "job %lld failed: %s", job_id, why.c_str());
    }
    if (field_out) std::copy(sj->result.get(), sj->result.get() + sj->result_n, field_out);
    if (stats) *stats = sj->stats;
    s->jobs.erase(it);
    return MG_OK;
}

int mg_server_stats_get(mg_server_t* s, mg_server_stats* out)
{
    mg::clear_error();
    if (!s || !out) return fail(MG_EINVAL, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    mg_server_stats st{};
    st.submitted = s->submitted;
    st.completed = s->completed;
    st.failed = s->failed;
    st.running = (long long)s->running.size();
    st.step_s = s->step_s;
    st.admit_s = s->admit_s;
    st.retire_s = s->retire_s;
    st.ticks = s->ticks;
    st.rebuilds = s->eng.rebuilds();
    st.refreshes = s->eng.refreshes();
    st.queued = (long long)s->queue.size();
    if (!s->latencies_ms.empty()) {
        std::vector<double> v = s->latencies_ms;
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) {
            const double pos = q * (v.size() - 1);
            const size_t lo = (size_t)pos;
            const size_t hi = std::min(lo + 1, v.size() - 1);
            return v[lo] + (v[hi] - v[lo]) * (pos - lo);
        };
        st.p50_ms = pct(0.50);
        st.p99_ms = pct(0.99);
        double sum = 0;
        for (double x : v) sum += x;
        st.mean_ms = sum / v.size();
    }
    if (s->have_first && s->completed > 0) {
        const double wall = std::chrono::duration<double>(s->t_last - s->t_first).count();
        if (wall > 0) {
            st.sims_per_hour = s->completed / wall * 3600.0;
            st.site_updates_per_s = s->site_updates / wall;
        }
    }
    st.sat_ticks = s->sat_ticks;
    st.gpu_s = s->gpu_s;
    st.sat_site_updates_per_s = s->sat_s > 0 ? s->sat_updates / s->sat_s : 0.0;
    st.hbm_in_use_gb = s->in_use / 1e9;
    st.hbm_peak_gb = s->peak / 1e9;
    *out = st;
    return MG_OK;
}

void mg_server_destroy(mg_server_t* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    for (cudaEvent_t ev : s->ev_tick)
        if (ev) cudaEventDestroy(ev);
    delete s;
}

}  // extern "C"
