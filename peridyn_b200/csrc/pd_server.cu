// pd_server.cu -- the serving loop (pd_server_* in include/peridyn_b200.h).
//
// Jobs queue in arrival order; two admission threads take the head of the
// queue while the sum of the resident jobs' HBM footprints stays within the
// budget (and fewer than max_active run) and finalize the job's
// environment; a stepping thread advances the resident jobs in chunks of
// velocity-Verlet steps.
//
// Continuous batching: a job's first chunk runs on its own CUDA stream
// (the deformed gate is decided there).  Once every block of a job has
// deformed, a job of at most 64 k particles without contacts, boundary
// conditions or elasto-plastic blocks joins the batch of its precision at
// the batch's next chunk: the batch's jobs advance together in shared
// launches (one job-table kernel per step, kernel shape and 16 jobs,
// pd_fast.cu k_step_jobs), each chunk as long as
// the shortest remaining run among them; membership changes between
// chunks, without graph capture.  Other jobs keep running chunk after chunk
// on their own streams, overlapping with the batch on the device.  A job's
// numbers are the same alone and in any mix: its kernel shape is fixed
// from its size, and a run split into chunks computes what one run does.
// A finished job's state is downloaded and its device memory released at
// once, which frees its share of the budget for the next admission.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pd_env_impl.h"

using namespace pd;
using Clock = std::chrono::steady_clock;

namespace {

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
    int64_t id = 0;
    pd_env *env = nullptr;
    int64_t nsteps = 0, chunk_now = 0;
    std::atomic<int64_t> done{0}, particles{0};  // read by pollers
    int32_t state = PD_JOB_QUEUED;
    pd_status status = PD_OK;
    std::string err;
    bool cancel = false, inflight = false;
    bool batched = false;  // advanced by a batch (not on its own stream)
    int64_t footprint = 0, bonds0 = 0, bond_updates = 0;
    Clock::time_point t_submit, t_admit, t_done;
    cudaEvent_t ev = nullptr;
    std::vector<double> y, v, damage;
};

// Kernel shape of a throughput-mode job from its size and the device's
// multiprocessor count alone (never timed, so the result of a job is the
// same whatever runs beside it): enough warps per slice for about 32
// resident warps per SM.
void fix_shape(pd_env *env) {
    if (env->precision == PD_PREC_FP64_SERIAL) return;
    const int64_t slices = env->N / kSlice;
    int sms = env->sm_count;
    if (sms <= 0 && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, env->device) != cudaSuccess) sms = 148;
    int w = 1;
    while (w < 8 && slices * w < (int64_t)sms * 32) w *= 2;
    pd_env_set_kernel_shape(env, w, env->precision == PD_PREC_FP32C ? 4 : 2);
}

}  // namespace

struct pd_server {
    int device = 0;
    int64_t budget = 0, used = 0;
    int max_active = 1;
    int64_t chunk = 128;
    // shared launches for batchable jobs (PD_SERVE_BATCH=0: every job on
    // its own stream)
    bool batching = true;
    std::mutex mu;
    std::condition_variable wake, changed;
    std::deque<Job *> queue;
    std::map<int64_t, std::unique_ptr<Job>> jobs;
    int64_t next_id = 1;
    std::vector<Job *> ready;  // admitted, not yet picked up by the stepper
    int resident = 0;          // admitted and not finished
    bool stop = false;
    // Admission (family build, layout, initial forces) is mostly host work
    // of one job at a time; two admission threads finalize two jobs at once
    // while the stepping thread keeps the device busy.
    static constexpr int kAdmitters = 2;
    std::thread admitters[kAdmitters], stepper;
    // one batch per throughput precision (index 0: FP64, 1: FP32C), owned
    // by the stepping thread
    struct Batch {
        std::vector<Job *> members;
        std::vector<Job *> pending;  // idle, joining at the next chunk
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        bool inflight = false;
        int64_t chunk_now = 0;
    } batch[2];

    void admit_loop();
    void step_loop();
    bool step_batch(Batch &b);
    void admit(Job *j);
    void finish(Job *j, int32_t state);
};

void pd_server::finish(Job *j, int32_t state) {
    if (state == PD_JOB_DONE) {
        const int64_t n = j->env->N_env;
        j->y.resize(3 * n);
        j->v.resize(3 * n);
        j->damage.resize(n);
        pd_status s = pd_env_get_state(j->env, j->y.data(), j->v.data(), nullptr, nullptr);
        if (s == PD_OK) s = pd_env_damage(j->env, j->damage.data());
        int64_t b1 = 0;
        if (s == PD_OK) s = pd_env_num_bonds(j->env, &b1);
        if (s != PD_OK) {
            state = PD_JOB_FAILED;
            j->status = s;
            j->err = pd_last_error();
        } else {
            j->bond_updates = (j->bonds0 + b1) / 2 * j->nsteps;
        }
    }
    if (j->ev) cudaEventDestroy(j->ev);
    j->ev = nullptr;
    pd_env_destroy(j->env);
    j->env = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (j->state == PD_JOB_RUNNING) {
        used -= j->footprint;
        --resident;
    }
    j->state = state;
    j->t_done = Clock::now();
    changed.notify_all();
    wake.notify_all();  // room for the next admission
}

void pd_server::admit(Job *j) {
    pd_env *env = j->env;
    pd_status s = pd_env_finalize(env);
    if (s == PD_OK) {
        fix_shape(env);
        s = pd_env_apply_bc_at0(env);
    }
    if (s == PD_OK) s = pd_env_update_acc(env);  // save_state! at t0
    if (s == PD_OK) s = pd_env_num_bonds(env, &j->bonds0);
    if (s == PD_OK && cudaEventCreateWithFlags(&j->ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        s = fail(PD_ERR_CUDA, "event creation failed");
    }
    if (s != PD_OK) {
        j->status = s;
        j->err = pd_last_error();
        finish(j, PD_JOB_FAILED);
        return;
    }
    j->particles = env->N_env;
}

// Admission threads: each takes the head of the queue when its footprint fits
// (or nothing else is resident) and a slot is free, finalizes it (family
// build, BC snapshot, initial forces) and hands it to the stepping thread.
void pd_server::admit_loop() {
    cudaSetDevice(device);
    for (;;) {
        Job *j = nullptr;
        {
            std::unique_lock<std::mutex> lock(mu);
            for (;;) {
                while (!queue.empty() && queue.front()->cancel) {
                    Job *c = queue.front();
                    queue.pop_front();
                    pd_env_destroy(c->env);
                    c->env = nullptr;
                    c->state = PD_JOB_CANCELLED;
                    c->t_done = Clock::now();
                    changed.notify_all();
                }
                if (stop) return;
                if (!queue.empty() && resident < max_active &&
                    (used + queue.front()->footprint <= budget || resident == 0))
                    break;
                wake.wait(lock);
            }
            j = queue.front();
            queue.pop_front();
            used += j->footprint;
            ++resident;
            j->state = PD_JOB_RUNNING;
            j->t_admit = Clock::now();
        }
        admit(j);
        std::lock_guard<std::mutex> lock(mu);
        if (j->env) ready.push_back(j);
        wake.notify_all();
    }
}

// One batch: when its chunk has finished, credit the steps and retire the
// finished and cancelled members; when idle, take in the jobs waiting to
// join and launch the next chunk.  Returns true when anything changed.
bool pd_server::step_batch(Batch &b) {
    bool progressed = false;
    if (b.inflight) {
        const cudaError_t q = cudaEventQuery(b.ev);
        if (q == cudaErrorNotReady) return false;
        b.inflight = false;
        progressed = true;
        for (size_t k = 0; k < b.members.size();) {
            Job *j = b.members[k];
            if (q != cudaSuccess) {
                j->status = fail(PD_ERR_CUDA, "batch stream: %s", cudaGetErrorString(q));
                j->err = pd_last_error();
                finish(j, PD_JOB_FAILED);
                b.members.erase(b.members.begin() + k);
                continue;
            }
            j->done += b.chunk_now;
            ++k;
        }
    }
    if (!b.pending.empty()) {
        b.members.insert(b.members.end(), b.pending.begin(), b.pending.end());
        b.pending.clear();
        progressed = true;
    }
    for (size_t k = 0; k < b.members.size();) {
        Job *j = b.members[k];
        bool cancel;
        {
            std::lock_guard<std::mutex> lock(mu);
            cancel = j->cancel || stop;
        }
        if (cancel || j->done >= j->nsteps) {
            finish(j, cancel ? PD_JOB_CANCELLED : PD_JOB_DONE);
            b.members.erase(b.members.begin() + k);
            progressed = true;
            continue;
        }
        ++k;
    }
    if (b.members.empty()) return progressed;
    if (!b.st) {
        if (cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            for (Job *j : b.members) {
                j->status = fail(PD_ERR_CUDA, "batch stream creation failed");
                j->err = pd_last_error();
                finish(j, PD_JOB_FAILED);
            }
            b.members.clear();
            return true;
        }
    }
    int64_t n = chunk;
    for (Job *j : b.members) n = std::min(n, j->nsteps - j->done);
    std::vector<pd_env *> envs;
    for (Job *j : b.members) envs.push_back(j->env);
    pd_status s = fast_batch_steps(envs.data(), (int)envs.size(), n, b.st);
    if (s == PD_OK && cudaEventRecord(b.ev, b.st) != cudaSuccess) {
        cudaGetLastError();
        s = fail(PD_ERR_CUDA, "event record failed");
    }
    if (s != PD_OK) {
        const std::string err = pd_last_error();
        for (Job *j : b.members) {
            j->status = s;
            j->err = err;
            finish(j, PD_JOB_FAILED);
        }
        b.members.clear();
        return true;
    }
    b.chunk_now = n;
    b.inflight = true;
    return true;
}

// Stepping thread: every resident job on its own stream gets its next chunk
// as soon as its previous one has finished; the batches advance theirs.
void pd_server::step_loop() {
    cudaSetDevice(device);
    std::vector<Job *> active;
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(mu);
            for (Job *j : ready) active.push_back(j);
            ready.clear();
            if (active.empty() && batch[0].members.empty() && batch[1].members.empty() && batch[0].pending.empty() &&
                batch[1].pending.empty()) {
                if (stop) {
                    for (Batch &b : batch) {
                        if (b.st) cudaStreamDestroy(b.st);
                        if (b.ev) cudaEventDestroy(b.ev);
                        b = Batch{};
                    }
                    return;
                }
                wake.wait(lock);
                continue;
            }
        }
        bool progressed = false;
        for (Batch &b : batch) progressed |= step_batch(b);
        for (size_t k = 0; k < active.size();) {
            Job *j = active[k];
            if (j->inflight) {
                const cudaError_t q = cudaEventQuery(j->ev);
                if (q == cudaErrorNotReady) {
                    ++k;
                    continue;
                }
                j->inflight = false;
                if (q != cudaSuccess) {
                    j->status = fail(PD_ERR_CUDA, "job stream: %s", cudaGetErrorString(q));
                    j->err = pd_last_error();
                    finish(j, PD_JOB_FAILED);
                    active.erase(active.begin() + k);
                    progressed = true;
                    continue;
                }
                j->done += j->chunk_now;
            }
            bool cancel;
            {
                std::lock_guard<std::mutex> lock(mu);
                cancel = j->cancel || stop;
            }
            if (cancel || j->done >= j->nsteps) {
                finish(j, cancel ? PD_JOB_CANCELLED : PD_JOB_DONE);
                active.erase(active.begin() + k);
                progressed = true;
                continue;
            }
            // past its first chunk, a job that may share launches waits for
            // the next chunk of its precision's batch
            if (batching && j->done > 0 && j->env->precision != PD_PREC_FP64_SERIAL &&
                fast_land_flags(j->env) == PD_OK && fast_batchable(j->env)) {
                j->batched = true;
                batch[j->env->precision == PD_PREC_FP32C ? 1 : 0].pending.push_back(j);
                active.erase(active.begin() + k);
                progressed = true;
                continue;
            }
            const int64_t n = std::min(chunk, j->nsteps - j->done);
            pd_status s = j->env->precision == PD_PREC_FP64_SERIAL ? pd_env_vv_steps(j->env, n)
                                                                     : fast_vv_enqueue(j->env, n);
            if (s == PD_OK && cudaEventRecord(j->ev, j->env->st) != cudaSuccess) {
                cudaGetLastError();
                s = fail(PD_ERR_CUDA, "event record failed");
            }
            if (s != PD_OK) {
                j->status = s;
                j->err = pd_last_error();
                finish(j, PD_JOB_FAILED);
                active.erase(active.begin() + k);
                progressed = true;
                continue;
            }
            j->chunk_now = n;
            j->inflight = true;
            progressed = true;
            ++k;
        }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

namespace {
pd_status job_of(pd_server *srv, int64_t id, Job **out) {
    auto it = srv->jobs.find(id);
    if (it == srv->jobs.end()) return fail(PD_ERR_ARG, "no job %lld", (long long)id);
    *out = it->second.get();
    return PD_OK;
}

void fill_info(const Job *j, pd_job_info *info) {
    if (!info) return;
    std::memset(info, 0, sizeof(*info));
    info->state = j->state;
    info->status = j->status;
    info->steps_done = j->state == PD_JOB_DONE ? j->nsteps : j->done.load();
    info->particles = j->particles.load();
    info->footprint_bytes = j->footprint;
    info->bond_updates = j->bond_updates;
    if (j->state != PD_JOB_QUEUED) info->queue_ms = ms_between(j->t_submit, j->t_admit);
    if (j->state >= PD_JOB_DONE) info->latency_ms = ms_between(j->t_submit, j->t_done);
}
}  // namespace

extern "C" pd_status pd_server_create(pd_server **out, int32_t device, int64_t hbm_budget_bytes, int32_t max_active,
                                      int64_t chunk_steps) {
    if (!out) return fail(PD_ERR_ARG, "out is NULL");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(PD_ERR_NO_DEVICE, "no CUDA device is visible; libperidyn_b200 has no CPU path");
    }
    if (device < 0 || device >= n) return fail(PD_ERR_ARG, "device %d out of range (%d visible)", device, n);
    if (max_active < 1 || chunk_steps < 1) return fail(PD_ERR_ARG, "max_active and chunk_steps must be >= 1");
    CK(cudaSetDevice(device));
    if (hbm_budget_bytes <= 0) {
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        hbm_budget_bytes = (int64_t)(0.9 * (double)fr);
    }
    std::unique_ptr<pd_server> s(new (std::nothrow) pd_server());
    if (!s) return fail(PD_ERR_OOM, "host allocation failed");
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->max_active = max_active;
    s->chunk = chunk_steps;
    if (const char *e = std::getenv("PD_SERVE_BATCH")) s->batching = std::strcmp(e, "0") != 0;
    try {
        s->stepper = std::thread([p = s.get()] { p->step_loop(); });
        for (auto &t : s->admitters) t = std::thread([p = s.get()] { p->admit_loop(); });
    } catch (...) {
        {
            std::lock_guard<std::mutex> lock(s->mu);
            s->stop = true;
            s->wake.notify_all();
        }
        for (auto &t : s->admitters)
            if (t.joinable()) t.join();
        if (s->stepper.joinable()) s->stepper.join();
        return fail(PD_ERR_OOM, "cannot start the server threads");
    }
    *out = s.release();
    return PD_OK;
}

extern "C" pd_status pd_server_submit(pd_server *srv, pd_env *env, int64_t nsteps, int64_t *job) {
    if (!srv || !env || !job) return fail(PD_ERR_ARG, "NULL server, environment or job");
    if (env->finalized) return fail(PD_ERR_STATE, "submit an assembled environment before pd_env_finalize");
    if (env->device != srv->device)
        return fail(PD_ERR_ARG, "environment is on device %d, server on %d", env->device, srv->device);
    if (env->hb.empty()) return fail(PD_ERR_STATE, "environment has no material blocks");
    if (nsteps < 0) return fail(PD_ERR_ARG, "nsteps < 0");
    std::unique_ptr<Job> j(new (std::nothrow) Job());
    if (!j) return fail(PD_ERR_OOM, "host allocation failed");
    j->env = env;
    j->nsteps = nsteps;
    j->footprint = footprint_estimate(env);
    j->t_submit = Clock::now();
    std::lock_guard<std::mutex> lock(srv->mu);
    if (srv->stop) return fail(PD_ERR_STATE, "server is shutting down");
    j->id = srv->next_id++;
    *job = j->id;
    srv->queue.push_back(j.get());
    srv->jobs[j->id] = std::move(j);
    srv->wake.notify_all();
    return PD_OK;
}

extern "C" pd_status pd_server_poll(pd_server *srv, int64_t job, pd_job_info *info) {
    if (!srv) return fail(PD_ERR_ARG, "server is NULL");
    std::lock_guard<std::mutex> lock(srv->mu);
    Job *j = nullptr;
    PD_TRY(job_of(srv, job, &j));
    fill_info(j, info);
    if (j->state == PD_JOB_FAILED) return fail(j->status, "job %lld failed: %s", (long long)job, j->err.c_str());
    return PD_OK;
}

extern "C" pd_status pd_server_wait(pd_server *srv, int64_t job, double timeout_s, pd_job_info *info) {
    if (!srv) return fail(PD_ERR_ARG, "server is NULL");
    std::unique_lock<std::mutex> lock(srv->mu);
    Job *j = nullptr;
    PD_TRY(job_of(srv, job, &j));
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 0.0));
    while (j->state < PD_JOB_DONE) {
        if (srv->changed.wait_until(lock, until) == std::cv_status::timeout && j->state < PD_JOB_DONE) {
            fill_info(j, info);
            return fail(PD_ERR_TIMEOUT, "job %lld not finished after %.3f s", (long long)job, timeout_s);
        }
    }
    fill_info(j, info);
    if (j->state == PD_JOB_FAILED) return fail(j->status, "job %lld failed: %s", (long long)job, j->err.c_str());
    return PD_OK;
}

extern "C" pd_status pd_server_result(pd_server *srv, int64_t job, double *y, double *v, double *damage) {
    if (!srv) return fail(PD_ERR_ARG, "server is NULL");
    std::lock_guard<std::mutex> lock(srv->mu);
    Job *j = nullptr;
    PD_TRY(job_of(srv, job, &j));
    if (j->state != PD_JOB_DONE) return fail(PD_ERR_STATE, "job %lld is not done (state %d)", (long long)job, j->state);
    if (y) std::memcpy(y, j->y.data(), j->y.size() * sizeof(double));
    if (v) std::memcpy(v, j->v.data(), j->v.size() * sizeof(double));
    if (damage) std::memcpy(damage, j->damage.data(), j->damage.size() * sizeof(double));
    srv->jobs.erase(job);
    return PD_OK;
}

extern "C" pd_status pd_server_cancel(pd_server *srv, int64_t job) {
    if (!srv) return fail(PD_ERR_ARG, "server is NULL");
    std::lock_guard<std::mutex> lock(srv->mu);
    Job *j = nullptr;
    PD_TRY(job_of(srv, job, &j));
    j->cancel = true;
    srv->wake.notify_all();
    return PD_OK;
}

extern "C" pd_status pd_server_destroy(pd_server *srv) {
    if (!srv) return PD_OK;
    {
        std::lock_guard<std::mutex> lock(srv->mu);
        srv->stop = true;
        for (Job *j : srv->queue) j->cancel = true;
        srv->wake.notify_all();
    }
    for (auto &t : srv->admitters)
        if (t.joinable()) t.join();
    if (srv->stepper.joinable()) srv->stepper.join();
    for (auto &kv : srv->jobs)
        if (kv.second->env) pd_env_destroy(kv.second->env);
    delete srv;
    return PD_OK;
}
