// The serving loop: admission by HBM budget, continuous batching of direct
// jobs, overlapped tree jobs, latency accounting.
//
// One host thread owns every device object. API threads only touch the job
// table and the queues, under one mutex, and wait on a condition variable.
// The loop never blocks on the device while steps are in flight: it polls one
// event per running entity, retires finished steps and launches the next ones:
//   * direct jobs are grouped by (integrator, dt); each group is one Batch
//     whose step is a replayed graph; members join or leave only while the
//     group has no step in flight, so membership changes fall between steps;
//   * each tree job is a System (the full Barnes-Hut pipeline captured as one
//     graph per step).
// Every entity issues its work on the server's single device stream. Each
// step runs the whole GPU (the batched kernel is persistent: its CTAs hold
// every SM until its queue drains), so steps of different entities are
// ordered on one stream, not interleaved kernel by kernel: an entity puts its
// next step at the back of the stream when its previous one retires, which
// gives round-robin service with the stream never empty while work remains.
// With fake_device set, nothing touches CUDA: a step "runs" for a modelled
// time, so the admission, queueing and latency logic is testable on a CPU.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "batch.hpp"
#include "orrery_b200.h"
#include "runtime.hpp"
#include "system.hpp"

namespace ob {
namespace {

using Clock = std::chrono::steady_clock;

// The moment `seconds` from now. The wait is clamped to [0, 1e9 s] so that the
// conversion to the clock's integer ticks cannot overflow: a negative or NaN
// timeout waits not at all, an infinite one about 31 years.
Clock::time_point deadline_after(double seconds) {
    const double clamped = std::min(std::max(0.0, seconds), 1e9);
    return Clock::now() +
           std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(clamped));
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) {
        return 0.0;
    }
    std::sort(v.begin(), v.end());
    const double pos = q * static_cast<double>(v.size() - 1);
    const size_t lo = static_cast<size_t>(std::floor(pos));
    const size_t hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - static_cast<double>(lo));
}

// Device bytes a tree job holds: state (80 B per particle), ordering, sorted
// copy and leaf records (88 B per particle) and about 0.75 N + 1024 nodes at
// 188 B (FP64 node 64, quadrupole 48, walk record 64, first particle 4, child
// and arrival counts 8).
uint64_t tree_job_bytes(uint64_t n) { return n * 80 + n * 88 + (n * 3 / 4 + 1024) * 188; }

uint64_t direct_job_bytes(uint64_t n) {
    return Batch::footprint(static_cast<uint32_t>(n)) * Batch::kBytesPerParticle;
}

struct Job {
    uint64_t id = 0;
    ob_job_spec spec{};
    int status = OB_JOB_QUEUED;
    double submitted = 0, admitted = 0, finished = 0;
    uint64_t steps_done = 0;
    uint64_t bytes = 0;
    double work = 0;             // work units (work_units below)
    std::vector<double> input;   // x y z vx vy vz m (7n)
    std::vector<double> output;  // x y z vx vy vz ax ay az (9n)
    bool cancel_requested = false;
    // Device side (loop thread only).
    std::unique_ptr<System> system; // tree jobs
    int64_t member = -1;            // direct jobs: id in its group's batch
    bool in_flight = false;
    Clock::time_point launched;
    double fake_end = 0;            // fake mode: when the step in flight ends
    cudaEvent_t done = nullptr;     // recorded after the step in flight
};

struct Group {
    std::unique_ptr<Batch> batch;   // null in fake mode
    std::vector<Job *> members;
    std::vector<Job *> joining;
    bool in_flight = false;
    Clock::time_point launched;
    double fake_end = 0;
    uint64_t pairs = 0;             // sum N(N-1) of members (fake-mode cost)
    cudaEvent_t done = nullptr;     // recorded after the step in flight
};

} // namespace

class Server {
public:
    explicit Server(const ob_server_config &config) : config_(config), start_(Clock::now()) {
        if (config_.direct_arena_particles == 0) {
            config_.direct_arena_particles = 8u << 20;
        }
        if (config_.max_tree_jobs == 0) {
            config_.max_tree_jobs = 1;
        }
        if (!config_.fake_device) {
            check(cudaGetDevice(&device_), "cudaGetDevice");
        }
        worker_ = std::thread([this] { loop(); });
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stop_ = true;
        }
        cv_.notify_all();
        worker_.join();
    }

    uint64_t submit(const ob_job_spec &spec, const double *const *state) {
        validate(spec);
        auto job = std::make_unique<Job>();
        job->spec = spec;
        job->bytes = spec.kind == OB_SOLVER_DIRECT ? direct_job_bytes(spec.n)
                                                   : tree_job_bytes(spec.n);
        job->work = ob_work_units(spec.n, spec.steps, spec.kind);
        if (config_.max_job_work > 0 && job->work > config_.max_job_work) {
            std::lock_guard<std::mutex> lock(mutex_);
            ++rejected_;
            throw Error(OB_ERROR_CAPACITY, "the job's work exceeds the server's per-job ceiling");
        }
        if (job->bytes > config_.hbm_budget_bytes ||
            (spec.kind == OB_SOLVER_DIRECT &&
             (Batch::footprint(static_cast<uint32_t>(spec.n)) > config_.direct_arena_particles ||
              (config_.direct_pairs_cap > 0 &&
               spec.n * (spec.n - 1) > config_.direct_pairs_cap)))) {
            std::lock_guard<std::mutex> lock(mutex_);
            ++rejected_;
            throw Error(OB_ERROR_CAPACITY, "the job can never fit the server's budget");
        }
        const size_t n = spec.n;
        job->input.assign(7 * n, 0.0);
        for (int k = 0; k < 7; ++k) {
            if (state[k] != nullptr) {
                std::memcpy(job->input.data() + k * n, state[k], sizeof(double) * n);
            }
        }
        std::lock_guard<std::mutex> lock(mutex_);
        job->id = ++next_id_;
        job->submitted = now();
        const uint64_t id = job->id;
        (spec.kind == OB_SOLVER_DIRECT ? direct_queue_ : tree_queue_).push_back(job.get());
        jobs_[id] = std::move(job);
        ++submitted_;
        cv_.notify_all();
        return id;
    }

    void wait(uint64_t id, double timeout_s, ob_job_report *report, double *const *out) {
        std::unique_lock<std::mutex> lock(mutex_);
        const auto it = jobs_.find(id);
        if (it == jobs_.end()) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "no such job");
        }
        Job *job = it->second.get();
        const auto deadline = deadline_after(timeout_s);
        while (job->status == OB_JOB_QUEUED || job->status == OB_JOB_RUNNING) {
            if (cv_.wait_until(lock, deadline) == std::cv_status::timeout &&
                (job->status == OB_JOB_QUEUED || job->status == OB_JOB_RUNNING)) {
                throw Error(OB_ERROR_TIMEOUT, "the job did not finish in time");
            }
        }
        if (report != nullptr) {
            *report = ob_job_report{job->id,        job->status,    0,
                                    job->steps_done, job->submitted, job->admitted,
                                    job->finished};
        }
        const size_t n = job->spec.n;
        if (job->status == OB_JOB_DONE && job->output.size() == 9 * n) {
            for (int k = 0; k < 9; ++k) {
                if (out[k] != nullptr) {
                    std::memcpy(out[k], job->output.data() + k * n, sizeof(double) * n);
                }
            }
        }
    }

    void cancel(uint64_t id) {
        std::lock_guard<std::mutex> lock(mutex_);
        const auto it = jobs_.find(id);
        if (it == jobs_.end()) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "no such job");
        }
        it->second->cancel_requested = true;
        cv_.notify_all();
    }

    void drain(double timeout_s) {
        std::unique_lock<std::mutex> lock(mutex_);
        const auto deadline = deadline_after(timeout_s);
        while (!idle_locked()) {
            if (cv_.wait_until(lock, deadline) == std::cv_status::timeout && !idle_locked()) {
                throw Error(OB_ERROR_TIMEOUT, "the server did not drain in time");
            }
        }
    }

    ob_server_summary stats() {
        std::lock_guard<std::mutex> lock(mutex_);
        ob_server_summary s{};
        s.submitted = submitted_;
        s.admitted = admitted_;
        s.completed = completed_;
        s.failed = failed_;
        s.cancelled = cancelled_;
        s.rejected = rejected_;
        s.queued = direct_queue_.size() + tree_queue_.size();
        s.running = running_;
        s.elapsed_s = now();
        s.jobs_per_s = s.elapsed_s > 0 ? static_cast<double>(completed_) / s.elapsed_s : 0.0;
        s.job_latency_p50_s = percentile(job_latency_, 0.50);
        s.job_latency_p99_s = percentile(job_latency_, 0.99);
        s.step_latency_p50_ms = percentile(step_latency_, 0.50) * 1e3;
        s.step_latency_p99_ms = percentile(step_latency_, 0.99) * 1e3;
        s.hbm_in_use = hbm_in_use_;
        s.hbm_peak = hbm_peak_;
        return s;
    }

private:
    double now() const {
        return std::chrono::duration<double>(Clock::now() - start_).count();
    }

    bool idle_locked() const {
        return direct_queue_.empty() && tree_queue_.empty() && running_ == 0;
    }

    static void validate(const ob_job_spec &spec) {
        if (spec.kind != OB_SOLVER_DIRECT && spec.kind != OB_SOLVER_TREE) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "unknown job kind");
        }
        if (spec.integrator == OB_INTEGRATOR_RK4) {
            throw Error(OB_ERROR_UNSUPPORTED, "served jobs step with VV or Yoshida-4");
        }
        if (spec.integrator != OB_INTEGRATOR_VV && spec.integrator != OB_INTEGRATOR_YOSHIDA4) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "unknown integrator");
        }
        if (spec.n == 0 || spec.n > 0x3fffffffull) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "a job needs 1 .. 2^30-1 particles");
        }
        if (!std::isfinite(spec.dt) || spec.steps == 0) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "a job needs a finite timestep and steps");
        }
        if (!(spec.softening_squared >= 0.0) || !std::isfinite(spec.softening_squared) ||
            (spec.kind == OB_SOLVER_DIRECT && !(spec.softening_squared > 0.0))) {
            throw Error(OB_ERROR_INVALID_ARGUMENT,
                        "softening squared must be finite (and positive for direct jobs)");
        }
    }

    // ---------------------------------------------------------------- loop

    void loop() {
        if (!config_.fake_device) {
            cudaSetDevice(device_);
            if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) {
                stream_ = nullptr;
            }
        }
        while (true) {
            {
                std::unique_lock<std::mutex> lock(mutex_);
                if (stop_) {
                    break;
                }
            }
            bool progress = false;
            try {
                progress |= admit();
                progress |= service_trees();
                progress |= service_groups();
            } catch (const std::exception &) {
                fail_everything();
                progress = true;
            }
            if (!progress) {
                std::unique_lock<std::mutex> lock(mutex_);
                if (stop_) {
                    break;
                }
                cv_.wait_for(lock, std::chrono::microseconds(200));
            }
        }
        shutdown();
    }

    // Moves queued jobs to running while the budget and the caps allow, in
    // arrival order per solver kind.
    bool admit() {
        std::vector<Job *> direct, tree;
        {
            std::lock_guard<std::mutex> lock(mutex_);
            drop_cancelled_queued(direct_queue_);
            drop_cancelled_queued(tree_queue_);
            while (!tree_queue_.empty() && running_trees_ < config_.max_tree_jobs &&
                   hbm_in_use_ + tree_queue_.front()->bytes <= config_.hbm_budget_bytes &&
                   work_allows(tree_queue_.front())) {
                Job *job = tree_queue_.front();
                tree_queue_.pop_front();
                start_job_locked(job);
                ++running_trees_;
                tree.push_back(job);
            }
            while (!direct_queue_.empty()) {
                Job *job = direct_queue_.front();
                const uint64_t pairs = job->spec.n * (job->spec.n - 1);
                if (hbm_in_use_ + job->bytes > config_.hbm_budget_bytes) {
                    break;
                }
                if (config_.direct_pairs_cap > 0 && direct_pairs_ > 0 &&
                    direct_pairs_ + pairs > config_.direct_pairs_cap) {
                    break;
                }
                if (!work_allows(job)) {
                    break;
                }
                direct_queue_.pop_front();
                start_job_locked(job);
                direct_pairs_ += pairs;
                direct.push_back(job);
            }
        }
        for (Job *job : tree) {
            begin_tree(job);
        }
        for (Job *job : direct) {
            const auto key = std::make_tuple(job->spec.integrator, job->spec.dt);
            Group &g = groups_[key];
            if (!g.batch && !config_.fake_device) {
                g.batch = std::make_unique<Batch>(config_.direct_arena_particles, device_stream());
                check(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming), "an event");
            }
            g.joining.push_back(job);
        }
        return !tree.empty() || !direct.empty();
    }

    void drop_cancelled_queued(std::deque<Job *> &queue) {
        for (auto it = queue.begin(); it != queue.end();) {
            if ((*it)->cancel_requested) {
                (*it)->status = OB_JOB_CANCELLED;
                (*it)->finished = now();
                ++cancelled_;
                it = queue.erase(it);
                cv_.notify_all();
            } else {
                ++it;
            }
        }
    }

    // The running jobs' work units leave room for this one (a job alone
    // always runs: the per-job ceiling is checked at submission).
    bool work_allows(const Job *job) const {
        return config_.max_running_work <= 0 || running_ == 0 ||
               running_work_ + job->work <= config_.max_running_work;
    }

    void start_job_locked(Job *job) {
        job->status = OB_JOB_RUNNING;
        job->admitted = now();
        running_work_ += job->work;
        hbm_in_use_ += job->bytes;
        hbm_peak_ = std::max(hbm_peak_, hbm_in_use_);
        ++admitted_;
        ++running_;
    }

    void begin_tree(Job *job) {
        const ob_job_spec &s = job->spec;
        if (!config_.fake_device) {
            ob_solver_params p{OB_SOLVER_TREE, OB_PRECISION_FP32, s.softening_squared,
                               s.opening_angle, s.leaf_capacity, s.quadrupole, 0};
            job->system = std::make_unique<System>(p, static_cast<uint32_t>(s.n), device_stream());
            check(cudaEventCreateWithFlags(&job->done, cudaEventDisableTiming), "an event");
            const size_t n = s.n;
            const double *in = job->input.data();
            job->system->set_state(in, in + n, in + 2 * n, in + 3 * n, in + 4 * n, in + 5 * n,
                                   in + 6 * n);
        }
        launch_tree(job);
    }

    void launch_tree(Job *job) {
        job->launched = Clock::now();
        job->in_flight = true;
        if (config_.fake_device) {
            const double evals = job->spec.integrator == OB_INTEGRATOR_YOSHIDA4 ? 3.0 : 1.0;
            job->fake_end = now() + evals * static_cast<double>(job->spec.n) *
                                        config_.fake_tree_ns_per_particle * 1e-9;
        } else {
            job->system->step_async(job->spec.integrator, job->spec.dt, 1);
            check(cudaEventRecord(job->done, device_stream()), "recording a step");
        }
    }

    cudaStream_t device_stream() const {
        if (stream_ == nullptr) {
            throw Error(OB_ERROR_CUDA, "the server has no device stream");
        }
        return stream_;
    }

    bool step_done(cudaEvent_t done, double fake_end) const {
        if (config_.fake_device) {
            return now() >= fake_end;
        }
        const cudaError_t q = cudaEventQuery(done);
        if (q == cudaErrorNotReady) {
            return false;
        }
        check(q, "a serving step");
        return true;
    }

    static void release(cudaEvent_t &event) {
        if (event != nullptr) {
            cudaEventDestroy(event);
            event = nullptr;
        }
    }

    bool service_trees() {
        bool progress = false;
        std::vector<Job *> running;
        {
            std::lock_guard<std::mutex> lock(mutex_);
            for (auto &entry : jobs_) {
                Job *j = entry.second.get();
                if (j->status == OB_JOB_RUNNING && j->spec.kind == OB_SOLVER_TREE && j->in_flight) {
                    running.push_back(j);
                }
            }
        }
        for (Job *job : running) {
            if (!step_done(job->done, job->fake_end)) {
                continue;
            }
            progress = true;
            job->in_flight = false;
            const double latency =
                std::chrono::duration<double>(Clock::now() - job->launched).count();
            bool finished, cancelled;
            {
                std::lock_guard<std::mutex> lock(mutex_);
                ++job->steps_done;
                step_latency_.push_back(latency);
                finished = job->steps_done >= job->spec.steps;
                cancelled = job->cancel_requested;
            }
            if (finished || cancelled) {
                if (finished && job->system) {
                    job->system->synchronize();
                    collect_output(job, [&](double *const *out) { job->system->get_state(out); });
                } else if (finished) {
                    fake_output(job);
                }
                job->system.reset();
                release(job->done);
                finish(job, finished ? OB_JOB_DONE : OB_JOB_CANCELLED);
                std::lock_guard<std::mutex> lock(mutex_);
                --running_trees_;
            } else {
                launch_tree(job);
            }
        }
        return progress;
    }

    template <typename F> void collect_output(Job *job, F &&download) {
        const size_t n = job->spec.n;
        job->output.assign(9 * n, 0.0);
        double *out[9];
        for (int k = 0; k < 9; ++k) {
            out[k] = job->output.data() + k * n;
        }
        download(out);
    }

    void fake_output(Job *job) {
        const size_t n = job->spec.n;
        job->output.assign(9 * n, 0.0);
        std::memcpy(job->output.data(), job->input.data(), sizeof(double) * 6 * n);
    }

    bool service_groups() {
        bool progress = false;
        for (auto &entry : groups_) {
            Group &g = entry.second;
            const int integrator = std::get<0>(entry.first);
            const double dt = std::get<1>(entry.first);
            if (g.in_flight) {
                if (!step_done(g.done, g.fake_end)) {
                    continue;
                }
                g.in_flight = false;
                progress = true;
                const double latency =
                    std::chrono::duration<double>(Clock::now() - g.launched).count();
                std::vector<Job *> leaving;
                {
                    std::lock_guard<std::mutex> lock(mutex_);
                    for (Job *job : g.members) {
                        ++job->steps_done;
                        step_latency_.push_back(latency);
                        if (job->steps_done >= job->spec.steps || job->cancel_requested) {
                            leaving.push_back(job);
                        }
                    }
                }
                if (g.batch && !leaving.empty()) {
                    g.batch->synchronize(); // also reports a device-side wait that ran out
                }
                for (Job *job : leaving) {
                    const bool done = job->steps_done >= job->spec.steps;
                    if (g.batch) {
                        if (done) {
                            collect_output(job, [&](double *const *out) {
                                g.batch->get_state(static_cast<uint32_t>(job->member), out);
                            });
                        }
                        g.batch->remove(static_cast<uint32_t>(job->member));
                    } else if (done) {
                        fake_output(job);
                    }
                    g.members.erase(std::find(g.members.begin(), g.members.end(), job));
                    g.pairs -= job->spec.n * (job->spec.n - 1);
                    {
                        std::lock_guard<std::mutex> lock(mutex_);
                        direct_pairs_ -= job->spec.n * (job->spec.n - 1);
                    }
                    finish(job, done ? OB_JOB_DONE : OB_JOB_CANCELLED);
                }
            }
            // Between steps: new members join.
            if (!g.joining.empty()) {
                std::vector<uint32_t> ids;
                std::vector<Job *> still_waiting;
                for (Job *job : g.joining) {
                    const size_t n = job->spec.n;
                    if (g.batch) {
                        const int64_t id = g.batch->add(static_cast<uint32_t>(n),
                                                        job->spec.softening_squared);
                        if (id < 0) {
                            still_waiting.push_back(job); // arena full for now
                            continue;
                        }
                        job->member = id;
                        const double *in = job->input.data();
                        g.batch->set_state(static_cast<uint32_t>(id), in, in + n, in + 2 * n,
                                           in + 3 * n, in + 4 * n, in + 5 * n, in + 6 * n);
                        ids.push_back(static_cast<uint32_t>(id));
                    }
                    g.members.push_back(job);
                    g.pairs += n * (n - 1);
                }
                if (g.batch && !ids.empty()) {
                    g.batch->refresh_members(ids);
                }
                g.joining.swap(still_waiting);
                progress = true;
            }
            if (!g.in_flight && !g.members.empty()) {
                g.launched = Clock::now();
                g.in_flight = true;
                if (g.batch) {
                    g.batch->step_async(integrator, dt, 1);
                    check(cudaEventRecord(g.done, device_stream()), "recording a step");
                } else {
                    const double evals = integrator == OB_INTEGRATOR_YOSHIDA4 ? 3.0 : 1.0;
                    g.fake_end = now() + evals * static_cast<double>(g.pairs) /
                                             (config_.fake_direct_gint_s * 1e9);
                }
                progress = true;
            }
        }
        return progress;
    }

    void finish(Job *job, int status) {
        std::lock_guard<std::mutex> lock(mutex_);
        job->status = status;
        job->finished = now();
        job->in_flight = false;
        hbm_in_use_ -= job->bytes;
        --running_;
        running_work_ = running_ == 0 ? 0.0 : running_work_ - job->work;
        if (status == OB_JOB_DONE) {
            ++completed_;
            job_latency_.push_back(job->finished - job->submitted);
        } else if (status == OB_JOB_CANCELLED) {
            ++cancelled_;
        } else {
            ++failed_;
        }
        job->input.clear();
        job->input.shrink_to_fit();
        cv_.notify_all();
    }

    // A device error: every running job fails; queued jobs stay queued.
    void fail_everything() {
        for (auto &entry : groups_) {
            for (Job *job : entry.second.members) {
                finish(job, OB_JOB_FAILED);
                std::lock_guard<std::mutex> lock(mutex_);
                direct_pairs_ -= job->spec.n * (job->spec.n - 1);
            }
            for (Job *job : entry.second.joining) {
                finish(job, OB_JOB_FAILED);
                std::lock_guard<std::mutex> lock(mutex_);
                direct_pairs_ -= job->spec.n * (job->spec.n - 1);
            }
        }
        for (auto &entry : groups_) {
            release(entry.second.done);
        }
        groups_.clear();
        std::vector<Job *> trees;
        {
            std::lock_guard<std::mutex> lock(mutex_);
            for (auto &entry : jobs_) {
                if (entry.second->status == OB_JOB_RUNNING &&
                    entry.second->spec.kind == OB_SOLVER_TREE) {
                    trees.push_back(entry.second.get());
                }
            }
        }
        for (Job *job : trees) {
            job->system.reset();
            release(job->done);
            finish(job, OB_JOB_FAILED);
            std::lock_guard<std::mutex> lock(mutex_);
            --running_trees_;
        }
        cudaGetLastError();
    }

    void shutdown() {
        std::vector<Job *> running;
        {
            std::lock_guard<std::mutex> lock(mutex_);
            for (auto &entry : jobs_) {
                Job *j = entry.second.get();
                if (j->status == OB_JOB_QUEUED) {
                    j->status = OB_JOB_CANCELLED;
                    ++cancelled_;
                } else if (j->status == OB_JOB_RUNNING) {
                    running.push_back(j);
                }
            }
        }
        if (stream_ != nullptr) {
            cudaStreamSynchronize(stream_);
        }
        for (Job *j : running) {
            j->system.reset();
            release(j->done);
            finish(j, OB_JOB_CANCELLED);
        }
        for (auto &entry : groups_) {
            release(entry.second.done);
        }
        groups_.clear();
        if (stream_ != nullptr) {
            cudaStreamDestroy(stream_);
            stream_ = nullptr;
        }
        cv_.notify_all();
    }

    ob_server_config config_;
    Clock::time_point start_;
    int device_ = 0;
    cudaStream_t stream_ = nullptr; // the device stream of every entity (loop thread)
    std::thread worker_;
    std::mutex mutex_;
    std::condition_variable cv_;
    bool stop_ = false;
    uint64_t next_id_ = 0;
    std::map<uint64_t, std::unique_ptr<Job>> jobs_;
    std::deque<Job *> direct_queue_, tree_queue_;
    std::map<std::tuple<int, double>, Group> groups_; // loop thread only
    uint64_t submitted_ = 0, admitted_ = 0, completed_ = 0, failed_ = 0, cancelled_ = 0,
             rejected_ = 0, running_ = 0;
    uint32_t running_trees_ = 0;
    uint64_t direct_pairs_ = 0;
    double running_work_ = 0; // work units of the running jobs
    uint64_t hbm_in_use_ = 0, hbm_peak_ = 0;
    std::vector<double> job_latency_, step_latency_;
};

} // namespace ob

struct ob_server {
    std::unique_ptr<ob::Server> impl;
};

namespace {
template <typename F> int server_call(F &&body) {
    try {
        body();
        return OB_OK;
    } catch (const ob::Error &e) {
        return ob::set_error(e.code(), e.what());
    } catch (const std::exception &e) {
        return ob::set_error(OB_ERROR_INVALID_ARGUMENT, e.what());
    }
}
void need(bool condition, const char *message) {
    if (!condition) {
        throw ob::Error(OB_ERROR_INVALID_ARGUMENT, message);
    }
}
} // namespace

extern "C" double ob_work_units(uint64_t count, uint64_t steps, int32_t kind) {
    // The reference service's cost model (service/orrery_service/limits.py:82-111):
    // count^2 per step for the direct sum, count log2(count) for the tree.
    if (count < 2) {
        return 0.0;
    }
    const double c = static_cast<double>(count);
    const double per_step = kind == OB_SOLVER_DIRECT ? c * c : c * std::log2(c);
    return per_step * static_cast<double>(steps);
}

extern "C" {

int ob_server_create(const ob_server_config *config, ob_server **out) {
    return server_call([&] {
        need(config != nullptr && out != nullptr, "NULL argument");
        *out = nullptr;
        need(config->hbm_budget_bytes > 0, "the server needs an HBM budget");
        if (config->fake_device) {
            need(config->fake_direct_gint_s > 0 && config->fake_tree_ns_per_particle > 0,
                 "fake mode needs its cost model");
        } else {
            int count = 0;
            if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
                cudaGetLastError();
                throw ob::Error(OB_ERROR_NO_DEVICE, "no CUDA device is visible");
            }
        }
        auto s = std::make_unique<ob_server>();
        s->impl = std::make_unique<ob::Server>(*config);
        *out = s.release();
    });
}

void ob_server_destroy(ob_server *server) { delete server; }

int ob_server_submit(ob_server *server, const ob_job_spec *spec, const double *x,
                     const double *y, const double *z, const double *vx, const double *vy,
                     const double *vz, const double *m, uint64_t *job_id) {
    return server_call([&] {
        need(server != nullptr && spec != nullptr && job_id != nullptr, "NULL argument");
        need(x && y && z && m, "positions and masses are required");
        const double *state[7] = {x, y, z, vx, vy, vz, m};
        *job_id = server->impl->submit(*spec, state);
    });
}

int ob_server_wait(ob_server *server, uint64_t job_id, double timeout_s, ob_job_report *report,
                   double *x, double *y, double *z, double *vx, double *vy, double *vz,
                   double *ax, double *ay, double *az) {
    return server_call([&] {
        need(server != nullptr, "server is NULL");
        double *out[9] = {x, y, z, vx, vy, vz, ax, ay, az};
        server->impl->wait(job_id, timeout_s, report, out);
    });
}

int ob_server_cancel(ob_server *server, uint64_t job_id) {
    return server_call([&] {
        need(server != nullptr, "server is NULL");
        server->impl->cancel(job_id);
    });
}

int ob_server_stats(ob_server *server, ob_server_summary *stats) {
    return server_call([&] {
        need(server != nullptr && stats != nullptr, "NULL argument");
        *stats = server->impl->stats();
    });
}

int ob_server_drain(ob_server *server, double timeout_s) {
    return server_call([&] {
        need(server != nullptr, "server is NULL");
        server->impl->drain(timeout_s);
    });
}

} // extern "C"
