// Served mode: continuous batching of window-solve requests (see the
// cgmli_server_* declarations in cgmli_backend.h).
//
// Two solvers, each with its own CUDA stream, and two threads.  The scheduler
// takes the queued requests that fit the next batch (arrival order, window cap,
// device-footprint budget) as soon as a solver is free, builds and uploads that
// batch and launches its LM solve and marginalization.  The completion thread
// waits for each launched batch in order, writes the states back into the
// callers' windows, records the reports and priors, and frees the solver.  The
// host work of one batch therefore overlaps both the device work and the
// read-back of the other, and requests arriving meanwhile join the next batch.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/cgmli_backend.h"
#include "topology.h"

namespace cgmli {
int setLastError(int code, const char* message);
}  // namespace cgmli

namespace {
using Clock = std::chrono::steady_clock;

struct Request {
    long long ticket = 0;
    cgmli_window window{};
    int victim = -1;
    Clock::time_point submitted, completed;
    bool complete = false;
    cgmli_solve_report report{};
    // prior of a request with a victim
    int rank = 0, cols = 0, numBlocks = 0;
    std::vector<int> kinds, index;
    std::vector<double> reference, A, r0;
    // gated solve: the window's gate report and rejected factors
    cgmli_gate_report gate{};
    std::vector<unsigned char> rejected;
    // IMU samples for the refresh before the solve (num_imu_samples 0: none) and the
    // factors after it
    cgmli_server_request extra{};
    std::vector<cgmli_frozen_imu> imu;
    int imuRefreshed = 0;
    // calibration information at the solved states (extra.calibration_information)
    int calibStatus = CGMLI_E_INVALID, calibSize = 0, calibBlocks = 0;
    // CGMLI_MARGIN_SECOND_NEW_IMU_MERGE: the merge's outcome and, when re-integrated,
    // the merged factor (mergeStatus: the read's code when it failed)
    int mergeState = CGMLI_IMU_MERGE_NONE, mergeStatus = CGMLI_OK;
    cgmli_frozen_imu merged{};
    std::vector<int> calibKind, calibIndex;
    std::vector<double> calibConditional, calibEvals;
};

// Device bytes a window occupies in a batch (observation arrays and the uploaded
// payload they are gathered from, landmark and dense per-window arrays, both state
// buffers, the staged rows and the marginalization; with deterministic sums, the
// slots of its pair units (about 256 observations each) and of its Schur units
// (estimated at 64 landmarks each), at most 128 of each kind).
// The solvers' device arrays are grow-only and grow by at least half their size,
// so a batch whose windows need N bytes can leave a solver holding up to 1.5 N:
// admission counts kGrowth times the footprint.
constexpr double kGrowth = 1.5;
long long footprint(const cgmli_window& w, bool deterministic) {
    const long long F = w.num_observations, L = w.num_landmarks, K = w.num_keyframes;
    const long long ncal = (w.estimate_extrinsics ? 6ll * w.num_extrinsics : 0) + (w.estimate_td ? 1 : 0);
    const long long Nr = 15 * K + ncal, Npc = 6 * K + ncal, m = 15 * K + 6ll * w.num_extrinsics + 1;
    long long bytes = F * (120 + 108 + 448) + L * (160 + 8 * (6 * 12 + 7)) + 8 * (3 * Nr * Nr + Npc * Npc + 4 * m * m) + 4096;
    if (deterministic) {
        const long long units = std::min(128ll, (F + 255) / 256) + std::min(128ll, L / 64 + 1);
        bytes += 8 * units * (Npc * (Npc + 1) / 2 + Npc);
    }
    return bytes;
}
}  // namespace

struct cgmli_server {
    cgmli_server_options opt{};
    cgmli_solver* solver[2] = {nullptr, nullptr};
    std::mutex mu;
    std::condition_variable work, done, freed, launchedCv;
    std::deque<Request*> queue;
    // shared: a poller waiting on a request keeps it alive if another thread releases it
    std::unordered_map<long long, std::shared_ptr<Request>> requests;
    long long nextTicket = 1;
    bool stopping = false;
    std::thread worker;

    struct Batch {
        std::vector<Request*> reqs;
        std::vector<cgmli_window> windows;
        int solver = 0;
        bool marg = false;
        int status = CGMLI_OK;
        bool imu = false;  // the batch carries IMU samples (refreshed factors are read back)
        double launchMs = 0;
        double phaseMs[3] = {0, 0, 0};  // host time of set_windows, the solve launch, the marginalization launch
    };
    bool busy[2] = {false, false};                 // solver has a launched, uncompleted batch
    long long solverBytes[2] = {0, 0};             // device bytes each solver holds (after its last launch)
    std::deque<std::unique_ptr<Batch>> launched;   // scheduler -> completion thread
    bool schedulerDone = false;
    bool trace = false;

    // Launches a batch on solver s (asynchronous on its stream).
    void launch(Batch& b) {
        cgmli_solver* S = solver[b.solver];
        const int n = (int)b.reqs.size();
        b.windows.resize(n);
        std::vector<int> victims(n, -1);
        for (int i = 0; i < n; ++i) {
            b.windows[i] = b.reqs[i]->window;
            victims[i] = b.reqs[i]->victim;
            b.marg = b.marg || victims[i] >= 0;
        }
        const auto t0 = Clock::now();
        b.status = cgmli_solver_set_windows(S, b.windows.data(), n);
        if (b.status == CGMLI_OK) b.status = refreshImu(b);
        const auto t1 = Clock::now();
        if (b.status == CGMLI_OK)
            b.status = opt.nis_threshold > 0 ? cgmli_solver_solve_gated(S, opt.iterations, opt.nis_threshold, opt.max_refits, opt.pre_gate)
                                             : cgmli_solver_solve(S, opt.iterations);
        if (b.status == CGMLI_OK) calibration(b);
        const auto t2 = Clock::now();
        if (b.status == CGMLI_OK && b.marg) b.status = cgmli_solver_marginalize(S, victims.data(), opt.policy);
        const auto t3 = Clock::now();
        b.phaseMs[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
        b.phaseMs[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
        b.phaseMs[2] = std::chrono::duration<double, std::milli>(t3 - t2).count();
    }

    // The batch's IMU samples, when a request brought some: every IMU factor of the
    // batch in order, a request's ranges moved into the concatenated samples, the
    // factors of windows without samples with empty ranges (kept as given); then the
    // refresh, enqueued before the solve.
    int refreshImu(Batch& b) {
        bool any = false;
        for (Request* r : b.reqs) any = any || r->extra.num_imu_samples > 0;
        if (!any) return CGMLI_OK;
        std::vector<long long> times, t0, t1;
        std::vector<double> readings;
        std::vector<int> range;
        for (Request* r : b.reqs) {
            const cgmli_server_request& x = r->extra;
            const int nimu = r->window.num_imu, base = (int)times.size();
            if (x.num_imu_samples > 0) {
                times.insert(times.end(), x.imu_sample_time_ns, x.imu_sample_time_ns + x.num_imu_samples);
                readings.insert(readings.end(), x.imu_sample_readings, x.imu_sample_readings + 6ll * x.num_imu_samples);
            }
            for (int q = 0; q < nimu; ++q) {
                const bool has = x.num_imu_samples > 0;
                range.push_back(has ? base + x.imu_range[2 * q] : 0);
                range.push_back(has ? base + x.imu_range[2 * q + 1] : 0);
                t0.push_back(has ? x.imu_t0_ns[q] : 0);
                t1.push_back(has ? x.imu_t1_ns[q] : 0);
            }
        }
        cgmli_solver* S = solver[b.solver];
        int st = cgmli_solver_set_imu_samples(S, &opt.imu_params, times.data(), readings.data(), (int)times.size(), range.data(),
                                              t0.data(), t1.data());
        if (st == CGMLI_OK) st = cgmli_solver_refresh_imu(S, opt.imu_gyro_threshold, opt.imu_accel_threshold, nullptr);
        b.imu = true;
        return st;
    }
    // The conditional calibration information of the windows that asked for it, read
    // back before the marginalization reuses the same device buffers (this waits for
    // the batch's solve).
    void calibration(Batch& b) {
        bool any = false;
        for (Request* r : b.reqs) any = any || r->extra.calibration_information;
        if (!any) return;
        cgmli_solver* S = solver[b.solver];
        const int st = cgmli_solver_calibration_information(S, opt.calibration_include_prior);
        for (int i = 0; i < (int)b.reqs.size(); ++i) {
            Request* r = b.reqs[i];
            if (!r->extra.calibration_information) continue;
            r->calibStatus = st;
            if (st != CGMLI_OK) continue;
            int size = 0, nb = 0;
            int rs = cgmli_solver_read_calibration_information(S, i, &size, &nb, nullptr, nullptr, nullptr, nullptr);
            if (rs == CGMLI_OK) {
                r->calibKind.resize(nb);
                r->calibIndex.resize(nb);
                r->calibConditional.resize((size_t)size * size);
                r->calibEvals.resize(size);
                rs = cgmli_solver_read_calibration_information(S, i, &size, &nb, r->calibKind.data(), r->calibIndex.data(),
                                                               r->calibConditional.data(), r->calibEvals.data());
            }
            r->calibStatus = rs;
            r->calibSize = size;
            r->calibBlocks = nb;
        }
    }

    // Waits for a launched batch and records its results.
    void complete(Batch& b, double* waitMs = nullptr, double* readMs = nullptr) {
        cgmli_solver* S = solver[b.solver];
        const int n = (int)b.reqs.size();
        std::vector<cgmli_solve_report> reps(n);
        int st = b.status;
        const auto w0 = Clock::now();
        if (st == CGMLI_OK) st = cgmli_solver_synchronize(S);
        const auto w1 = Clock::now();
        if (waitMs) *waitMs = std::chrono::duration<double, std::milli>(w1 - w0).count();
        if (st == CGMLI_OK) st = cgmli_solver_read_states(S, b.windows.data(), n);
        if (st == CGMLI_OK) st = cgmli_solver_read_reports(S, reps.data(), n);
        for (int i = 0; i < n; ++i) {
            Request* r = b.reqs[i];
            if (st != CGMLI_OK) {
                r->report = cgmli_solve_report{};
                r->report.status = st;
                continue;
            }
            r->report = reps[i];
            if (b.imu && r->extra.num_imu_samples > 0 && r->window.num_imu > 0) {
                r->imu.resize(r->window.num_imu);
                const int is = cgmli_solver_read_imu(S, i, r->imu.data());
                if (is != CGMLI_OK && r->report.status == CGMLI_OK) r->report.status = is;
                r->imuRefreshed = 0;
                for (int q = 0; q < r->window.num_imu; ++q)
                    r->imuRefreshed += std::memcmp(&r->imu[q], &r->window.imu[q], sizeof(cgmli_frozen_imu)) != 0 ? 1 : 0;
            }
            if (opt.nis_threshold > 0) {
                r->rejected.resize(r->window.num_observations);
                const int gs = cgmli_solver_read_gate(S, i, &r->gate, r->rejected.data());
                if (gs != CGMLI_OK && r->report.status == CGMLI_OK) r->report.status = gs;
            }
            if (r->victim >= 0 && r->report.status == CGMLI_OK && opt.policy == CGMLI_MARGIN_SECOND_NEW_IMU_MERGE)
                r->mergeStatus = cgmli_solver_read_merged_imu(S, i, &r->mergeState, &r->merged);
            if (r->victim >= 0 && r->report.status == CGMLI_OK) {
                int rank = 0, cols = 0, nb = 0;
                int ps = cgmli_solver_read_prior(S, i, &rank, &cols, &nb, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
                if (ps == CGMLI_OK) {
                    r->kinds.resize(nb);
                    r->index.resize(nb);
                    r->reference.resize(9ull * nb + 1);
                    r->A.resize((size_t)rank * cols);
                    r->r0.resize(rank);
                    ps = cgmli_solver_read_prior(S, i, &rank, &cols, &nb, r->kinds.data(), r->index.data(), r->reference.data(),
                                                 r->A.data(), r->r0.data(), nullptr);
                }
                if (ps != CGMLI_OK) r->report.status = ps;
                r->rank = rank;
                r->cols = cols;
                r->numBlocks = nb;
            }
        }
        const auto now = Clock::now();
        if (readMs) *readMs = std::chrono::duration<double, std::milli>(now - w1).count();
        {
            std::lock_guard<std::mutex> lock(mu);
            for (Request* r : b.reqs) {
                r->completed = now;
                r->complete = true;
            }
        }
        done.notify_all();
        b.reqs.clear();
    }

    // Scheduler: forms the next batch from the queue as soon as a solver is
    // free, builds and launches it, and hands it to the completion thread.
    void run() {
        int cur = 0;
        // each solver keeps its device arrays between batches, so the budget is
        // split: a batch may hold at most half of it, growth headroom included,
        // and the two solvers together stay within the whole budget (a single
        // window above that half still runs, alone in its batch)
        const long long perSolver = opt.memory_budget_bytes / 2;
        // CGMLI_SERVER_TRACE set: one line per batch on stderr (size, host launch
        // time and its set_windows / solve / marginalize parts, the completion
        // thread's wait and read-back; milliseconds)
        trace = std::getenv("CGMLI_SERVER_TRACE") != nullptr;
        std::thread completer([this] { completeLoop(); });
        for (;;) {
            auto next = std::make_unique<Batch>();
            {
                std::unique_lock<std::mutex> lock(mu);
                work.wait(lock, [&] { return stopping || (!queue.empty() && !busy[cur]); });
                if (stopping && queue.empty()) break;
                if (busy[cur]) freed.wait(lock, [&] { return !busy[cur]; });  // stopping with queued requests
                long long bytes = 0;
                while (!queue.empty() && (int)next->reqs.size() < opt.max_batch_windows) {
                    const long long f = (long long)(kGrowth * (double)footprint(queue.front()->window, opt.deterministic != 0));
                    if (!next->reqs.empty() && bytes + f > perSolver) break;
                    bytes += f;
                    next->reqs.push_back(queue.front());
                    queue.pop_front();
                }
                busy[cur] = true;
            }
            const auto c0 = Clock::now();
            next->solver = cur;
            launch(*next);
            next->launchMs = std::chrono::duration<double, std::milli>(Clock::now() - c0).count();
            long long held = 0;  // the solver's device arrays after this batch's allocations (only this thread launches)
            if (cgmli_solver_device_bytes(solver[cur], &held) != CGMLI_OK) held = 0;
            {
                std::lock_guard<std::mutex> lock(mu);
                solverBytes[cur] = held;
                launched.push_back(std::move(next));
            }
            launchedCv.notify_one();
            cur ^= 1;
        }
        {
            std::lock_guard<std::mutex> lock(mu);
            schedulerDone = true;
        }
        launchedCv.notify_one();
        completer.join();
    }
    // Completion thread: waits for each launched batch in launch order, records
    // its results and frees its solver.
    void completeLoop() {
        for (;;) {
            std::unique_ptr<Batch> b;
            {
                std::unique_lock<std::mutex> lock(mu);
                launchedCv.wait(lock, [&] { return schedulerDone || !launched.empty(); });
                if (launched.empty()) return;
                b = std::move(launched.front());
                launched.pop_front();
            }
            double waitMs = 0, readMs = 0;
            const int size = (int)b->reqs.size();
            const int sv = b->solver;
            complete(*b, trace ? &waitMs : nullptr, trace ? &readMs : nullptr);
            if (trace)
                std::fprintf(stderr, "batch %d launch %.3f (set %.3f solve %.3f marg %.3f) wait %.3f read %.3f\n", size, b->launchMs,
                             b->phaseMs[0], b->phaseMs[1], b->phaseMs[2], waitMs, readMs);
            {
                std::lock_guard<std::mutex> lock(mu);
                busy[sv] = false;
            }
            freed.notify_all();
            work.notify_all();
        }
    }
};

using cgmli::setLastError;

extern "C" {

int cgmli_server_create(const cgmli_server_options* options, cgmli_server** out) {
    if (!options || !out) return setLastError(CGMLI_E_INVALID, "server: null options or output handle");
    *out = nullptr;
    if (options->iterations < 1) return setLastError(CGMLI_E_INVALID, "server: iterations < 1");
    if (options->policy != CGMLI_MARGIN_OLD && options->policy != CGMLI_MARGIN_SECOND_NEW &&
        options->policy != CGMLI_MARGIN_SECOND_NEW_IMU_MERGE)
        return setLastError(CGMLI_E_INVALID, "server: unknown marginalization policy");
    if (!(options->nis_threshold >= 0) || options->max_refits < 0 || options->max_refits > 64)
        return setLastError(CGMLI_E_INVALID, "server: nis_threshold < 0 or max_refits outside 0..64");
    if (!(options->imu_gyro_threshold >= 0) || !(options->imu_accel_threshold >= 0))
        return setLastError(CGMLI_E_INVALID, "server: negative or NaN IMU refresh threshold");
    if (options->precision != CGMLI_PRECISION_FP64 && options->precision != CGMLI_PRECISION_MIXED)
        return setLastError(CGMLI_E_INVALID, "server: unknown precision");
    if (options->deterministic != 0 && options->deterministic != 1)
        return setLastError(CGMLI_E_INVALID, "server: deterministic not 0 or 1");
    auto* s = new cgmli_server();
    s->opt = *options;
    if (s->opt.max_batch_windows <= 0) s->opt.max_batch_windows = 512;
    if (s->opt.memory_budget_bytes <= 0) s->opt.memory_budget_bytes = 40ll << 30;
    cgmli_solver_options so;
    cgmli_default_options(&so);
    so.precision = options->precision;
    for (int k = 0; k < 2; ++k) {
        int st = cgmli_solver_create(options->device, &so, &s->solver[k]);
        if (st == CGMLI_OK && options->deterministic) {
            cgmli_tuning t{};
            t.deterministic = 1;
            st = cgmli_solver_set_tuning(s->solver[k], &t);
        }
        if (st != CGMLI_OK) {
            for (auto* sv : s->solver) cgmli_solver_destroy(sv);
            delete s;
            return st;
        }
    }
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return CGMLI_OK;
}

void cgmli_server_destroy(cgmli_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
    }
    s->work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto* sv : s->solver) cgmli_solver_destroy(sv);
    delete s;
}

namespace {
int submitAt(cgmli_server* s, cgmli_window* window, int victim_kf, Clock::time_point arrival, long long* ticket,
             const cgmli_server_request* extra = nullptr);
}

int cgmli_server_submit(cgmli_server* s, cgmli_window* window, int victim_kf, long long* ticket) {
    return submitAt(s, window, victim_kf, Clock::now(), ticket);
}

int cgmli_server_submit_request(cgmli_server* s, const cgmli_server_request* request, long long* ticket) {
    if (!request) return setLastError(CGMLI_E_INVALID, "server: null request");
    return submitAt(s, request->window, request->victim_kf, Clock::now(), ticket, request);
}

namespace {
// The IMU part of a request: every factor's range inside the request's samples.
int validateImuPart(const cgmli_window& w, const cgmli_server_request& x, std::string& why) {
    if (x.num_imu_samples == 0) return CGMLI_OK;
    if (x.num_imu_samples < 2 || !x.imu_sample_time_ns || !x.imu_sample_readings || (w.num_imu > 0 && (!x.imu_range || !x.imu_t0_ns || !x.imu_t1_ns))) {
        why = "server: IMU samples need times, readings, ranges and interval ends (and at least 2 samples)";
        return CGMLI_E_INVALID;
    }
    for (int q = 0; q < w.num_imu; ++q) {
        const int b = x.imu_range[2 * q], e = x.imu_range[2 * q + 1];
        if (b < 0 || e > x.num_imu_samples || e - b < 2) {
            why = "server: IMU factor " + std::to_string(q) + ": sample range outside the request's samples or shorter than 2";
            return CGMLI_E_INVALID;
        }
    }
    return CGMLI_OK;
}

int submitAt(cgmli_server* s, cgmli_window* window, int victim_kf, Clock::time_point arrival, long long* ticket,
             const cgmli_server_request* extra) {
    if (!s || !window || !ticket) return setLastError(CGMLI_E_INVALID, "server: null server, window or ticket");
    std::string why;
    int st = cgmli::validateWindow(*window, 0, why);
    if (st == CGMLI_OK && extra) st = validateImuPart(*window, *extra, why);
    if (st != CGMLI_OK) return setLastError(st, why.c_str());
    if (victim_kf < -1 || victim_kf >= window->num_keyframes) return setLastError(CGMLI_E_INVALID, "server: victim keyframe out of range");
    auto r = std::make_shared<Request>();
    r->window = *window;
    r->victim = victim_kf;
    r->submitted = arrival;
    if (extra) r->extra = *extra;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stopping) return setLastError(CGMLI_E_INVALID, "server: stopping");
        r->ticket = s->nextTicket++;
        *ticket = r->ticket;
        s->queue.push_back(r.get());
        s->requests.emplace(r->ticket, r);
    }
    s->work.notify_one();
    return CGMLI_OK;
}
}  // namespace

int cgmli_server_replay(cgmli_server* s, cgmli_window* const* windows, const int* victims, const double* arrival_s, int count,
                        double* latency_ms, int* status, double* span_s) {
    if (!s || !windows || !victims || !arrival_s || !latency_ms || !status || count < 1)
        return setLastError(CGMLI_E_INVALID, "server replay: null arrays or empty trace");
    for (int i = 0; i < count; ++i)
        if (!windows[i] || (i > 0 && arrival_s[i] < arrival_s[i - 1]))
            return setLastError(CGMLI_E_INVALID, "server replay: null window or arrival times not sorted");
    std::vector<long long> tickets(count, 0);
    std::mutex qmu;
    std::condition_variable qcv;
    int submitted = 0;
    bool failed = false;
    std::unordered_map<const cgmli_window*, int> lastUse;  // window -> last request using it
    std::vector<char> finished(count, 0);
    std::mutex fmu;
    std::condition_variable fcv;
    // collector: waits for the requests in submission order
    std::thread collector([&] {
        for (int i = 0; i < count; ++i) {
            long long t = 0;
            {
                std::unique_lock<std::mutex> lock(qmu);
                qcv.wait(lock, [&] { return submitted > i || failed; });
                if (submitted <= i) break;
                t = tickets[i];
            }
            cgmli_solve_report rep{};
            double ms = 0;
            cgmli_server_poll(s, t, 1, &rep, &ms);
            latency_ms[i] = ms;
            status[i] = rep.status;
            cgmli_server_release(s, t);
            {
                std::lock_guard<std::mutex> lock(fmu);
                finished[i] = 1;
            }
            fcv.notify_all();
        }
    });
    const auto t0 = Clock::now();
    int rc = CGMLI_OK;
    for (int i = 0; i < count; ++i) {
        const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
        std::this_thread::sleep_until(due);
        // a window is reused only after its earlier request completed
        auto it = lastUse.find(windows[i]);
        if (it != lastUse.end()) {
            const int prev = it->second;
            std::unique_lock<std::mutex> lock(fmu);
            fcv.wait(lock, [&] { return finished[prev] != 0; });
        }
        lastUse[windows[i]] = i;
        long long t = 0;
        rc = submitAt(s, windows[i], victims[i], due, &t);
        {
            std::lock_guard<std::mutex> lock(qmu);
            if (rc != CGMLI_OK) { failed = true; }
            else { tickets[i] = t; ++submitted; }
        }
        qcv.notify_all();
        if (rc != CGMLI_OK) break;
    }
    collector.join();
    if (span_s) *span_s = std::chrono::duration<double>(Clock::now() - t0).count();
    return rc;
}

int cgmli_server_poll(cgmli_server* s, long long ticket, int wait, cgmli_solve_report* report, double* latency_ms) {
    if (!s) return setLastError(CGMLI_E_INVALID, "server: null server");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return setLastError(CGMLI_E_INVALID, "server: unknown ticket");
    const std::shared_ptr<Request> r = it->second;  // stays valid if the request is released while we wait
    if (!r->complete) {
        if (!wait) return CGMLI_E_PENDING;
        s->done.wait(lock, [&] { return r->complete; });
    }
    if (report) *report = r->report;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->completed - r->submitted).count();
    return CGMLI_OK;
}

int cgmli_server_read_prior(cgmli_server* s, long long ticket, int* rank, int* cols, int* num_blocks, int* block_kind,
                            int* block_index, double* reference, double* A, double* r0) {
    if (!s || !rank || !cols || !num_blocks) return setLastError(CGMLI_E_INVALID, "server: null server or size outputs");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return setLastError(CGMLI_E_INVALID, "server: unknown ticket");
    const Request* r = it->second.get();
    if (!r->complete) return CGMLI_E_PENDING;
    if (r->victim < 0) return setLastError(CGMLI_E_INVALID, "server: request had no victim keyframe");
    if (r->report.status != CGMLI_OK) return setLastError(r->report.status, "server: request failed");
    *rank = r->rank;
    *cols = r->cols;
    *num_blocks = r->numBlocks;
    if (block_kind) std::copy(r->kinds.begin(), r->kinds.end(), block_kind);
    if (block_index) std::copy(r->index.begin(), r->index.end(), block_index);
    if (reference) {
        size_t amb = 0;
        for (int k : r->kinds) amb += k == CGMLI_PRIOR_SPEED_BIAS ? 9 : k == CGMLI_PRIOR_TIME_OFFSET ? 1 : 7;
        std::copy(r->reference.begin(), r->reference.begin() + amb, reference);
    }
    if (A) std::copy(r->A.begin(), r->A.end(), A);
    if (r0) std::copy(r->r0.begin(), r->r0.end(), r0);
    return CGMLI_OK;
}

int cgmli_server_read_gate(cgmli_server* s, long long ticket, cgmli_gate_report* report, unsigned char* rejected) {
    if (!s || !report) return setLastError(CGMLI_E_INVALID, "server: null server or report");
    if (!(s->opt.nis_threshold > 0)) return setLastError(CGMLI_E_INVALID, "server: the gate is off (nis_threshold 0)");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return setLastError(CGMLI_E_INVALID, "server: unknown ticket");
    const Request& r = *it->second;
    if (!r.complete) return setLastError(CGMLI_E_PENDING, "server: request not complete");
    *report = r.gate;
    if (rejected && !r.rejected.empty()) std::copy(r.rejected.begin(), r.rejected.end(), rejected);
    return CGMLI_OK;
}

int cgmli_server_read_imu(cgmli_server* s, long long ticket, cgmli_frozen_imu* imu, int* refreshed) {
    if (!s || !imu) return setLastError(CGMLI_E_INVALID, "server: null server or buffer");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return setLastError(CGMLI_E_INVALID, "server: unknown ticket");
    const Request& r = *it->second;
    if (!r.complete) return setLastError(CGMLI_E_PENDING, "server: request not complete");
    if (r.extra.num_imu_samples == 0) return setLastError(CGMLI_E_INVALID, "server: the request brought no IMU samples");
    if (r.imu.size() != (size_t)r.window.num_imu) return setLastError(r.report.status ? r.report.status : CGMLI_E_INVALID,
                                                                      "server: the request's IMU factors were not read back");
    std::copy(r.imu.begin(), r.imu.end(), imu);
    if (refreshed) *refreshed = r.imuRefreshed;
    return CGMLI_OK;
}

int cgmli_server_read_merged_imu(cgmli_server* s, long long ticket, int* state, cgmli_frozen_imu* imu) {
    if (!s || !state) return setLastError(CGMLI_E_INVALID, "server: null server or state output");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return setLastError(CGMLI_E_INVALID, "server: unknown ticket");
    const Request& r = *it->second;
    if (!r.complete) return setLastError(CGMLI_E_PENDING, "server: request not complete");
    if (s->opt.policy != CGMLI_MARGIN_SECOND_NEW_IMU_MERGE || r.victim < 0)
        return setLastError(CGMLI_E_INVALID, "server: the request had no IMU-merge marginalization");
    if (r.report.status != CGMLI_OK) return setLastError(r.report.status, "server: request failed");
    if (r.mergeStatus != CGMLI_OK) return setLastError(r.mergeStatus, "server: the merged factor could not be read");
    *state = r.mergeState;
    if (imu && r.mergeState == CGMLI_IMU_MERGE_REINTEGRATED) *imu = r.merged;
    return CGMLI_OK;
}

int cgmli_server_read_calibration_information(cgmli_server* s, long long ticket, int* size, int* num_blocks, int* block_kind,
                                              int* block_index, double* conditional, double* eigenvalues) {
    if (!s || !size || !num_blocks) return setLastError(CGMLI_E_INVALID, "server: null server or size outputs");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return setLastError(CGMLI_E_INVALID, "server: unknown ticket");
    const Request& r = *it->second;
    if (!r.complete) return setLastError(CGMLI_E_PENDING, "server: request not complete");
    if (!r.extra.calibration_information) return setLastError(CGMLI_E_INVALID, "server: the request did not ask for the calibration information");
    if (r.calibStatus != CGMLI_OK) return setLastError(r.calibStatus, "server: the calibration information failed for this window");
    *size = r.calibSize;
    *num_blocks = r.calibBlocks;
    if (block_kind) std::copy(r.calibKind.begin(), r.calibKind.end(), block_kind);
    if (block_index) std::copy(r.calibIndex.begin(), r.calibIndex.end(), block_index);
    if (conditional) std::copy(r.calibConditional.begin(), r.calibConditional.end(), conditional);
    if (eigenvalues) std::copy(r.calibEvals.begin(), r.calibEvals.end(), eigenvalues);
    return CGMLI_OK;
}

int cgmli_server_device_bytes(cgmli_server* s, long long* bytes) {
    if (!s || !bytes) return setLastError(CGMLI_E_INVALID, "server: null server or output");
    std::lock_guard<std::mutex> lock(s->mu);
    *bytes = s->solverBytes[0] + s->solverBytes[1];
    return CGMLI_OK;
}

int cgmli_server_release(cgmli_server* s, long long ticket) {
    if (!s) return setLastError(CGMLI_E_INVALID, "server: null server");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return setLastError(CGMLI_E_INVALID, "server: unknown ticket");
    if (!it->second->complete) return setLastError(CGMLI_E_PENDING, "server: request not complete");
    s->requests.erase(it);
    return CGMLI_OK;
}

}  // extern "C"
