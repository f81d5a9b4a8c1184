// Host-side device layout of a batch of windows (no CUDA calls).
//
// buildHostBatch turns the caller's windows into the concatenated arrays the
// kernels read: landmarks reordered by support, observations of a landmark
// sorted by observer keyframe, the key order of the J^T J pass, the warp work
// units (runs of tiles, pair chunks, Schur chunks) and the per-window
// descriptors.  Windows are independent, so the build runs on host threads in
// parallel; every array position is known from the windows' sizes except the
// support lists and cross-vector offsets, which are fixed up after a prefix sum.
#pragma once
#include <cuda_runtime.h>  // int2 / int4

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <cstdlib>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cgmli_backend.h"
#include "backend_internal.h"

namespace cgmli {

// Process-wide worker threads for parallelFor, created on first use and kept
// (thread start-up is a sizable part of a small batch's host build).  One loop
// runs on the pool at a time; a concurrent caller gets false and spawns its own.
class WorkPool {
public:
    static WorkPool& get() {
        static WorkPool pool;
        return pool;
    }
    bool run(int count, int threads, const std::function<void(int)>& fn) {
        std::unique_lock<std::mutex> use(use_, std::try_to_lock);
        if (!use.owns_lock()) return false;
        const int helpers = std::min(threads, count) - 1;
        {
            std::lock_guard<std::mutex> lock(m_);
            while ((int)workers_.size() < helpers) {
                const int id = (int)workers_.size();
                workers_.emplace_back([this, id] { loop(id); });
            }
            job_ = &fn;
            count_ = count;
            next_ = 0;
            want_ = helpers;
            active_ = helpers;
            ++gen_;
        }
        cv_.notify_all();
        for (int i = next_++; i < count; i = next_++) fn(i);
        std::unique_lock<std::mutex> lock(m_);
        done_.wait(lock, [&] { return active_ == 0; });
        job_ = nullptr;
        return true;
    }
    ~WorkPool() {
        {
            std::lock_guard<std::mutex> lock(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

private:
    void loop(int id) {
        unsigned long long seen = 0;
        for (;;) {
            const std::function<void(int)>* job;
            int count;
            {
                std::unique_lock<std::mutex> lock(m_);
                cv_.wait(lock, [&] { return stop_ || (gen_ != seen && id < want_); });
                if (stop_) return;
                seen = gen_;
                job = job_;
                count = count_;
            }
            for (int i = next_++; i < count; i = next_++) (*job)(i);
            std::lock_guard<std::mutex> lock(m_);
            if (--active_ == 0) done_.notify_all();
        }
    }
    std::mutex use_, m_;
    std::condition_variable cv_, done_;
    std::vector<std::thread> workers_;
    const std::function<void(int)>* job_ = nullptr;
    int count_ = 0, want_ = 0, active_ = 0;
    std::atomic<int> next_{0};
    unsigned long long gen_ = 0;
    bool stop_ = false;
};

// Runs fn(i) for i in [0, n) on up to `threads` host threads (0: all cores).
template <class Fn>
void parallelFor(int n, int threads, Fn&& fn) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (threads <= 1 || n <= 1) {
        for (int i = 0; i < n; ++i) fn(i);
        return;
    }
    const std::function<void(int)> job = [&](int i) { fn(i); };
    if (WorkPool::get().run(n, threads, job)) return;
    std::atomic<int> next{0};
    auto body = [&] {
        for (int i = next++; i < n; i = next++) fn(i);
    };
    std::vector<std::thread> pool;
    const int t = std::min(threads, n);
    for (int k = 1; k < t; ++k) pool.emplace_back(body);
    body();
    for (auto& th : pool) th.join();
}

// Page-locked host memory for the arrays uploaded to (and read back from) the
// device, so that the copies run at DMA speed; plain memory where no CUDA
// device is present (the host-only diagnostic path).  Elements are
// default-initialized: every position is written by the builder, and a batch
// of the same size reuses the capacity without touching it first.
void* pinnedAllocate(size_t bytes);
void pinnedFree(void* p);
template <class T>
struct PinnedAllocator {
    using value_type = T;
    PinnedAllocator() = default;
    template <class U>
    PinnedAllocator(const PinnedAllocator<U>&) {}
    T* allocate(size_t n) {
        void* p = pinnedAllocate(n * sizeof(T));
        if (!p) throw std::bad_alloc();
        return static_cast<T*>(p);
    }
    void deallocate(T* p, size_t) { pinnedFree(p); }
    template <class U>
    void construct(U* p) { ::new ((void*)p) U; }
    template <class U, class... A>
    void construct(U* p, A&&... a) { ::new ((void*)p) U(static_cast<A&&>(a)...); }
    template <class U>
    bool operator==(const PinnedAllocator<U>&) const { return true; }
    template <class U>
    bool operator!=(const PinnedAllocator<U>&) const { return false; }
};
template <class T>
using HVec = std::vector<T, PinnedAllocator<T>>;
// Resize with 1.5x headroom on growth: pinned memory is freed with
// cudaFreeHost, which waits for the whole device, so a batch slightly larger
// than every earlier one must not reallocate the staging again.
template <class V>
void sizeTo(V& v, size_t n) {
    if (n > v.capacity()) v.reserve(std::max(n, v.capacity() + v.capacity() / 2));
    v.resize(n);
}

// Work decomposition chosen by the caller or the autotuner (cgmli_tuning).
struct PlanParams {
    int runLandmarks = 0;  // 0: from the batch size
    int pairChunk = 32;
    int schurRows = kSchurMaxRows;
    int linShape = 0;      // kLinShapeTable entry of the landmark pass
    int trialShape = 0;    // kTrialShapeTable entry of the trial pass
    int deterministic = 0; // 1: per-unit slots of the visual sums (WinDesc::det0)
};

struct HostBatch {
    PlanParams plan;  // the decomposition the batch was built with
    std::vector<WinDesc> win;
    HVec<int4> runs;         // {window, first tile, end tile, -}
    HVec<int2> tiles;        // {first landmark, end landmark}
    HVec<int4> pairChunks;   // {window, first key-ordered position, end, -}
    HVec<int4> schurChunks;  // {window, first landmark, end landmark, offset in schurCols}
    HVec<int4> detPairs;     // deterministic mode: {window, first key-ordered position, end, slot}
    HVec<int4> detSchur;     // deterministic mode: {first Schur chunk, end chunk, slot, window}
    long long detSlots = 0;  // doubles of all windows' slots
    HVec<int> schurCols;     // per Schur chunk: count, then the ascending visual columns of its landmarks
    HVec<unsigned short> lmUmap;  // per cross-vector entry: position of its column in the chunk's list
    HVec<int> lmPerm;        // device landmark -> landmark index within its window
    // cameras
    HVec<double> camR, camT;
    HVec<int> camExt;        // global extrinsic of each global camera
    // landmarks (device order)
    HVec<int> lmWin, lmKf, lmCam, lmObsBegin, lmNs, lmNx, lmSupp0, supp;
    HVec<long long> lmC0;
    HVec<double> lmBearing, lmVel, lmTime;
    // observations (device order)
    HVec<int> obKf, obCam, obSlot, obXslot, obLm, keyOrder;
    HVec<int> obOrig;        // device observation -> observation index within its window
    // observation payload in each window's caller order (from WinDesc::obs0); the
    // device gathers it into device order through obOrig
    HVec<double> obBearing, obP, obVel, obTime;
    // states
    HVec<double> pose, sb, ext, td, rho;
    HVec<signed char> colChart;   // per retained column of each window (at WinDesc::vec0): kCol*
    HVec<unsigned char> lmFixed;  // per device landmark: 1 = inverse distance held constant
    // IMU and priors
    HVec<double> imu;
    HVec<int> imuKf;
    HVec<int> priorKind, priorIndex, priorCol, priorOff;
    HVec<double> priorA, priorR0, priorRef;
    // totals
    int totalKf = 0, totalExt = 0, totalCam = 0, totalLm = 0, totalObs = 0, totalImu = 0;
    int maxNpc = 0, maxNr = 0, maxNs = 1;
    long long vec = 0, dense = 0, acc = 0, sch = 0, imuScratch = 0, priorScratch = 0, cross = 0;
};

// Structural checks of one window (sizes, index ranges, limits).  Returns a
// CGMLI_* code and the reason.
int validateWindow(const cgmli_window& w, int index, std::string& why);

// Builds the batch with up to `threads` host threads (0: hardware concurrency).
// Returns a CGMLI_* code and the reason.
// `ready`, when given, is called (on the calling thread) each time the windows
// [w0, w1) have their landmark and observation arrays final, before the rest of
// the batch is built, so that their uploads can overlap the remaining host work.
int buildHostBatch(const cgmli_window* windows, int count, int threads, HostBatch& out, std::string& why,
                   const std::function<void(int, int)>* ready = nullptr, const PlanParams& plan = PlanParams());

// Invariants of a built batch (used by the diagnostic entry point and tests).
int checkHostBatch(const cgmli_window* windows, int count, const HostBatch& hb, std::string& why);

}  // namespace cgmli
