// Host runtime of the B200 backend solver: topology preprocessing, device
// buffers, the launch sequence and the C ABI of include/cgmli_backend.h.
//
// The reference rebuilds CSR rows, columns and per-point support sets on the
// host for every new topology (VisualCudaBatch.cu:450-490) and ping-pongs
// the host every LM iteration (:595-597).  Here the topology is built once per
// set of windows (support sets, landmarks sorted by support, tiles of <= 32
// observations, warp runs of tiles)
// and the whole LM loop runs on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cgmli_backend.h"
#include "backend_internal.h"
#include "imu_preintegration.h"
#include "topology.h"

namespace cgmli {
size_t linearizeSmemBytes(int maxNs, bool mixed);
size_t factorSmemBytes(int maxNr);
size_t wideFinishSmemBytes(int maxNr);
cudaError_t configureKernels(size_t linSmem, size_t facSmem, size_t wideSmem);
int launchIteration(const DevBatch& B, const LaunchPlan& P, int refinement, int maxIterations, int probe, double* Sdebug,
                    cudaStream_t s, LaunchHook hook, void* ctx);
int launchIterationParts(const DevBatch& B, const LaunchPlan& P, int refinement, int maxIterations, int probe, double* Sdebug,
                         cudaStream_t s, LaunchHook hook, void* ctx, int parts);
void launchEvaluate(const DevBatch& B, int derivatives, double* out, int* valid, cudaStream_t s);
void launchGatherObservations(const DevBatch& B, const int* obOrig, const double* const src[4], double* const dst[4],
                              cudaStream_t s);
void launchAddHost(const DevBatch& B, const double* hostH, const double* hostG, const double* hostCost, const unsigned char* flag,
                   int trial, cudaStream_t s);
int launchLmInit(const DevBatch& B, double lambda0, cudaStream_t s);
int launchGate(const DevBatch& B, const LaunchPlan& P, int pass, int pre, double threshold, double* obP, unsigned char* rejected,
               double* gateStats, int* gateCounts, cudaStream_t s);
int launchRefit(const DevBatch& B, int pass, double lambda0, int maxIterations, const int* gateCounts, cudaStream_t s);
size_t margVisualSmemBytes(int maxNc);
size_t margRowsSmemBytes(int maxNv);
int margRowsCap(int nv);
cudaError_t configureMarginalization(size_t visualSmem, size_t rowsSmem, int maxNr, int maxFastNr, long long* eigenSmem,
                                     long long* fastSmem, long long* triSmem);
int launchMarginalization(const DevBatch& B, const MargBatch& M, size_t visualSmem, cudaStream_t s);
int launchCalibration(const DevBatch& B, const MargBatch& M, size_t visualSmem, double* work, const long long* work0, double* cond,
                      double* evals, int maxNuisance, cudaStream_t s);
void launchDenseEigen(const double* H, int n, double* work, double* evals, double* evecs, int* status, cudaStream_t s);
void launchDensePsd(const double* evals, const double* U, const double* rhs, int n, int columns, double absCut, double relCut,
                    double* projected, double* solution, int* status, cudaStream_t s);
void launchDenseSubtract(const double* coupling, const double* solution, int nm, int nr, double* Hg, cudaStream_t s);
}  // namespace cgmli

using namespace cgmli;

namespace cgmli {
int setLastError(int code, const char* message);
}

namespace {
thread_local std::string g_error = "ok";

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}
int cudaFail(cudaError_t e, const char* what) {
    g_error = std::string(what) + ": " + cudaGetErrorString(e);
    return CGMLI_E_CUDA;
}
#define CK(call)                                                 \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cudaFail(e_, #call);      \
    } while (0)

// Stream the calling solver entry point works on, for stream-ordered growth of its
// arrays (nullptr: plain cudaMalloc / cudaFree).  cudaFree waits for the whole
// device, so a solver growing an array in one thread would stall behind another
// solver's work; ordered on the solver's own stream, the old block is released
// after the solver's earlier kernels and the new one is ready for its later ones.
thread_local cudaStream_t tlsAllocStream = nullptr;
struct AllocStreamScope {
    cudaStream_t prev;
    explicit AllocStreamScope(cudaStream_t s) : prev(tlsAllocStream) { tlsAllocStream = s; }
    ~AllocStreamScope() { tlsAllocStream = prev; }
};

// Grow-only device array (src/common/CudaArray.hpp:10-39 keeps the same policy);
// it grows by at least half its size, so batches of slowly rising size do not
// reallocate at every call.
template <class T>
struct DArray {
    T* p = nullptr;
    size_t cap = 0;
    bool pooled = false;  // allocated stream-ordered (freed the same way)
    cudaError_t reserve(size_t n) {
        if (n <= cap) return cudaSuccess;
        free(tlsAllocStream);
        const size_t want = std::max<size_t>(std::max(n, cap + cap / 2), 1);
        cudaError_t e;
        if (tlsAllocStream) {
            e = cudaMallocAsync(reinterpret_cast<void**>(&p), want * sizeof(T), tlsAllocStream);
            pooled = e == cudaSuccess;
        } else {
            e = cudaMalloc(&p, want * sizeof(T));
        }
        if (e == cudaSuccess) cap = want;
        else p = nullptr;
        return e;
    }
    template <class V>
    cudaError_t upload(const V& v, cudaStream_t s) {
        cudaError_t e = reserve(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    }
    void release() { free(nullptr); }
    void free(cudaStream_t s) {
        if (p) {
            if (pooled && s) cudaFreeAsync(p, s);
            else cudaFree(p);
        }
        p = nullptr;
        cap = 0;
        pooled = false;
    }
};
}  // namespace

struct cgmli_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // ev0 / ev1 bracket the last timed call; before the first one they were never
    // recorded, and querying them would leave an error for the next launch check
    bool timed = false;
    void readTiming() {
        float ms = 0;
        if (timed && cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) lastMs = ms;
    }
    // CUDA graph of a whole solve: captured when the same launch sequence (device
    // pointers, work decomposition, iteration budget, options) is solved a second
    // time in a row, replayed while it stays the same; a new topology is solved
    // eagerly, so a batch solved once pays no capture
    PlanParams tune;  // work decomposition of the next set_windows (cgmli_tuning)
    cudaGraphExec_t graphExec = nullptr;
    std::vector<char> graphKey, lastKey;
    int graphLaunches = 0;
    cgmli_solver_options opt{};
    // topology (host copies)
    std::vector<WinDesc> win;
    int maxNpc = 0, maxNr = 0, maxNs = 1;
    size_t linSmem = 0, facSmem = 0;
    // wide windows (isWideWindow): factored by the multi-launch sequence
    int numWide = 0, wideCols = 0, wideCharts = 0;
    size_t wideFinishSmem = 0;
    HVec<int> hWideList;
    DArray<int> wideList, facFailed;
    DArray<double> facVec, wideProd, wideL21;
    int totalKf = 0, totalExt = 0, totalCam = 0, totalLm = 0, totalObs = 0, totalImu = 0;
    // device arrays
    DArray<WinDesc> dWin;
    DArray<WinLM> dLm;
    DArray<int4> dRuns;
    DArray<int2> dTiles;
    DArray<int4> dPairChunks, dSchurChunks, dDetPairs, dDetSchur;
    DArray<double> detSlots;  // deterministic mode: per-unit partial sums
    DArray<int> schurCols;
    DArray<unsigned short> lmUmap;
    DArray<int> obLm, keyOrder, bigFirst;
    HVec<int> hBigFirst;
    DArray<double> keyRows;
    DArray<double> sch;
    DArray<double> camR, camT;
    DArray<int> camExt;
    DArray<int> lmWin, lmKf, lmCam, lmObsBegin, lmNs, lmNx, lmSupp0, supp;
    DArray<long long> lmC0;
    DArray<double> lmBearing, lmVel, lmTime, lmC, lmD, lmG, lmCost, lmDelta, lmPred, lmTrial, lmMaxInc;
    DArray<int> lmValid, lmTrialValid;
    DArray<int> obKf, obCam, obSlot, obXslot;
    DArray<double> obBearing, obP, obVel, obTime;
    // the payload as uploaded (each window's caller order) and its device-order map
    DArray<double> obSrcBearing, obSrcP, obSrcVel, obSrcTime;
    DArray<int> obOrig;
    DArray<double> pose[2], sb[2], ext[2], td[2], rho[2], rotKf[2], rotExt[2];
    DArray<double> imu;
    DArray<int> imuKf;
    DArray<int> priorKind, priorIndex, priorCol, priorOff;
    DArray<double> priorA, priorR0, priorRef;
    DArray<double> Hret, gret, costRet, trialRet, acc, dr, rhs, Sglob, imuScratch, priorScratch, predState, out, Sdebug;
    DArray<int> retValid, solveStatus;
    DArray<signed char> colChart;  // solve-time chart of every retained column
    DArray<unsigned char> lmFixed;
    // per-factor evaluation (cgmli_solver_evaluate) and caller-evaluated factors (cgmli_solver_solve_host)
    DArray<double> evalOut;
    DArray<int> evalValid;
    bool haveEval = false, evalDerivatives = false;
    DArray<double> hostH, hostG, hostCost;
    DArray<unsigned char> hostFlag;
    DevBatch B{};
    double lastMs = 0;
    int lastLaunches = 0;
    // host side of the batch (pinned; also the host copies of the topology the
    // elimination sets are built from, and the staging of state read-back)
    HostBatch hb;
    // marginalization
    std::vector<MargWin> margWin;
    std::vector<std::vector<int>> sepKind, sepIndex;  // separator blocks per window (window-local index)
    DArray<MargWin> dMargWin;
    DArray<MargElim> dMargElim;
    DArray<int> margCols, margObsMap, margPoseCol, margSbCol, margExtCol, margRank, margStatus, margFast;
    DArray<int> margVisCol, margVisPose, margVisExt, margSlow;
    DArray<int4> margChunks, margItems;
    DArray<double> margH, margB, margSepH, margSepV, margSepB, margEvals, margA, margR0, margX, margMaxD, margStats;
    MargBatch MB{};
    bool haveMarg = false;
    // host copy of every window's marginalization result, made by the first
    // read_prior after a marginalization (one pass instead of copies per window)
    bool margCached = false;
    long long margSepTotal = 0, margVecTotal = 0;
    HVec<double> hMargA, hMargR0, hMargStats;
    HVec<int> hMargRank, hMargStatus;
    // pinned staging of the marginalization's inputs, and the event after their uploads
    HVec<MargElim> hMargElim;
    HVec<MargWin> hMargWin;      // pinned: a pageable upload would first wait for the stream's solve
    HVec<int> hMargOrder;
    DArray<int> dMargOrder;
    HVec<WinDesc> hWin;
    HVec<int> hMargCols, hMargObsMap, hMargPoseCol, hMargSbCol, hMargExtCol;
    HVec<int> hMargVisCol, hMargVisPose, hMargVisExt, hMargSlow;
    HVec<int4> hMargChunks, hMargItems;
    int numSMs = 0;
    cudaEvent_t margUploaded = nullptr;
    // NIS gate: rejected observations (device order), per-window counters
    // (kGateCounts each) and energies {sum, max} of the last gate
    DArray<unsigned char> obRejected;
    DArray<int> gateCounts;
    DArray<double> gateStats;
    // IMU samples of the batch's factors, kept for cgmli_solver_refresh_imu
    bool haveImuSamples = false;
    cgmli_imu_parameters imuParams{};
    int imuSampleOffset = 0;
    DArray<long long> imuTimes, imuT0, imuT1;
    DArray<double> imuReadings;
    DArray<int> imuRanges, imuStatus, imuRefreshed;
    DArray<cgmli_frozen_imu> imuRefreshScratch;
    std::vector<int> hImuStatus, hImuRefreshed;
    std::vector<int> hImuRange;            // host copies of the factors' sample ranges and ends
    std::vector<long long> hImuT0, hImuT1;
    // SECOND_NEW with the IMU merge: per window its outcome (CGMLI_IMU_MERGE_*)
    // and job index; per job the merged interval and the merged factor
    double mergeMaxInterval = 10.0;
    int mergeMaxSamples = 10000;
    std::vector<int> mergeState, mergeJob;
    HVec<int> hMergeRange, hMergeKf;
    HVec<long long> hMergeT0, hMergeT1;
    DArray<int> mergeRange, mergeKf, mergeStatus, mergeFlag;
    DArray<long long> mergeT0, mergeT1;
    DArray<cgmli_frozen_imu> mergeOut;
    std::vector<int> hMergeStatus;
    bool mergeRead = false;
    // conditional calibration information (the marginalization's formation in
    // calibration mode): per-window work offsets, results
    bool haveCalib = false;
    HVec<long long> hCalibWork0;
    DArray<long long> calibWork0;
    DArray<double> calibWork, calibCond, calibEvals;
    // checkpoint of the accepted states
    DArray<double> snapPose, snapSb, snapExt, snapTd, snapRho;
    bool haveSnapshot = false;
    // per-kernel event timing
    bool profile = false;
    std::vector<cudaEvent_t> evPool;
    std::vector<std::pair<int, int>> evUsed;  // (kind, index of start event)
    size_t evNext = 0;
    double kernelMs[CGMLI_KERNEL_KINDS] = {};
    int kernelCalls[CGMLI_KERNEL_KINDS] = {};
    cudaEvent_t nextEvent() {
        if (evNext == evPool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            evPool.push_back(e);
        }
        return evPool[evNext++];
    }
    // device bytes held by the solver's arrays (grow-only: they stay until destruction)
    long long deviceBytes() const {
        long long t = 0;
        auto add = [&](const auto&... a) { ((t += (long long)(a.cap * sizeof(*a.p))), ...); };
        add(dDetPairs, dDetSchur, detSlots);
        add(dWin, dLm, dRuns, dTiles, dPairChunks, dSchurChunks, schurCols, lmUmap, obLm, keyOrder, bigFirst, keyRows, sch, camR, camT,
            camExt, lmWin, lmKf, lmCam, lmObsBegin, lmNs, lmNx, lmSupp0, supp, lmC0, lmBearing, lmVel, lmTime, lmC, lmD, lmG, lmCost,
            lmDelta, lmPred, lmTrial, lmMaxInc, lmValid, lmTrialValid, obKf, obCam, obSlot, obXslot, obBearing, obP, obVel, obTime,
            obSrcBearing, obSrcP, obSrcVel, obSrcTime, obOrig);
        for (int k = 0; k < 2; ++k) add(pose[k], sb[k], ext[k], td[k], rho[k], rotKf[k], rotExt[k]);
        add(imu, imuKf, priorKind, priorIndex, priorCol, priorOff, priorA, priorR0, priorRef, Hret, gret, costRet, trialRet, acc, dr,
            rhs, Sglob, imuScratch, priorScratch, predState, out, Sdebug, retValid, solveStatus);
        add(dMargWin, dMargElim, margCols, margObsMap, margPoseCol, margSbCol, margExtCol, margRank, margStatus, margFast, margVisCol,
            margVisPose, margVisExt, margSlow, margChunks, margItems, margH, margB, margSepH, margSepV, margSepB, margEvals, margA,
            margR0, margX, margMaxD, margStats, dMargOrder);
        add(colChart, lmFixed, evalOut, evalValid, hostH, hostG, hostCost, hostFlag, wideList, facFailed, facVec, wideProd, wideL21);
        add(obRejected, gateCounts, gateStats, imuTimes, imuT0, imuT1, imuReadings, imuRanges, imuStatus, imuRefreshed,
            imuRefreshScratch, mergeRange, mergeKf, mergeStatus, mergeFlag, mergeT0, mergeT1, mergeOut, calibWork0, calibWork, calibCond,
            calibEvals, snapPose, snapSb, snapExt, snapTd, snapRho);
        return t;
    }
    LaunchPlan plan() const {
        LaunchPlan P{};
        P.runs = dRuns.p; P.tiles = dTiles.p; P.numTiles = (int)hb.tiles.size();
        P.pairChunks = dPairChunks.p; P.numPairChunks = (int)hb.pairChunks.size();
        P.schurChunks = dSchurChunks.p; P.numSchurChunks = (int)hb.schurChunks.size();
        P.detPairs = dDetPairs.p; P.numDetPairs = (int)hb.detPairs.size();
        P.detSchur = dDetSchur.p; P.numDetSchur = (int)hb.detSchur.size();
        P.facSmem = facSmem; P.maxNs = maxNs;
        P.linShape = hb.plan.linShape; P.trialShape = hb.plan.trialShape;
        P.numWide = numWide; P.wideCols = wideCols; P.wideCharts = wideCharts;
        P.wideFinishSmem = wideFinishSmem;
        return P;
    }
    void collectKernelTimes() {
        for (const auto& u : evUsed) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, evPool[u.second], evPool[u.second + 1]) == cudaSuccess) {
                kernelMs[u.first] += ms;
                kernelCalls[u.first] += 1;
            }
        }
        evUsed.clear();
        evNext = 0;
    }

    ~cgmli_solver() {
        if (stream) cudaStreamSynchronize(stream);
        if (graphExec) cudaGraphExecDestroy(graphExec);
        DArray<double>* dbl[] = {&camR, &camT, &lmBearing, &lmVel, &lmTime, &lmC, &lmD, &lmG, &lmCost, &lmDelta, &lmPred, &lmTrial,
                                 &lmMaxInc, &obBearing, &obP, &obVel, &obTime, &obSrcBearing, &obSrcP, &obSrcVel, &obSrcTime,
                                 &pose[0], &pose[1], &sb[0], &sb[1], &ext[0], &ext[1],
                                 &rotKf[0], &rotKf[1], &rotExt[0], &rotExt[1],
                                 &td[0], &td[1], &rho[0], &rho[1], &imu, &priorA, &priorR0, &priorRef, &Hret, &gret, &costRet,
                                 &trialRet, &acc, &dr, &rhs, &Sglob, &imuScratch, &priorScratch, &predState, &out, &Sdebug};
        for (auto* a : dbl) a->release();
        DArray<int>* ints[] = {&camExt, &lmWin, &lmKf, &lmCam, &lmObsBegin, &lmNs, &lmSupp0, &supp, &lmValid, &lmTrialValid, &obKf,
                               &obCam, &obSlot, &imuKf, &priorKind, &priorIndex, &priorCol, &priorOff, &retValid,
                               &solveStatus, &lmNx, &obXslot, &obOrig};
        for (auto* a : ints) a->release();
        lmC0.release(); dWin.release(); dLm.release(); dRuns.release(); dTiles.release();
        dDetPairs.release(); dDetSchur.release(); detSlots.release();
        dPairChunks.release(); dSchurChunks.release(); schurCols.release(); lmUmap.release(); obLm.release(); keyOrder.release(); bigFirst.release(); keyRows.release(); sch.release();
        snapPose.release(); snapSb.release(); snapExt.release(); snapTd.release(); snapRho.release();
        wideList.release(); facFailed.release(); facVec.release(); wideProd.release(); wideL21.release();
        imuTimes.release(); imuT0.release(); imuT1.release(); imuReadings.release(); imuRanges.release(); imuStatus.release();
        imuRefreshed.release(); imuRefreshScratch.release();
        obRejected.release(); gateCounts.release(); gateStats.release();
        mergeRange.release(); mergeKf.release(); mergeStatus.release(); mergeFlag.release(); mergeT0.release(); mergeT1.release();
        mergeOut.release();
        calibWork0.release(); calibWork.release(); calibCond.release(); calibEvals.release();
        colChart.release(); lmFixed.release(); evalOut.release(); evalValid.release();
        hostH.release(); hostG.release(); hostCost.release(); hostFlag.release();
        dMargWin.release(); dMargElim.release(); dMargOrder.release();
        DArray<int>* mi[] = {&margCols, &margObsMap, &margPoseCol, &margSbCol, &margExtCol, &margRank, &margStatus, &margFast,
                             &margVisCol, &margVisPose, &margVisExt, &margSlow};
        for (auto* a : mi) a->release();
        margChunks.release(); margItems.release();
        DArray<double>* md[] = {&margH, &margB, &margSepH, &margSepV, &margSepB, &margEvals, &margA, &margR0, &margX, &margMaxD, &margStats};
        for (auto* a : md) a->release();
        for (auto e : evPool) cudaEventDestroy(e);
        if (margUploaded) cudaEventDestroy(margUploaded);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {
int ambientOf(int kind) { return kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 7; }

}  // namespace

extern "C" {

const char* cgmli_last_error(void) { return g_error.c_str(); }

static int planOf(const cgmli_tuning* t, PlanParams& p) {
    p = PlanParams();
    if (!t) return CGMLI_OK;
    if (t->run_landmarks < 0 || t->run_landmarks > 4096) return fail(CGMLI_E_INVALID, "tuning: run_landmarks outside 0..4096");
    if (t->pair_chunk != 0 && (t->pair_chunk < 8 || t->pair_chunk > 1024)) return fail(CGMLI_E_INVALID, "tuning: pair_chunk outside 8..1024");
    if (t->schur_rows != 0 && (t->schur_rows < 8 || t->schur_rows > kSchurMaxRows))
        return fail(CGMLI_E_INVALID, "tuning: schur_rows outside 8..128");
    if (t->lin_shape < 0 || t->lin_shape >= kLinShapes) return fail(CGMLI_E_INVALID, "tuning: lin_shape outside 0..3");
    if (t->trial_shape < 0 || t->trial_shape >= kTrialShapes) return fail(CGMLI_E_INVALID, "tuning: trial_shape outside 0..2");
    if (t->deterministic != 0 && t->deterministic != 1) return fail(CGMLI_E_INVALID, "tuning: deterministic not 0 or 1");
    p.deterministic = t->deterministic;
    p.linShape = t->lin_shape;
    p.trialShape = t->trial_shape;
    p.runLandmarks = t->run_landmarks;
    if (t->pair_chunk) p.pairChunk = t->pair_chunk;
    if (t->schur_rows) p.schurRows = t->schur_rows;
    return CGMLI_OK;
}

int cgmli_topology_check(const cgmli_window* windows, int count, int threads, double* seconds) {
    return cgmli_topology_check_tuned(windows, count, threads, nullptr, seconds);
}

int cgmli_topology_check_tuned(const cgmli_window* windows, int count, int threads, const cgmli_tuning* tuning, double* seconds) {
    if (!windows || count < 1) return fail(CGMLI_E_INVALID, "empty window list");
    PlanParams plan;
    if (planOf(tuning, plan) != CGMLI_OK) return CGMLI_E_INVALID;
    const auto t0 = std::chrono::steady_clock::now();
    HostBatch hb;
    std::string why;
    int st = buildHostBatch(windows, count, threads, hb, why, nullptr, plan);
    const auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (st != CGMLI_OK) return fail(st, why);
    st = checkHostBatch(windows, count, hb, why);
    if (st != CGMLI_OK) return fail(st, why);
    return CGMLI_OK;
}

int cgmli_topology_digest(const cgmli_window* windows, int count, int threads, const cgmli_tuning* tuning,
                          unsigned long long* digest) {
    if (!windows || count < 1 || !digest) return fail(CGMLI_E_INVALID, "empty window list or null digest");
    PlanParams plan;
    if (planOf(tuning, plan) != CGMLI_OK) return CGMLI_E_INVALID;
    HostBatch hb;
    std::string why;
    const int st = buildHostBatch(windows, count, threads, hb, why, nullptr, plan);
    if (st != CGMLI_OK) return fail(st, why);
    unsigned long long h = 1469598103934665603ull;
    auto mix = [&](const auto& v) {
        const unsigned char* b = reinterpret_cast<const unsigned char*>(v.data());
        for (size_t i = 0; i < v.size() * sizeof(v[0]); ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    };
    mix(hb.runs); mix(hb.tiles); mix(hb.pairChunks); mix(hb.schurChunks); mix(hb.schurCols); mix(hb.lmUmap);
    mix(hb.lmPerm); mix(hb.camR); mix(hb.camT); mix(hb.camExt); mix(hb.lmWin); mix(hb.lmKf); mix(hb.lmCam); mix(hb.lmObsBegin);
    mix(hb.lmNs); mix(hb.lmNx); mix(hb.lmSupp0); mix(hb.supp); mix(hb.lmC0); mix(hb.lmBearing); mix(hb.lmVel); mix(hb.lmTime);
    mix(hb.obKf); mix(hb.obCam); mix(hb.obSlot); mix(hb.obXslot); mix(hb.obLm); mix(hb.keyOrder); mix(hb.obOrig);
    mix(hb.obBearing); mix(hb.obP); mix(hb.obVel); mix(hb.obTime); mix(hb.pose); mix(hb.sb); mix(hb.ext); mix(hb.td);
    mix(hb.rho); mix(hb.colChart); mix(hb.lmFixed); mix(hb.imu); mix(hb.imuKf); mix(hb.priorKind); mix(hb.priorIndex);
    mix(hb.priorCol); mix(hb.priorOff); mix(hb.priorA); mix(hb.priorR0); mix(hb.priorRef);
    mix(hb.detPairs); mix(hb.detSchur);
    for (const WinDesc& d : hb.win) {
        const long long det[3] = {d.det0, d.detPairs, d.detSchur};
        mix(std::vector<long long>(det, det + 3));
    }
    *digest = h;
    return CGMLI_OK;
}

void cgmli_default_options(cgmli_solver_options* o) {
    o->precision = CGMLI_PRECISION_FP64;
    o->refinement_steps = 0;
    o->initial_lambda = 1e-4;
    o->min_iterations = 0;
    o->time_budget_s = 0.0;
}

int cgmli_solver_create(int device, const cgmli_solver_options* options, cgmli_solver** out) {
    if (!out) return fail(CGMLI_E_INVALID, "null output handle");
    *out = nullptr;
    if (options) {
        if (options->precision != CGMLI_PRECISION_FP64 && options->precision != CGMLI_PRECISION_MIXED)
            return fail(CGMLI_E_INVALID, "unknown precision");
        if (options->refinement_steps < 0 || options->refinement_steps > 2) return fail(CGMLI_E_INVALID, "refinement_steps outside 0..2");
        if (!(options->initial_lambda > 0)) return fail(CGMLI_E_INVALID, "initial_lambda must be positive");
        if (options->min_iterations < 0) return fail(CGMLI_E_INVALID, "min_iterations < 0");
        if (!std::isfinite(options->time_budget_s)) return fail(CGMLI_E_INVALID, "time_budget_s not finite");
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(CGMLI_E_CUDA, "no CUDA device available");
    if (device < 0 || device >= count) return fail(CGMLI_E_INVALID, "device index out of range");
    CK(cudaSetDevice(device));
    auto* s = new cgmli_solver();
    s->device = device;
    if (options) s->opt = *options; else cgmli_default_options(&s->opt);
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&s->ev0)) != cudaSuccess || (e = cudaEventCreate(&s->ev1)) != cudaSuccess) {
        delete s;
        return cudaFail(e, "stream/event creation");
    }
    *out = s;
    return CGMLI_OK;
}

void cgmli_solver_destroy(cgmli_solver* s) { delete s; }

int cgmli_solver_set_windows(cgmli_solver* S, const cgmli_window* windows, int count) {
    if (!S || !windows || count < 1) return fail(CGMLI_E_INVALID, "null solver or empty window list");
    CK(cudaSetDevice(S->device));
    cudaStream_t st = S->stream;
    const AllocStreamScope ordered(st);
    // the previous batch's uploads read the pinned host arrays that are rebuilt now
    CK(cudaStreamSynchronize(st));
    S->haveSnapshot = false;
    S->haveMarg = false;
    S->haveImuSamples = false;
    S->haveEval = false;
    S->win.clear();
    HostBatch& hb = S->hb;
    std::string why;
    // the landmark and observation arrays (most of the bytes) are uploaded range
    // by range as the builder finishes them, overlapping the rest of the build
    cudaError_t streamErr = cudaSuccess;
    bool reserved = false;
    auto part = [&](auto& dev, const auto& host, size_t first, size_t n) {
        if (streamErr != cudaSuccess || n == 0) return;
        streamErr = cudaMemcpyAsync(dev.p + first, host.data() + first, n * sizeof(host[0]), cudaMemcpyHostToDevice, st);
    };
    const std::function<void(int, int)> ready = [&](int w0, int w1) {
        if (!reserved) {
            reserved = true;
            const size_t ob = hb.obKf.size(), lmn = hb.lmKf.size();
            cudaError_t e = cudaSuccess;
            auto res = [&](auto& dev, size_t n) { if (e == cudaSuccess) e = dev.reserve(n); };
            res(S->obBearing, 3 * ob); res(S->obP, 6 * ob); res(S->obVel, 3 * ob); res(S->obTime, ob);
            res(S->obSrcBearing, 3 * ob); res(S->obSrcP, 6 * ob); res(S->obSrcVel, 3 * ob); res(S->obSrcTime, ob);
            res(S->obOrig, ob);
            res(S->obKf, ob); res(S->obCam, ob); res(S->obSlot, ob); res(S->obXslot, ob); res(S->obLm, ob); res(S->keyOrder, ob);
            res(S->lmWin, lmn); res(S->lmKf, lmn); res(S->lmCam, lmn); res(S->lmNs, lmn); res(S->lmNx, lmn);
            res(S->lmBearing, 3 * lmn); res(S->lmVel, 3 * lmn); res(S->lmTime, lmn); res(S->rho[0], lmn);
            streamErr = e;
        }
        const WinDesc& a = hb.win[w0];
        const WinDesc& b = hb.win[w1 - 1];
        const size_t o0 = a.obs0, on = (size_t)b.obs0 + b.F - o0, l0 = a.lm0, ln = (size_t)b.lm0 + b.L - l0;
        part(S->obSrcBearing, hb.obBearing, 3 * o0, 3 * on); part(S->obSrcP, hb.obP, 6 * o0, 6 * on);
        part(S->obSrcVel, hb.obVel, 3 * o0, 3 * on); part(S->obSrcTime, hb.obTime, o0, on); part(S->obOrig, hb.obOrig, o0, on);
        part(S->obKf, hb.obKf, o0, on); part(S->obCam, hb.obCam, o0, on); part(S->obSlot, hb.obSlot, o0, on);
        part(S->obXslot, hb.obXslot, o0, on); part(S->obLm, hb.obLm, o0, on); part(S->keyOrder, hb.keyOrder, o0, on);
        part(S->lmWin, hb.lmWin, l0, ln); part(S->lmKf, hb.lmKf, l0, ln); part(S->lmCam, hb.lmCam, l0, ln);
        part(S->lmNs, hb.lmNs, l0, ln); part(S->lmNx, hb.lmNx, l0, ln); part(S->lmBearing, hb.lmBearing, 3 * l0, 3 * ln);
        part(S->lmVel, hb.lmVel, 3 * l0, 3 * ln); part(S->lmTime, hb.lmTime, l0, ln); part(S->rho[0], hb.rho, l0, ln);
    };
    const int built = buildHostBatch(windows, count, 0, hb, why, &ready, S->tune);
    if (built != CGMLI_OK) return fail(built, why);
    CK(streamErr);
    S->win = hb.win;
    S->totalKf = hb.totalKf; S->totalExt = hb.totalExt; S->totalCam = hb.totalCam; S->totalLm = hb.totalLm;
    S->totalObs = hb.totalObs; S->totalImu = hb.totalImu;
    S->maxNpc = hb.maxNpc; S->maxNr = hb.maxNr; S->maxNs = hb.maxNs;
    S->linSmem = linearizeSmemBytes(S->maxNs, S->opt.precision == CGMLI_PRECISION_MIXED);
    {
        // windows of at least kWideCols retained columns take the wide sequence; k_factor's
        // shared memory is sized by the others
        int narrow = 0, wide = 0;
        for (int i = 0; i < count; ++i) wide += isWideWindow(S->win[i].Nr) ? 1 : 0;
        auto& wl = S->hWideList;
        sizeTo(wl, wide);  // pinned staging: the upload stays asynchronous
        S->wideCols = 0; S->wideCharts = 0;
        for (int i = 0, k = 0; i < count; ++i) {
            const WinDesc& d = S->win[i];
            if (isWideWindow(d.Nr)) {
                wl[k++] = i;
                S->wideCols = std::max(S->wideCols, d.Nr);
                S->wideCharts |= d.charts ? 1 : 0;
            } else {
                narrow = std::max(narrow, d.Nr);
            }
        }
        S->numWide = wide;
        S->facSmem = factorSmemBytes(narrow);
        S->wideFinishSmem = S->numWide ? wideFinishSmemBytes(S->wideCols) : 0;
    }
    CK(configureKernels(S->linSmem, S->facSmem, S->wideFinishSmem));
    const long long lm = hb.totalLm;
    S->hWin.assign(S->win.begin(), S->win.end());  // pinned staging: the copy stays asynchronous
    CK(S->dWin.upload(S->hWin, st));
    CK(S->dLm.reserve(count));
    {
        auto& order = S->hBigFirst;
        sizeTo(order, count);
        for (int i = 0; i < count; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return S->win[a].Nr > S->win[b].Nr; });
        CK(S->bigFirst.reserve(count));
        CK(cudaMemcpyAsync(S->bigFirst.p, order.data(), count * sizeof(int), cudaMemcpyHostToDevice, st));
    }
    CK(S->dRuns.upload(hb.runs, st));
    CK(S->dTiles.upload(hb.tiles, st));
    CK(S->dPairChunks.upload(hb.pairChunks, st));
    CK(S->dSchurChunks.upload(hb.schurChunks, st));
    if (hb.plan.deterministic) {
        CK(S->dDetPairs.upload(hb.detPairs, st));
        CK(S->dDetSchur.upload(hb.detSchur, st));
        CK(S->detSlots.reserve(hb.detSlots));
    }
    CK(S->schurCols.upload(hb.schurCols, st));
    CK(S->lmUmap.upload(hb.lmUmap, st));
    CK(S->camR.upload(hb.camR, st)); CK(S->camT.upload(hb.camT, st)); CK(S->camExt.upload(hb.camExt, st));
    CK(S->lmObsBegin.upload(hb.lmObsBegin, st));
    CK(S->lmSupp0.upload(hb.lmSupp0, st));
    CK(S->supp.upload(hb.supp, st)); CK(S->lmC0.upload(hb.lmC0, st));
    CK(S->keyRows.reserve((size_t)hb.totalObs * 56));
    CK(S->pose[0].upload(hb.pose, st)); CK(S->sb[0].upload(hb.sb, st)); CK(S->ext[0].upload(hb.ext, st));
    CK(S->td[0].upload(hb.td, st));
    CK(S->pose[1].reserve(hb.pose.size())); CK(S->sb[1].reserve(hb.sb.size())); CK(S->ext[1].reserve(hb.ext.size()));
    for (int k = 0; k < 2; ++k) { CK(S->rotKf[k].reserve(9ull * hb.totalKf)); CK(S->rotExt[k].reserve(9ull * hb.totalExt)); }
    CK(S->td[1].reserve(hb.td.size())); CK(S->rho[1].reserve(hb.rho.size()));
    CK(S->imu.upload(hb.imu, st)); CK(S->imuKf.upload(hb.imuKf, st));
    CK(S->colChart.upload(hb.colChart, st)); CK(S->lmFixed.upload(hb.lmFixed, st));
    CK(S->priorKind.upload(hb.priorKind, st)); CK(S->priorIndex.upload(hb.priorIndex, st));
    CK(S->priorCol.upload(hb.priorCol, st)); CK(S->priorOff.upload(hb.priorOff, st));
    CK(S->priorA.upload(hb.priorA, st)); CK(S->priorR0.upload(hb.priorR0, st)); CK(S->priorRef.upload(hb.priorRef, st));
    CK(S->lmC.reserve(hb.cross)); CK(S->lmD.reserve(lm)); CK(S->lmG.reserve(lm)); CK(S->lmCost.reserve(lm));
    CK(S->lmDelta.reserve(lm)); CK(S->lmPred.reserve(lm)); CK(S->lmTrial.reserve(lm)); CK(S->lmMaxInc.reserve(lm));
    CK(S->lmValid.reserve(lm)); CK(S->lmTrialValid.reserve(lm));
    CK(S->Hret.reserve(hb.dense)); CK(S->Sglob.reserve(hb.dense)); CK(S->gret.reserve(hb.vec)); CK(S->dr.reserve(hb.vec));
    CK(S->rhs.reserve(hb.vec));
    if (S->numWide) {
        CK(S->wideList.upload(S->hWideList, st));
        CK(S->facVec.reserve(3 * (size_t)hb.vec));
        CK(S->facFailed.reserve(count));
        CK(S->wideProd.reserve((size_t)S->numWide * ((S->wideCols + 31) / 32 + 1) * S->wideCols));
        CK(S->wideL21.reserve((size_t)S->numWide * 2 * 32 * S->wideCols));
    }
    CK(S->acc.reserve(hb.acc)); CK(S->sch.reserve(hb.sch)); CK(S->imuScratch.reserve(hb.imuScratch));
    CK(S->priorScratch.reserve(hb.priorScratch));
    CK(S->costRet.reserve(count)); CK(S->trialRet.reserve(count)); CK(S->retValid.reserve(count));
    CK(S->predState.reserve(count)); CK(S->solveStatus.reserve(count)); CK(S->out.reserve(4ll * count));
    DevBatch& B = S->B;
    B = DevBatch{};
    B.numWindows = count; B.numLandmarks = hb.totalLm; B.numObs = hb.totalObs; B.numKf = hb.totalKf; B.numExt = hb.totalExt;
    B.numCam = hb.totalCam; B.numImu = hb.totalImu;
    B.numRuns = (int)hb.runs.size();
    B.mixed = S->opt.precision == CGMLI_PRECISION_MIXED ? 1 : 0;
    B.win = S->dWin.p; B.lm = S->dLm.p; B.bigFirst = S->bigFirst.p;
    B.camR = S->camR.p; B.camT = S->camT.p; B.camExt = S->camExt.p;
    B.lmWin = S->lmWin.p; B.lmKf = S->lmKf.p; B.lmCam = S->lmCam.p; B.lmObsBegin = S->lmObsBegin.p;
    B.lmBearing = S->lmBearing.p; B.lmVel = S->lmVel.p; B.lmTime = S->lmTime.p;
    B.lmNs = S->lmNs.p; B.lmNx = S->lmNx.p; B.lmSupp0 = S->lmSupp0.p; B.supp = S->supp.p; B.lmC0 = S->lmC0.p;
    B.lmUmap = S->lmUmap.p; B.schurCols = S->schurCols.p;
    B.obXslot = S->obXslot.p;
    B.lmC = S->lmC.p; B.lmD = S->lmD.p; B.lmG = S->lmG.p; B.lmCost = S->lmCost.p; B.lmValid = S->lmValid.p;
    B.lmDelta = S->lmDelta.p; B.lmPred = S->lmPred.p; B.lmTrial = S->lmTrial.p; B.lmMaxInc = S->lmMaxInc.p;
    B.lmTrialValid = S->lmTrialValid.p;
    B.obKf = S->obKf.p; B.obCam = S->obCam.p; B.obSlot = S->obSlot.p;
    B.obLm = S->obLm.p; B.keyOrder = S->keyOrder.p; B.keyRows = S->keyRows.p;
    B.obBearing = S->obBearing.p; B.obP = S->obP.p; B.obVel = S->obVel.p; B.obTime = S->obTime.p;
    for (int k = 0; k < 2; ++k) {
        B.pose[k] = S->pose[k].p; B.sb[k] = S->sb[k].p; B.ext[k] = S->ext[k].p; B.td[k] = S->td[k].p; B.rho[k] = S->rho[k].p;
        B.rotKf[k] = S->rotKf[k].p; B.rotExt[k] = S->rotExt[k].p;
    }
    B.imu = S->imu.p; B.imuKf = S->imuKf.p;
    B.colChart = S->colChart.p; B.lmFixed = S->lmFixed.p;
    B.minIterations = S->opt.min_iterations;
    B.budgetNs = S->opt.time_budget_s > 0 ? std::max(1ll, (long long)std::llround(S->opt.time_budget_s * 1e9)) : 0;
    B.priorKind = S->priorKind.p; B.priorIndex = S->priorIndex.p; B.priorCol = S->priorCol.p; B.priorOff = S->priorOff.p;
    B.priorA = S->priorA.p; B.priorR0 = S->priorR0.p; B.priorRef = S->priorRef.p;
    B.Hret = S->Hret.p; B.gret = S->gret.p; B.costRet = S->costRet.p; B.trialRet = S->trialRet.p; B.retValid = S->retValid.p;
    B.acc = S->acc.p; B.sch = S->sch.p; B.dr = S->dr.p; B.rhs = S->rhs.p; B.Sglob = S->Sglob.p;
    B.imuScratch = S->imuScratch.p; B.priorScratch = S->priorScratch.p; B.predState = S->predState.p;
    B.solveStatus = S->solveStatus.p; B.out = S->out.p;
    B.wideList = S->numWide ? S->wideList.p : nullptr;
    B.facVec = S->numWide ? S->facVec.p : nullptr;
    B.facFailed = S->numWide ? S->facFailed.p : nullptr;
    B.wideProd = S->numWide ? S->wideProd.p : nullptr;
    B.wideL21 = S->numWide ? S->wideL21.p : nullptr;
    B.detSlots = hb.plan.deterministic ? S->detSlots.p : nullptr;
    {
        // the observation payload into device order (after every upload above on this stream)
        const double* const src[4] = {S->obSrcBearing.p, S->obSrcP.p, S->obSrcVel.p, S->obSrcTime.p};
        double* const dst[4] = {S->obBearing.p, S->obP.p, S->obVel.p, S->obTime.p};
        launchGatherObservations(B, S->obOrig.p, src, dst, st);
        CK(cudaGetLastError());
    }
    CK(cudaMemsetAsync(S->costRet.p, 0, count * sizeof(double), st));
    CK(cudaMemsetAsync(S->trialRet.p, 0, count * sizeof(double), st));
    CK(S->obRejected.reserve(std::max(1, S->totalObs))); CK(S->gateCounts.reserve((size_t)kGateCounts * count));
    CK(S->gateStats.reserve(2ull * count));
    CK(cudaMemsetAsync(S->obRejected.p, 0, std::max(1, S->totalObs), st));
    CK(cudaMemsetAsync(S->gateCounts.p, 0, (size_t)kGateCounts * count * sizeof(int), st));
    CK(cudaMemsetAsync(S->gateStats.p, 0, 2ull * count * sizeof(double), st));
    return CGMLI_OK;
}

int cgmli_solver_upload_states(cgmli_solver* S, const cgmli_window* windows, int count) {
    if (!S || !windows || count != (int)S->win.size()) return fail(CGMLI_E_INVALID, "window count differs from the configured batch");
    for (int i = 0; i < count; ++i) {
        const WinDesc& d = S->win[i];
        const auto& w = windows[i];
        if (w.num_keyframes != d.K || w.num_landmarks != d.L || w.num_extrinsics != d.E || (w.td != nullptr) != (d.hasTd != 0))
            return fail(CGMLI_E_INVALID, "state upload with a different topology");
    }
    CK(cudaSetDevice(S->device));
    cudaStream_t st = S->stream;
    CK(cudaStreamSynchronize(st));  // the pinned host arrays are the staging of earlier copies
    HostBatch& hb = S->hb;
    for (int i = 0; i < count; ++i) {
        const WinDesc& d = S->win[i];
        const auto& w = windows[i];
        std::memcpy(&hb.pose[7ll * d.kf0], w.poses, 7ull * d.K * sizeof(double));
        std::memcpy(&hb.sb[9ll * d.kf0], w.speed_bias, 9ull * d.K * sizeof(double));
        std::memcpy(&hb.ext[7ll * d.ext0], w.extrinsics, 7ull * d.E * sizeof(double));
        hb.td[i] = w.td ? *w.td : 0.0;
        // device order is sorted by support; lmPerm maps it back to the caller's order
        for (int q = 0; q < d.L; ++q) hb.rho[d.lm0 + q] = w.rho[hb.lmPerm[d.lm0 + q]];
    }
    CK(S->pose[0].upload(hb.pose, st)); CK(S->sb[0].upload(hb.sb, st)); CK(S->ext[0].upload(hb.ext, st));
    CK(S->td[0].upload(hb.td, st)); CK(S->rho[0].upload(hb.rho, st));
    return CGMLI_OK;
}

static void profileHook(void* ctx, int kind, int phase) {
    auto* S = static_cast<cgmli_solver*>(ctx);
    cudaEvent_t e = S->nextEvent();
    if (phase == 0) S->evUsed.push_back({kind, (int)S->evNext - 1});
    cudaEventRecord(e, S->stream);
}

// Everything a captured solve depends on: the batch's device pointers and counts,
// its work decomposition, the iteration budget and the options the kernels read.
static std::vector<char> solveKey(const cgmli_solver* S, int iterations) {
    const LaunchPlan P = S->plan();
    const int ints[2] = {iterations, S->opt.refinement_steps};
    const double lambda0 = S->opt.initial_lambda;
    std::vector<char> k(sizeof(DevBatch) + sizeof(LaunchPlan) + sizeof(ints) + sizeof(lambda0));
    char* p = k.data();
    std::memcpy(p, &S->B, sizeof(DevBatch)); p += sizeof(DevBatch);
    std::memcpy(p, &P, sizeof(LaunchPlan)); p += sizeof(LaunchPlan);
    std::memcpy(p, ints, sizeof(ints)); p += sizeof(ints);
    std::memcpy(p, &lambda0, sizeof(lambda0));
    return k;
}

static int runIterations(cgmli_solver* S, int iterations, int probe, double* Sdebug) {
    cudaStream_t st = S->stream;
    if (S->profile) S->collectKernelTimes();
    if (!probe && !Sdebug && !S->profile) {
        std::vector<char> key = solveKey(S, iterations);
        if (!(S->graphExec && key == S->graphKey) && key == S->lastKey) {
            // second solve of the same sequence: capture it
            if (S->graphExec) { cudaGraphExecDestroy(S->graphExec); S->graphExec = nullptr; }
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int launches = launchLmInit(S->B, S->opt.initial_lambda, st);
            for (int it = 0; it < iterations; ++it)
                launches += launchIteration(S->B, S->plan(), S->opt.refinement_steps, iterations, 0, nullptr, st, nullptr, nullptr);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (e == cudaSuccess) e = cudaGraphInstantiate(&S->graphExec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                S->graphExec = nullptr;
                return cudaFail(e, "solve graph capture");
            }
            S->graphKey = key;
            S->graphLaunches = launches;
        }
        S->lastKey = std::move(key);
        if (S->graphExec && S->lastKey == S->graphKey) {
            CK(cudaEventRecord(S->ev0, st));
            CK(cudaGraphLaunch(S->graphExec, st));
            CK(cudaEventRecord(S->ev1, st));
            S->timed = true;
            S->lastLaunches = S->graphLaunches;
            return CGMLI_OK;
        }
    }
    CK(cudaEventRecord(S->ev0, st));
    int launches = launchLmInit(S->B, S->opt.initial_lambda, st);
    for (int it = 0; it < iterations; ++it)
        launches += launchIteration(S->B, S->plan(), S->opt.refinement_steps, iterations, probe, Sdebug, st,
                                    S->profile ? profileHook : nullptr, S);
    CK(cudaGetLastError());
    CK(cudaEventRecord(S->ev1, st));
    S->timed = true;
    S->lastLaunches = launches;
    return CGMLI_OK;
}

int cgmli_solver_solve(cgmli_solver* S, int max_iterations) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    if (max_iterations < 1) return fail(CGMLI_E_INVALID, "max_iterations < 1");
    CK(cudaSetDevice(S->device));
    return runIterations(S, max_iterations, 0, nullptr);
}

int cgmli_solver_set_tuning(cgmli_solver* S, const cgmli_tuning* tuning) {
    if (!S || !tuning) return fail(CGMLI_E_INVALID, "set_tuning: null solver or tuning");
    PlanParams p;
    if (planOf(tuning, p) != CGMLI_OK) return CGMLI_E_INVALID;
    S->tune = p;
    return CGMLI_OK;
}

int cgmli_solver_get_tuning(cgmli_solver* S, cgmli_tuning* tuning) {
    if (!S || !tuning) return fail(CGMLI_E_INVALID, "get_tuning: null solver or tuning");
    tuning->run_landmarks = S->tune.runLandmarks;
    tuning->pair_chunk = S->tune.pairChunk;
    tuning->schur_rows = S->tune.schurRows;
    tuning->lin_shape = S->tune.linShape;
    tuning->trial_shape = S->tune.trialShape;
    tuning->deterministic = S->tune.deterministic;
    tuning->ms = 0.0;
    return CGMLI_OK;
}

// Coordinate search: each parameter mainly shapes one pass (runs: the landmark
// and trial passes; pair chunks: the J^T J pass; Schur rows: the Schur pass), so
// they are tuned one after the other, each over a few multiples of the current
// value; then the kernel shapes of the landmark and trial passes, each over all
// of its compiled variants.
int cgmli_solver_autotune(cgmli_solver* S, const cgmli_window* windows, int count, int iterations, cgmli_tuning* best) {
    if (!S || !windows || count < 1) return fail(CGMLI_E_INVALID, "autotune: null solver or empty window list");
    if (iterations < 1) return fail(CGMLI_E_INVALID, "autotune: iterations < 1");
    const bool profiled = S->profile;
    S->profile = false;
    auto measure = [&](const PlanParams& p, double& ms) -> int {
        S->tune = p;
        int st = cgmli_solver_set_windows(S, windows, count);
        if (st == CGMLI_OK) st = cgmli_solver_checkpoint(S);
        for (int rep = 0; rep < 2 && st == CGMLI_OK; ++rep) {  // the first solve warms caches and clocks
            if (rep > 0) st = cgmli_solver_rollback(S);
            if (st == CGMLI_OK) st = runIterations(S, iterations, 0, nullptr);
            if (st == CGMLI_OK) {
                float t = 0;
                cudaError_t e = cudaEventSynchronize(S->ev1);
                if (e == cudaSuccess) e = cudaEventElapsedTime(&t, S->ev0, S->ev1);
                if (e != cudaSuccess) st = cudaFail(e, "autotune timing");
                ms = t;
            }
        }
        return st;
    };
    PlanParams cur = S->tune;
    if (cur.runLandmarks <= 0) {
        long long lm = 0;
        for (int i = 0; i < count; ++i) lm += windows[i].num_landmarks;
        cur.runLandmarks = std::max<long long>(4, std::min<long long>(64, lm / (148ll * 6 * 4)));
    }
    double bestMs = 0;
    int st = measure(cur, bestMs);
    for (int param = 0; param < 3 && st == CGMLI_OK; ++param) {
        const int base = param == 0 ? cur.runLandmarks : param == 1 ? cur.pairChunk : cur.schurRows;
        const int lo = param == 0 ? 2 : 8, hi = param == 0 ? 4096 : param == 1 ? 1024 : kSchurMaxRows;
        for (const int v : {base / 2, base * 2}) {
            if (v < lo || v > hi) continue;
            PlanParams p = cur;
            (param == 0 ? p.runLandmarks : param == 1 ? p.pairChunk : p.schurRows) = v;
            double ms = 0;
            if ((st = measure(p, ms)) != CGMLI_OK) break;
            if (ms < bestMs) { bestMs = ms; cur = p; }
        }
    }
    for (int shape = 0; shape < kLinShapes && st == CGMLI_OK; ++shape) {
        if (shape == cur.linShape) continue;
        PlanParams p = cur;
        p.linShape = shape;
        double ms = 0;
        if ((st = measure(p, ms)) != CGMLI_OK) break;
        if (ms < bestMs) { bestMs = ms; cur = p; }
    }
    const int linBest = cur.linShape;
    for (int shape = 0; shape < kTrialShapes && st == CGMLI_OK; ++shape) {
        if (shape == cur.trialShape) continue;
        PlanParams p = cur;
        p.trialShape = shape;
        p.linShape = linBest;
        double ms = 0;
        if ((st = measure(p, ms)) != CGMLI_OK) break;
        if (ms < bestMs) { bestMs = ms; cur = p; }
    }
    S->profile = profiled;
    S->tune = cur;
    if (st != CGMLI_OK) return st;
    if ((st = cgmli_solver_set_windows(S, windows, count)) != CGMLI_OK) return st;
    if (best) {
        best->run_landmarks = cur.runLandmarks;
        best->pair_chunk = cur.pairChunk;
        best->schur_rows = cur.schurRows;
        best->lin_shape = cur.linShape;
        best->trial_shape = cur.trialShape;
        best->deterministic = cur.deterministic;
        best->ms = bestMs;
    }
    return CGMLI_OK;
}

int cgmli_solver_solve_gated(cgmli_solver* S, int max_iterations, double nis_threshold, int max_refits, int pre_gate) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    if (max_iterations < 1) return fail(CGMLI_E_INVALID, "max_iterations < 1");
    if (!(nis_threshold > 0)) return fail(CGMLI_E_INVALID, "solve_gated: nis_threshold must be positive");
    if (max_refits < 0 || max_refits > 64) return fail(CGMLI_E_INVALID, "solve_gated: max_refits outside 0..64");
    CK(cudaSetDevice(S->device));
    cudaStream_t st = S->stream;
    if (S->profile) S->collectKernelTimes();
    const LaunchPlan P = S->plan();
    CK(cudaEventRecord(S->ev0, st));
    int launches = launchLmInit(S->B, S->opt.initial_lambda, st);
    // the gate at the initial states removes factors before the first solve
    if (pre_gate)
        launches += launchGate(S->B, P, 0, 1, nis_threshold, S->obP.p, S->obRejected.p, S->gateStats.p, S->gateCounts.p, st);
    for (int pass = 0; pass <= max_refits; ++pass) {
        // pass 0 solves every window; a refit pass restarts the windows whose gate
        // rejected factors (the others return at once from every kernel)
        if (pass > 0) launches += launchRefit(S->B, pass, S->opt.initial_lambda, max_iterations, S->gateCounts.p, st);
        for (int it = 0; it < max_iterations; ++it)
            launches += launchIteration(S->B, P, S->opt.refinement_steps, max_iterations, 0, nullptr, st,
                                        S->profile ? profileHook : nullptr, S);
        launches += launchGate(S->B, P, pass, 0, nis_threshold, S->obP.p, S->obRejected.p, S->gateStats.p, S->gateCounts.p, st);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(S->ev1, st));
    S->timed = true;
    S->lastLaunches = launches;
    return CGMLI_OK;
}

int cgmli_solver_read_gate(cgmli_solver* S, int window, cgmli_gate_report* report, unsigned char* rejected) {
    if (!S || window < 0 || window >= (int)S->win.size() || !report) return fail(CGMLI_E_INVALID, "read_gate: bad window or null report");
    CK(cudaSetDevice(S->device));
    const WinDesc& d = S->win[window];
    WinLM lm;
    int counts[kGateCounts];
    double stats[2];
    std::vector<unsigned char> mask(rejected ? d.F : 0);
    CK(cudaMemcpyAsync(&lm, S->dLm.p + window, sizeof(WinLM), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaMemcpyAsync(counts, S->gateCounts.p + (long long)kGateCounts * window, sizeof(counts), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaMemcpyAsync(stats, S->gateStats.p + 2ll * window, sizeof(stats), cudaMemcpyDeviceToHost, S->stream));
    if (rejected && d.F)
        CK(cudaMemcpyAsync(mask.data(), S->obRejected.p + d.obs0, d.F, cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    report->passes = lm.pass + 1;
    report->evaluated = counts[0];
    report->rejected_last = counts[1];
    report->rejected_total = counts[2];
    report->rejected_pre = counts[4];
    report->nis_sum = stats[0];
    report->nis_max = stats[1];
    if (rejected)
        for (int o = 0; o < d.F; ++o) rejected[S->hb.obOrig[d.obs0 + o]] = mask[o];
    return counts[3] ? fail(CGMLI_E_NONFINITE, "read_gate: a gated residual was not finite") : CGMLI_OK;
}

int cgmli_solver_set_imu_samples(cgmli_solver* S, const cgmli_imu_parameters* params, const long long* sample_time_ns,
                                 const double* sample_readings, int num_samples, const int* range, const long long* t0_ns,
                                 const long long* t1_ns) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    const int count = S->totalImu;
    if (!params) return fail(CGMLI_E_INVALID, "set_imu_samples: null parameters");
    if (count == 0) {
        S->haveImuSamples = false;
        return CGMLI_OK;
    }
    if (!sample_time_ns || !sample_readings || !range || !t0_ns || !t1_ns || num_samples < 2)
        return fail(CGMLI_E_INVALID, "set_imu_samples: null buffers or fewer than 2 samples");
    int lo = num_samples, hi = 0;
    for (int i = 0; i < count; ++i) {
        const int b = range[2 * i], e = range[2 * i + 1];
        if (b == e && b >= 0 && b <= num_samples) continue;  // no samples: the refresh keeps the factor
        if (b < 0 || e > num_samples || e - b < 2)
            return fail(CGMLI_E_INVALID, "set_imu_samples: factor " + std::to_string(i) + ": sample range outside the samples or shorter than 2");
        lo = std::min(lo, b);
        hi = std::max(hi, e);
    }
    if (hi <= lo) lo = hi = 0;  // every factor without samples
    CK(cudaSetDevice(S->device));
    cudaStream_t st = S->stream;
    const size_t span = (size_t)(hi - lo);
    CK(S->imuTimes.reserve(span)); CK(S->imuReadings.reserve(6 * span));
    CK(S->imuRanges.reserve(2 * (size_t)count)); CK(S->imuT0.reserve(count)); CK(S->imuT1.reserve(count));
    CK(S->imuStatus.reserve(count)); CK(S->imuRefreshed.reserve(count)); CK(S->imuRefreshScratch.reserve(count));
    if (span) {
        CK(cudaMemcpyAsync(S->imuTimes.p, sample_time_ns + lo, span * sizeof(long long), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S->imuReadings.p, sample_readings + 6 * (size_t)lo, 6 * span * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemcpyAsync(S->imuRanges.p, range, 2 * (size_t)count * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S->imuT0.p, t0_ns, count * sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S->imuT1.p, t1_ns, count * sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(S->imuStatus.p, 0, count * sizeof(int), st));
    CK(cudaMemsetAsync(S->imuRefreshed.p, 0, count * sizeof(int), st));
    // the caller's arrays may change once this returns (pageable copies are staged
    // before cudaMemcpyAsync returns, so no wait is needed for them)
    S->imuParams = *params;
    S->imuSampleOffset = lo;
    S->haveImuSamples = true;
    S->hImuRange.assign(range, range + 2 * (size_t)count);
    S->hImuT0.assign(t0_ns, t0_ns + count);
    S->hImuT1.assign(t1_ns, t1_ns + count);
    return CGMLI_OK;
}

int cgmli_solver_refresh_imu(cgmli_solver* S, double gyro_threshold, double accel_threshold, int* refreshed) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    if (!(gyro_threshold >= 0) || !(accel_threshold >= 0)) return fail(CGMLI_E_INVALID, "refresh_imu: negative or NaN threshold");
    const int count = S->totalImu;
    if (count > 0 && !S->haveImuSamples) return fail(CGMLI_E_INVALID, "refresh_imu: no IMU samples for this batch (set_imu_samples)");
    CK(cudaSetDevice(S->device));
    if (count > 0) {
        ImuLaunch L{};
        L.prm = S->imuParams;
        L.times = S->imuTimes.p; L.readings = S->imuReadings.p; L.sampleOffset = S->imuSampleOffset;
        L.ranges = S->imuRanges.p; L.t0s = S->imuT0.p; L.t1s = S->imuT1.p;
        L.out = reinterpret_cast<cgmli_frozen_imu*>(S->imu.p);
        L.status = S->imuStatus.p;
        L.biases = nullptr;
        L.sb = S->sb[0].p; L.kf = S->imuKf.p;
        L.gyroThreshold = gyro_threshold; L.accelThreshold = accel_threshold;
        L.scratch = S->imuRefreshScratch.p; L.refreshed = S->imuRefreshed.p;
        CK(launchImuPreintegration(L, count, S->stream));
    }
    if (!refreshed) return CGMLI_OK;
    *refreshed = 0;
    if (count == 0) return CGMLI_OK;
    sizeTo(S->hImuStatus, count);
    sizeTo(S->hImuRefreshed, count);
    CK(cudaMemcpyAsync(S->hImuStatus.data(), S->imuStatus.p, count * sizeof(int), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaMemcpyAsync(S->hImuRefreshed.data(), S->imuRefreshed.p, count * sizeof(int), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    for (int i = 0; i < count; ++i) *refreshed += S->hImuRefreshed[i];
    for (int i = 0; i < count; ++i)
        if (S->hImuStatus[i] != CGMLI_OK)
            return fail(S->hImuStatus[i], "refresh_imu: factor " + std::to_string(i) +
                                              (S->hImuStatus[i] == CGMLI_E_INVALID ? ": invalid samples" : ": result not finite") +
                                              "; it keeps its previous value");
    return CGMLI_OK;
}

int cgmli_solver_read_imu(cgmli_solver* S, int window, cgmli_frozen_imu* imu) {
    if (!S || window < 0 || window >= (int)S->win.size()) return fail(CGMLI_E_INVALID, "read_imu: bad window");
    const WinDesc& d = S->win[window];
    if (d.nImu == 0) return CGMLI_OK;
    if (!imu) return fail(CGMLI_E_INVALID, "read_imu: null buffer");
    CK(cudaSetDevice(S->device));
    CK(cudaMemcpyAsync(imu, reinterpret_cast<const cgmli_frozen_imu*>(S->imu.p) + d.imu0, d.nImu * sizeof(cgmli_frozen_imu),
                       cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return CGMLI_OK;
}

int cgmli_solver_synchronize(cgmli_solver* S) {
    if (!S) return fail(CGMLI_E_INVALID, "null solver");
    CK(cudaStreamSynchronize(S->stream));
    S->readTiming();
    if (S->profile) S->collectKernelTimes();
    return CGMLI_OK;
}

int cgmli_solver_checkpoint(cgmli_solver* S) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    CK(cudaSetDevice(S->device));
    const size_t np = 7ull * S->totalKf, ns = 9ull * S->totalKf, ne = 7ull * S->totalExt, nt = S->win.size(), nl = S->totalLm;
    CK(S->snapPose.reserve(np)); CK(S->snapSb.reserve(ns)); CK(S->snapExt.reserve(ne)); CK(S->snapTd.reserve(nt));
    CK(S->snapRho.reserve(nl));
    CK(cudaMemcpyAsync(S->snapPose.p, S->pose[0].p, np * 8, cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaMemcpyAsync(S->snapSb.p, S->sb[0].p, ns * 8, cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaMemcpyAsync(S->snapExt.p, S->ext[0].p, ne * 8, cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaMemcpyAsync(S->snapTd.p, S->td[0].p, nt * 8, cudaMemcpyDeviceToDevice, S->stream));
    if (nl) CK(cudaMemcpyAsync(S->snapRho.p, S->rho[0].p, nl * 8, cudaMemcpyDeviceToDevice, S->stream));
    S->haveSnapshot = true;
    return CGMLI_OK;
}

int cgmli_solver_rollback(cgmli_solver* S) {
    if (!S || !S->haveSnapshot) return fail(CGMLI_E_INVALID, "no checkpoint to roll back to");
    CK(cudaSetDevice(S->device));
    const size_t np = 7ull * S->totalKf, ns = 9ull * S->totalKf, ne = 7ull * S->totalExt, nt = S->win.size(), nl = S->totalLm;
    CK(cudaMemcpyAsync(S->pose[0].p, S->snapPose.p, np * 8, cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaMemcpyAsync(S->sb[0].p, S->snapSb.p, ns * 8, cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaMemcpyAsync(S->ext[0].p, S->snapExt.p, ne * 8, cudaMemcpyDeviceToDevice, S->stream));
    CK(cudaMemcpyAsync(S->td[0].p, S->snapTd.p, nt * 8, cudaMemcpyDeviceToDevice, S->stream));
    if (nl) CK(cudaMemcpyAsync(S->rho[0].p, S->snapRho.p, nl * 8, cudaMemcpyDeviceToDevice, S->stream));
    return CGMLI_OK;
}

int cgmli_solver_kernel_times(cgmli_solver* S, int enable, double* ms, int* calls) {
    if (!S) return fail(CGMLI_E_INVALID, "null solver");
    if (enable >= 0) {
        S->profile = enable != 0;
        for (int k = 0; k < CGMLI_KERNEL_KINDS; ++k) { S->kernelMs[k] = 0; S->kernelCalls[k] = 0; }
        S->evUsed.clear();
        S->evNext = 0;
    }
    for (int k = 0; k < CGMLI_KERNEL_KINDS; ++k) {
        if (ms) ms[k] = S->kernelMs[k];
        if (calls) calls[k] = S->kernelCalls[k];
    }
    return CGMLI_OK;
}

int cgmli_solver_step(cgmli_solver* S, double lambda) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    if (!(lambda > 0) || !std::isfinite(lambda)) return fail(CGMLI_E_INVALID, "lambda must be positive");
    CK(cudaSetDevice(S->device));
    long long dense = 0;
    for (const auto& d : S->win) dense += (long long)d.Nr * d.Nr;
    CK(S->Sdebug.reserve(dense));
    const double saved = S->opt.initial_lambda;
    S->opt.initial_lambda = lambda;
    const int r = runIterations(S, 1, 1, S->Sdebug.p);
    S->opt.initial_lambda = saved;
    if (r != CGMLI_OK) return r;
    return cgmli_solver_synchronize(S);
}

int cgmli_solver_window_dims(cgmli_solver* S, int w, int* retained, int* landmarks) {
    if (!S || w < 0 || w >= (int)S->win.size()) return fail(CGMLI_E_INVALID, "window index");
    if (retained) *retained = S->win[w].Nr;
    if (landmarks) *landmarks = S->win[w].L;
    return CGMLI_OK;
}

int cgmli_solver_read_step(cgmli_solver* S, int w, double* increment, double* cost, double* predicted, double* trial_cost,
                           int* trial_valid) {
    if (!S || w < 0 || w >= (int)S->win.size()) return fail(CGMLI_E_INVALID, "window index");
    CK(cudaSetDevice(S->device));
    const WinDesc& d = S->win[w];
    WinLM lmst;
    CK(cudaMemcpy(&lmst, S->dLm.p + w, sizeof(WinLM), cudaMemcpyDeviceToHost));
    if (increment) {
        CK(cudaMemcpy(increment, S->dr.p + d.vec0, d.Nr * sizeof(double), cudaMemcpyDeviceToHost));
        if (d.L) {
            std::vector<double> r(d.L);
            CK(cudaMemcpy(r.data(), S->lmDelta.p + d.lm0, d.L * sizeof(double), cudaMemcpyDeviceToHost));
            for (int q = 0; q < d.L; ++q) increment[d.Nr + S->hb.lmPerm[d.lm0 + q]] = r[q];
        }
    }
    if (cost) *cost = lmst.linCost;
    if (predicted) *predicted = lmst.predicted;
    if (trial_cost) *trial_cost = lmst.trialCost;
    if (trial_valid) *trial_valid = lmst.trialValid;
    if (lmst.status != CGMLI_OK) return fail(lmst.status, "window step failed");
    return CGMLI_OK;
}

int cgmli_solver_read_reduced(cgmli_solver* S, int w, double* Sout, double* rhs) {
    if (!S || w < 0 || w >= (int)S->win.size() || !S->Sdebug.p) return fail(CGMLI_E_INVALID, "no reduced system recorded");
    CK(cudaSetDevice(S->device));
    const WinDesc& d = S->win[w];
    if (Sout) CK(cudaMemcpy(Sout, S->Sdebug.p + d.dense0, (size_t)d.Nr * d.Nr * sizeof(double), cudaMemcpyDeviceToHost));
    // the right-hand side the factorization solved: -(g_r - B_v), restricted by the solve-time charts
    if (rhs) CK(cudaMemcpy(rhs, S->rhs.p + d.vec0, d.Nr * sizeof(double), cudaMemcpyDeviceToHost));
    return CGMLI_OK;
}

int cgmli_solver_read_states(cgmli_solver* S, cgmli_window* windows, int count) {
    if (!S || !windows || count != (int)S->win.size()) return fail(CGMLI_E_INVALID, "window count differs from the configured batch");
    CK(cudaSetDevice(S->device));
    // one copy per state array into the pinned host arrays, then a scatter to the windows
    HostBatch& hb = S->hb;
    cudaStream_t st = S->stream;
    CK(cudaMemcpyAsync(hb.pose.data(), S->pose[0].p, hb.pose.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hb.sb.data(), S->sb[0].p, hb.sb.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hb.ext.data(), S->ext[0].p, hb.ext.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hb.td.data(), S->td[0].p, hb.td.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (!hb.rho.empty()) CK(cudaMemcpyAsync(hb.rho.data(), S->rho[0].p, hb.rho.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int i = 0; i < count; ++i) {
        const WinDesc& d = S->win[i];
        auto& w = windows[i];
        std::memcpy(w.poses, &hb.pose[7ll * d.kf0], 7ull * d.K * sizeof(double));
        std::memcpy(w.speed_bias, &hb.sb[9ll * d.kf0], 9ull * d.K * sizeof(double));
        std::memcpy(w.extrinsics, &hb.ext[7ll * d.ext0], 7ull * d.E * sizeof(double));
        if (w.td) *w.td = hb.td[i];
        for (int q = 0; q < d.L; ++q) w.rho[hb.lmPerm[d.lm0 + q]] = hb.rho[d.lm0 + q];
    }
    return CGMLI_OK;
}

int cgmli_solver_read_reports(cgmli_solver* S, cgmli_solve_report* reports, int count) {
    if (!S || !reports || count != (int)S->win.size()) return fail(CGMLI_E_INVALID, "report count differs from the configured batch");
    CK(cudaSetDevice(S->device));
    std::vector<WinLM> lm(count);
    CK(cudaMemcpyAsync(lm.data(), S->dLm.p, count * sizeof(WinLM), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    for (int i = 0; i < count; ++i) {
        auto& r = reports[i];
        r.initial_cost = lm[i].initialCost; r.final_cost = lm[i].cost; r.lambda = lm[i].lambda;
        r.predicted_reduction = lm[i].predicted; r.max_increment = lm[i].maxInc;
        r.iterations = lm[i].iterations; r.accepted_steps = lm[i].accepted; r.converged = lm[i].converged; r.status = lm[i].status;
    }
    return CGMLI_OK;
}

int cgmli_solver_device_bytes(cgmli_solver* S, long long* bytes) {
    if (!S || !bytes) return fail(CGMLI_E_INVALID, "null solver or output");
    *bytes = S->deviceBytes();
    return CGMLI_OK;
}

int cgmli_solver_evaluate(cgmli_solver* S, int derivatives) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    CK(cudaSetDevice(S->device));
    const size_t F = std::max(1, S->totalObs);
    CK(S->evalOut.reserve(F * (2 + CGMLI_FACTOR_JACOBIAN)));
    CK(S->evalValid.reserve(F));
    launchEvaluate(S->B, derivatives ? 1 : 0, S->evalOut.p, S->evalValid.p, S->stream);
    CK(cudaGetLastError());
    S->haveEval = true;
    S->evalDerivatives = derivatives != 0;
    return CGMLI_OK;
}

int cgmli_solver_read_factors(cgmli_solver* S, int w, double* residuals, int* valid, double* jacobians) {
    if (!S || w < 0 || w >= (int)S->win.size()) return fail(CGMLI_E_INVALID, "window index out of range");
    if (!S->haveEval) return fail(CGMLI_E_INVALID, "read_factors before cgmli_solver_evaluate");
    if (jacobians && !S->evalDerivatives) return fail(CGMLI_E_INVALID, "read_factors: Jacobians requested but evaluated without derivatives");
    const WinDesc& d = S->win[w];
    if (d.F == 0) return CGMLI_OK;
    constexpr int rec = 2 + CGMLI_FACTOR_JACOBIAN;
    std::vector<double> out((size_t)rec * d.F);
    std::vector<int> ok(d.F);
    CK(cudaSetDevice(S->device));
    CK(cudaMemcpyAsync(out.data(), S->evalOut.p + (size_t)rec * d.obs0, out.size() * sizeof(double), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaMemcpyAsync(ok.data(), S->evalValid.p + d.obs0, d.F * sizeof(int), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    for (int q = 0; q < d.F; ++q) {
        const int f = S->hb.obOrig[d.obs0 + q];  // caller's observation index
        const double* src = out.data() + (size_t)rec * q;
        if (residuals) { residuals[2 * f] = src[0]; residuals[2 * f + 1] = src[1]; }
        if (valid) valid[f] = ok[q];
        if (jacobians) std::memcpy(jacobians + (size_t)CGMLI_FACTOR_JACOBIAN * f, src + 2, CGMLI_FACTOR_JACOBIAN * sizeof(double));
    }
    return CGMLI_OK;
}

int cgmli_solver_solve_host(cgmli_solver* S, int max_iterations, const unsigned char* has_host, cgmli_host_factor_fn fn, void* ctx) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    if (max_iterations < 1) return fail(CGMLI_E_INVALID, "max_iterations < 1");
    if (!fn) return fail(CGMLI_E_INVALID, "solve_host: null factor callback");
    CK(cudaSetDevice(S->device));
    cudaStream_t st = S->stream;
    const int W = (int)S->win.size();
    HostBatch& hb = S->hb;
    CK(S->hostH.reserve(std::max<long long>(1, hb.dense)));
    CK(S->hostG.reserve(std::max<long long>(1, hb.vec)));
    CK(S->hostCost.reserve(W));
    CK(S->hostFlag.reserve(W));
    std::vector<unsigned char> flag(W);
    for (int w = 0; w < W; ++w) flag[w] = has_host ? (has_host[w] ? 1 : 0) : 1;
    CK(cudaMemcpyAsync(S->hostFlag.p, flag.data(), W, cudaMemcpyHostToDevice, st));
    // host staging of the callbacks' states and results
    std::vector<WinLM> lm(W);
    std::vector<double> Hh((size_t)std::max<long long>(1, hb.dense)), gh((size_t)std::max<long long>(1, hb.vec)), cost(W);
    std::vector<double> pose(hb.pose.size()), sbv(hb.sb.size()), extv(hb.ext.size()), tdv(W);
    auto download = [&](int buf) -> int {
        CK(cudaMemcpyAsync(lm.data(), S->dLm.p, W * sizeof(WinLM), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(pose.data(), S->pose[buf].p, pose.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(sbv.data(), S->sb[buf].p, sbv.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(extv.data(), S->ext[buf].p, extv.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(tdv.data(), S->td[buf].p, W * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return CGMLI_OK;
    };
    const double nan = std::numeric_limits<double>::quiet_NaN();
    CK(cudaEventRecord(S->ev0, st));
    int launches = launchLmInit(S->B, S->opt.initial_lambda, st);
    for (int it = 0; it < max_iterations; ++it) {
        launches += launchIterationParts(S->B, S->plan(), S->opt.refinement_steps, max_iterations, 0, nullptr, st, nullptr, nullptr,
                                         kIterLinearize);
        int r = download(0);
        if (r != CGMLI_OK) return r;
        bool live = false;
        for (int w = 0; w < W; ++w) live = live || lm[w].mode != kModeDone;
        if (!live) break;  // every window has finished
        bool any = false;
        for (int w = 0; w < W; ++w) {
            cost[w] = 0.0;
            if (!flag[w] || lm[w].mode != kModeLinearize) continue;
            any = true;
            const WinDesc& d = S->win[w];
            double* H = Hh.data() + d.dense0;
            double* g = gh.data() + d.vec0;
            std::fill(H, H + (size_t)d.Nr * d.Nr, 0.0);
            std::fill(g, g + d.Nr, 0.0);
            double c = 0;
            const int rc = fn(ctx, w, 0, pose.data() + 7ll * d.kf0, sbv.data() + 9ll * d.kf0, extv.data() + 7ll * d.ext0, &tdv[w], H, g, &c);
            cost[w] = rc == 0 && std::isfinite(c) ? c : nan;  // a failed evaluation fails the window (non-finite cost)
            CK(cudaMemcpyAsync(S->hostH.p + d.dense0, H, (size_t)d.Nr * d.Nr * sizeof(double), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(S->hostG.p + d.vec0, g, d.Nr * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        if (any) {
            CK(cudaMemcpyAsync(S->hostCost.p, cost.data(), W * sizeof(double), cudaMemcpyHostToDevice, st));
            launchAddHost(S->B, S->hostH.p, S->hostG.p, S->hostCost.p, S->hostFlag.p, 0, st);
            ++launches;
        }
        launches += launchIterationParts(S->B, S->plan(), S->opt.refinement_steps, max_iterations, 0, nullptr, st, nullptr, nullptr,
                                         kIterStep);
        if ((r = download(1)) != CGMLI_OK) return r;
        any = false;
        for (int w = 0; w < W; ++w) {
            cost[w] = 0.0;
            if (!flag[w] || lm[w].mode == kModeDone) continue;
            any = true;
            const WinDesc& d = S->win[w];
            double c = 0;
            const int rc = fn(ctx, w, 1, pose.data() + 7ll * d.kf0, sbv.data() + 9ll * d.kf0, extv.data() + 7ll * d.ext0, &tdv[w], nullptr,
                              nullptr, &c);
            cost[w] = rc == 0 && std::isfinite(c) ? c : nan;  // a failed trial evaluation rejects the step
        }
        if (any) {
            CK(cudaMemcpyAsync(S->hostCost.p, cost.data(), W * sizeof(double), cudaMemcpyHostToDevice, st));
            launchAddHost(S->B, S->hostH.p, S->hostG.p, S->hostCost.p, S->hostFlag.p, 1, st);
            ++launches;
        }
        launches += launchIterationParts(S->B, S->plan(), S->opt.refinement_steps, max_iterations, 0, nullptr, st, nullptr, nullptr,
                                         kIterDecide);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(S->ev1, st));
    S->timed = true;
    S->lastLaunches = launches;
    S->lastKey.clear();  // the next plain solve of this batch is not a repeat of a captured one
    return CGMLI_OK;
}

int cgmli_solver_last_timing(cgmli_solver* S, double* ms, int* launches) {
    if (!S) return fail(CGMLI_E_INVALID, "null solver");
    if (ms) *ms = S->lastMs;
    if (launches) *launches = S->lastLaunches;
    return CGMLI_OK;
}

// Elimination set (SlidingWindowManager.cpp:627-652): landmarks anchored at the
// victim, plus under OLD those observed at it; all their observations, the IMU
// factors touching the victim and the prior are consumed.  Every block a
// consumed factor touches joins the system, frozen calibration included
// (BackendProblem.hpp:75-80 with honorConstant=false).
int cgmli_solver_set_imu_merge_limits(cgmli_solver* S, double max_interval_s, int max_samples) {
    if (!S) return fail(CGMLI_E_INVALID, "null solver");
    if (!(max_interval_s > 0) || !std::isfinite(max_interval_s) || max_samples < 4)
        return fail(CGMLI_E_INVALID, "set_imu_merge_limits: interval must be positive and finite, samples >= 4");
    S->mergeMaxInterval = max_interval_s;
    S->mergeMaxSamples = max_samples;
    return CGMLI_OK;
}

int cgmli_solver_read_merged_imu(cgmli_solver* S, int window, int* state, cgmli_frozen_imu* imu) {
    if (!S || !S->haveMarg || !state) return fail(CGMLI_E_INVALID, "read_merged_imu: no marginalization recorded or null state");
    if (window < 0 || window >= (int)S->mergeState.size()) return fail(CGMLI_E_INVALID, "read_merged_imu: window index");
    CK(cudaSetDevice(S->device));
    *state = S->mergeState[window];
    const int job = S->mergeJob[window];
    if (job < 0) return CGMLI_OK;
    if (!S->mergeRead) {
        sizeTo(S->hMergeStatus, S->hMergeKf.size());
        CK(cudaMemcpyAsync(S->hMergeStatus.data(), S->mergeStatus.p, S->hMergeStatus.size() * sizeof(int), cudaMemcpyDeviceToHost,
                           S->stream));
        CK(cudaStreamSynchronize(S->stream));
        S->mergeRead = true;
    }
    if (S->hMergeStatus[job] != CGMLI_OK)
        return fail(S->hMergeStatus[job], S->hMergeStatus[job] == CGMLI_E_INVALID ? "merged IMU interval: invalid samples"
                                                                                   : "merged IMU interval: result not finite");
    if (imu) {
        CK(cudaMemcpyAsync(imu, S->mergeOut.p + job, sizeof(cgmli_frozen_imu), cudaMemcpyDeviceToHost, S->stream));
        CK(cudaStreamSynchronize(S->stream));
    }
    return CGMLI_OK;
}

// The Schur formation shared by the marginalization and the calibration
// information.  calib: every landmark eliminated, every IMU factor (and the
// prior when includePrior) consumed, poses and speed/biases as the nuisance
// block [0, nm), the calibration blocks as the separator; no victim.
static int marginalizeImpl(cgmli_solver* S, const int* victim_kf, int policy, bool calib, bool includePrior);

int cgmli_solver_marginalize(cgmli_solver* S, const int* victim_kf, int policy) {
    if (!S || S->win.empty() || !victim_kf) return fail(CGMLI_E_INVALID, "solver has no windows or no victim list");
    if (policy != CGMLI_MARGIN_OLD && policy != CGMLI_MARGIN_SECOND_NEW && policy != CGMLI_MARGIN_SECOND_NEW_IMU_MERGE)
        return fail(CGMLI_E_INVALID, "unknown marginalization policy");
    const int W = (int)S->win.size();
    for (int w = 0; w < W; ++w)
        if (victim_kf[w] < -1 || victim_kf[w] >= S->win[w].K) return fail(CGMLI_E_INVALID, "victim keyframe out of range");
    return marginalizeImpl(S, victim_kf, policy, false, false);
}

int cgmli_solver_calibration_information(cgmli_solver* S, int include_prior) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    return marginalizeImpl(S, nullptr, CGMLI_MARGIN_OLD, true, include_prior != 0);
}

int cgmli_solver_read_calibration_information(cgmli_solver* S, int window, int* size, int* num_blocks, int* block_kind,
                                              int* block_index, double* conditional, double* eigenvalues) {
    if (!S || !S->haveCalib) return fail(CGMLI_E_INVALID, "no calibration information recorded");
    if (window < 0 || window >= (int)S->margWin.size() || !size || !num_blocks) return fail(CGMLI_E_INVALID, "read_calibration_information: window index or null sizes");
    CK(cudaSetDevice(S->device));
    const MargWin& mw = S->margWin[window];
    int status = CGMLI_OK;
    CK(cudaMemcpyAsync(&status, S->margStatus.p + window, sizeof(int), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    if (status != CGMLI_OK)
        return fail(status, status == CGMLI_E_INDEFINITE ? "calibration information is indefinite"
                            : status == CGMLI_E_INVALID ? "no calibration Jacobians in the window's factors"
                                                        : "calibration information: invalid factor or non-finite result");
    *size = mw.m ? mw.nr : 0;
    *num_blocks = mw.m ? (int)S->sepKind[window].size() : 0;
    if (!mw.m) return CGMLI_OK;
    if (block_kind) std::copy(S->sepKind[window].begin(), S->sepKind[window].end(), block_kind);
    if (block_index) std::copy(S->sepIndex[window].begin(), S->sepIndex[window].end(), block_index);
    if (conditional)
        CK(cudaMemcpyAsync(conditional, S->calibCond.p + mw.sep0, (size_t)mw.nr * mw.nr * sizeof(double), cudaMemcpyDeviceToHost, S->stream));
    if (eigenvalues)
        CK(cudaMemcpyAsync(eigenvalues, S->calibEvals.p + 2 * mw.vec0, mw.nr * sizeof(double), cudaMemcpyDeviceToHost, S->stream));
    CK(cudaStreamSynchronize(S->stream));
    return CGMLI_OK;
}

static int marginalizeImpl(cgmli_solver* S, const int* victim_kf, int policy, bool calib, bool includePrior) {
    const int W = (int)S->win.size();
    CK(cudaSetDevice(S->device));
    const AllocStreamScope ordered(S->stream);
    // ---- phase A (parallel over windows): elimination set, columns, local maps
    struct Part {
        std::vector<MargElim> elims;   // col0 / obs0 window-local
        std::vector<int> cols, obsMap;
        std::vector<int> visCols;      // visual column -> marginalization column
        std::vector<int4> chunks;      // window-local eliminated landmarks and staged observations
        int maxNc = 0, status = CGMLI_OK;
        const char* why = "";
    };
    std::vector<MargWin> mwv(W);
    std::vector<Part> part(W);
    // IMU merge: per window the outcome and the two edges of the victim
    S->mergeState.assign(W, CGMLI_IMU_MERGE_NONE);
    S->mergeJob.assign(W, -1);
    std::vector<int2> mergeEdges(W, int2{-1, -1});
    S->sepKind.assign(W, {});
    S->sepIndex.assign(W, {});
    const HostBatch& hb = S->hb;
    HVec<int>& poseCol = S->hMargPoseCol;
    HVec<int>& sbCol = S->hMargSbCol;
    HVec<int>& extCol = S->hMargExtCol;
    HVec<int>& visPose = S->hMargVisPose;
    HVec<int>& visExt = S->hMargVisExt;
    // the staging arrays may still feed the previous marginalization's uploads
    if (S->margUploaded) CK(cudaEventSynchronize(S->margUploaded));
    sizeTo(poseCol, S->totalKf);
    sizeTo(sbCol, S->totalKf);
    sizeTo(extCol, S->totalExt);
    sizeTo(visPose, S->totalKf);
    sizeTo(visExt, S->totalExt);
    parallelFor(W, 0, [&](int w) {
        const WinDesc& d = S->win[w];
        const int v = calib ? -1 : victim_kf[w];
        MargWin& mw = mwv[w];
        Part& P = part[w];
        mw = MargWin{};
        mw.imu[0] = mw.imu[1] = -1;
        mw.tdCol = -1;
        mw.visTd = -1;
        mw.huber = d.huber;
        mw.hasPrior = (!calib || includePrior) && d.priorRank > 0;
        std::fill(&poseCol[d.kf0], &poseCol[d.kf0] + d.K, -1);
        std::fill(&sbCol[d.kf0], &sbCol[d.kf0] + d.K, -1);
        std::fill(&extCol[d.ext0], &extCol[d.ext0] + d.E, -1);
        std::fill(&visPose[d.kf0], &visPose[d.kf0] + d.K, -1);
        std::fill(&visExt[d.ext0], &visExt[d.ext0] + d.E, -1);
        if (v < 0 && !calib) return;
        std::vector<char> poseUsed(d.K, 0), sbUsed(d.K, 0), extUsed(d.E, 0);
        bool tdUsed = false;
        std::vector<int> elimLm;
        for (int q = 0; q < d.L; ++q) {
            const int g = d.lm0 + q, a = hb.lmKf[g] - d.kf0;
            bool e = calib ? hb.lmObsBegin[g + 1] > hb.lmObsBegin[g] : a == v;
            for (int f = hb.lmObsBegin[g]; f < hb.lmObsBegin[g + 1] && !e && !calib && policy == CGMLI_MARGIN_OLD; ++f)
                e = hb.obKf[f] - d.kf0 == v;
            if (!e) continue;
            elimLm.push_back(g);
            for (int f = hb.lmObsBegin[g]; f < hb.lmObsBegin[g + 1]; ++f) {
                poseUsed[a] = 1;
                poseUsed[hb.obKf[f] - d.kf0] = 1;
                extUsed[hb.camExt[hb.lmCam[g]] - d.ext0] = 1;
                extUsed[hb.camExt[hb.obCam[f]] - d.ext0] = 1;
                tdUsed = true;
            }
        }
        // SECOND_NEW with the IMU merge (SlidingWindowManager::prepareEviction,
        // SlidingWindowManager.cpp:275-310): when the victim has exactly its two IMU
        // edges left -> victim -> right, its speed/bias is not in the prior, and the
        // edges' samples are on the device, the edges are re-integrated into one
        // left -> right factor (mergeBodyImuRecords, BodyImuFactor.cpp:306-388) and
        // do not enter the Schur step; otherwise they are consumed by it.
        bool skipImu = false;
        if (policy == CGMLI_MARGIN_SECOND_NEW_IMU_MERGE) {
            int left = -1, right = -1, incident = 0;
            for (int i = 0; i < d.nImu; ++i) {
                const int k = hb.imuKf[d.imu0 + i] - d.kf0;
                if (k + 1 == v) { left = d.imu0 + i; ++incident; }
                else if (k == v) { right = d.imu0 + i; ++incident; }
            }
            bool sbInPrior = false;
            for (int b = 0; b < d.priorBlocks; ++b)
                sbInPrior = sbInPrior || (hb.priorKind[d.priorBlk0 + b] == CGMLI_PRIOR_SPEED_BIAS && hb.priorIndex[d.priorBlk0 + b] == d.kf0 + v);
            S->mergeState[w] = CGMLI_IMU_MERGE_BRIDGE;
            const auto hasSamples = [&](int q) { return q >= 0 && S->hImuRange[2 * q + 1] > S->hImuRange[2 * q]; };
            if (incident == 2 && left >= 0 && right >= 0 && !sbInPrior && S->haveImuSamples && hasSamples(left) && hasSamples(right)) {
                const int lb = S->hImuRange[2 * left], le = S->hImuRange[2 * left + 1];
                const int rb = S->hImuRange[2 * right], re = S->hImuRange[2 * right + 1];
                if (S->hImuT1[left] != S->hImuT0[right] || rb < lb || rb > le || re < le) {
                    P.status = CGMLI_E_INVALID;
                    P.why = "IMU merge: the victim's two edges must meet at its time and share one contiguous sample range";
                    return;
                }
                const long long span = S->hImuT1[right] - S->hImuT0[left];
                const bool suppressed = (double)span * 1e-9 > S->mergeMaxInterval;
                if (!suppressed && re - lb > S->mergeMaxSamples) {
                    P.status = CGMLI_E_LIMIT;
                    P.why = "IMU merge: merged interval exceeds the sample budget";
                    return;
                }
                S->mergeState[w] = suppressed ? CGMLI_IMU_MERGE_SUPPRESSED : CGMLI_IMU_MERGE_REINTEGRATED;
                mergeEdges[w] = int2{left, right};
                skipImu = true;
            }
        }
        if (calib) {
            mw.imuAll = 1;
            skipImu = true;
            for (int i = 0; i < d.nImu; ++i) {
                const int k = hb.imuKf[d.imu0 + i] - d.kf0;
                poseUsed[k] = poseUsed[k + 1] = sbUsed[k] = sbUsed[k + 1] = 1;
            }
        }
        int nImu = 0;
        for (int i = 0; i < d.nImu && !skipImu; ++i) {
            const int k = hb.imuKf[d.imu0 + i] - d.kf0;
            if (k != v && k + 1 != v) continue;
            if (nImu == 2) { P.status = CGMLI_E_LIMIT; P.why = "more than two IMU factors touch the victim keyframe"; return; }
            mw.imu[nImu++] = d.imu0 + i;
            poseUsed[k] = poseUsed[k + 1] = sbUsed[k] = sbUsed[k + 1] = 1;
        }
        for (int b = 0; b < (mw.hasPrior ? d.priorBlocks : 0); ++b) {
            const int kind = hb.priorKind[d.priorBlk0 + b], gi = hb.priorIndex[d.priorBlk0 + b];
            if (kind == CGMLI_PRIOR_POSE) poseUsed[gi - d.kf0] = 1;
            else if (kind == CGMLI_PRIOR_SPEED_BIAS) sbUsed[gi - d.kf0] = 1;
            else if (kind == CGMLI_PRIOR_EXTRINSIC) extUsed[gi - d.ext0] = 1;
            else tdUsed = true;
        }
        // columns: victim first, then the separator in block order (calibration
        // information: every pose and speed/bias first, the calibration as separator)
        int n = 0;
        auto sep = [&](int kind, int index) { S->sepKind[w].push_back(kind); S->sepIndex[w].push_back(index); };
        if (calib) {
            for (int k = 0; k < d.K; ++k) {
                if (poseUsed[k]) { poseCol[d.kf0 + k] = n; n += 6; }
                if (sbUsed[k]) { sbCol[d.kf0 + k] = n; n += 9; }
            }
            mw.nm = n;
        } else {
            if (poseUsed[v]) { poseCol[d.kf0 + v] = n; n += 6; }
            if (sbUsed[v]) { sbCol[d.kf0 + v] = n; n += 9; }
            mw.nm = n;
            for (int k = 0; k < d.K; ++k) {
                if (k == v) continue;
                if (poseUsed[k]) { poseCol[d.kf0 + k] = n; n += 6; sep(CGMLI_PRIOR_POSE, k); }
                if (sbUsed[k]) { sbCol[d.kf0 + k] = n; n += 9; sep(CGMLI_PRIOR_SPEED_BIAS, k); }
            }
        }
        for (int e = 0; e < d.E; ++e)
            if (extUsed[e]) { extCol[d.ext0 + e] = n; n += 6; sep(CGMLI_PRIOR_EXTRINSIC, e); }
        if (tdUsed && d.hasTd) { mw.tdCol = n; n += 1; sep(CGMLI_PRIOR_TIME_OFFSET, 0); }
        mw.m = n;
        mw.nr = n - mw.nm;
        if (mw.nr > kMargMaxSep) { P.status = CGMLI_E_LIMIT; P.why = "marginalization separator above 1024 columns"; return; }
        if (calib && mw.nm > kMargMaxSep) { P.status = CGMLI_E_LIMIT; P.why = "calibration information: more than 1024 nuisance columns"; return; }
        // visual columns (poses, extrinsics, td) in column order
        auto addVis = [&](int col, int width) {
            for (int c = 0; c < width; ++c) P.visCols.push_back(col + c);
            return (int)P.visCols.size() - width;
        };
        if (v >= 0 && poseUsed[v]) visPose[d.kf0 + v] = addVis(poseCol[d.kf0 + v], 6);
        for (int k = 0; k < d.K; ++k)
            if (k != v && poseUsed[k]) visPose[d.kf0 + k] = addVis(poseCol[d.kf0 + k], 6);
        for (int e = 0; e < d.E; ++e)
            if (extUsed[e]) visExt[d.ext0 + e] = addVis(extCol[d.ext0 + e], 6);
        if (mw.tdCol >= 0) mw.visTd = addVis(mw.tdCol, 1);
        mw.nv = (int)P.visCols.size();
        mw.rowsPath = mw.nv <= kRowsMaxN;
        // eliminated landmarks: local column blocks in order of first use; a block is
        // known by its first column, stamped with the landmark that last used it.  The
        // anchor's pose and extrinsic and td are first met in a landmark's first
        // observation, so later observations look up only the observer's blocks.
        int obsCount = 0;
        std::vector<int> stamp(n, -1), local(n, 0);
        long long nob = 0, colBound = 0;
        for (int g : elimLm) {
            const int k = hb.lmObsBegin[g + 1] - hb.lmObsBegin[g];
            nob += k;
            colBound += 13 + 12ll * k;
        }
        P.obsMap.resize(5 * nob);
        P.cols.resize(colBound);
        P.elims.reserve(elimLm.size());
        int* om = P.obsMap.data();
        int* cp = P.cols.data();
        for (int g : elimLm) {
            MargElim me{g, w, 0, (int)(cp - P.cols.data()), obsCount};
            auto localOf = [&](int start, int size) {
                if (start < 0) return -1;
                if (stamp[start] == g) return local[start];
                stamp[start] = g;
                local[start] = me.nc;
                for (int c = 0; c < size; ++c) *cp++ = start + c;
                me.nc += size;
                return me.nc - size;
            };
            const int a = hb.lmKf[g], ea = hb.camExt[hb.lmCam[g]];
            const int f0 = hb.lmObsBegin[g], f1 = hb.lmObsBegin[g + 1];
            int la = -1, lea = -1, ltd = -1;
            for (int f = f0; f < f1; ++f) {
                const int b = hb.obKf[f], eb = hb.camExt[hb.obCam[f]];
                if (f == f0) {
                    la = localOf(poseCol[a], 6);
                    om[1] = localOf(poseCol[b], 6);
                    lea = localOf(extCol[ea], 6);
                    om[3] = localOf(extCol[eb], 6);
                    ltd = localOf(mw.tdCol, 1);
                } else {
                    om[1] = localOf(poseCol[b], 6);
                    om[3] = localOf(extCol[eb], 6);
                }
                om[0] = la;
                om[2] = lea;
                om[4] = ltd;
                om += 5;
                ++obsCount;
            }
            if (me.nc > kMargMaxNc) {
                P.status = CGMLI_E_LIMIT;
                P.why = "eliminated landmark touches more than 200 marginalization columns";
                return;
            }
            P.maxNc = std::max(P.maxNc, me.nc);
            P.elims.push_back(me);
        }
        P.cols.resize(cp - P.cols.data());
        // dense-row chunks: 2 rows per observation and 1 per landmark, at most
        // 96 (72 above 192 visual columns)
        if (mw.rowsPath && !P.elims.empty()) {
            const int cap = margRowsCap(mw.nv);
            int4 ch{0, 0, 0, 0};
            for (int e = 0; e < (int)P.elims.size(); ++e) {
                const int nob = hb.lmObsBegin[P.elims[e].lm + 1] - hb.lmObsBegin[P.elims[e].lm];
                const int rows = 2 * (ch.w - ch.z) + (ch.y - ch.x);
                if (ch.y > ch.x && rows + 2 * nob + 1 > cap) {
                    P.chunks.push_back(ch);
                    ch = int4{e, e, ch.w, ch.w};
                }
                ch.y = e + 1;
                ch.w += nob;
            }
            P.chunks.push_back(ch);
        }
    });
    // ---- prefix sums over the windows, then one concatenation (parallel)
    std::vector<long long> colBase(W + 1, 0), obsBase(W + 1, 0);
    std::vector<int> elimBase(W + 1, 0), visBase(W + 1, 0), chunkBase(W + 1, 0);
    long long H0 = 0, sep0 = 0, vec0 = 0, x0 = 0;
    int maxNc = 0, maxNv = 0, numSlow = 0;
    for (int w = 0; w < W; ++w) {
        if (part[w].status != CGMLI_OK) return fail(part[w].status, part[w].why);
        MargWin& mw = mwv[w];
        mw.H0 = H0; mw.sep0 = sep0; mw.vec0 = vec0; mw.x0 = x0;
        mw.elim0 = elimBase[w];
        mw.nElim = (int)part[w].elims.size();
        elimBase[w + 1] = elimBase[w] + mw.nElim;
        mw.vis0 = visBase[w];
        visBase[w + 1] = visBase[w] + mw.nv;
        chunkBase[w + 1] = chunkBase[w] + (int)part[w].chunks.size();
        if (!part[w].chunks.empty()) maxNv = std::max(maxNv, mw.nv);
        if (!mw.rowsPath) numSlow += mw.nElim;
        colBase[w + 1] = colBase[w] + (long long)part[w].cols.size();
        obsBase[w + 1] = obsBase[w] + (long long)part[w].obsMap.size() / 5;
        maxNc = std::max(maxNc, part[w].maxNc);
        H0 += (long long)mw.m * mw.m;
        sep0 += (long long)mw.nr * mw.nr;
        vec0 += mw.m;
        x0 += 2ll * 15 * (mw.nr + 1);
    }
    HVec<MargElim>& elims = S->hMargElim;
    HVec<int>& cols = S->hMargCols;
    HVec<int>& obsMap = S->hMargObsMap;
    HVec<int>& visCol = S->hMargVisCol;
    HVec<int4>& chunks = S->hMargChunks;
    sizeTo(elims, elimBase[W]);
    sizeTo(cols, colBase[W]);
    sizeTo(obsMap, 5 * obsBase[W]);
    sizeTo(visCol, std::max(visBase[W], 1));
    sizeTo(chunks, std::max(chunkBase[W], 1));
    parallelFor(W, 0, [&](int w) {
        const Part& P = part[w];
        for (size_t e = 0; e < P.elims.size(); ++e) {
            MargElim me = P.elims[e];
            me.col0 += (int)colBase[w];
            me.obs0 += (int)obsBase[w];
            elims[elimBase[w] + e] = me;
        }
        std::copy(P.cols.begin(), P.cols.end(), cols.begin() + colBase[w]);
        std::copy(P.obsMap.begin(), P.obsMap.end(), obsMap.begin() + 5 * obsBase[w]);
        std::copy(P.visCols.begin(), P.visCols.end(), visCol.begin() + visBase[w]);
        for (size_t c = 0; c < P.chunks.size(); ++c) {
            const int4 ch = P.chunks[c];
            chunks[chunkBase[w] + c] = int4{ch.x + elimBase[w], ch.y + elimBase[w], ch.z + (int)obsBase[w], ch.w + (int)obsBase[w]};
        }
    });
    // items: runs of one window's chunks of about equal work (rows x upper tiles),
    // four per SM over the batch
    if (!S->numSMs) CK(cudaDeviceGetAttribute(&S->numSMs, cudaDevAttrMultiProcessorCount, S->device));
    auto chunkWork = [&](int w, const int4& ch) {
        const long long nb = (mwv[w].nv + 31) / 32;
        return (long long)(2 * (ch.w - ch.z) + (ch.y - ch.x)) * (nb * (nb + 1) / 2);
    };
    long long totalWork = 0;
    for (int w = 0; w < W; ++w)
        for (int c = chunkBase[w]; c < chunkBase[w + 1]; ++c) totalWork += chunkWork(w, chunks[c]);
    const long long target = std::max(1ll, totalWork / (4ll * std::max(S->numSMs, 1)));
    HVec<int4>& items = S->hMargItems;
    HVec<int>& slow = S->hMargSlow;
    items.clear();
    sizeTo(slow, std::max(numSlow, 1));
    numSlow = 0;
    for (int w = 0; w < W; ++w) {
        if (!mwv[w].rowsPath) {
            for (int e = elimBase[w]; e < elimBase[w + 1]; ++e) slow[numSlow++] = e;
            continue;
        }
        int c0 = chunkBase[w];
        long long work = 0;
        for (int c = chunkBase[w]; c < chunkBase[w + 1]; ++c) {
            const long long cw = chunkWork(w, chunks[c]);
            if (c > c0 && work + cw > target) {
                items.push_back(int4{w, c0, c, 0});
                c0 = c;
                work = 0;
            }
            work += cw;
        }
        if (chunkBase[w + 1] > c0) items.push_back(int4{w, c0, chunkBase[w + 1], 0});
    }
    const int numItems = (int)items.size();
    if (items.empty()) items.push_back(int4{0, 0, 0, 0});
    cudaStream_t st = S->stream;
    const size_t smem = margVisualSmemBytes(std::max(maxNc, 1));
    const size_t rowsSmem = margRowsSmemBytes(std::max(maxNv, 1));
    int maxNr = 1, maxFastNr = 0;
    for (const auto& mw : mwv) {
        maxNr = std::max(maxNr, mw.nr);
        maxFastNr = std::max(maxFastNr, mw.nr);
    }
    long long eigenSmem = 0, fastSmem = 0, triSmem = 0;
    CK(configureMarginalization(smem, rowsSmem, maxNr, maxFastNr, &eigenSmem, &fastSmem, &triSmem));
    S->hMargWin.assign(mwv.begin(), mwv.end());  // guarded by margUploaded like the other staging
    CK(S->dMargWin.upload(S->hMargWin, st));
    {
        auto& order = S->hMargOrder;
        sizeTo(order, mwv.size());
        for (size_t i = 0; i < mwv.size(); ++i) order[i] = (int)i;
        // the wider of the eliminated and kept blocks sets the CTA's work
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return std::max(mwv[a].nr, mwv[a].nm) > std::max(mwv[b].nr, mwv[b].nm); });
        CK(S->dMargOrder.reserve(std::max<size_t>(1, mwv.size())));
        CK(cudaMemcpyAsync(S->dMargOrder.p, order.data(), mwv.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    }
    CK(S->dMargElim.upload(elims, st));
    CK(S->margCols.upload(cols, st));
    CK(S->margObsMap.upload(obsMap, st));
    CK(S->margPoseCol.upload(poseCol, st));
    CK(S->margSbCol.upload(sbCol, st));
    CK(S->margExtCol.upload(extCol, st));
    CK(S->margVisCol.upload(visCol, st));
    CK(S->margVisPose.upload(visPose, st));
    CK(S->margVisExt.upload(visExt, st));
    CK(S->margChunks.upload(chunks, st));
    CK(S->margItems.upload(items, st));
    CK(S->margSlow.upload(slow, st));
    if (!S->margUploaded) CK(cudaEventCreateWithFlags(&S->margUploaded, cudaEventDisableTiming));
    CK(S->margH.reserve(H0)); CK(S->margB.reserve(vec0)); CK(S->margSepH.reserve(sep0)); CK(S->margSepV.reserve(sep0));
    CK(S->margSepB.reserve(vec0)); CK(S->margEvals.reserve(vec0)); CK(S->margA.reserve(sep0)); CK(S->margR0.reserve(vec0));
    CK(S->margX.reserve(x0)); CK(S->margMaxD.reserve(W)); CK(S->margStats.reserve(4ll * W));
    CK(S->margRank.reserve(W)); CK(S->margStatus.reserve(W)); CK(S->margFast.reserve(W));
    if (H0) CK(cudaMemsetAsync(S->margH.p, 0, H0 * sizeof(double), st));
    if (vec0) CK(cudaMemsetAsync(S->margB.p, 0, vec0 * sizeof(double), st));
    CK(cudaMemsetAsync(S->margMaxD.p, 0, W * sizeof(double), st));
    CK(cudaMemsetAsync(S->margStats.p, 0, 4ll * W * sizeof(double), st));
    CK(cudaMemsetAsync(S->margStatus.p, 0, W * sizeof(int), st));
    CK(cudaMemsetAsync(S->margRank.p, 0, W * sizeof(int), st));
    MargBatch& M = S->MB;
    M = MargBatch{};
    M.numWindows = W;
    M.numElim = (int)elims.size();
    M.eigenSmem = eigenSmem;
    M.fastSmem = fastSmem;
    M.triSmem = triSmem;
    M.win = S->dMargWin.p; M.bigFirst = S->dMargOrder.p; M.elim = S->dMargElim.p; M.cols = S->margCols.p; M.obsMap = S->margObsMap.p;
    M.poseCol = S->margPoseCol.p; M.sbCol = S->margSbCol.p; M.extCol = S->margExtCol.p;
    M.H = S->margH.p; M.b = S->margB.p; M.sepH = S->margSepH.p; M.sepV = S->margSepV.p; M.sepB = S->margSepB.p;
    M.evals = S->margEvals.p; M.A = S->margA.p; M.r0 = S->margR0.p; M.X = S->margX.p;
    M.maxD = S->margMaxD.p; M.stats = S->margStats.p; M.rank = S->margRank.p; M.status = S->margStatus.p;
    M.fast = S->margFast.p;
    M.rows = S->keyRows.p;
    M.visCol = S->margVisCol.p; M.visPose = S->margVisPose.p; M.visExt = S->margVisExt.p;
    M.chunks = S->margChunks.p;
    M.items = S->margItems.p;
    M.numItems = numItems;
    M.rowsSmem = (long long)rowsSmem;
    M.slowElim = S->margSlow.p;
    M.numSlowElim = numSlow;
    S->margWin = mwv;
    S->margSepTotal = sep0;
    S->margVecTotal = vec0;
    S->margCached = false;
    // merged IMU intervals: one job per reintegrated window
    S->hMergeRange.clear(); S->hMergeKf.clear(); S->hMergeT0.clear(); S->hMergeT1.clear();
    for (int w = 0; w < W; ++w) {
        if (S->mergeState[w] != CGMLI_IMU_MERGE_REINTEGRATED) continue;
        const int left = mergeEdges[w].x, right = mergeEdges[w].y;
        S->mergeJob[w] = (int)S->hMergeKf.size();
        S->hMergeRange.push_back(S->hImuRange[2 * left]);
        S->hMergeRange.push_back(S->hImuRange[2 * right + 1]);
        S->hMergeT0.push_back(S->hImuT0[left]);
        S->hMergeT1.push_back(S->hImuT1[right]);
        S->hMergeKf.push_back(hb.imuKf[left]);
    }
    const int jobs = (int)S->hMergeKf.size();
    S->mergeRead = false;
    if (jobs) {
        CK(S->mergeRange.upload(S->hMergeRange, st)); CK(S->mergeKf.upload(S->hMergeKf, st));
        CK(S->mergeT0.upload(S->hMergeT0, st)); CK(S->mergeT1.upload(S->hMergeT1, st));
        CK(S->mergeStatus.reserve(jobs)); CK(S->mergeFlag.reserve(jobs)); CK(S->mergeOut.reserve(jobs));
    }
    int calibMaxNx = 0;
    if (calib) {
        // per window 2 nx^2 + 2 nx nc + 4 nc^2 doubles of work; results at the
        // separator offsets (nc^2) and 2x the vector offsets (eigenvalues)
        sizeTo(S->hCalibWork0, W);
        long long work = 0;
        for (int w = 0; w < W; ++w) {
            const long long nx = mwv[w].nm, nc = mwv[w].nr;
            calibMaxNx = std::max(calibMaxNx, (int)nx);
            S->hCalibWork0[w] = work;
            work += 2 * nx * nx + 2 * nx * nc + 4 * nc * nc;
        }
        CK(S->calibWork0.upload(S->hCalibWork0, st));
        CK(S->calibWork.reserve(std::max(work, 1ll)));
        CK(S->calibCond.reserve(std::max(sep0, 1ll)));
        CK(S->calibEvals.reserve(std::max(2 * vec0, 1ll)));
    }
    CK(cudaEventRecord(S->margUploaded, st));
    CK(cudaEventRecord(S->ev0, st));
    if (calib)
        S->lastLaunches =
            launchCalibration(S->B, M, smem, S->calibWork.p, S->calibWork0.p, S->calibCond.p, S->calibEvals.p, calibMaxNx, st);
    else
        S->lastLaunches = launchMarginalization(S->B, M, smem, st);
    if (jobs) {
        // at the left keyframe's accepted bias, as BodyImuCost builds the merged factor
        ImuLaunch L{};
        L.prm = S->imuParams;
        L.times = S->imuTimes.p; L.readings = S->imuReadings.p; L.sampleOffset = S->imuSampleOffset;
        L.ranges = S->mergeRange.p; L.t0s = S->mergeT0.p; L.t1s = S->mergeT1.p;
        L.out = S->mergeOut.p; L.status = S->mergeStatus.p; L.biases = nullptr;
        L.sb = S->sb[0].p; L.kf = S->mergeKf.p; L.force = 1;
        L.scratch = nullptr; L.refreshed = S->mergeFlag.p;
        CK(launchImuPreintegration(L, jobs, st));
        S->lastLaunches += 1;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(S->ev1, st));
    S->timed = true;
    // the formation buffers now hold one or the other result
    S->haveMarg = !calib;
    S->haveCalib = calib;
    return CGMLI_OK;
}

int cgmli_solver_read_prior(cgmli_solver* S, int window, int* rank, int* cols, int* num_blocks, int* block_kind, int* block_index,
                            double* reference, double* A, double* r0, double* formation) {
    if (!S || !S->haveMarg) return fail(CGMLI_E_INVALID, "no marginalization recorded");
    if (window < 0 || window >= (int)S->margWin.size()) return fail(CGMLI_E_INVALID, "window index");
    if (!rank || !cols || !num_blocks) return fail(CGMLI_E_INVALID, "null size outputs");
    CK(cudaSetDevice(S->device));
    const int W = (int)S->margWin.size();
    if (!S->margCached) {
        CK(cudaStreamSynchronize(S->stream));
        S->readTiming();
        HostBatch& hb = S->hb;
        sizeTo(S->hMargA, S->margSepTotal);
        sizeTo(S->hMargR0, S->margVecTotal);
        sizeTo(S->hMargStats, 4ll * W);
        sizeTo(S->hMargRank, W);
        sizeTo(S->hMargStatus, W);
        cudaStream_t st = S->stream;
        if (S->margSepTotal)
            CK(cudaMemcpyAsync(S->hMargA.data(), S->margA.p, S->margSepTotal * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (S->margVecTotal)
            CK(cudaMemcpyAsync(S->hMargR0.data(), S->margR0.p, S->margVecTotal * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(S->hMargStats.data(), S->margStats.p, 4ll * W * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(S->hMargRank.data(), S->margRank.p, W * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(S->hMargStatus.data(), S->margStatus.p, W * sizeof(int), cudaMemcpyDeviceToHost, st));
        // the states the separator references come from (the accepted states)
        CK(cudaMemcpyAsync(hb.pose.data(), S->pose[0].p, hb.pose.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hb.sb.data(), S->sb[0].p, hb.sb.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hb.ext.data(), S->ext[0].p, hb.ext.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hb.td.data(), S->td[0].p, hb.td.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        S->margCached = true;
    }
    const MargWin& mw = S->margWin[window];
    const WinDesc& d = S->win[window];
    const int status = S->hMargStatus[window], rk = S->hMargRank[window];
    if (status != CGMLI_OK) return fail(status, "window marginalization failed (invalid factor or indefinite information)");
    *rank = mw.m ? rk : 0;
    *cols = mw.m ? mw.nr : 0;
    *num_blocks = mw.m ? (int)S->sepKind[window].size() : 0;
    if (!mw.m) return CGMLI_OK;
    const auto& kinds = S->sepKind[window];
    const auto& idx = S->sepIndex[window];
    if (block_kind) std::copy(kinds.begin(), kinds.end(), block_kind);
    if (block_index) std::copy(idx.begin(), idx.end(), block_index);
    if (reference) {
        const HostBatch& hb = S->hb;
        double* out = reference;
        for (size_t b = 0; b < kinds.size(); ++b) {
            const double* src = kinds[b] == CGMLI_PRIOR_POSE ? &hb.pose[7ull * (d.kf0 + idx[b])]
                                : kinds[b] == CGMLI_PRIOR_SPEED_BIAS ? &hb.sb[9ull * (d.kf0 + idx[b])]
                                : kinds[b] == CGMLI_PRIOR_EXTRINSIC ? &hb.ext[7ull * (d.ext0 + idx[b])] : &hb.td[window];
            const int n = ambientOf(kinds[b]);
            std::copy(src, src + n, out);
            out += n;
        }
    }
    if (A && rk) std::copy(&S->hMargA[mw.sep0], &S->hMargA[mw.sep0] + (size_t)rk * mw.nr, A);
    if (r0 && rk) std::copy(&S->hMargR0[mw.vec0], &S->hMargR0[mw.vec0] + rk, r0);
    if (formation) std::copy(&S->hMargStats[4ll * window], &S->hMargStats[4ll * window] + 4, formation);
    return CGMLI_OK;
}

// ---- dense helpers: one process-wide workspace on the current device, serialized
namespace {
struct DenseWorkspace {
    std::mutex mu;
    int device = -1;
    cudaStream_t stream = nullptr;
    DArray<double> H, work, evals, U, rhs, projected, solution;
    DArray<int> status;
};
DenseWorkspace g_dense;

int denseBegin(int n) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (g_dense.device != dev) {
        if (g_dense.stream) cudaStreamDestroy(g_dense.stream);
        g_dense.stream = nullptr;
        DArray<double>* a[] = {&g_dense.H, &g_dense.work, &g_dense.evals, &g_dense.U, &g_dense.rhs, &g_dense.projected, &g_dense.solution};
        for (auto* x : a) x->release();
        g_dense.status.release();
        CK(cudaStreamCreateWithFlags(&g_dense.stream, cudaStreamNonBlocking));
        g_dense.device = dev;
    }
    CK(g_dense.status.reserve(1));
    CK(cudaMemsetAsync(g_dense.status.p, 0, sizeof(int), g_dense.stream));
    (void)n;
    return CGMLI_OK;
}
// eigen-decomposition of H into g_dense.evals (ascending) / g_dense.U
int denseDecompose(const double* H, int n) {
    const size_t nn = (size_t)n * n;
    CK(g_dense.H.reserve(nn)); CK(g_dense.work.reserve(2 * nn)); CK(g_dense.evals.reserve(2ull * n)); CK(g_dense.U.reserve(nn));
    CK(cudaMemcpyAsync(g_dense.H.p, H, nn * sizeof(double), cudaMemcpyHostToDevice, g_dense.stream));
    launchDenseEigen(g_dense.H.p, n, g_dense.work.p, g_dense.evals.p, g_dense.U.p, g_dense.status.p, g_dense.stream);
    CK(cudaGetLastError());
    return CGMLI_OK;
}
int denseStatus() {
    int st = 0;
    CK(cudaMemcpyAsync(&st, g_dense.status.p, sizeof(int), cudaMemcpyDeviceToHost, g_dense.stream));
    CK(cudaStreamSynchronize(g_dense.stream));
    return st;
}
}  // namespace

int cgmli_marg_eigen(const double* H, int n, double* eigenvalues, double* eigenvectors) {
    if (!H || !eigenvalues || !eigenvectors || n < 1) return fail(CGMLI_E_INVALID, "eigen: null buffers or n < 1");
    if (n > kMargMaxSep) return fail(CGMLI_E_LIMIT, "eigen: n above 1024");
    std::lock_guard<std::mutex> lock(g_dense.mu);
    int r = denseBegin(n);
    if (r != CGMLI_OK || (r = denseDecompose(H, n)) != CGMLI_OK) return r;
    CK(cudaMemcpyAsync(eigenvalues, g_dense.evals.p, n * sizeof(double), cudaMemcpyDeviceToHost, g_dense.stream));
    CK(cudaMemcpyAsync(eigenvectors, g_dense.U.p, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToHost, g_dense.stream));
    const int st = denseStatus();
    if (st == CGMLI_E_CUDA) return st;
    if (st != CGMLI_OK) return fail(st, "eigen: non-finite eigenvalue");
    return CGMLI_OK;
}

int cgmli_marg_psd_solve(const double* H, const double* rhs, int n, int columns, double absolute_cutoff, double relative_cutoff,
                         double* solution) {
    if (!H || !rhs || !solution || n < 1) return fail(CGMLI_E_INVALID, "psd_solve: null buffers or n < 1");
    if (columns < 1 || columns > 4001) return fail(CGMLI_E_INVALID, "psd_solve: columns outside 1..4001");
    if (n > kMargMaxSep) return fail(CGMLI_E_LIMIT, "psd_solve: n above 1024");
    std::lock_guard<std::mutex> lock(g_dense.mu);
    int r = denseBegin(n);
    if (r != CGMLI_OK || (r = denseDecompose(H, n)) != CGMLI_OK) return r;
    const size_t count = (size_t)n * columns;
    CK(g_dense.rhs.reserve(count)); CK(g_dense.projected.reserve(count)); CK(g_dense.solution.reserve(count));
    CK(cudaMemcpyAsync(g_dense.rhs.p, rhs, count * sizeof(double), cudaMemcpyHostToDevice, g_dense.stream));
    launchDensePsd(g_dense.evals.p, g_dense.U.p, g_dense.rhs.p, n, columns, absolute_cutoff, relative_cutoff, g_dense.projected.p,
                   g_dense.solution.p, g_dense.status.p, g_dense.stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(solution, g_dense.solution.p, count * sizeof(double), cudaMemcpyDeviceToHost, g_dense.stream));
    const int st = denseStatus();
    if (st != CGMLI_OK) return fail(st, "psd_solve: indefinite or non-finite information");
    return CGMLI_OK;
}

int cgmli_marg_subtract(const double* coupling, const double* solution, int nm, int nr, double* H, double* g) {
    if (!coupling || !solution || !H || !g) return fail(CGMLI_E_INVALID, "subtract: null buffers");
    if (nm < 1 || nr < 1 || nm > 4000 || nr > 4000) return fail(CGMLI_E_INVALID, "subtract: sizes outside 1..4000");
    std::lock_guard<std::mutex> lock(g_dense.mu);
    int r = denseBegin(nr);
    if (r != CGMLI_OK) return r;
    const size_t nc = (size_t)nm * nr, ns = (size_t)nm * (nr + 1), nh = (size_t)nr * nr;
    CK(g_dense.U.reserve(nc)); CK(g_dense.rhs.reserve(ns)); CK(g_dense.solution.reserve(nh + nr));
    CK(cudaMemcpyAsync(g_dense.U.p, coupling, nc * sizeof(double), cudaMemcpyHostToDevice, g_dense.stream));
    CK(cudaMemcpyAsync(g_dense.rhs.p, solution, ns * sizeof(double), cudaMemcpyHostToDevice, g_dense.stream));
    CK(cudaMemcpyAsync(g_dense.solution.p, H, nh * sizeof(double), cudaMemcpyHostToDevice, g_dense.stream));
    CK(cudaMemcpyAsync(g_dense.solution.p + nh, g, nr * sizeof(double), cudaMemcpyHostToDevice, g_dense.stream));
    launchDenseSubtract(g_dense.U.p, g_dense.rhs.p, nm, nr, g_dense.solution.p, g_dense.stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(H, g_dense.solution.p, nh * sizeof(double), cudaMemcpyDeviceToHost, g_dense.stream));
    CK(cudaMemcpyAsync(g, g_dense.solution.p + nh, nr * sizeof(double), cudaMemcpyDeviceToHost, g_dense.stream));
    CK(cudaStreamSynchronize(g_dense.stream));
    return CGMLI_OK;
}

}  // extern "C"

// Message of a failure reported by another translation unit of the library.
int cgmli::setLastError(int code, const char* message) { return fail(code, message); }
