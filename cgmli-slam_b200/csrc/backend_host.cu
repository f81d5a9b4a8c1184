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
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cgmli_backend.h"
#include "backend_internal.h"

namespace cgmli {
size_t linearizeSmemBytes(int maxNs);
size_t factorSmemBytes(int maxNr);
cudaError_t configureKernels(size_t linSmem, size_t facSmem);
int schurRowsPerChunk(int Npc);
int launchIteration(const DevBatch& B, const LaunchPlan& P, int refinement, int maxIterations, int probe, double* Sdebug,
                    cudaStream_t s, LaunchHook hook, void* ctx);
int launchLmInit(const DevBatch& B, double lambda0, cudaStream_t s);
size_t margVisualSmemBytes(int maxNc);
cudaError_t configureMarginalization(size_t visualSmem, int maxNr, long long* eigenSmem);
int launchMarginalization(const DevBatch& B, const MargBatch& M, size_t visualSmem, cudaStream_t s);
void launchDenseEigen(const double* H, int n, double* work, double* evals, double* evecs, int* status, cudaStream_t s);
void launchDensePsd(const double* evals, const double* U, const double* rhs, int n, int columns, double absCut, double relCut,
                    double* projected, double* solution, int* status, cudaStream_t s);
void launchDenseSubtract(const double* coupling, const double* solution, int nm, int nr, double* Hg, cudaStream_t s);
}  // namespace cgmli

using namespace cgmli;

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

// Grow-only device array (src/common/CudaArray.hpp:10-39 keeps the same policy).
template <class T>
struct DArray {
    T* p = nullptr;
    size_t cap = 0;
    cudaError_t reserve(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) cap = n;
        return e;
    }
    cudaError_t upload(const std::vector<T>& v, cudaStream_t s) {
        cudaError_t e = reserve(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    }
    void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};
}  // namespace

struct cgmli_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cgmli_solver_options opt{};
    // topology (host copies)
    std::vector<WinDesc> win;
    std::vector<int4> runs;       // {window, first tile, end tile, -}
    std::vector<int2> tiles;      // {first landmark, end landmark} (device order)
    std::vector<int> lmPerm;      // device landmark -> landmark index within its window
    std::vector<int4> pairChunks; // {window, first key-ordered observation, end, -}
    std::vector<int4> schurChunks;// {window, first landmark, end landmark, -}
    int maxNpc = 0, maxNr = 0, maxNs = 1;
    size_t linSmem = 0, facSmem = 0;
    int totalKf = 0, totalExt = 0, totalCam = 0, totalLm = 0, totalObs = 0, totalImu = 0;
    // device arrays
    DArray<WinDesc> dWin;
    DArray<WinLM> dLm;
    DArray<int4> dRuns;
    DArray<int2> dTiles;
    DArray<int4> dPairChunks, dSchurChunks;
    DArray<int> obLm, keyOrder;
    DArray<double> sch;
    DArray<double> camR, camT;
    DArray<int> camExt;
    DArray<int> lmWin, lmKf, lmCam, lmObsBegin, lmNs, lmNx, lmSupp0, supp, lmGroup;
    DArray<long long> lmC0;
    DArray<double> lmBearing, lmVel, lmTime, lmC, lmD, lmG, lmCost, lmDelta, lmPred, lmTrial, lmMaxInc;
    DArray<int> lmValid, lmTrialValid;
    DArray<int> obKf, obKfl, obCam, obSlot, obXslot;
    DArray<double> obBearing, obP, obVel, obTime;
    DArray<double> pose[2], sb[2], ext[2], td[2], rho[2];
    DArray<double> imu;
    DArray<int> imuKf;
    DArray<int> priorKind, priorIndex, priorCol, priorOff;
    DArray<double> priorA, priorR0, priorRef;
    DArray<double> Hret, gret, costRet, trialRet, acc, dr, rhs, Sglob, imuScratch, priorScratch, predState, out, Sdebug;
    DArray<int> retValid, solveStatus;
    DevBatch B{};
    double lastMs = 0;
    int lastLaunches = 0;
    // host copies of the topology (device order, global indices) for elimination sets
    std::vector<int> hLmKf, hLmCam, hLmObsBegin, hObKf, hObCam, hCamExt, hImuKf, hPriorKind, hPriorIndex;
    // marginalization
    std::vector<MargWin> margWin;
    std::vector<std::vector<int>> sepKind, sepIndex;  // separator blocks per window (window-local index)
    DArray<MargWin> dMargWin;
    DArray<MargElim> dMargElim;
    DArray<int> margCols, margObsMap, margPoseCol, margSbCol, margExtCol, margRank, margStatus;
    DArray<double> margH, margB, margSepH, margSepV, margSepB, margEvals, margA, margR0, margX, margMaxD, margStats;
    MargBatch MB{};
    bool haveMarg = false;
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
    LaunchPlan plan() const {
        LaunchPlan P{};
        P.runs = dRuns.p; P.tiles = dTiles.p;
        P.pairChunks = dPairChunks.p; P.numPairChunks = (int)pairChunks.size();
        P.schurChunks = dSchurChunks.p; P.numSchurChunks = (int)schurChunks.size();
        P.linSmem = linSmem; P.facSmem = facSmem; P.maxNs = maxNs;
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
        DArray<double>* dbl[] = {&camR, &camT, &lmBearing, &lmVel, &lmTime, &lmC, &lmD, &lmG, &lmCost, &lmDelta, &lmPred, &lmTrial,
                                 &lmMaxInc, &obBearing, &obP, &obVel, &obTime, &pose[0], &pose[1], &sb[0], &sb[1], &ext[0], &ext[1],
                                 &td[0], &td[1], &rho[0], &rho[1], &imu, &priorA, &priorR0, &priorRef, &Hret, &gret, &costRet,
                                 &trialRet, &acc, &dr, &rhs, &Sglob, &imuScratch, &priorScratch, &predState, &out, &Sdebug};
        for (auto* a : dbl) a->release();
        DArray<int>* ints[] = {&camExt, &lmWin, &lmKf, &lmCam, &lmObsBegin, &lmNs, &lmSupp0, &supp, &lmValid, &lmTrialValid, &obKf,
                               &obKfl, &obCam, &obSlot, &imuKf, &priorKind, &priorIndex, &priorCol, &priorOff, &retValid,
                               &solveStatus, &lmGroup, &lmNx, &obXslot};
        for (auto* a : ints) a->release();
        lmC0.release(); dWin.release(); dLm.release(); dRuns.release(); dTiles.release();
        dPairChunks.release(); dSchurChunks.release(); obLm.release(); keyOrder.release(); sch.release();
        snapPose.release(); snapSb.release(); snapExt.release(); snapTd.release(); snapRho.release();
        dMargWin.release(); dMargElim.release();
        DArray<int>* mi[] = {&margCols, &margObsMap, &margPoseCol, &margSbCol, &margExtCol, &margRank, &margStatus};
        for (auto* a : mi) a->release();
        DArray<double>* md[] = {&margH, &margB, &margSepH, &margSepV, &margSepB, &margEvals, &margA, &margR0, &margX, &margMaxD, &margStats};
        for (auto* a : md) a->release();
        for (auto e : evPool) cudaEventDestroy(e);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {
int tangentOf(int kind) { return kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 6; }
int ambientOf(int kind) { return kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 7; }

int validateWindow(const cgmli_window& w, int index) {
    char buf[256];
    auto bad = [&](const char* what) {
        std::snprintf(buf, sizeof buf, "window %d: %s", index, what);
        return fail(CGMLI_E_INVALID, buf);
    };
    if (w.num_keyframes < 1 || w.num_cameras < 1 || w.num_extrinsics < 1 || w.num_landmarks < 0 || w.num_observations < 0 ||
        w.num_imu < 0 || w.prior_rank < 0)
        return bad("negative or empty sizes");
    if (!w.poses || !w.speed_bias || !w.extrinsics || (w.num_landmarks && !w.rho) || !w.cam_R || !w.cam_t || !w.cam_ext)
        return bad("missing state or rig arrays");
    if (w.num_landmarks && (!w.lm_anchor_kf || !w.lm_anchor_cam || !w.lm_obs_begin || !w.lm_anchor_bearing))
        return bad("missing landmark arrays");
    if (w.num_observations && (!w.obs_kf || !w.obs_cam || !w.obs_bearing || !w.obs_P)) return bad("missing observation arrays");
    if (w.num_imu && (!w.imu || !w.imu_kf)) return bad("missing IMU arrays");
    if (w.estimate_td && !w.td) return bad("estimate_td requires a td value");
    for (int c = 0; c < w.num_cameras; ++c)
        if (w.cam_ext[c] < 0 || w.cam_ext[c] >= w.num_extrinsics) return bad("camera extrinsic index out of range");
    if (w.num_landmarks && (w.lm_obs_begin[0] != 0 || w.lm_obs_begin[w.num_landmarks] != w.num_observations))
        return bad("landmark observation ranges do not cover the observations");
    for (int l = 0; l < w.num_landmarks; ++l) {
        if (w.lm_obs_begin[l + 1] < w.lm_obs_begin[l]) return bad("landmark observation ranges not sorted");
        if (w.lm_obs_begin[l + 1] - w.lm_obs_begin[l] > kMaxTrackChunk) return bad("more than 32 observations of one landmark");
        if (w.lm_anchor_kf[l] < 0 || w.lm_anchor_kf[l] >= w.num_keyframes) return bad("anchor keyframe out of range");
        if (w.lm_anchor_cam[l] < 0 || w.lm_anchor_cam[l] >= w.num_cameras) return bad("anchor camera out of range");
    }
    for (int f = 0; f < w.num_observations; ++f) {
        if (w.obs_kf[f] < 0 || w.obs_kf[f] >= w.num_keyframes) return bad("observer keyframe out of range");
        if (w.obs_cam[f] < 0 || w.obs_cam[f] >= w.num_cameras) return bad("observer camera out of range");
    }
    for (int i = 0; i < w.num_imu; ++i)
        if (w.imu_kf[i] < 0 || w.imu_kf[i] + 1 >= w.num_keyframes) return bad("IMU keyframe out of range");
    if (w.prior_rank > 0) {
        if (!w.prior_block_kind || !w.prior_block_index || !w.prior_ref || !w.prior_A || !w.prior_r0 || w.prior_num_blocks < 1)
            return bad("missing prior arrays");
        for (int b = 0; b < w.prior_num_blocks; ++b) {
            const int k = w.prior_block_kind[b], i = w.prior_block_index[b];
            if (k < 0 || k > 3) return bad("prior block kind");
            if ((k <= 1 && (i < 0 || i >= w.num_keyframes)) || (k == 2 && (i < 0 || i >= w.num_extrinsics)) || (k == 3 && !w.td))
                return bad("prior block index");
        }
    }
    const int ncal = (w.estimate_extrinsics ? 6 * w.num_extrinsics : 0) + (w.estimate_td ? 1 : 0);
    if (6 * w.num_keyframes + ncal > 400) return fail(CGMLI_E_LIMIT, "window visual dimension above 400");
    return CGMLI_OK;
}
}  // namespace

extern "C" {

const char* cgmli_last_error(void) { return g_error.c_str(); }

void cgmli_default_options(cgmli_solver_options* o) {
    o->precision = CGMLI_PRECISION_FP64;
    o->refinement_steps = 0;
    o->initial_lambda = 1e-4;
    o->slabs_per_window = 0;
    o->threads_per_block = 0;
}

int cgmli_solver_create(int device, const cgmli_solver_options* options, cgmli_solver** out) {
    if (!out) return fail(CGMLI_E_INVALID, "null output handle");
    *out = nullptr;
    if (options) {
        if (options->precision != CGMLI_PRECISION_FP64 && options->precision != CGMLI_PRECISION_MIXED)
            return fail(CGMLI_E_INVALID, "unknown precision");
        if (options->precision == CGMLI_PRECISION_MIXED) return fail(CGMLI_E_UNSUPPORTED, "mixed precision is not built");
        if (options->refinement_steps < 0 || options->refinement_steps > 2) return fail(CGMLI_E_INVALID, "refinement_steps outside 0..2");
        if (!(options->initial_lambda > 0)) return fail(CGMLI_E_INVALID, "initial_lambda must be positive");
        if (options->slabs_per_window != 0 || options->threads_per_block != 0)
            return fail(CGMLI_E_UNSUPPORTED, "slabs_per_window / threads_per_block are reserved and must be 0");
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
    for (int i = 0; i < count; ++i) {
        const int st = validateWindow(windows[i], i);
        if (st != CGMLI_OK) return st;
    }
    CK(cudaSetDevice(S->device));
    cudaStream_t st = S->stream;
    S->win.assign(count, WinDesc{});
    S->haveSnapshot = false;
    S->runs.clear(); S->tiles.clear(); S->lmPerm.clear(); S->pairChunks.clear(); S->schurChunks.clear();
    int kf = 0, ex = 0, cam = 0, lm = 0, ob = 0, im = 0, pblk = 0, vec = 0, groups = 0;
    long long dense = 0, acc = 0, schOff = 0, pA = 0, pR = 0, pRef = 0, imuS = 0, priS = 0, cOff = 0;
    std::vector<int> obLmv, keyOrderv;
    S->maxNpc = 0; S->maxNr = 0;
    std::vector<double> camR, camT, lmBearing, lmVel, lmTime, obBearing, obP, obVel, obTime;
    std::vector<int> camExt, lmWin, lmKf, lmCam, lmObsBegin, lmNs, lmNx, lmSupp0, supp, lmGroup, obKf, obKfl, obCam, obSlot, obXslot, imuKf;
    std::vector<long long> lmC0;
    std::vector<int> priorKind, priorIndex, priorCol, priorOff;
    std::vector<double> priorA, priorR0, priorRef, imuData;
    std::vector<double> pose, sbv, extv, tdv, rhov;
    long long totalLm = 0;
    for (int i = 0; i < count; ++i) totalLm += windows[i].num_landmarks;
    // landmarks per warp run: enough runs to fill the GPU, long runs for large batches
    const long long targetRuns = 148ll * 6 * 4;
    const int runLen = (int)std::max<long long>(4, std::min<long long>(64, totalLm / targetRuns));
    for (int i = 0; i < count; ++i) {
        const auto& w = windows[i];
        WinDesc& d = S->win[i];
        d.K = w.num_keyframes; d.E = w.num_extrinsics; d.C = w.num_cameras; d.L = w.num_landmarks; d.F = w.num_observations;
        d.nImu = w.num_imu;
        d.estExt = w.estimate_extrinsics != 0; d.estTd = w.estimate_td != 0 && w.td; d.hasTd = w.td != nullptr;
        d.ncalib = (d.estExt ? 6 * d.E : 0) + (d.estTd ? 1 : 0);
        d.Npc = 6 * d.K + d.ncalib;
        d.Nr = 15 * d.K + d.ncalib;
        d.kf0 = kf; d.ext0 = ex; d.cam0 = cam; d.lm0 = lm; d.obs0 = ob; d.imu0 = im;
        d.vec0 = vec; d.dense0 = dense; d.acc0 = acc; d.sch0 = schOff;
        d.huber = w.huber_scale; d.minInv = w.min_inverse_distance;
        S->maxNpc = std::max(S->maxNpc, d.Npc);
        S->maxNr = std::max(S->maxNr, d.Nr);
        vec += d.Nr;
        dense += (long long)d.Nr * d.Nr;
        acc += (long long)d.Npc * (d.Npc + 1) / 2 + 3ll * d.Npc;
        schOff += (long long)d.Npc * (d.Npc + 1) / 2;
        pose.insert(pose.end(), w.poses, w.poses + 7 * d.K);
        sbv.insert(sbv.end(), w.speed_bias, w.speed_bias + 9 * d.K);
        extv.insert(extv.end(), w.extrinsics, w.extrinsics + 7 * d.E);
        tdv.push_back(w.td ? *w.td : 0.0);
        camR.insert(camR.end(), w.cam_R, w.cam_R + 9 * d.C);
        camT.insert(camT.end(), w.cam_t, w.cam_t + 3 * d.C);
        for (int c = 0; c < d.C; ++c) camExt.push_back(ex + w.cam_ext[c]);
        // support of each landmark: keyframes (anchor first, then observers
        // ascending), then the extrinsic blocks its observations touch (the
        // anchor camera's first, then the others ascending) when estimated
        std::vector<std::vector<int>> sup(d.L);
        std::vector<int> nkf(d.L), nx(d.L);
        for (int l = 0; l < d.L; ++l) {
            const int a = w.lm_anchor_kf[l];
            std::vector<int> kfs{a}, exs;
            if (d.estExt) exs.push_back(w.cam_ext[w.lm_anchor_cam[l]]);
            for (int f = w.lm_obs_begin[l]; f < w.lm_obs_begin[l + 1]; ++f) {
                if (std::find(kfs.begin(), kfs.end(), w.obs_kf[f]) == kfs.end()) kfs.push_back(w.obs_kf[f]);
                const int e = w.cam_ext[w.obs_cam[f]];
                if (d.estExt && std::find(exs.begin(), exs.end(), e) == exs.end()) exs.push_back(e);
            }
            std::sort(kfs.begin() + 1, kfs.end());
            if (exs.size() > 1) std::sort(exs.begin() + 1, exs.end());
            if ((int)kfs.size() > kMaxSupport) return fail(CGMLI_E_LIMIT, "landmark support above 64 keyframes");
            nkf[l] = (int)kfs.size();
            nx[l] = (int)exs.size();
            sup[l] = kfs;
            sup[l].push_back(-1);  // separator keeps keyframe and extrinsic lists distinct in the sort key
            sup[l].insert(sup[l].end(), exs.begin(), exs.end());
        }
        // device order: landmarks sorted by support (stable), so that equal supports are adjacent
        std::vector<int> order(d.L);
        for (int l = 0; l < d.L; ++l) order[l] = l;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            if (sup[x].size() != sup[y].size()) return sup[x].size() < sup[y].size();
            return sup[x] < sup[y];
        });
        int tileObs = 0, runTiles = 0, runLms = 0;
        for (int q = 0; q < d.L; ++q) {
            const int l = order[q];
            const auto& key = sup[l];
            const int ns = 6 * (nkf[l] + nx[l]) + (d.estTd ? 1 : 0);
            const bool newGroup = q == 0 || sup[order[q - 1]] != key;
            if (newGroup) ++groups;
            const int b = w.lm_obs_begin[l], e = w.lm_obs_begin[l + 1], nobs = e - b;
            // run / tile bookkeeping: runs end at group boundaries once long enough
            if (q == 0 || (runLms >= runLen && newGroup) || runLms >= 4 * runLen) {
                if (!S->runs.empty() && S->runs.back().z < 0) S->runs.back().z = (int)S->tiles.size();
                if (!S->tiles.empty() && S->tiles.back().y < 0) S->tiles.back().y = lm + q;
                S->runs.push_back(make_int4(i, (int)S->tiles.size(), -1, 0));
                S->tiles.push_back(make_int2(lm + q, -1));
                tileObs = 0; runLms = 0; runTiles = 1;
            } else if (tileObs + nobs > kMaxTrackChunk) {
                S->tiles.back().y = lm + q;
                S->tiles.push_back(make_int2(lm + q, -1));
                tileObs = 0; ++runTiles;
            }
            tileObs += nobs;
            ++runLms;
            S->lmPerm.push_back(l);
            lmGroup.push_back(groups);
            lmWin.push_back(i);
            lmKf.push_back(kf + w.lm_anchor_kf[l]);
            lmCam.push_back(cam + w.lm_anchor_cam[l]);
            lmObsBegin.push_back(ob + (int)obKf.size() - ob);
            for (int k = 0; k < 3; ++k) lmBearing.push_back(w.lm_anchor_bearing[3 * l + k]);
            for (int k = 0; k < 3; ++k) lmVel.push_back(w.lm_anchor_velocity ? w.lm_anchor_velocity[3 * l + k] : 0.0);
            lmTime.push_back(w.lm_anchor_time ? w.lm_anchor_time[l] : 0.0);
            lmNs.push_back(nkf[l]);
            lmNx.push_back(nx[l]);
            lmSupp0.push_back((int)supp.size());
            supp.insert(supp.end(), key.begin(), key.begin() + nkf[l]);
            supp.insert(supp.end(), key.begin() + nkf[l] + 1, key.end());
            lmC0.push_back(cOff);
            cOff += ns;
            rhov.push_back(w.rho[l]);
            // observations of the landmark sorted by observer keyframe (slot order)
            std::vector<int> fo(nobs);
            for (int k = 0; k < nobs; ++k) fo[k] = b + k;
            std::stable_sort(fo.begin(), fo.end(), [&](int x, int y) { return w.obs_kf[x] < w.obs_kf[y]; });
            for (int f : fo) {
                obLmv.push_back(lm + q);
                obKf.push_back(kf + w.obs_kf[f]);
                obKfl.push_back(w.obs_kf[f]);
                obCam.push_back(cam + w.obs_cam[f]);
                obSlot.push_back((int)(std::find(key.begin(), key.begin() + nkf[l], w.obs_kf[f]) - key.begin()));
                {
                    const auto xb = key.begin() + nkf[l] + 1;
                    obXslot.push_back(d.estExt ? (int)(std::find(xb, key.end(), w.cam_ext[w.obs_cam[f]]) - xb) : 0);
                }
                for (int k = 0; k < 3; ++k) obBearing.push_back(w.obs_bearing[3 * f + k]);
                for (int k = 0; k < 6; ++k) obP.push_back(w.obs_P[6 * f + k]);
                for (int k = 0; k < 3; ++k) obVel.push_back(w.obs_velocity ? w.obs_velocity[3 * f + k] : 0.0);
                obTime.push_back(w.obs_time ? w.obs_time[f] : 0.0);
            }
        }
        if (d.L) {
            S->tiles.back().y = lm + d.L;
            S->runs.back().z = (int)S->tiles.size();
        }
        // observations of the window in key order (anchor kf, observer kf, anchor ext,
        // observer ext): the J^T J pass sums the observations of one key together
        {
            const int F = (int)obKf.size() - ob;  // device observations of this window: [ob, ob + F)
            auto keyOf = [&](int g) {
                const int l = obLmv[g] - lm;  // device landmark within the window
                const int a = lmKf[lm + l] - kf, b = obKf[g] - kf;
                const int ea = camExt[lmCam[lm + l]] - ex, eb = camExt[obCam[g]] - ex;
                return ((long long)(a * d.K + b) * d.E + ea) * d.E + eb;
            };
            const long long buckets = (long long)d.K * d.K * d.E * d.E;
            std::vector<int> order(F);
            if (buckets <= 4ll * F + 4096) {
                std::vector<int> count(buckets + 1, 0);
                for (int g = 0; g < F; ++g) ++count[keyOf(ob + g) + 1];
                for (long long k = 0; k < buckets; ++k) count[k + 1] += count[k];
                for (int g = 0; g < F; ++g) order[count[keyOf(ob + g)]++] = ob + g;
            } else {
                std::vector<std::pair<long long, int>> kv(F);
                for (int g = 0; g < F; ++g) kv[g] = {keyOf(ob + g), ob + g};
                std::sort(kv.begin(), kv.end());
                for (int g = 0; g < F; ++g) order[g] = kv[g].second;
            }
            const int base = (int)keyOrderv.size();
            keyOrderv.insert(keyOrderv.end(), order.begin(), order.end());
            for (int c0 = 0; c0 < F; c0 += 32)
                S->pairChunks.push_back(make_int4(i, base + c0, base + std::min(F, c0 + 32), 0));
            const int rows = schurRowsPerChunk(d.Npc);
            for (int l0 = 0; l0 < d.L; l0 += rows)
                S->schurChunks.push_back(make_int4(i, lm + l0, lm + std::min(d.L, l0 + rows), 0));
        }
        (void)runTiles;
        // IMU
        for (int q = 0; q < d.nImu; ++q) {
            const double* raw = reinterpret_cast<const double*>(&w.imu[q]);
            imuData.insert(imuData.end(), raw, raw + sizeof(cgmli_frozen_imu) / sizeof(double));
            imuKf.push_back(kf + w.imu_kf[q]);
        }
        d.imuScratch0 = imuS;
        imuS += 465ll * d.nImu;
        // prior
        d.priorRank = w.prior_rank;
        d.priorBlk0 = pblk;
        d.priorBlocks = w.prior_rank > 0 ? w.prior_num_blocks : 0;
        int cols = 0, amb = 0;
        for (int b2 = 0; b2 < d.priorBlocks; ++b2) {
            const int kind = w.prior_block_kind[b2], idx = w.prior_block_index[b2];
            priorKind.push_back(kind);
            int gidx = idx, col = -1;
            if (kind == CGMLI_PRIOR_POSE) { gidx = kf + idx; col = 15 * idx; }
            else if (kind == CGMLI_PRIOR_SPEED_BIAS) { gidx = kf + idx; col = 15 * idx + 6; }
            else if (kind == CGMLI_PRIOR_EXTRINSIC) { gidx = ex + idx; col = d.estExt ? 15 * d.K + 6 * idx : -1; }
            else { gidx = i; col = d.estTd ? 15 * d.K + (d.estExt ? 6 * d.E : 0) : -1; }
            priorIndex.push_back(gidx);
            priorCol.push_back(col);
            priorOff.push_back(cols);
            cols += tangentOf(kind);
            amb += ambientOf(kind);
        }
        d.priorCols = cols;
        d.priorA0 = pA; d.priorR00 = pR; d.priorRef0 = pRef;
        if (d.priorRank > 0) {
            priorA.insert(priorA.end(), w.prior_A, w.prior_A + (long long)d.priorRank * cols);
            priorR0.insert(priorR0.end(), w.prior_r0, w.prior_r0 + d.priorRank);
            priorRef.insert(priorRef.end(), w.prior_ref, w.prior_ref + amb);
        }
        pA += (long long)d.priorRank * cols;
        pR += d.priorRank;
        pRef += d.priorRank > 0 ? amb : 0;
        pblk += d.priorBlocks;
        d.priorScratch0 = priS;
        priS += d.priorRank > 0 ? (long long)cols * 7 + d.priorRank + (long long)d.priorRank * cols : 0;
        kf += d.K; ex += d.E; cam += d.C; lm += d.L; ob += d.F; im += d.nImu;
    }
    lmObsBegin.push_back((int)obKf.size());
    S->totalKf = kf; S->totalExt = ex; S->totalCam = cam; S->totalLm = lm; S->totalObs = ob; S->totalImu = im;
    S->maxNs = 1;
    for (size_t q = 0; q < lmNs.size(); ++q)
        S->maxNs = std::max(S->maxNs, 6 * (lmNs[q] + lmNx[q]) + (S->win[lmWin[q]].estTd ? 1 : 0));
    S->linSmem = linearizeSmemBytes(S->maxNs);
    S->facSmem = factorSmemBytes(S->maxNr);
    CK(configureKernels(S->linSmem, S->facSmem));
    CK(S->dWin.upload(S->win, st));
    CK(S->dLm.reserve(count));
    CK(S->dRuns.upload(S->runs, st));
    CK(S->dTiles.upload(S->tiles, st));
    CK(S->camR.upload(camR, st)); CK(S->camT.upload(camT, st)); CK(S->camExt.upload(camExt, st));
    CK(S->lmWin.upload(lmWin, st)); CK(S->lmKf.upload(lmKf, st)); CK(S->lmCam.upload(lmCam, st));
    CK(S->lmObsBegin.upload(lmObsBegin, st)); CK(S->lmNs.upload(lmNs, st)); CK(S->lmSupp0.upload(lmSupp0, st));
    CK(S->supp.upload(supp, st)); CK(S->lmC0.upload(lmC0, st)); CK(S->lmGroup.upload(lmGroup, st));
    CK(S->lmNx.upload(lmNx, st)); CK(S->obXslot.upload(obXslot, st));
    CK(S->lmBearing.upload(lmBearing, st)); CK(S->lmVel.upload(lmVel, st)); CK(S->lmTime.upload(lmTime, st));
    CK(S->obKf.upload(obKf, st)); CK(S->obKfl.upload(obKfl, st)); CK(S->obCam.upload(obCam, st)); CK(S->obSlot.upload(obSlot, st));
    CK(S->obBearing.upload(obBearing, st)); CK(S->obP.upload(obP, st)); CK(S->obVel.upload(obVel, st));
    CK(S->obTime.upload(obTime, st));
    CK(S->pose[0].upload(pose, st)); CK(S->sb[0].upload(sbv, st)); CK(S->ext[0].upload(extv, st));
    CK(S->td[0].upload(tdv, st)); CK(S->rho[0].upload(rhov, st));
    CK(S->pose[1].reserve(pose.size())); CK(S->sb[1].reserve(sbv.size())); CK(S->ext[1].reserve(extv.size()));
    CK(S->td[1].reserve(tdv.size())); CK(S->rho[1].reserve(rhov.size()));
    CK(S->imu.upload(imuData, st)); CK(S->imuKf.upload(imuKf, st));
    CK(S->priorKind.upload(priorKind, st)); CK(S->priorIndex.upload(priorIndex, st));
    CK(S->priorCol.upload(priorCol, st)); CK(S->priorOff.upload(priorOff, st));
    CK(S->priorA.upload(priorA, st)); CK(S->priorR0.upload(priorR0, st)); CK(S->priorRef.upload(priorRef, st));
    CK(S->lmC.reserve(cOff)); CK(S->lmD.reserve(lm)); CK(S->lmG.reserve(lm)); CK(S->lmCost.reserve(lm));
    CK(S->lmDelta.reserve(lm)); CK(S->lmPred.reserve(lm)); CK(S->lmTrial.reserve(lm)); CK(S->lmMaxInc.reserve(lm));
    CK(S->lmValid.reserve(lm)); CK(S->lmTrialValid.reserve(lm));
    CK(S->Hret.reserve(dense)); CK(S->Sglob.reserve(dense)); CK(S->gret.reserve(vec)); CK(S->dr.reserve(vec)); CK(S->rhs.reserve(vec));
    CK(S->acc.reserve(acc)); CK(S->sch.reserve(schOff)); CK(S->imuScratch.reserve(imuS)); CK(S->priorScratch.reserve(priS));
    CK(S->obLm.upload(obLmv, st)); CK(S->keyOrder.upload(keyOrderv, st));
    CK(S->dPairChunks.upload(S->pairChunks, st)); CK(S->dSchurChunks.upload(S->schurChunks, st));
    CK(S->costRet.reserve(count)); CK(S->trialRet.reserve(count)); CK(S->retValid.reserve(count));
    CK(S->predState.reserve(count)); CK(S->solveStatus.reserve(count)); CK(S->out.reserve(4ll * count));
    DevBatch& B = S->B;
    B = DevBatch{};
    B.numWindows = count; B.numLandmarks = lm; B.numObs = ob; B.numKf = kf; B.numExt = ex; B.numCam = cam; B.numImu = im;
    B.numRuns = (int)S->runs.size();
    B.win = S->dWin.p; B.lm = S->dLm.p;
    B.camR = S->camR.p; B.camT = S->camT.p; B.camExt = S->camExt.p;
    B.lmWin = S->lmWin.p; B.lmKf = S->lmKf.p; B.lmCam = S->lmCam.p; B.lmObsBegin = S->lmObsBegin.p;
    B.lmBearing = S->lmBearing.p; B.lmVel = S->lmVel.p; B.lmTime = S->lmTime.p;
    B.lmNs = S->lmNs.p; B.lmNx = S->lmNx.p; B.lmSupp0 = S->lmSupp0.p; B.supp = S->supp.p; B.lmC0 = S->lmC0.p;
    B.lmGroup = S->lmGroup.p; B.obXslot = S->obXslot.p;
    B.lmC = S->lmC.p; B.lmD = S->lmD.p; B.lmG = S->lmG.p; B.lmCost = S->lmCost.p; B.lmValid = S->lmValid.p;
    B.lmDelta = S->lmDelta.p; B.lmPred = S->lmPred.p; B.lmTrial = S->lmTrial.p; B.lmMaxInc = S->lmMaxInc.p;
    B.lmTrialValid = S->lmTrialValid.p;
    B.obKf = S->obKf.p; B.obKfl = S->obKfl.p; B.obCam = S->obCam.p; B.obSlot = S->obSlot.p;
    B.obLm = S->obLm.p; B.keyOrder = S->keyOrder.p;
    B.obBearing = S->obBearing.p; B.obP = S->obP.p; B.obVel = S->obVel.p; B.obTime = S->obTime.p;
    for (int k = 0; k < 2; ++k) {
        B.pose[k] = S->pose[k].p; B.sb[k] = S->sb[k].p; B.ext[k] = S->ext[k].p; B.td[k] = S->td[k].p; B.rho[k] = S->rho[k].p;
    }
    B.imu = S->imu.p; B.imuKf = S->imuKf.p;
    B.priorKind = S->priorKind.p; B.priorIndex = S->priorIndex.p; B.priorCol = S->priorCol.p; B.priorOff = S->priorOff.p;
    B.priorA = S->priorA.p; B.priorR0 = S->priorR0.p; B.priorRef = S->priorRef.p;
    B.Hret = S->Hret.p; B.gret = S->gret.p; B.costRet = S->costRet.p; B.trialRet = S->trialRet.p; B.retValid = S->retValid.p;
    B.acc = S->acc.p; B.sch = S->sch.p; B.dr = S->dr.p; B.rhs = S->rhs.p; B.Sglob = S->Sglob.p;
    B.imuScratch = S->imuScratch.p; B.priorScratch = S->priorScratch.p; B.predState = S->predState.p;
    B.solveStatus = S->solveStatus.p; B.out = S->out.p;
    S->hLmKf = lmKf; S->hLmCam = lmCam; S->hLmObsBegin = lmObsBegin; S->hObKf = obKf; S->hObCam = obCam;
    S->hCamExt = camExt; S->hImuKf = imuKf; S->hPriorKind = priorKind; S->hPriorIndex = priorIndex;
    S->haveMarg = false;
    CK(cudaMemsetAsync(S->costRet.p, 0, count * sizeof(double), st));
    CK(cudaMemsetAsync(S->trialRet.p, 0, count * sizeof(double), st));
    CK(cudaStreamSynchronize(st));
    return CGMLI_OK;
}

int cgmli_solver_upload_states(cgmli_solver* S, const cgmli_window* windows, int count) {
    if (!S || !windows || count != (int)S->win.size()) return fail(CGMLI_E_INVALID, "window count differs from the configured batch");
    CK(cudaSetDevice(S->device));
    for (int i = 0; i < count; ++i) {
        const WinDesc& d = S->win[i];
        const auto& w = windows[i];
        if (w.num_keyframes != d.K || w.num_landmarks != d.L || w.num_extrinsics != d.E)
            return fail(CGMLI_E_INVALID, "state upload with a different topology");
        CK(cudaMemcpyAsync(S->pose[0].p + 7ll * d.kf0, w.poses, 7ll * d.K * sizeof(double), cudaMemcpyHostToDevice, S->stream));
        CK(cudaMemcpyAsync(S->sb[0].p + 9ll * d.kf0, w.speed_bias, 9ll * d.K * sizeof(double), cudaMemcpyHostToDevice, S->stream));
        CK(cudaMemcpyAsync(S->ext[0].p + 7ll * d.ext0, w.extrinsics, 7ll * d.E * sizeof(double), cudaMemcpyHostToDevice, S->stream));
        if (w.td) CK(cudaMemcpyAsync(S->td[0].p + i, w.td, sizeof(double), cudaMemcpyHostToDevice, S->stream));
        if (d.L) {
            // device order is sorted by support; lmPerm maps it back to the caller's order
            std::vector<double> r(d.L);
            for (int q = 0; q < d.L; ++q) r[q] = w.rho[S->lmPerm[d.lm0 + q]];
            CK(cudaMemcpy(S->rho[0].p + d.lm0, r.data(), d.L * sizeof(double), cudaMemcpyHostToDevice));
        }
    }
    return CGMLI_OK;
}

static void profileHook(void* ctx, int kind, int phase) {
    auto* S = static_cast<cgmli_solver*>(ctx);
    cudaEvent_t e = S->nextEvent();
    if (phase == 0) S->evUsed.push_back({kind, (int)S->evNext - 1});
    cudaEventRecord(e, S->stream);
}

static int runIterations(cgmli_solver* S, int iterations, int probe, double* Sdebug) {
    cudaStream_t st = S->stream;
    if (S->profile) S->collectKernelTimes();
    CK(cudaEventRecord(S->ev0, st));
    int launches = launchLmInit(S->B, S->opt.initial_lambda, st);
    for (int it = 0; it < iterations; ++it)
        launches += launchIteration(S->B, S->plan(), S->opt.refinement_steps, iterations, probe, Sdebug, st,
                                    S->profile ? profileHook : nullptr, S);
    CK(cudaGetLastError());
    CK(cudaEventRecord(S->ev1, st));
    S->lastLaunches = launches;
    return CGMLI_OK;
}

int cgmli_solver_solve(cgmli_solver* S, int max_iterations) {
    if (!S || S->win.empty()) return fail(CGMLI_E_INVALID, "solver has no windows");
    if (max_iterations < 1) return fail(CGMLI_E_INVALID, "max_iterations < 1");
    CK(cudaSetDevice(S->device));
    return runIterations(S, max_iterations, 0, nullptr);
}

int cgmli_solver_synchronize(cgmli_solver* S) {
    if (!S) return fail(CGMLI_E_INVALID, "null solver");
    CK(cudaStreamSynchronize(S->stream));
    float ms = 0;
    if (cudaEventElapsedTime(&ms, S->ev0, S->ev1) == cudaSuccess) S->lastMs = ms;
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
            for (int q = 0; q < d.L; ++q) increment[d.Nr + S->lmPerm[d.lm0 + q]] = r[q];
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
    if (rhs) {
        // rhs is recomputed from the accumulators (it equals -(g_r - B_v))
        std::vector<double> g(d.Nr), accv((size_t)d.Npc * (d.Npc + 1) / 2 + 3 * d.Npc);
        CK(cudaMemcpy(g.data(), S->gret.p + d.vec0, d.Nr * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(accv.data(), S->acc.p + d.acc0, accv.size() * sizeof(double), cudaMemcpyDeviceToHost));
        const size_t nS = (size_t)d.Npc * (d.Npc + 1) / 2;
        for (int i = 0; i < d.Nr; ++i) {
            double v = g[i];
            int p = -1;
            if (i >= 15 * d.K) p = 6 * d.K + (i - 15 * d.K);
            else if (i % 15 < 6) p = 6 * (i / 15) + i % 15;
            if (p >= 0) v += accv[nS + d.Npc + p] - accv[nS + 2 * d.Npc + p];
            rhs[i] = -v;
        }
    }
    return CGMLI_OK;
}

int cgmli_solver_read_states(cgmli_solver* S, cgmli_window* windows, int count) {
    if (!S || !windows || count != (int)S->win.size()) return fail(CGMLI_E_INVALID, "window count differs from the configured batch");
    CK(cudaSetDevice(S->device));
    CK(cudaStreamSynchronize(S->stream));
    for (int i = 0; i < count; ++i) {
        const WinDesc& d = S->win[i];
        auto& w = windows[i];
        CK(cudaMemcpy(w.poses, S->pose[0].p + 7ll * d.kf0, 7ll * d.K * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(w.speed_bias, S->sb[0].p + 9ll * d.kf0, 9ll * d.K * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(w.extrinsics, S->ext[0].p + 7ll * d.ext0, 7ll * d.E * sizeof(double), cudaMemcpyDeviceToHost));
        if (w.td) CK(cudaMemcpy(w.td, S->td[0].p + i, sizeof(double), cudaMemcpyDeviceToHost));
        if (d.L) {
            std::vector<double> r(d.L);
            CK(cudaMemcpy(r.data(), S->rho[0].p + d.lm0, d.L * sizeof(double), cudaMemcpyDeviceToHost));
            for (int q = 0; q < d.L; ++q) w.rho[S->lmPerm[d.lm0 + q]] = r[q];
        }
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
int cgmli_solver_marginalize(cgmli_solver* S, const int* victim_kf, int policy) {
    if (!S || S->win.empty() || !victim_kf) return fail(CGMLI_E_INVALID, "solver has no windows or no victim list");
    if (policy != CGMLI_MARGIN_OLD && policy != CGMLI_MARGIN_SECOND_NEW) return fail(CGMLI_E_INVALID, "unknown marginalization policy");
    const int W = (int)S->win.size();
    for (int w = 0; w < W; ++w)
        if (victim_kf[w] < -1 || victim_kf[w] >= S->win[w].K) return fail(CGMLI_E_INVALID, "victim keyframe out of range");
    CK(cudaSetDevice(S->device));
    std::vector<MargWin> mwv(W);
    std::vector<MargElim> elims;
    std::vector<int> cols, obsMap;
    std::vector<int> poseCol(S->totalKf, -1), sbCol(S->totalKf, -1), extCol(S->totalExt, -1);
    S->sepKind.assign(W, {});
    S->sepIndex.assign(W, {});
    long long H0 = 0, sep0 = 0, vec0 = 0, x0 = 0;
    int maxNc = 0;
    for (int w = 0; w < W; ++w) {
        const WinDesc& d = S->win[w];
        const int v = victim_kf[w];
        MargWin& mw = mwv[w];
        mw = MargWin{};
        mw.imu[0] = mw.imu[1] = -1;
        mw.tdCol = -1;
        mw.huber = d.huber;
        mw.H0 = H0; mw.sep0 = sep0; mw.vec0 = vec0; mw.x0 = x0;
        mw.elim0 = (int)elims.size();
        if (v < 0) continue;
        std::vector<char> poseUsed(d.K, 0), sbUsed(d.K, 0), extUsed(d.E, 0);
        bool tdUsed = false;
        std::vector<int> elimLm;
        for (int q = 0; q < d.L; ++q) {
            const int g = d.lm0 + q, a = S->hLmKf[g] - d.kf0;
            bool e = a == v;
            for (int f = S->hLmObsBegin[g]; f < S->hLmObsBegin[g + 1] && !e && policy == CGMLI_MARGIN_OLD; ++f)
                e = S->hObKf[f] - d.kf0 == v;
            if (!e) continue;
            elimLm.push_back(g);
            for (int f = S->hLmObsBegin[g]; f < S->hLmObsBegin[g + 1]; ++f) {
                poseUsed[a] = 1;
                poseUsed[S->hObKf[f] - d.kf0] = 1;
                extUsed[S->hCamExt[S->hLmCam[g]] - d.ext0] = 1;
                extUsed[S->hCamExt[S->hObCam[f]] - d.ext0] = 1;
                tdUsed = true;
            }
        }
        int nImu = 0;
        for (int i = 0; i < d.nImu; ++i) {
            const int k = S->hImuKf[d.imu0 + i] - d.kf0;
            if (k != v && k + 1 != v) continue;
            if (nImu == 2) return fail(CGMLI_E_LIMIT, "more than two IMU factors touch the victim keyframe");
            mw.imu[nImu++] = d.imu0 + i;
            poseUsed[k] = poseUsed[k + 1] = sbUsed[k] = sbUsed[k + 1] = 1;
        }
        for (int b = 0; b < d.priorBlocks; ++b) {
            const int kind = S->hPriorKind[d.priorBlk0 + b], gi = S->hPriorIndex[d.priorBlk0 + b];
            if (kind == CGMLI_PRIOR_POSE) poseUsed[gi - d.kf0] = 1;
            else if (kind == CGMLI_PRIOR_SPEED_BIAS) sbUsed[gi - d.kf0] = 1;
            else if (kind == CGMLI_PRIOR_EXTRINSIC) extUsed[gi - d.ext0] = 1;
            else tdUsed = true;
        }
        // columns: victim first, then the separator in block order
        int n = 0;
        if (poseUsed[v]) { poseCol[d.kf0 + v] = n; n += 6; }
        if (sbUsed[v]) { sbCol[d.kf0 + v] = n; n += 9; }
        mw.nm = n;
        auto sep = [&](int kind, int index) { S->sepKind[w].push_back(kind); S->sepIndex[w].push_back(index); };
        for (int k = 0; k < d.K; ++k) {
            if (k == v) continue;
            if (poseUsed[k]) { poseCol[d.kf0 + k] = n; n += 6; sep(CGMLI_PRIOR_POSE, k); }
            if (sbUsed[k]) { sbCol[d.kf0 + k] = n; n += 9; sep(CGMLI_PRIOR_SPEED_BIAS, k); }
        }
        for (int e = 0; e < d.E; ++e)
            if (extUsed[e]) { extCol[d.ext0 + e] = n; n += 6; sep(CGMLI_PRIOR_EXTRINSIC, e); }
        if (tdUsed && d.hasTd) { mw.tdCol = n; n += 1; sep(CGMLI_PRIOR_TIME_OFFSET, 0); }
        mw.m = n;
        mw.nr = n - mw.nm;
        if (mw.nr > kMargMaxSep) return fail(CGMLI_E_LIMIT, "marginalization separator above 1024 columns");
        // eliminated landmarks: local column blocks in order of first use
        for (int g : elimLm) {
            MargElim me{g, w, 0, (int)cols.size(), (int)(obsMap.size() / 5)};
            std::vector<int> blkStart, blkLocal;
            auto localOf = [&](int start, int size) {
                if (start < 0) return -1;
                for (size_t i = 0; i < blkStart.size(); ++i)
                    if (blkStart[i] == start) return blkLocal[i];
                blkStart.push_back(start);
                blkLocal.push_back(me.nc);
                for (int c = 0; c < size; ++c) cols.push_back(start + c);
                me.nc += size;
                return blkLocal.back();
            };
            const int a = S->hLmKf[g], ea = S->hCamExt[S->hLmCam[g]];
            for (int f = S->hLmObsBegin[g]; f < S->hLmObsBegin[g + 1]; ++f) {
                const int b = S->hObKf[f], eb = S->hCamExt[S->hObCam[f]];
                obsMap.push_back(localOf(poseCol[a], 6));
                obsMap.push_back(localOf(poseCol[b], 6));
                obsMap.push_back(localOf(extCol[ea], 6));
                obsMap.push_back(localOf(extCol[eb], 6));
                obsMap.push_back(mw.tdCol >= 0 ? localOf(mw.tdCol, 1) : -1);
            }
            if (me.nc > kMargMaxNc) return fail(CGMLI_E_LIMIT, "eliminated landmark touches more than 200 marginalization columns");
            maxNc = std::max(maxNc, me.nc);
            elims.push_back(me);
        }
        mw.nElim = (int)elims.size() - mw.elim0;
        H0 += (long long)mw.m * mw.m;
        sep0 += (long long)mw.nr * mw.nr;
        vec0 += mw.m;
        x0 += 2ll * 15 * (mw.nr + 1);
    }
    cudaStream_t st = S->stream;
    const size_t smem = margVisualSmemBytes(std::max(maxNc, 1));
    int maxNr = 1;
    for (const auto& mw : mwv) maxNr = std::max(maxNr, mw.nr);
    long long eigenSmem = 0;
    CK(configureMarginalization(smem, maxNr, &eigenSmem));
    CK(S->dMargWin.upload(mwv, st));
    CK(S->dMargElim.upload(elims, st));
    CK(S->margCols.upload(cols, st));
    CK(S->margObsMap.upload(obsMap, st));
    CK(S->margPoseCol.upload(poseCol, st));
    CK(S->margSbCol.upload(sbCol, st));
    CK(S->margExtCol.upload(extCol, st));
    CK(S->margH.reserve(H0)); CK(S->margB.reserve(vec0)); CK(S->margSepH.reserve(sep0)); CK(S->margSepV.reserve(sep0));
    CK(S->margSepB.reserve(vec0)); CK(S->margEvals.reserve(vec0)); CK(S->margA.reserve(sep0)); CK(S->margR0.reserve(vec0));
    CK(S->margX.reserve(x0)); CK(S->margMaxD.reserve(W)); CK(S->margStats.reserve(4ll * W));
    CK(S->margRank.reserve(W)); CK(S->margStatus.reserve(W));
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
    M.win = S->dMargWin.p; M.elim = S->dMargElim.p; M.cols = S->margCols.p; M.obsMap = S->margObsMap.p;
    M.poseCol = S->margPoseCol.p; M.sbCol = S->margSbCol.p; M.extCol = S->margExtCol.p;
    M.H = S->margH.p; M.b = S->margB.p; M.sepH = S->margSepH.p; M.sepV = S->margSepV.p; M.sepB = S->margSepB.p;
    M.evals = S->margEvals.p; M.A = S->margA.p; M.r0 = S->margR0.p; M.X = S->margX.p;
    M.maxD = S->margMaxD.p; M.stats = S->margStats.p; M.rank = S->margRank.p; M.status = S->margStatus.p;
    S->margWin = mwv;
    CK(cudaEventRecord(S->ev0, st));
    S->lastLaunches = launchMarginalization(S->B, M, smem, st);
    CK(cudaGetLastError());
    CK(cudaEventRecord(S->ev1, st));
    S->haveMarg = true;
    return CGMLI_OK;
}

int cgmli_solver_read_prior(cgmli_solver* S, int window, int* rank, int* cols, int* num_blocks, int* block_kind, int* block_index,
                            double* reference, double* A, double* r0, double* formation) {
    if (!S || !S->haveMarg) return fail(CGMLI_E_INVALID, "no marginalization recorded");
    if (window < 0 || window >= (int)S->margWin.size()) return fail(CGMLI_E_INVALID, "window index");
    if (!rank || !cols || !num_blocks) return fail(CGMLI_E_INVALID, "null size outputs");
    CK(cudaSetDevice(S->device));
    CK(cudaStreamSynchronize(S->stream));
    float ms = 0;
    if (cudaEventElapsedTime(&ms, S->ev0, S->ev1) == cudaSuccess) S->lastMs = ms;
    const MargWin& mw = S->margWin[window];
    const WinDesc& d = S->win[window];
    int status = CGMLI_OK, rk = 0;
    CK(cudaMemcpy(&status, S->margStatus.p + window, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&rk, S->margRank.p + window, sizeof(int), cudaMemcpyDeviceToHost));
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
        std::vector<double> pose(7ull * d.K), sb(9ull * d.K), ext(7ull * d.E);
        double td = 0;
        CK(cudaMemcpy(pose.data(), S->pose[0].p + 7ll * d.kf0, pose.size() * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(sb.data(), S->sb[0].p + 9ll * d.kf0, sb.size() * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ext.data(), S->ext[0].p + 7ll * d.ext0, ext.size() * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&td, S->td[0].p + window, 8, cudaMemcpyDeviceToHost));
        double* out = reference;
        for (size_t b = 0; b < kinds.size(); ++b) {
            const double* src = kinds[b] == CGMLI_PRIOR_POSE ? &pose[7ull * idx[b]] : kinds[b] == CGMLI_PRIOR_SPEED_BIAS ? &sb[9ull * idx[b]]
                                : kinds[b] == CGMLI_PRIOR_EXTRINSIC ? &ext[7ull * idx[b]] : &td;
            const int n = ambientOf(kinds[b]);
            std::copy(src, src + n, out);
            out += n;
        }
    }
    if (A && rk) CK(cudaMemcpy(A, S->margA.p + mw.sep0, (size_t)rk * mw.nr * sizeof(double), cudaMemcpyDeviceToHost));
    if (r0 && rk) CK(cudaMemcpy(r0, S->margR0.p + mw.vec0, (size_t)rk * sizeof(double), cudaMemcpyDeviceToHost));
    if (formation) CK(cudaMemcpy(formation, S->margStats.p + 4ll * window, 4 * sizeof(double), cudaMemcpyDeviceToHost));
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
