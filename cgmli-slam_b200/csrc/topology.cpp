// Host-side device layout of a batch of windows; see topology.h.
#include "topology.h"

#include <algorithm>
#include <memory>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <thread>

namespace cgmli {

// A 64-byte header records how the block was obtained.
void* pinnedAllocate(size_t bytes) {
    constexpr size_t kHeader = 64;
    void* raw = nullptr;
    long long kind = 1;
    if (cudaHostAlloc(&raw, bytes + kHeader, cudaHostAllocPortable) != cudaSuccess) {
        (void)cudaGetLastError();
        raw = std::malloc(bytes + kHeader);
        kind = 0;
        if (!raw) return nullptr;
    }
    *static_cast<long long*>(raw) = kind;
    return static_cast<char*>(raw) + kHeader;
}
void pinnedFree(void* p) {
    if (!p) return;
    void* raw = static_cast<char*>(p) - 64;
    if (*static_cast<long long*>(raw) == 1) cudaFreeHost(raw);
    else std::free(raw);
}

namespace {
int tangentOf(int kind) { return kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 6; }
int ambientOf(int kind) { return kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 7; }

// Landmarks per warp run: enough runs to fill the GPU, long runs for large batches.
int runLength(long long totalLm) {
    const long long targetRuns = 148ll * 6 * 4;
    return (int)std::max<long long>(4, std::min<long long>(64, totalLm / targetRuns));
}

// Per-window results whose global position is only known after a prefix sum.
struct WindowPart {
    std::vector<int> supp;          // support lists (keyframes then extrinsics), window-local offsets
    std::vector<int2> tiles;        // global landmark indices
    std::vector<int4> runs;         // window-local tile indices
    std::vector<int4> pairChunks;
    std::vector<int4> schurChunks;  // .w: window-local offset in schurCols
    std::vector<int> schurCols;     // per chunk: count, then ascending visual columns
    // per cross-vector entry (window-local): position in its chunk's columns; every
    // entry is written by the chunking, so the array is not zero-filled first
    std::unique_ptr<unsigned short[]> umap;
    long long cross = 0;            // sum of support widths
    int maxNs = 1;
    int status = CGMLI_OK;
    std::string why;
    // scratch of the build
    int ranges = 1;                      // landmark ranges of kBuildRange (steps A and C)
    std::vector<int> nkf, nx;            // per landmark: support keyframes, support extrinsics
    std::vector<const int*> sup;         // per landmark: its support list (in flat)
    std::vector<std::vector<int>> flat;  // per landmark range: the support lists of its landmarks
    std::vector<int> order;              // device position -> landmark
    std::vector<int> obStart;            // device position -> its first observation in the batch
    std::vector<int> rangeStatus;        // per landmark range
    // support order: length, keyframes, then extrinsics (the shorter keyframe list
    // first where one is a prefix of the other)
    bool less(int a, int b) const {
        const int la = nkf[a] + nx[a], lb = nkf[b] + nx[b];
        if (la != lb) return la < lb;
        const int* pa = sup[a];
        const int* pb = sup[b];
        const int n = std::min(nkf[a], nkf[b]);
        for (int j = 0; j < n; ++j)
            if (pa[j] != pb[j]) return pa[j] < pb[j];
        if (nkf[a] != nkf[b]) return nkf[a] < nkf[b];
        for (int j = nkf[a]; j < la; ++j)
            if (pa[j] != pb[j]) return pa[j] < pb[j];
        return false;
    }
    bool same(int a, int b) const {
        return nkf[a] == nkf[b] && nx[a] == nx[b] && std::equal(sup[a], sup[a] + nkf[a] + nx[a], sup[b]);
    }
};
// Landmarks per work item of the build's range steps: a large window is split
// over several threads.
constexpr int kBuildRange = 256;
}  // namespace

int validateWindow(const cgmli_window& w, int index, std::string& why) {
    char buf[256];
    auto bad = [&](const char* what) {
        std::snprintf(buf, sizeof buf, "window %d: %s", index, what);
        why = buf;
        return CGMLI_E_INVALID;
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
    if (!w.num_landmarks && w.num_observations) return bad("observations without landmarks");
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
        int cols = 0;
        for (int b = 0; b < w.prior_num_blocks; ++b) {
            const int k = w.prior_block_kind[b], i = w.prior_block_index[b];
            if (k < 0 || k > 3) return bad("prior block kind");
            if ((k <= 1 && (i < 0 || i >= w.num_keyframes)) || (k == 2 && (i < 0 || i >= w.num_extrinsics)) || (k == 3 && !w.td))
                return bad("prior block index");
            cols += tangentOf(k);
        }
        if (cols > kPriorMaxCols) {
            std::snprintf(buf, sizeof buf, "window %d: prior above 1024 tangent columns", index);
            why = buf;
            return CGMLI_E_LIMIT;
        }
    }
    if (w.kf_fixed)
        for (int k = 0; k < w.num_keyframes; ++k)
            if (w.kf_fixed[k] & ~(CGMLI_FIX_POSE | CGMLI_FIX_VELOCITY | CGMLI_FIX_BIAS)) return bad("kf_fixed has unknown bits");
    if (w.ext_chart && w.estimate_extrinsics)
        for (int e = 0; e < w.num_extrinsics; ++e)
            if (w.ext_chart[e] > CGMLI_CHART_FIXED) return bad("ext_chart outside CGMLI_CHART_*");
    if (w.lm_fixed)
        for (int l = 0; l < w.num_landmarks; ++l)
            if (w.lm_fixed[l] > 1) return bad("lm_fixed entries must be 0 or 1");
    const int ncal = (w.estimate_extrinsics ? 6 * w.num_extrinsics : 0) + (w.estimate_td ? 1 : 0);
    if (6 * w.num_keyframes + ncal > 400) {
        std::snprintf(buf, sizeof buf, "window %d: visual dimension above 400", index);
        why = buf;
        return CGMLI_E_LIMIT;
    }
    return CGMLI_OK;
}

int buildHostBatch(const cgmli_window* windows, int count, int threads, HostBatch& hb, std::string& why,
                   const std::function<void(int, int)>* ready, const PlanParams& plan) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    threads = std::min(threads, 64);
    // ---- validation (parallel)
    std::vector<int> vst(count, CGMLI_OK);
    std::vector<std::string> vwhy(count);
    parallelFor(count, threads, [&](int i) { vst[i] = validateWindow(windows[i], i, vwhy[i]); });
    for (int i = 0; i < count; ++i)
        if (vst[i] != CGMLI_OK) { why = vwhy[i]; return vst[i]; }
    // ---- phase 0: offsets from the windows' sizes
    hb.win.assign(count, WinDesc{});
    hb.plan = plan;
    hb.maxNpc = 0; hb.maxNr = 0; hb.maxNs = 1;
    std::vector<long long> pA0(count), pR0(count), pRef0(count);
    std::vector<int> pblk0(count);
    int kf = 0, ex = 0, cam = 0, lm = 0, ob = 0, im = 0, pblk = 0;
    long long vec = 0, dense = 0, acc = 0, sch = 0, imuS = 0, priS = 0, pA = 0, pR = 0, pRef = 0;
    for (int i = 0; i < count; ++i) {
        const auto& w = windows[i];
        WinDesc& d = hb.win[i];
        d.K = w.num_keyframes; d.E = w.num_extrinsics; d.C = w.num_cameras; d.L = w.num_landmarks; d.F = w.num_observations;
        d.nImu = w.num_imu;
        d.estExt = w.estimate_extrinsics != 0; d.estTd = w.estimate_td != 0 && w.td; d.hasTd = w.td != nullptr;
        d.ncalib = (d.estExt ? 6 * d.E : 0) + (d.estTd ? 1 : 0);
        d.Npc = 6 * d.K + d.ncalib;
        d.Nr = 15 * d.K + d.ncalib;
        d.kf0 = kf; d.ext0 = ex; d.cam0 = cam; d.lm0 = lm; d.obs0 = ob; d.imu0 = im;
        d.vec0 = (int)vec; d.dense0 = dense; d.acc0 = acc; d.sch0 = sch;
        d.huber = w.huber_scale; d.minInv = w.min_inverse_distance;
        d.charts = 0;
        if (w.kf_fixed)
            for (int k = 0; k < d.K; ++k) d.charts |= w.kf_fixed[k] ? 1 : 0;
        if (d.estExt && w.ext_chart)
            for (int e = 0; e < d.E; ++e) d.charts |= w.ext_chart[e] ? 1 : 0;
        d.fixedLm = 0;
        if (w.lm_fixed)
            for (int l = 0; l < d.L; ++l) d.fixedLm |= w.lm_fixed[l];
        hb.maxNpc = std::max(hb.maxNpc, d.Npc);
        hb.maxNr = std::max(hb.maxNr, d.Nr);
        vec += d.Nr;
        dense += (long long)d.Nr * d.Nr;
        acc += (long long)d.Npc * (d.Npc + 1) / 2 + 3ll * d.Npc;
        sch += (long long)d.Npc * (d.Npc + 1) / 2;
        d.imuScratch0 = imuS;
        imuS += 930ll * d.nImu;
        d.priorRank = w.prior_rank;
        d.priorBlk0 = pblk;
        d.priorBlocks = w.prior_rank > 0 ? w.prior_num_blocks : 0;
        int cols = 0, amb = 0;
        for (int b = 0; b < d.priorBlocks; ++b) {
            cols += tangentOf(w.prior_block_kind[b]);
            amb += ambientOf(w.prior_block_kind[b]);
        }
        d.priorCols = cols;
        d.priorA0 = pA; d.priorR00 = pR; d.priorRef0 = pRef;
        pA0[i] = pA; pR0[i] = pR; pRef0[i] = pRef; pblk0[i] = pblk;
        pA += (long long)d.priorRank * cols;
        pR += d.priorRank;
        pRef += d.priorRank > 0 ? amb : 0;
        pblk += d.priorBlocks;
        d.priorScratch0 = priS;
        priS += d.priorRank > 0 ? (long long)cols * 7 + d.priorRank + (long long)d.priorRank * cols : 0;
        kf += d.K; ex += d.E; cam += d.C; lm += d.L; ob += d.F; im += d.nImu;
    }
    hb.totalKf = kf; hb.totalExt = ex; hb.totalCam = cam; hb.totalLm = lm; hb.totalObs = ob; hb.totalImu = im;
    hb.vec = vec; hb.dense = dense; hb.acc = acc; hb.sch = sch; hb.imuScratch = imuS; hb.priorScratch = priS;
    constexpr int kImuDoubles = sizeof(cgmli_frozen_imu) / sizeof(double);
    sizeTo(hb.camR, 9ll * cam); sizeTo(hb.camT, 3ll * cam); sizeTo(hb.camExt, cam);
    sizeTo(hb.lmWin, lm); sizeTo(hb.lmKf, lm); sizeTo(hb.lmCam, lm); sizeTo(hb.lmObsBegin, lm + 1ll); sizeTo(hb.lmNs, lm); sizeTo(hb.lmNx, lm);
    sizeTo(hb.lmSupp0, lm); sizeTo(hb.lmC0, lm); sizeTo(hb.lmPerm, lm);
    sizeTo(hb.lmBearing, 3ll * lm); sizeTo(hb.lmVel, 3ll * lm); sizeTo(hb.lmTime, lm);
    sizeTo(hb.obKf, ob); sizeTo(hb.obCam, ob); sizeTo(hb.obSlot, ob); sizeTo(hb.obXslot, ob); sizeTo(hb.obLm, ob); sizeTo(hb.obOrig, ob);
    sizeTo(hb.keyOrder, ob);
    sizeTo(hb.obBearing, 3ll * ob); sizeTo(hb.obP, 6ll * ob); sizeTo(hb.obVel, 3ll * ob); sizeTo(hb.obTime, ob);
    sizeTo(hb.pose, 7ll * kf); sizeTo(hb.sb, 9ll * kf); sizeTo(hb.ext, 7ll * ex); sizeTo(hb.td, count); sizeTo(hb.rho, lm);
    sizeTo(hb.colChart, vec); sizeTo(hb.lmFixed, lm);
    sizeTo(hb.imu, (size_t)kImuDoubles * im); sizeTo(hb.imuKf, im);
    sizeTo(hb.priorKind, pblk); sizeTo(hb.priorIndex, pblk); sizeTo(hb.priorCol, pblk); sizeTo(hb.priorOff, pblk);
    sizeTo(hb.priorA, pA); sizeTo(hb.priorR0, pR); sizeTo(hb.priorRef, pRef);
    hb.lmObsBegin[lm] = ob;
    const int runLen = plan.runLandmarks > 0 ? plan.runLandmarks : runLength(lm);
    // ---- phase 1, in four steps so that a large window is built by several threads:
    //  A (ranges of a window's landmarks): support lists, and the range sorted by support;
    //  B (per window): states and rig; the sorted ranges merged into the device order;
    //    runs and tiles; offsets of each landmark's support, cross-vector entries and
    //    observations;
    //  C (ranges of the device order): landmark and observation arrays;
    //  D (two items per window): the key order of the J^T J pass; the Schur chunks.
    std::vector<WindowPart> part(count);
    for (int i = 0; i < count; ++i) {
        const int L = hb.win[i].L;
        WindowPart& P = part[i];
        P.ranges = std::max(1, (L + kBuildRange - 1) / kBuildRange);
        P.nkf.resize(L);
        P.nx.resize(L);
        P.sup.resize(L);
        P.order.resize(L);
        P.obStart.resize(L);
        P.flat.resize(P.ranges);
        P.rangeStatus.assign(P.ranges, CGMLI_OK);
    }
    auto stepA = [&](int i, int r) {
        const auto& w = windows[i];
        const WinDesc& d = hb.win[i];
        WindowPart& P = part[i];
        const int l0 = r * kBuildRange, l1 = std::min(d.L, l0 + kBuildRange);
        if (l0 >= l1) return;
        // supports: keyframes (anchor first, then observers ascending), then the
        // extrinsic blocks the observations touch (anchor camera's first, then ascending)
        std::vector<int>& flat = P.flat[r];
        flat.clear();
        flat.reserve((size_t)2 * (w.lm_obs_begin[l1] - w.lm_obs_begin[l0]) + 2 * (l1 - l0) + 1);
        for (int l = l0; l < l1; ++l) {
            const int b = w.lm_obs_begin[l], e = w.lm_obs_begin[l + 1];
            const int s0 = (int)flat.size();
            flat.push_back(w.lm_anchor_kf[l]);
            for (int f = b; f < e; ++f) {
                const int k = w.obs_kf[f];
                bool seen = false;
                for (int j = s0; j < (int)flat.size(); ++j) seen = seen || flat[j] == k;
                if (!seen) {  // insertion into the sorted tail (after the anchor)
                    flat.push_back(k);
                    for (int j = (int)flat.size() - 1; j > s0 + 1 && flat[j - 1] > flat[j]; --j) std::swap(flat[j - 1], flat[j]);
                }
            }
            P.nkf[l] = (int)flat.size() - s0;
            if (P.nkf[l] > kMaxSupport) {
                P.rangeStatus[r] = CGMLI_E_LIMIT;
                return;
            }
            const int x0 = (int)flat.size();
            if (d.estExt) {
                flat.push_back(w.cam_ext[w.lm_anchor_cam[l]]);
                for (int f = b; f < e; ++f) {
                    const int x = w.cam_ext[w.obs_cam[f]];
                    bool seen = false;
                    for (int j = x0; j < (int)flat.size(); ++j) seen = seen || flat[j] == x;
                    if (!seen) {
                        flat.push_back(x);
                        for (int j = (int)flat.size() - 1; j > x0 + 1 && flat[j - 1] > flat[j]; --j) std::swap(flat[j - 1], flat[j]);
                    }
                }
            }
            P.nx[l] = (int)flat.size() - x0;
        }
        // the observation payload of these landmarks in the caller's order (one
        // contiguous range); the device gathers it into device order through obOrig
        {
            const long long b0 = w.lm_obs_begin[l0], n = w.lm_obs_begin[l1] - b0, o0 = d.obs0 + b0;
            std::memcpy(&hb.obBearing[3 * o0], &w.obs_bearing[3 * b0], sizeof(double) * 3 * n);
            std::memcpy(&hb.obP[6 * o0], &w.obs_P[6 * b0], sizeof(double) * 6 * n);
            if (w.obs_velocity) std::memcpy(&hb.obVel[3 * o0], &w.obs_velocity[3 * b0], sizeof(double) * 3 * n);
            else std::memset(&hb.obVel[3 * o0], 0, sizeof(double) * 3 * n);
            if (w.obs_time) std::memcpy(&hb.obTime[o0], &w.obs_time[b0], sizeof(double) * n);
            else std::memset(&hb.obTime[o0], 0, sizeof(double) * n);
        }
        // the list is final: point each landmark at its support
        for (int l = l0, s = 0; l < l1; ++l) {
            P.sup[l] = flat.data() + s;
            s += P.nkf[l] + P.nx[l];
        }
        // the range in support order (stable); step B merges the ranges
        for (int l = l0; l < l1; ++l) P.order[l] = l;
        std::stable_sort(P.order.begin() + l0, P.order.begin() + l1, [&P](int a, int b) { return P.less(a, b); });
    };
    auto stepB = [&](int i) {
        const auto& w = windows[i];
        const WinDesc& d = hb.win[i];
        WindowPart& P = part[i];
        for (int r = 0; r < P.ranges; ++r)
            if (P.rangeStatus[r] != CGMLI_OK) {
                P.status = P.rangeStatus[r];
                P.why = "landmark support above 64 keyframes";
                return;
            }
        // states, rig, IMU, prior
        std::memcpy(&hb.pose[7ll * d.kf0], w.poses, sizeof(double) * 7 * d.K);
        {
            // solve-time chart of every retained column (kColFree / kColFixed / the rotation-only pair)
            signed char* cc = &hb.colChart[d.vec0];
            for (int c = 0; c < d.Nr; ++c) cc[c] = kColFree;
            if (w.kf_fixed)
                for (int k = 0; k < d.K; ++k) {
                    const int m = w.kf_fixed[k];
                    for (int c = 0; c < 6; ++c) if (m & CGMLI_FIX_POSE) cc[15 * k + c] = kColFixed;
                    for (int c = 6; c < 9; ++c) if (m & CGMLI_FIX_VELOCITY) cc[15 * k + c] = kColFixed;
                    for (int c = 9; c < 15; ++c) if (m & CGMLI_FIX_BIAS) cc[15 * k + c] = kColFixed;
                }
            if (d.estExt && w.ext_chart)
                for (int e = 0; e < d.E; ++e) {
                    const int c0 = 15 * d.K + 6 * e;
                    for (int c = 0; c < 6; ++c)
                        cc[c0 + c] = w.ext_chart[e] == CGMLI_CHART_FIXED ? kColFixed
                                     : w.ext_chart[e] == CGMLI_CHART_ROTATION_ONLY ? (c < 3 ? kColRotRho : kColRotTheta) : kColFree;
                }
        }
        std::memcpy(&hb.sb[9ll * d.kf0], w.speed_bias, sizeof(double) * 9 * d.K);
        std::memcpy(&hb.ext[7ll * d.ext0], w.extrinsics, sizeof(double) * 7 * d.E);
        hb.td[i] = w.td ? *w.td : 0.0;
        std::memcpy(&hb.camR[9ll * d.cam0], w.cam_R, sizeof(double) * 9 * d.C);
        std::memcpy(&hb.camT[3ll * d.cam0], w.cam_t, sizeof(double) * 3 * d.C);
        for (int c = 0; c < d.C; ++c) hb.camExt[d.cam0 + c] = d.ext0 + w.cam_ext[c];
        if (d.nImu) std::memcpy(&hb.imu[(size_t)kImuDoubles * d.imu0], w.imu, sizeof(cgmli_frozen_imu) * d.nImu);
        for (int q = 0; q < d.nImu; ++q) hb.imuKf[d.imu0 + q] = d.kf0 + w.imu_kf[q];
        {
            int cols = 0, amb = 0;
            for (int b = 0; b < d.priorBlocks; ++b) {
                const int kind = w.prior_block_kind[b], idx = w.prior_block_index[b], g = pblk0[i] + b;
                int gidx = idx, col = -1;
                if (kind == CGMLI_PRIOR_POSE) { gidx = d.kf0 + idx; col = 15 * idx; }
                else if (kind == CGMLI_PRIOR_SPEED_BIAS) { gidx = d.kf0 + idx; col = 15 * idx + 6; }
                else if (kind == CGMLI_PRIOR_EXTRINSIC) { gidx = d.ext0 + idx; col = d.estExt ? 15 * d.K + 6 * idx : -1; }
                else { gidx = i; col = d.estTd ? 15 * d.K + (d.estExt ? 6 * d.E : 0) : -1; }
                hb.priorKind[g] = kind; hb.priorIndex[g] = gidx; hb.priorCol[g] = col; hb.priorOff[g] = cols;
                cols += tangentOf(kind);
                amb += ambientOf(kind);
            }
            if (d.priorRank > 0) {
                std::memcpy(&hb.priorA[pA0[i]], w.prior_A, sizeof(double) * (size_t)d.priorRank * cols);
                std::memcpy(&hb.priorR0[pR0[i]], w.prior_r0, sizeof(double) * d.priorRank);
                std::memcpy(&hb.priorRef[pRef0[i]], w.prior_ref, sizeof(double) * amb);
            }
        }
        // device order: landmarks sorted (stably) by support, so that equal supports are
        // adjacent; merging the stably sorted ranges pairwise, the left range first on
        // ties, gives the stable sort of the whole window
        const int L = d.L;
        auto less = [&P](int a, int b) { return P.less(a, b); };
        for (int width = 1; width < P.ranges; width *= 2)
            for (int r = 0; r + width < P.ranges; r += 2 * width) {
                const auto first = P.order.begin() + (long long)r * kBuildRange;
                const auto mid = P.order.begin() + (long long)(r + width) * kBuildRange;
                const auto last = P.order.begin() + std::min<long long>(L, (long long)(r + 2 * width) * kBuildRange);
                std::inplace_merge(first, mid, last, less);
            }
        // runs of landmarks (a new run at a support change once a run holds runLen
        // landmarks, and at 4 runLen), tiles of at most kMaxTrackChunk observations,
        // and the window-local offsets of supports and cross-vector entries
        int obPos = d.obs0, tileObs = 0, runLms = 0;
        long long suppSize = 0;
        for (int q = 0; q < L; ++q) {
            const int l = P.order[q], g = d.lm0 + q;
            const int nobs = w.lm_obs_begin[l + 1] - w.lm_obs_begin[l];
            const bool newGroup = q == 0 || !P.same(P.order[q - 1], l);
            if (q == 0 || (runLms >= runLen && newGroup) || runLms >= 4 * runLen) {
                if (!P.runs.empty()) P.runs.back().z = (int)P.tiles.size();
                if (!P.tiles.empty()) P.tiles.back().y = g;
                P.runs.push_back(make_int4(i, (int)P.tiles.size(), -1, 0));
                P.tiles.push_back(make_int2(g, -1));
                tileObs = 0;
                runLms = 0;
            } else if (tileObs + nobs > kMaxTrackChunk) {
                P.tiles.back().y = g;
                P.tiles.push_back(make_int2(g, -1));
                tileObs = 0;
            }
            tileObs += nobs;
            ++runLms;
            const int width = P.nkf[l] + P.nx[l];
            hb.lmSupp0[g] = (int)suppSize;  // window-local, fixed up after the prefix sum
            suppSize += width;
            const int ns = 6 * width + (d.estTd ? 1 : 0);
            hb.lmC0[g] = P.cross;  // window-local
            P.cross += ns;
            P.maxNs = std::max(P.maxNs, ns);
            P.obStart[q] = obPos;
            obPos += nobs;
        }
        if (L) {
            P.tiles.back().y = d.lm0 + L;
            P.runs.back().z = (int)P.tiles.size();
        }
        P.supp.resize(suppSize);
    };
    auto stepC = [&](int i, int r) {
        const auto& w = windows[i];
        const WinDesc& d = hb.win[i];
        WindowPart& P = part[i];
        const int L = d.L;
        const int q0 = r * kBuildRange, q1 = std::min(L, q0 + kBuildRange);
        for (int q = q0; q < q1; ++q) {
            if (q + 8 < L) {  // the support order jumps through the caller's arrays: fetch ahead
                const int lp = P.order[q + 8], bp = w.lm_obs_begin[lp];
                __builtin_prefetch(&w.obs_kf[bp]);
                __builtin_prefetch(&w.obs_cam[bp]);
                __builtin_prefetch(&w.lm_anchor_bearing[3ll * lp]);
                __builtin_prefetch(&w.rho[lp]);
                __builtin_prefetch(P.sup[lp]);
            }
            const int l = P.order[q], g = d.lm0 + q;
            const int b = w.lm_obs_begin[l], nobs = w.lm_obs_begin[l + 1] - b;
            const int nk = P.nkf[l], nxl = P.nx[l];
            const int* sl = P.sup[l];
            hb.lmPerm[g] = l;
            hb.lmWin[g] = i;
            hb.lmKf[g] = d.kf0 + w.lm_anchor_kf[l];
            hb.lmCam[g] = d.cam0 + w.lm_anchor_cam[l];
            hb.lmObsBegin[g] = P.obStart[q];
            for (int k = 0; k < 3; ++k) {
                hb.lmBearing[3ll * g + k] = w.lm_anchor_bearing[3 * l + k];
                hb.lmVel[3ll * g + k] = w.lm_anchor_velocity ? w.lm_anchor_velocity[3 * l + k] : 0.0;
            }
            hb.lmTime[g] = w.lm_anchor_time ? w.lm_anchor_time[l] : 0.0;
            hb.lmNs[g] = nk;
            hb.lmNx[g] = nxl;
            std::copy(sl, sl + nk + nxl, P.supp.begin() + hb.lmSupp0[g]);
            hb.rho[g] = w.rho[l];
            hb.lmFixed[g] = w.lm_fixed ? w.lm_fixed[l] : 0;
            // observations sorted by observer keyframe (slot order), stable
            int fo[kMaxTrackChunk];
            for (int k = 0; k < nobs; ++k) {
                int j = k;
                fo[j] = b + k;
                while (j > 0 && w.obs_kf[fo[j - 1]] > w.obs_kf[fo[j]]) { std::swap(fo[j - 1], fo[j]); --j; }
            }
            int obPos = P.obStart[q];
            for (int k = 0; k < nobs; ++k) {
                const int f = fo[k], o = obPos++;
                hb.obLm[o] = g;
                hb.obOrig[o] = f;
                hb.obKf[o] = d.kf0 + w.obs_kf[f];
                hb.obCam[o] = d.cam0 + w.obs_cam[f];
                int slot = 0;
                while (sl[slot] != w.obs_kf[f]) ++slot;
                hb.obSlot[o] = slot;
                int xs = 0;
                if (d.estExt) {
                    const int x = w.cam_ext[w.obs_cam[f]];
                    while (sl[nk + xs] != x) ++xs;
                }
                hb.obXslot[o] = xs;
            }
        }
    };
    auto stepD = [&](int i, int which) {
        const WinDesc& d = hb.win[i];
        WindowPart& P = part[i];
        const int L = d.L;
        (void)L;
        if (which == 0) {
            // key order (anchor kf, observer kf, anchor ext, observer ext) of the J^T J pass
            const int F = d.F;
            auto keyOf = [&](int o) {
                const int g = hb.obLm[o];
                const int a = hb.lmKf[g] - d.kf0, bkf = hb.obKf[o] - d.kf0;
                const int ea = hb.camExt[hb.lmCam[g]] - d.ext0, eb = hb.camExt[hb.obCam[o]] - d.ext0;
                return ((long long)(a * d.K + bkf) * d.E + ea) * d.E + eb;
            };
            const long long buckets = (long long)d.K * d.K * d.E * d.E;
            int* ko = F ? &hb.keyOrder[d.obs0] : nullptr;
            if (buckets <= 4ll * F + 4096) {
                std::vector<int> cnt(buckets + 1, 0);
                for (int g = 0; g < F; ++g) ++cnt[keyOf(d.obs0 + g) + 1];
                for (long long k = 0; k < buckets; ++k) cnt[k + 1] += cnt[k];
                for (int g = 0; g < F; ++g) ko[cnt[keyOf(d.obs0 + g)]++] = d.obs0 + g;
            } else {
                std::vector<std::pair<long long, int>> kv(F);
                for (int g = 0; g < F; ++g) kv[g] = {keyOf(d.obs0 + g), d.obs0 + g};
                std::sort(kv.begin(), kv.end());
                for (int g = 0; g < F; ++g) ko[g] = kv[g].second;
            }
            for (int c0 = 0; c0 < F; c0 += plan.pairChunk)
                P.pairChunks.push_back(make_int4(i, d.obs0 + c0, d.obs0 + std::min(F, c0 + plan.pairChunk), 0));
            return;
        }
        // Schur chunks: runs of consecutive landmarks whose support columns
        // together fit the chunk's shared rows (schurChunkFits); the column
        // union of each chunk and every landmark's map into it.  Unions are kept
        // as bit sets of column blocks: keyframe k, extrinsic K + e, td K + E.
        {
            const int tdCol = 6 * d.K + (d.estExt ? 6 * d.E : 0);
            const int tdBlk = d.K + d.E, nBlk = tdBlk + 1;
            const int words = (nBlk + 63) / 64;
            std::vector<unsigned long long> U(words, 0), Ul(words, 0);
            std::vector<int> blkPos(nBlk, 0);
            P.umap.reset(new unsigned short[P.cross > 0 ? P.cross : 1]);
            auto blocksOf = [&](int q) {
                std::fill(Ul.begin(), Ul.end(), 0ull);
                const int g = d.lm0 + q, ns_ = hb.lmNs[g], nx_ = hb.lmNx[g];
                const int* sk = &P.supp[hb.lmSupp0[g]];
                for (int j = 0; j < ns_; ++j) Ul[sk[j] >> 6] |= 1ull << (sk[j] & 63);
                for (int j = 0; j < nx_; ++j) {
                    const int b = d.K + sk[ns_ + j];
                    Ul[b >> 6] |= 1ull << (b & 63);
                }
                if (d.estTd) Ul[tdBlk >> 6] |= 1ull << (tdBlk & 63);
            };
            auto columnsIn = [&](const std::vector<unsigned long long>& a, const std::vector<unsigned long long>* b) {
                int blocks = 0;
                for (int wi = 0; wi < words; ++wi) blocks += __builtin_popcountll(a[wi] | (b ? (*b)[wi] : 0ull));
                return d.estTd ? 6 * (blocks - 1) + 1 : 6 * blocks;
            };
            int q0 = 0, nu = 0;
            auto closeChunk = [&](int q1) {
                const int off = (int)P.schurCols.size();
                P.schurCols.push_back(nu);
                int k = 0;
                for (int wi = 0; wi < words; ++wi)
                    for (unsigned long long bits = U[wi]; bits; bits &= bits - 1) {
                        const int blk = 64 * wi + __builtin_ctzll(bits);
                        blkPos[blk] = k;
                        if (blk == tdBlk && d.estTd) {
                            P.schurCols.push_back(tdCol);
                            k += 1;
                        } else {
                            const int col0 = blk < d.K ? 6 * blk : 6 * d.K + 6 * (blk - d.K);
                            for (int c = 0; c < 6; ++c) P.schurCols.push_back(col0 + c);
                            k += 6;
                        }
                    }
                for (int q = q0; q < q1; ++q) {
                    const int g = d.lm0 + q, ns_ = hb.lmNs[g], nx_ = hb.lmNx[g];
                    const int* sk = &P.supp[hb.lmSupp0[g]];
                    const long long c0 = hb.lmC0[g];  // window-local here
                    for (int j = 0; j < ns_; ++j)
                        for (int c = 0; c < 6; ++c) P.umap[c0 + 6 * j + c] = (unsigned short)(blkPos[sk[j]] + c);
                    for (int j = 0; j < nx_; ++j)
                        for (int c = 0; c < 6; ++c) P.umap[c0 + 6 * (ns_ + j) + c] = (unsigned short)(blkPos[d.K + sk[ns_ + j]] + c);
                    if (d.estTd) P.umap[c0 + 6 * (ns_ + nx_)] = (unsigned short)blkPos[tdBlk];
                }
                P.schurChunks.push_back(make_int4(i, d.lm0 + q0, d.lm0 + q1, off));
                std::fill(U.begin(), U.end(), 0ull);
                nu = 0;
                q0 = q1;
            };
            for (int q = 0; q < L; ++q) {
                blocksOf(q);
                int nuNew = columnsIn(U, &Ul);
                if (q > q0 && (q - q0 + 1 > plan.schurRows || !schurChunkFits(q - q0 + 1, nuNew))) {
                    closeChunk(q);
                    nuNew = columnsIn(Ul, nullptr);
                }
                for (int wi = 0; wi < words; ++wi) U[wi] |= Ul[wi];
                nu = nuNew;
            }
            if (L > q0) closeChunk(L);
        }
    };
    // A batch of at least two windows per thread, or of small windows only, keeps the
    // threads busy with whole windows, largest first so that no thread is left with a
    // large one at the end; otherwise the steps run one after the other, each split
    // over the threads.  In up to four ranges of windows when a caller streams the
    // finished ranges.
    int maxL = 0;
    for (int i = 0; i < count; ++i) maxL = std::max(maxL, hb.win[i].L);
    const bool whole = count >= 2 * threads || maxL <= 4 * kBuildRange;
    const int ranges = ready && count >= 4 * threads ? 4 : 1;
    std::vector<int2> items;
    std::vector<int> bySize;
    for (int rg = 0; rg < ranges; ++rg) {
        const int w0 = (int)((long long)count * rg / ranges), w1 = (int)((long long)count * (rg + 1) / ranges);
        if (whole) {
            bySize.resize(w1 - w0);
            for (int k = 0; k < w1 - w0; ++k) bySize[k] = w0 + k;
            std::stable_sort(bySize.begin(), bySize.end(), [&](int a, int b) {
                return hb.win[a].F + hb.win[a].L > hb.win[b].F + hb.win[b].L;
            });
            parallelFor(w1 - w0, threads, [&](int k) {
                const int i = bySize[k];
                for (int r = 0; r < part[i].ranges; ++r) stepA(i, r);
                stepB(i);
                if (part[i].status != CGMLI_OK) return;
                for (int r = 0; r < part[i].ranges; ++r) stepC(i, r);
                stepD(i, 0);
                stepD(i, 1);
            });
        } else {
            items.clear();
            for (int i = w0; i < w1; ++i)
                for (int r = 0; r < part[i].ranges; ++r) items.push_back(make_int2(i, r));
            parallelFor((int)items.size(), threads, [&](int k) { stepA(items[k].x, items[k].y); });
            parallelFor(w1 - w0, threads, [&](int k) { stepB(w0 + k); });
            bool failed = false;
            for (int i = w0; i < w1; ++i) failed = failed || part[i].status != CGMLI_OK;
            if (failed) break;
            parallelFor((int)items.size(), threads, [&](int k) { stepC(items[k].x, items[k].y); });
            parallelFor(2 * (w1 - w0), threads, [&](int k) { stepD(w0 + k / 2, k % 2); });
        }
        bool failed = false;
        for (int i = w0; i < w1; ++i) failed = failed || part[i].status != CGMLI_OK;
        if (failed) break;
        if (ready) (*ready)(w0, w1);
    }
    for (int i = 0; i < count; ++i)
        if (part[i].status != CGMLI_OK) {
            char buf[256];
            std::snprintf(buf, sizeof buf, "window %d: %s", i, part[i].why.c_str());
            why = buf;
            return part[i].status;
        }
    // ---- phase 2: prefix sums and fix-ups
    std::vector<long long> suppBase(count + 1, 0), crossBase(count + 1, 0);
    std::vector<int> tileBase(count + 1, 0), runBase(count + 1, 0), pairBase(count + 1, 0), schurBase(count + 1, 0),
        schurColBase(count + 1, 0);
    for (int i = 0; i < count; ++i) {
        suppBase[i + 1] = suppBase[i] + (long long)part[i].supp.size();
        crossBase[i + 1] = crossBase[i] + part[i].cross;
        tileBase[i + 1] = tileBase[i] + (int)part[i].tiles.size();
        runBase[i + 1] = runBase[i] + (int)part[i].runs.size();
        pairBase[i + 1] = pairBase[i] + (int)part[i].pairChunks.size();
        schurBase[i + 1] = schurBase[i] + (int)part[i].schurChunks.size();
        schurColBase[i + 1] = schurColBase[i] + (int)part[i].schurCols.size();
        hb.maxNs = std::max(hb.maxNs, part[i].maxNs);
    }
    hb.cross = crossBase[count];
    sizeTo(hb.supp, suppBase[count]);
    sizeTo(hb.tiles, tileBase[count]);
    sizeTo(hb.runs, runBase[count]);
    sizeTo(hb.pairChunks, pairBase[count]);
    sizeTo(hb.schurChunks, schurBase[count]);
    sizeTo(hb.schurCols, std::max(schurColBase[count], 1));
    sizeTo(hb.lmUmap, std::max(hb.cross, 1ll));
    parallelFor(count, threads, [&](int i) {
        const WinDesc& d = hb.win[i];
        WindowPart& P = part[i];
        std::copy(P.supp.begin(), P.supp.end(), hb.supp.begin() + suppBase[i]);
        for (int q = 0; q < d.L; ++q) {
            hb.lmSupp0[d.lm0 + q] += (int)suppBase[i];
            hb.lmC0[d.lm0 + q] += crossBase[i];
        }
        std::copy(P.tiles.begin(), P.tiles.end(), hb.tiles.begin() + tileBase[i]);
        for (size_t r = 0; r < P.runs.size(); ++r) {
            int4 run = P.runs[r];
            run.y += tileBase[i];
            run.z += tileBase[i];
            hb.runs[runBase[i] + r] = run;
        }
        std::copy(P.pairChunks.begin(), P.pairChunks.end(), hb.pairChunks.begin() + pairBase[i]);
        for (size_t c = 0; c < P.schurChunks.size(); ++c) {
            int4 chunk = P.schurChunks[c];
            chunk.w += schurColBase[i];
            hb.schurChunks[schurBase[i] + c] = chunk;
        }
        std::copy(P.schurCols.begin(), P.schurCols.end(), hb.schurCols.begin() + schurColBase[i]);
        std::copy(P.umap.get(), P.umap.get() + P.cross, hb.lmUmap.begin() + crossBase[i]);
    });
    // ---- deterministic mode: each window's pair chunks and Schur chunks in contiguous
    // units (kDetUnitObs observations, kDetSchurChunksPerUnit chunks; at most kDetMaxSlots
    // of each), each with a slot of its own.  The units follow from the window alone, so
    // a window's sums are the same alone and in any batch.
    hb.detSlots = 0;
    if (!plan.deterministic) {
        sizeTo(hb.detPairs, 0);
        sizeTo(hb.detSchur, 0);
        return CGMLI_OK;
    }
    int nPairUnits = 0, nSchurUnits = 0;
    for (int i = 0; i < count; ++i) {
        WinDesc& d = hb.win[i];
        const int np = pairBase[i + 1] - pairBase[i], ns = schurBase[i + 1] - schurBase[i];
        d.detPairs = std::min({kDetMaxSlots, np, (d.F + kDetUnitObs - 1) / kDetUnitObs});
        d.detSchur = std::min(kDetMaxSlots, (ns + kDetSchurChunksPerUnit - 1) / kDetSchurChunksPerUnit);
        d.det0 = hb.detSlots;
        hb.detSlots += (long long)(d.detPairs + d.detSchur) * ((long long)d.Npc * (d.Npc + 1) / 2 + d.Npc);
        nPairUnits += d.detPairs;
        nSchurUnits += d.detSchur;
    }
    sizeTo(hb.detPairs, nPairUnits);
    sizeTo(hb.detSchur, nSchurUnits);
    for (int i = 0, pu = 0, su = 0; i < count; ++i) {
        const WinDesc& d = hb.win[i];
        const int np = pairBase[i + 1] - pairBase[i], ns = schurBase[i + 1] - schurBase[i];
        for (int g = 0; g < d.detPairs; ++g) {
            const int c0 = pairBase[i] + (int)((long long)g * np / d.detPairs);
            const int c1 = pairBase[i] + (int)((long long)(g + 1) * np / d.detPairs);
            hb.detPairs[pu++] = make_int4(i, hb.pairChunks[c0].y, hb.pairChunks[c1 - 1].z, g);
        }
        for (int g = 0; g < d.detSchur; ++g) {
            const int c0 = schurBase[i] + (int)((long long)g * ns / d.detSchur);
            const int c1 = schurBase[i] + (int)((long long)(g + 1) * ns / d.detSchur);
            hb.detSchur[su++] = make_int4(c0, c1, g, i);
        }
    }
    return CGMLI_OK;
}

int checkHostBatch(const cgmli_window* windows, int count, const HostBatch& hb, std::string& why) {
    char buf[256];
    auto bad = [&](int i, const char* what) {
        std::snprintf(buf, sizeof buf, "window %d: %s", i, what);
        why = buf;
        return CGMLI_E_INVALID;
    };
    for (int i = 0; i < count; ++i) {
        const auto& w = windows[i];
        const WinDesc& d = hb.win[i];
        // lmPerm is a permutation of the window's landmarks, the observation ranges
        // partition the window's observations and follow the caller's landmarks
        std::vector<char> seen(d.L, 0);
        for (int q = 0; q < d.L; ++q) {
            const int g = d.lm0 + q, l = hb.lmPerm[g];
            if (l < 0 || l >= d.L || seen[l]) return bad(i, "landmark order is not a permutation");
            seen[l] = 1;
            if (hb.lmObsBegin[g + 1] - hb.lmObsBegin[g] != w.lm_obs_begin[l + 1] - w.lm_obs_begin[l])
                return bad(i, "observation range of a landmark changed size");
            if (hb.lmKf[g] != d.kf0 + w.lm_anchor_kf[l]) return bad(i, "anchor keyframe");
            for (int o = hb.lmObsBegin[g]; o < hb.lmObsBegin[g + 1]; ++o) {
                if (hb.obLm[o] != g) return bad(i, "observation -> landmark map");
                if (o > hb.lmObsBegin[g] && hb.obKf[o - 1] > hb.obKf[o]) return bad(i, "observations not sorted by keyframe");
                const int* sl = &hb.supp[hb.lmSupp0[g]];
                if (d.kf0 + sl[hb.obSlot[o]] != hb.obKf[o]) return bad(i, "observation slot");
                if (d.estExt && d.ext0 + sl[hb.lmNs[g] + hb.obXslot[o]] != hb.camExt[hb.obCam[o]]) return bad(i, "extrinsic slot");
            }
            if (q > 0 && hb.lmNs[g] + hb.lmNx[g] < hb.lmNs[g - 1] + hb.lmNx[g - 1]) return bad(i, "landmarks not sorted by support");
        }
        if (d.L && (hb.lmObsBegin[d.lm0] != d.obs0 || hb.lmObsBegin[d.lm0 + d.L] != d.obs0 + d.F))
            return bad(i, "observation ranges do not cover the window");
        // key order: a permutation of the window's observations, keys non-decreasing
        std::vector<char> oseen(d.F, 0);
        long long prev = -1;
        for (int k = 0; k < d.F; ++k) {
            const int o = hb.keyOrder[d.obs0 + k];
            if (o < d.obs0 || o >= d.obs0 + d.F || oseen[o - d.obs0]) return bad(i, "key order is not a permutation");
            oseen[o - d.obs0] = 1;
            const int g = hb.obLm[o];
            const long long key = ((long long)((hb.lmKf[g] - d.kf0) * d.K + hb.obKf[o] - d.kf0) * d.E +
                                   (hb.camExt[hb.lmCam[g]] - d.ext0)) * d.E + (hb.camExt[hb.obCam[o]] - d.ext0);
            if (key < prev) return bad(i, "key order not sorted");
            prev = key;
        }
    }
    // work units cover every landmark / observation exactly once, within one window
    std::vector<int> lmCover(hb.totalLm, 0);
    for (const int4& r : hb.runs)
        for (int t = r.y; t < r.z; ++t) {
            const int2 tile = hb.tiles[t];
            const WinDesc& d = hb.win[r.x];
            if (tile.x < d.lm0 || tile.y > d.lm0 + d.L || tile.x >= tile.y) return bad(r.x, "tile outside its window");
            if (hb.lmObsBegin[tile.y] - hb.lmObsBegin[tile.x] > kMaxTrackChunk) return bad(r.x, "tile above 32 observations");
            for (int g = tile.x; g < tile.y; ++g) ++lmCover[g];
        }
    for (int g = 0; g < hb.totalLm; ++g)
        if (lmCover[g] != 1) return bad(-1, "runs do not cover every landmark once");
    std::vector<int> obCover(hb.totalObs, 0);
    for (const int4& c : hb.pairChunks) {
        const WinDesc& d = hb.win[c.x];
        if (c.y < d.obs0 || c.z > d.obs0 + d.F || c.z - c.y > hb.plan.pairChunk || c.y >= c.z) return bad(c.x, "pair chunk");
        for (int k = c.y; k < c.z; ++k) ++obCover[k];
    }
    for (int o = 0; o < hb.totalObs; ++o)
        if (obCover[o] != 1) return bad(-1, "pair chunks do not cover every observation once");
    std::vector<int> schCover(hb.totalLm, 0);
    for (const int4& c : hb.schurChunks) {
        const WinDesc& d = hb.win[c.x];
        if (c.y < d.lm0 || c.z > d.lm0 + d.L || c.y >= c.z || c.w < 0 || c.w >= (long long)hb.schurCols.size())
            return bad(c.x, "Schur chunk");
        const int nu = hb.schurCols[c.w];
        if (nu < 1 || nu > d.Npc || c.w + nu >= (long long)hb.schurCols.size() || !schurChunkFits(c.z - c.y, nu) ||
            c.z - c.y > hb.plan.schurRows)
            return bad(c.x, "Schur chunk columns");
        for (int k = 1; k <= nu; ++k) {
            const int col = hb.schurCols[c.w + k];
            if (col < 0 || col >= d.Npc || (k > 1 && col <= hb.schurCols[c.w + k - 1])) return bad(c.x, "Schur chunk column list");
        }
        for (int g = c.y; g < c.z; ++g) {
            ++schCover[g];
            const int ns = 6 * (hb.lmNs[g] + hb.lmNx[g]) + (d.estTd ? 1 : 0);
            for (int k = 0; k < ns; ++k)
                if (hb.lmUmap[hb.lmC0[g] + k] >= nu) return bad(c.x, "Schur chunk map");
        }
    }
    for (int g = 0; g < hb.totalLm; ++g)
        if (schCover[g] != 1) return bad(-1, "Schur chunks do not cover every landmark once");
    // deterministic units: a window's units tile its observations (pairs) and its Schur
    // chunks in slot order, and the slots stay inside the slot array
    if (hb.plan.deterministic) {
        std::vector<int> nextObs(count), nextChunk(count), nextPair(count, 0), nextSchur(count, 0);
        for (int i = 0; i < count; ++i) nextObs[i] = hb.win[i].obs0;
        for (int c = 0; c < (int)hb.schurChunks.size(); ++c)
            if (c == 0 || hb.schurChunks[c - 1].x != hb.schurChunks[c].x) nextChunk[hb.schurChunks[c].x] = c;
        for (const int4& u : hb.detPairs) {
            if (u.x < 0 || u.x >= count || u.w != nextPair[u.x] || u.y != nextObs[u.x] || u.z <= u.y) return bad(u.x, "pair unit");
            ++nextPair[u.x];
            nextObs[u.x] = u.z;
        }
        for (const int4& u : hb.detSchur) {
            if (u.w < 0 || u.w >= count || u.z != nextSchur[u.w] || u.x != nextChunk[u.w] || u.y <= u.x ||
                u.y > (int)hb.schurChunks.size() || hb.schurChunks[u.y - 1].x != u.w)
                return bad(u.w, "Schur unit");
            ++nextSchur[u.w];
            nextChunk[u.w] = u.y;
        }
        long long slots = 0;
        for (int i = 0; i < count; ++i) {
            const WinDesc& d = hb.win[i];
            if (nextPair[i] != d.detPairs || nextSchur[i] != d.detSchur || d.detPairs > kDetMaxSlots ||
                d.detSchur > kDetMaxSlots || (d.F > 0 && nextObs[i] != d.obs0 + d.F) || d.det0 != slots)
                return bad(i, "deterministic units do not cover the window");
            slots += (long long)(d.detPairs + d.detSchur) * ((long long)d.Npc * (d.Npc + 1) / 2 + d.Npc);
        }
        if (slots != hb.detSlots) return bad(-1, "deterministic slot array size");
    }
    return CGMLI_OK;
}

}  // namespace cgmli
