// sm_100a kernels of the sliding-window backend hot path.
//
// One LM iteration over a batch of windows is the launch sequence
//   zero_acc -> lin_landmark -> lin_pairs -> lin_schur -> retained -> factor
//   -> candidate -> backsub_trial -> retained_trial -> lm_update -> accept
// with every decision of the damped LM loop (BackendOptimizer.cpp:167-307)
// taken on the device from per-window state (WinLM), so that a whole solve
// runs without a host round trip and can be captured in a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "../../include/cgmli_backend.h"
#include "backend_internal.h"
#include "device_math.cuh"
#include "dense_tiles.cuh"
#include "factor_eval.cuh"

namespace cgmli {

__device__ __forceinline__ unsigned long long globalTimerNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warpMax(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// packed upper triangle, row-major: (i <= j)
__device__ __forceinline__ long long upIdx(int i, int j, int n) { return (long long)i * n - (long long)i * (i - 1) / 2 + (j - i); }
// packed lower triangle, column-major: (i >= j)
__device__ __forceinline__ int loIdx(int i, int j, int n) { return j * n - j * (j - 1) / 2 + (i - j); }

// Visual column of retained column c (or -1 for speed/bias columns).
__device__ __forceinline__ int pcOfRetained(int c, int K) {
    if (c >= 15 * K) return 6 * K + (c - 15 * K);
    const int w = c % 15;
    return w < 6 ? 6 * (c / 15) + w : -1;
}
__device__ __forceinline__ int retainedOfPc(int p, int K) {
    if (p >= 6 * K) return 15 * K + (p - 6 * K);
    return 15 * (p / 6) + (p % 6);
}

// ---------------------------------------------------------------------------------------
// Zeroes the visual accumulators: J^T J and J^T r of windows at a new point,
// the Schur term and B_v of every window still iterating (they depend on lambda).
// Accumulator of a window: [J^T J packed upper (Npc(Npc+1)/2) | unused Npc | G_v | B_v],
// Schur buffer: packed upper Npc(Npc+1)/2.
__global__ void k_zero_acc(DevBatch B) {
    const int w = blockIdx.x;
    const int mode = B.lm[w].mode;
    if (mode == kModeDone) return;
    const WinDesc& wd = B.win[w];
    const long long nS = (long long)wd.Npc * (wd.Npc + 1) / 2;
    double* acc = B.acc + wd.acc0;
    if (mode == kModeLinearize)
        for (long long i = threadIdx.x; i < nS + 2ll * wd.Npc; i += blockDim.x) acc[i] = 0.0;
    for (long long i = threadIdx.x; i < wd.Npc; i += blockDim.x) acc[nS + 2ll * wd.Npc + i] = 0.0;
    double* sch = B.sch + wd.sch0;
    for (long long i = threadIdx.x; i < nS; i += blockDim.x) sch[i] = 0.0;
    // rotations of the accepted state for this iteration's factors
    for (int k = threadIdx.x; k < wd.K; k += blockDim.x) poseRotation(B.pose[0] + 7ll * (wd.kf0 + k), B.rotKf[0] + 9ll * (wd.kf0 + k));
    for (int e = threadIdx.x; e < wd.E; e += blockDim.x) poseRotation(B.ext[0] + 7ll * (wd.ext0 + e), B.rotExt[0] + 9ll * (wd.ext0 + e));
}

// ---------------------------------------------------------------------------------------
// Linearization of the bearing factors and the per-landmark Schur complement
// at the window's current lambda (accumulateVisualPairs + subtractPointSchur,
// VisualCudaBatch.cu:74-96,149-161).  With J the weighted Jacobian rows over the
// visual columns and, per landmark l (scalar inverse distance),
//   d_l = sum J_rho^T J_rho,  g_l = sum J_rho^T r,  c_l = sum J_x^T J_rho,
//   dt_l = d_l + lambda max(d_l, 1e-6),
// the reduced visual system is
//   S_v = J^T J - sum_l c_l c_l^T / dt_l,   B_v = sum_l c_l g_l / dt_l.
// It is formed by three kernels:
//   k_lin_landmark  landmark order: c_l, d_l, g_l, cost, validity per landmark
//                   (no reductions into shared window state)
//   k_lin_pairs     observations sorted by (anchor keyframe, observer keyframe,
//                   anchor extrinsic, observer extrinsic): every observation of a
//                   key adds to the same entries of J^T J and J^T r, so a warp
//                   sums a key's observations in registers and adds them once
//   k_lin_schur     per window: the c_l / sqrt(dt_l) of a chunk of landmarks are
//                   expanded into dense shared-memory rows and the Schur term is
//                   a register-tiled FP64 SYRK (plus the B_v column)
// Only k_lin_schur depends on lambda, so a rejected step re-runs it alone.
constexpr int kCompact = 25;        // anchor pose 6 | observer pose 6 | ext_a 6 | ext_b 6 | td 1
constexpr int kPairWarps = 4;       // warps per CTA of k_lin_pairs
// A factor's FactorOut is staged per lane in shared memory with an odd stride
// (conflict-free lane rows); slot 54 carries the squared robust weight.
constexpr int kOut = 55;
static_assert(sizeof(FactorOut) == 54 * sizeof(double), "FactorOut layout: r, Ja, Jb, Jea, Jeb, Jtd, Jrho");
// Offset in FactorOut of row r of compact column c.
__device__ __forceinline__ int compactOff(int r, int c) { return c < 24 ? 2 + 12 * (c / 6) + 6 * r + c % 6 : 50 + r; }

// Local column -> visual column for a support (s keyframe slots, x extrinsic slots, td).
__device__ __forceinline__ int pcOfLocal(int i, int s, int x, const int* sk, int K, int tdCol) {
    if (i < 6 * s) return 6 * sk[i / 6] + i % 6;
    if (i < 6 * (s + x)) return 6 * K + 6 * sk[s + (i - 6 * s) / 6] + i % 6;
    return tdCol;
}

// ---- L1: per-landmark scalars and cross vectors --------------------------------------
// Work unit: a run = consecutive landmarks of one window processed by one warp in
// tiles of <= 32 observations (lane = observation for the evaluation).  Per-warp
// shared memory: 32 staged factors (overwritten in place by the weighted cross
// products J_x^T J_rho over the compact columns at [0, 25)), the compact -> local
// column maps, flags, and the landmark's cross vector (maxNs doubles, the batch's
// widest support).
//
// Mixed precision (Mixed = true): the factor is formed in FP64 as on the FP64 path,
// then its Jacobian blocks over the pose, extrinsic and td columns and its robust
// weight are rounded once to FP32.  Those FP32 values are what the linearization
// uses: the staged rows of the J^T J pass are stored in FP32 (half the bytes) and
// the landmark terms d_l, g_l and the cross products w^2 J_x^T J_rho are formed in
// FP64 from them, with the residual and the depth derivative J_rho kept FP64.  (An
// FP32 derivative chain, measured, saved 5% of this pass and put the configuration-2
// retained step 1.9e-6 away from FP64: its cancellations, not the storage rounding,
// set the error.)
__host__ __device__ constexpr size_t landmarkWarpBytes(int maxNs, bool) {
    return sizeof(double) * 32 * kOut + sizeof(double) * maxNs + sizeof(long long) * 32 + sizeof(short) * 32 * kCompact +
           sizeof(int) * 32;
}
// Staged row of one factor, written by k_lin_landmark (in observation order)
// and gathered in key order by k_lin_pairs.  FP64 (448 bytes): weighted J row 0
// over the compact columns [0, 25), row 1 [25, 50), weighted residual 50, 51, the
// packed key (anchor kf | observer kf << 16 | anchor ext << 32 | observer ext << 48,
// window-local) at 52; 53..55 pad.  Mixed (224 bytes): the weighted residual
// (2 doubles) at bytes [0, 16), the weighted J rows as 50 floats at [16, 216),
// the key at [216, 224).
constexpr int kKeyRow = 56;
constexpr int kKeyRowBytesF = 224;
__device__ __forceinline__ long long packKey(int a, int b, int ea, int eb) {
    return (long long)a | (long long)b << 16 | (long long)ea << 32 | (long long)eb << 48;
}

template <bool Mixed, int Warps, int MinBlocks>
__global__ void __launch_bounds__(Warps * 32, MinBlocks) k_lin_landmark(DevBatch B, const int4* runs, const int2* tiles, int maxNs) {
    extern __shared__ double smemRaw[];
    constexpr int kStride = kOut;
    using St = double;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int runIdx = blockIdx.x * Warps + warp;
    if (runIdx >= B.numRuns) return;
    const int4 run = runs[runIdx];  // {window, tile begin, tile end, -}
    const int wdx = run.x;
    if (B.lm[wdx].mode != kModeLinearize) return;
    char* base = reinterpret_cast<char*>(smemRaw) + landmarkWarpBytes(maxNs, Mixed) * warp;
    St* out = reinterpret_cast<St*>(base);
    double* cvec = out + 32 * kStride;
    long long* keys = reinterpret_cast<long long*>(cvec + maxNs);
    short* map = reinterpret_cast<short*>(keys + 32);
    int* flags = reinterpret_cast<int*>(map + 32 * kCompact);
    const WinDesc wd = B.win[wdx];
    for (int t = run.y; t < run.z; ++t) {
        const int2 tile = tiles[t];
        const int lb = tile.x, le = tile.y;
        const int ob = B.lmObsBegin[lb], oe = B.lmObsBegin[le];
        const int f = ob + lane;
        // per-landmark metadata of the tile, one landmark per lane (a tile holds <= 32 landmarks)
        const int nl = le - lb;
        int myBeg = 0, myEnd = 0, myNs = 0;
        long long myC0 = 0;
        if (lane < nl) {
            const int l = lb + lane;
            myBeg = B.lmObsBegin[l] - ob;
            myEnd = B.lmObsBegin[l + 1] - ob;
            myNs = 6 * (B.lmNs[l] + B.lmNx[l]) + (wd.estTd ? 1 : 0);
            myC0 = B.lmC0[l];
        }
        if (f < oe) {
            const int l = B.obLm[f];
            FactorIn in;
            int kfa, kfb, ea, eb;
            gatherFactor(B, wd, wdx, l, f, 0, in, kfa, kfb, ea, eb);
            St* st = out + kStride * lane;
            const bool ok = evalBearingFactor(in, true, *reinterpret_cast<FactorOut*>(st));
            const int s = B.lmNs[l], x = B.lmNx[l];
            const bool same = in.sameKf && !in.splitExt;
            const int obSlot = B.obSlot[f], obX = B.obXslot[f];
            short* mp = map + kCompact * lane;
            for (int c = 0; c < 6; ++c) {
                mp[c] = in.sameKf ? -1 : c;
                mp[6 + c] = in.sameKf ? -1 : 6 * obSlot + c;
                mp[12 + c] = (wd.estExt && !same) ? 6 * s + c : -1;  // anchor camera's extrinsic = ext slot 0
                mp[18 + c] = (wd.estExt && in.splitExt) ? 6 * (s + obX) + c : -1;
            }
            mp[24] = wd.estTd ? 6 * (s + x) : -1;
            flags[lane] = ok ? 1 : 0;
            keys[lane] = packKey(kfa - wd.kf0, kfb - wd.kf0, ea - wd.ext0, eb - wd.ext0);
            if (ok) {
                st[54] = huberWeight(wd.huber, st[0] * st[0] + st[1] * st[1]);
                if constexpr (Mixed) {  // the Jacobian blocks over the retained columns and the weight, rounded to FP32
#pragma unroll
                    for (int k = 2; k < 52; ++k) st[k] = (double)(float)st[k];
                    st[54] = (double)(float)st[54];
                }
            } else {
                for (int k = 0; k < kOut; ++k) st[k] = 0.0;
            }
        }
        __syncwarp();
        // weighted compact row of this lane's observation (unrolled: constant offsets)
        if (f < oe) {
            const St* st = out + kStride * lane;
            if constexpr (Mixed) {
                const float w = (float)st[54];
                char* row = reinterpret_cast<char*>(B.keyRows) + (size_t)f * kKeyRowBytesF;
                *reinterpret_cast<double2*>(row) = make_double2((double)w * st[0], (double)w * st[1]);
                float4* jr = reinterpret_cast<float4*>(row + 16);
                auto at = [&](int k) { return w * (float)st[k < 25 ? compactOff(0, k) : compactOff(1, k - 25)]; };
#pragma unroll
                for (int q = 0; q < 12; ++q) jr[q] = make_float4(at(4 * q), at(4 * q + 1), at(4 * q + 2), at(4 * q + 3));
                *reinterpret_cast<float2*>(row + 16 + 192) = make_float2(at(48), at(49));
                *reinterpret_cast<long long*>(row + 216) = keys[lane];
            } else {
                const double w = st[54];
                double2* row = reinterpret_cast<double2*>(B.keyRows + (size_t)f * kKeyRow);
#pragma unroll
                for (int q = 0; q < 25; ++q) {
                    const int c0 = 2 * q, c1 = 2 * q + 1;
                    row[q] = make_double2(w * st[c0 < 25 ? compactOff(0, c0) : compactOff(1, c0 - 25)],
                                          w * st[c1 < 25 ? compactOff(0, c1) : compactOff(1, c1 - 25)]);
                }
                row[25] = make_double2(w * st[0], w * st[1]);
                row[26] = make_double2(__longlong_as_double(keys[lane]), 0.0);
            }
        }
        __syncwarp();
        // this lane's contributions to d_l, g_l, the cost and (in place) the cross products
        const bool live = f < oe && flags[lane];
        double dD = 0.0, gD = 0.0, cost = 0.0;
        if (live) {
            St* st = out + kStride * lane;
            const double q0 = st[0], q1 = st[1], p0 = st[52], p1 = st[53];
            const double w = st[54], w2 = w * w;
            cost = huberCost(wd.huber, q0 * q0 + q1 * q1);
            dD = w2 * (p0 * p0 + p1 * p1);
            gD = w2 * (p0 * q0 + p1 * q1);
            // in place: column c reads offsets >= c + 2, all later than slot c
#pragma unroll
            for (int c = 0; c < kCompact; ++c) st[c] = w2 * (st[compactOff(0, c)] * p0 + st[compactOff(1, c)] * p1);
        }
        __syncwarp();
        // landmark sums of d, g, cost and validity: segmented inclusive scans over
        // the tile's lanes (observations of one landmark are consecutive lanes)
        {
            const int seg = B.obLm[f < oe ? f : ob] - lb;  // landmark of this lane (lanes past the tile: any)
            int bad = f < oe && !flags[lane] ? 1 : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double c2 = __shfl_up_sync(0xffffffffu, cost, o);
                const int b2 = __shfl_up_sync(0xffffffffu, bad, o), s2 = __shfl_up_sync(0xffffffffu, seg, o);
                const double d2 = __shfl_up_sync(0xffffffffu, dD, o), g2 = __shfl_up_sync(0xffffffffu, gD, o);
                if (lane >= o && s2 == seg) { dD += d2; gD += g2; cost += c2; bad |= b2; }
            }
            // the last lane of each landmark holds its sums
            const int nextSeg = __shfl_down_sync(0xffffffffu, seg, 1);
            if (f < oe && (lane == 31 || f + 1 >= oe || nextSeg != seg)) {
                const int l = lb + seg;
                B.lmD[l] = dD; B.lmG[l] = gD; B.lmCost[l] = cost; B.lmValid[l] = bad ? 0 : 1;
            }
        }
        // cross vectors c_l: lane c < 25 owns compact column c, whose local column
        // is the same run after run of observations (anchor pose, anchor
        // extrinsic, td) or changes only with the observer (observer pose and
        // extrinsic); different lanes never share a local column, so each lane
        // sums in a register and adds to the landmark's vector when its column changes
        for (int q = 0; q < nl; ++q) {
            const int fb = __shfl_sync(0xffffffffu, myBeg, q), fe = __shfl_sync(0xffffffffu, myEnd, q);
            const int ns = __shfl_sync(0xffffffffu, myNs, q);
            const long long c0 = __shfl_sync(0xffffffffu, myC0, q);
            if (fb == fe && lane == 0) {  // no observation in the window: nothing was summed above
                const int l = lb + q;
                B.lmD[l] = 0.0; B.lmG[l] = 0.0; B.lmCost[l] = 0.0; B.lmValid[l] = 1;
            }
            for (int i = lane; i < ns; i += 32) cvec[i] = 0.0;
            __syncwarp();
            if (lane < kCompact) {
                int cur = -1;
                double accv = 0.0;
                for (int k = fb; k < fe; ++k) {
                    const int li = map[kCompact * k + lane];
                    if (li != cur) {
                        if (cur >= 0) cvec[cur] += accv;
                        cur = li;
                        accv = 0.0;
                    }
                    if (li >= 0 && flags[k]) accv += out[kOut * k + lane];
                }
                if (cur >= 0) cvec[cur] += accv;
            }
            __syncwarp();
            for (int i = lane; i < ns; i += 32) B.lmC[c0 + i] = cvec[i];
            __syncwarp();
        }
    }
}

// ---- L2: J^T J and J^T r by observation key ------------------------------------------
// Work unit: a chunk of <= 32 consecutive positions of one window's key order.
// The warp gathers the chunk's staged rows (written by k_lin_landmark) into
// shared memory, kPairRows at a time.  For each run of equal keys the Gram matrix G = J'^T J' of the
// run's weighted rows is formed on the FP64 tensor path (mma.sync m8n8k4):
// J' is the 2x25 compact Jacobian of each observation with the weighted
// residual appended as column 25 and zero-padded to 32 columns, so that G's
// upper 25x25 block is J^T J and G[i][25] = (J^T r)_i.  One k-step of 4 rows
// covers two observations; the ten upper 8x8 tiles of the 32x32 G live in
// registers (two doubles per lane each) and are added to the window once per run.
constexpr int kPairStride = kKeyRow + 1;  // odd stride
constexpr int kPairRows = 16;             // rows staged per round: small staging, more resident warps
__host__ __device__ constexpr size_t pairCtaBytes() { return sizeof(double) * kPairWarps * kPairRows * kPairStride; }

__device__ __forceinline__ void mmaF64(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

//
// Det: the work unit is a deterministic unit {window, first position, end, slot}
// (several consecutive chunks of one window); its sums go with plain adds into the
// unit's own slot, which only this warp writes, and k_det_reduce adds a window's
// slots in unit order.
template <bool Mixed, bool Det>
__global__ void __launch_bounds__(kPairWarps * 32) k_lin_pairs(DevBatch B, const int4* chunks, int numChunks) {
    extern __shared__ double smemRaw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ci = blockIdx.x * kPairWarps + warp;
    if (ci >= numChunks) return;
    const int4 ch = chunks[ci];  // {window, first key-ordered position, end, - or slot}
    const int wdx = ch.x;
    if (B.lm[wdx].mode != kModeLinearize) return;
    double* rows = smemRaw + (size_t)warp * kPairRows * kPairStride;
    const WinDesc wd = B.win[wdx];
    const int K = wd.K, Npc = wd.Npc;
    const int tdCol = 6 * K + (wd.estExt ? 6 * wd.E : 0);
    const long long tri = (long long)Npc * (Npc + 1) / 2;
    double* JJ;
    double* Gv;
    if constexpr (Det) {
        JJ = B.detSlots + wd.det0 + (long long)ch.w * (tri + Npc);
        Gv = JJ + tri;
        for (long long e = lane; e < tri + Npc; e += 32) JJ[e] = 0.0;
        __syncwarp();
    } else {
        JJ = B.acc + wd.acc0;
        Gv = JJ + tri + Npc;
    }
    // fragment coordinates: k-step row kr = lane % 4 (observation kr / 2, row kr % 2),
    // column lane / 4 within an 8-column block; accumulator row lane / 4, columns 2 (lane % 4) + {0, 1}
    const int kr = lane & 3, cIn = lane >> 2;
    double g[10][2];
#pragma unroll
    for (int t = 0; t < 10; ++t) g[t][0] = g[t][1] = 0.0;
    long long cur = -1;  // key of the run held in g
    auto flush = [&]() {
        if (cur < 0) return;
        const int ka = (int)(cur & 0xffff), kb = (int)((cur >> 16) & 0xffff);
        const int xa = (int)((cur >> 32) & 0xffff), xb = (int)((cur >> 48) & 0xffff);
        const bool sameKf = ka == kb, split = xa != xb, same = sameKf && !split;
        auto colOf = [&](int c) -> int {
            if (c < 6) return sameKf ? -1 : 6 * ka + c;
            if (c < 12) return sameKf ? -1 : 6 * kb + c - 6;
            if (c < 18) return (wd.estExt && !same) ? 6 * K + 6 * xa + c - 12 : -1;
            if (c < 24) return (wd.estExt && split) ? 6 * K + 6 * xb + c - 18 : -1;
            return wd.estTd ? tdCol : -1;
        };
        if constexpr (!Det) {
            int t = 0;
#pragma unroll
            for (int I = 0; I < 4; ++I)
#pragma unroll
                for (int J = I; J < 4; ++J, ++t)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int i = 8 * I + cIn, j = 8 * J + 2 * kr + e;
                        const double v = g[t][e];
                        g[t][e] = 0.0;
                        if (v == 0.0 || i > j || i >= 25 || j > 25) continue;
                        const int ci2 = colOf(i);
                        if (ci2 < 0) continue;
                        if (j == 25) { atomicAdd(&Gv[ci2], v); continue; }
                        const int cj = colOf(j);
                        if (cj < 0) continue;
                        atomicAdd(&JJ[ci2 <= cj ? upIdx(ci2, cj, Npc) : upIdx(cj, ci2, Npc)], v);
                    }
            cur = -1;
            return;
        }
        // Det: destination of each held entry (offset from the slot: G_v follows the
        // triangle), -1: none
        int off[10][2];
        int t = 0;
#pragma unroll
        for (int I = 0; I < 4; ++I)
#pragma unroll
            for (int J = I; J < 4; ++J, ++t)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int i = 8 * I + cIn, j = 8 * J + 2 * kr + e;
                    off[t][e] = -1;
                    if (g[t][e] == 0.0 || i > j || i >= 25 || j > 25) continue;
                    const int ci2 = colOf(i);
                    if (ci2 < 0) continue;
                    if (j == 25) {
                        off[t][e] = (int)(Gv - JJ) + ci2;
                    } else {
                        const int cj = colOf(j);
                        if (cj >= 0) off[t][e] = (int)(ci2 <= cj ? upIdx(ci2, cj, Npc) : upIdx(cj, ci2, Npc));
                    }
                }
        // one run's entries land on distinct destinations (colOf is injective): every
        // load is issued before any store, so they overlap
        double old[10][2];
#pragma unroll
        for (int q = 0; q < 10; ++q)
#pragma unroll
            for (int e = 0; e < 2; ++e) old[q][e] = off[q][e] >= 0 ? JJ[off[q][e]] : 0.0;
#pragma unroll
        for (int q = 0; q < 10; ++q)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (off[q][e] >= 0) JJ[off[q][e]] = old[q][e] + g[q][e];
                g[q][e] = 0.0;
            }
        __syncwarp();  // the next run's adds may reach the same entries from other lanes
        cur = -1;
    };
    // the chunk is staged kPairRows rows at a time; a run of equal keys that
    // continues into the next round keeps its sums in registers
    for (int h0 = ch.y; h0 < ch.z; h0 += kPairRows) {
        const int n = min(kPairRows, ch.z - h0);
        if (lane < n) {  // gather: each lane loads its own key-ordered row (unrolled 16-byte loads)
            double* dst = rows + lane * kPairStride;
            if constexpr (Mixed) {  // FP32 rows widened to FP64 for the Gram matrices
                const char* src = reinterpret_cast<const char*>(B.keyRows) + (size_t)B.keyOrder[h0 + lane] * kKeyRowBytesF;
                const double2 rv = *reinterpret_cast<const double2*>(src);
                const float4* js = reinterpret_cast<const float4*>(src + 16);
#pragma unroll
                for (int q = 0; q < 12; ++q) {
                    const float4 v = js[q];
                    dst[4 * q] = v.x; dst[4 * q + 1] = v.y; dst[4 * q + 2] = v.z; dst[4 * q + 3] = v.w;
                }
                const float2 t = *reinterpret_cast<const float2*>(src + 16 + 192);
                dst[48] = t.x; dst[49] = t.y;
                dst[50] = rv.x; dst[51] = rv.y;
                dst[52] = __longlong_as_double(*reinterpret_cast<const long long*>(src + 216));
            } else {
                const double2* src = reinterpret_cast<const double2*>(B.keyRows + (size_t)B.keyOrder[h0 + lane] * kKeyRow);
#pragma unroll
                for (int q = 0; q < 27; ++q) {
                    const double2 v = src[q];
                    dst[2 * q] = v.x;
                    dst[2 * q + 1] = v.y;
                }
            }
        }
        __syncwarp();
        const long long key = lane < n ? __double_as_longlong(rows[lane * kPairStride + 52]) : -1ll;
        const long long prev = __shfl_up_sync(0xffffffffu, key, 1);
        unsigned starts = __ballot_sync(0xffffffffu, lane < n && (lane == 0 || prev != key));
        while (starts) {
            const int s0 = __ffs(starts) - 1;
            starts &= starts - 1;
            const int s1 = starts ? __ffs(starts) - 1 : n;
            const long long kk = __shfl_sync(0xffffffffu, key, s0);
            if (kk != cur) {
                flush();
                cur = kk;
            }
            for (int m = s0; m < s1; m += 2) {
                const int o = m + (kr >> 1), r = kr & 1;
                double frag[4];
#pragma unroll
                for (int I = 0; I < 4; ++I) {
                    const int col = 8 * I + cIn;
                    double v = 0.0;
                    if (o < s1) {
                        const double* st = rows + o * kPairStride;
                        v = col < 25 ? st[25 * r + col] : (col == 25 ? st[50 + r] : 0.0);
                    }
                    frag[I] = v;
                }
                int t = 0;
#pragma unroll
                for (int I = 0; I < 4; ++I)
#pragma unroll
                    for (int J = I; J < 4; ++J, ++t) mmaF64(g[t][0], g[t][1], frag[I], frag[J]);
            }
        }
        __syncwarp();  // the next round's gather overwrites the staged rows
    }
    flush();
}

// ---- L3: Schur term as a compact SYRK per chunk of landmarks -------------------------
// A chunk is a run of consecutive landmarks (support-sorted, so neighbours share
// most columns) with the ascending union U of their visual support columns.
// Each landmark's row c_l / sqrt(dt_l) is expanded over U in shared memory (its
// local -> U map is built on the host), with g_l / sqrt(dt_l) as column |U| for
// B_v.  The rank update uses 32 x 32 tiles, one per warp, on the FP64 tensor
// path (mma.sync m8n8k4, dense_tiles.cuh);
// spare warps split the rows when the tiles are fewer than the warps.  Every
// tile is added to the window's Schur sum once per chunk.
// One chunk into sch / Bv (the window's sums, or in Det mode the unit's slot: its
// tiles' parts then add in a fixed order with plain adds).
template <bool Det>
__device__ __forceinline__ void schurChunk(const DevBatch& B, const int4 ch, const WinDesc& wd, double lambda, double* sch,
                                           double* Bv, double* Rw) {
    const int nu = B.schurCols[ch.w];
    const int* U = B.schurCols + ch.w + 1;
    const int n = nu + 1, np = (n + 31) & ~31, nb = np >> 5, ntiles = nb * (nb + 1) / 2;
    const int rows = ch.z - ch.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int nw = kSchurThreads / 32;
    for (int r = warp; r < rows; r += nw) {
        const int l = ch.y + r;
        const int ns = 6 * (B.lmNs[l] + B.lmNx[l]) + (wd.estTd ? 1 : 0);
        const double d = B.lmD[l];
        // a landmark held constant is not eliminated: its row stays zero
        const double scale = wd.fixedLm && B.lmFixed[l] ? 0.0 : 1.0 / sqrt(d + lambda * fmax(d, 1e-6));
        const long long c0 = B.lmC0[l];
        double* row = Rw + (long long)r * np;
        for (int c = lane; c < np; c += 32) row[c] = 0.0;
        __syncwarp();
        for (int i = lane; i < ns; i += 32) row[B.lmUmap[c0 + i]] = scale * B.lmC[c0 + i];
        if (lane == 0) row[nu] = scale * B.lmG[l];
    }
    __syncthreads();
    const int wpt = ntiles < nw ? nw / ntiles : 1;  // warps per tile (row split)
    auto addTile = [&](const double (&acc)[4][8], int bi, int bj) {
        if constexpr (!Det) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int i = tileRowMma(bi, lane, r);
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int j = tileCol(bj, lane, c);
                    const double v = acc[r][c];
                    if (i > j || j >= n || i >= nu || v == 0.0) continue;
                    atomicAdd(j < nu ? sch + upIdx(U[i], U[j], wd.Npc) : Bv + U[i], v);
                }
            }
        } else {
            // a tile's entries land on distinct destinations: per half tile every load is
            // issued before any store, so they overlap
            const int bvOff = (int)(Bv - sch);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                int off[2][8];
                double old[2][8];
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                    const int i = tileRowMma(bi, lane, 2 * h + r);
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const int j = tileCol(bj, lane, c);
                        off[r][c] = (i > j || j >= n || i >= nu || acc[2 * h + r][c] == 0.0)
                                        ? -1
                                        : (j < nu ? (int)upIdx(U[i], U[j], wd.Npc) : bvOff + U[i]);
                    }
                }
#pragma unroll
                for (int r = 0; r < 2; ++r)
#pragma unroll
                    for (int c = 0; c < 8; ++c) old[r][c] = off[r][c] >= 0 ? sch[off[r][c]] : 0.0;
#pragma unroll
                for (int r = 0; r < 2; ++r)
#pragma unroll
                    for (int c = 0; c < 8; ++c)
                        if (off[r][c] >= 0) sch[off[r][c]] = old[r][c] + acc[2 * h + r][c];
            }
        }
    };
    if constexpr (!Det) {
        for (int u = warp; u < ntiles * wpt; u += nw) {
            const int t = u / wpt, part = u % wpt;
            int bi, bj;
            tileOf(t, nb, bi, bj);
            double acc[4][8];
            zeroTile(acc);
            rankUpdateMma<false>(acc, Rw, bi * 32, bj * 32, part, rows, wpt, np);
            addTile(acc, bi, bj);
        }
    } else {
        // every warp runs the same rounds; a tile's parts (wpt > 1: one round, one part
        // per warp) add in part order between barriers, distinct tiles never collide
        for (int u0 = 0; u0 < ntiles * wpt; u0 += nw) {
            const int u = u0 + warp;
            const bool active = u < ntiles * wpt;
            const int t = u / wpt, part = u % wpt;
            int bi = 0, bj = 0;
            double acc[4][8];
            zeroTile(acc);
            if (active) {
                tileOf(t, nb, bi, bj);
                rankUpdateMma<false>(acc, Rw, bi * 32, bj * 32, part, rows, wpt, np);
            }
            for (int p = 0; p < wpt; ++p) {
                __syncthreads();
                if (active && part == p) addTile(acc, bi, bj);
            }
        }
    }
}

__global__ void __launch_bounds__(kSchurThreads, 3) k_lin_schur(DevBatch B, const int4* chunks) {
    extern __shared__ __align__(16) double Rw[];
    const int4 ch = chunks[blockIdx.x];  // {window, first landmark, end landmark, offset of the column list}
    const int wdx = ch.x;
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const long long tri = (long long)wd.Npc * (wd.Npc + 1) / 2;
    schurChunk<false>(B, ch, wd, B.lm[wdx].lambda, B.sch + wd.sch0, B.acc + wd.acc0 + tri + 2ll * wd.Npc, Rw);
}

// Deterministic Schur pass: a unit {first chunk, end chunk, slot, window} of one
// window's consecutive chunks per CTA, summed in chunk order into the unit's slot.
__global__ void __launch_bounds__(kSchurThreads, 2) k_lin_schur_det(DevBatch B, const int4* chunks, const int4* units) {
    extern __shared__ __align__(16) double Rw[];
    const int4 un = units[blockIdx.x];
    const int wdx = un.w;
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const long long tri = (long long)wd.Npc * (wd.Npc + 1) / 2;
    double* slot = B.detSlots + wd.det0 + (long long)(wd.detPairs + un.z) * (tri + wd.Npc);
    for (long long e = threadIdx.x; e < tri + wd.Npc; e += blockDim.x) slot[e] = 0.0;
    const double lambda = B.lm[wdx].lambda;
    for (int c = un.x; c < un.y; ++c) {
        __syncthreads();  // the slot is cleared / the previous chunk's rows and adds are done
        schurChunk<true>(B, chunks[c], wd, lambda, slot, slot + tri, Rw);
    }
}

// Deterministic mode: a window's sums from its units' slots, added in unit order
// (J^T J and G_v of windows at a new point, the Schur term and B_v of every window
// still iterating: the entries k_zero_acc cleared).
__global__ void k_det_reduce(DevBatch B) {
    const int w = blockIdx.x;
    const int mode = B.lm[w].mode;
    if (mode == kModeDone) return;
    const WinDesc wd = B.win[w];
    const int Npc = wd.Npc;
    const long long tri = (long long)Npc * (Npc + 1) / 2, len = tri + Npc;
    const double* slots = B.detSlots + wd.det0;
    double* JJ = B.acc + wd.acc0;
    double* sch = B.sch + wd.sch0;
    for (long long e = (long long)blockIdx.y * blockDim.x + threadIdx.x; e < len; e += (long long)gridDim.y * blockDim.x) {
        if (mode == kModeLinearize && wd.detPairs > 0) {
            double v = 0.0;
            for (int k = 0; k < wd.detPairs; ++k) v += slots[(long long)k * len + e];
            if (e < tri) JJ[e] = v;
            else JJ[tri + Npc + (e - tri)] = v;  // G_v
        }
        if (wd.detSchur > 0) {
            double v = 0.0;
            for (int k = 0; k < wd.detSchur; ++k) v += slots[(long long)(wd.detPairs + k) * len + e];
            if (e < tri) sch[e] = v;
            else JJ[tri + 2ll * Npc + (e - tri)] = v;  // B_v
        }
    }
}

// ---------------------------------------------------------------------------------------
__device__ double blockSum(double v, double* red) {
    v = warpSum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0;
    for (int i = 0; i < nw; ++i) t += red[i];
    __syncthreads();
    return t;
}

// Retained (IMU + prior) normal blocks of each window that is at a new point:
// evaluateRetained + accumulateRetained (VisualCudaBatch.cu:626-642) written
// as block-structured accumulation.  Also evaluates the residual cost of the
// candidate state when `trial` is set (launchTrial, :715-721).
__global__ void __launch_bounds__(256, 2) k_retained(DevBatch B, int trial) {
    const int wdx = B.bigFirst[blockIdx.x];
    const int mode = B.lm[wdx].mode;
    if (mode == kModeDone || (!trial && mode != kModeLinearize)) return;
    const WinDesc wd = B.win[wdx];
    const int Nr = wd.Nr, buf = trial ? 1 : 0;
    __shared__ double red[32];
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    double* H = B.Hret + wd.dense0;
    double* g = B.gret + wd.vec0;
    // IMU factors: per factor 930 doubles of scratch, the raw error and Jacobian
    // [e 15 | U 450] (one thread each, U cleared beforehand by the whole CTA), then the
    // whitened [r 15 | J 450] = W [e | U] with one thread per output entry, which also
    // finds a non-finite U (every entry of U enters one of those sums)
    double* scratch = B.imuScratch + wd.imuScratch0;
    if (!trial) {
        for (long long i = threadIdx.x; i < (long long)Nr * Nr; i += blockDim.x) H[i] = 0.0;
        for (int i = threadIdx.x; i < Nr; i += blockDim.x) g[i] = 0.0;
        for (int t = threadIdx.x; t < 450 * wd.nImu; t += blockDim.x) scratch[930ll * (t / 450) + 15 + t % 450] = 0.0;
    }
    __syncthreads();
    double cost = 0;
    const cgmli_frozen_imu* imus = reinterpret_cast<const cgmli_frozen_imu*>(B.imu);
    for (int i = threadIdx.x; i < wd.nImu; i += blockDim.x) {
        const int gi = wd.imu0 + i;
        const int k = B.imuKf[gi];
        double* raw = scratch + 930ll * i;
        if (!evalImuRaw(imus[gi], B.pose[buf] + 7ll * k, B.sb[buf] + 9ll * k, B.pose[buf] + 7ll * (k + 1), B.sb[buf] + 9ll * (k + 1),
                        raw, trial ? nullptr : raw + 15, true))
            atomicOr(&bad, 1);
    }
    __syncthreads();
    {
        const int outs = trial ? 15 : 465;
        for (int t = threadIdx.x; t < wd.nImu * outs; t += blockDim.x) {
            const int f = t / outs, o = t % outs;
            const double* W = imus[wd.imu0 + f].whitening;  // column-major 15 x 15
            double* raw = scratch + 930ll * f;
            // o < 15: residual row o; else Jacobian entry (row, column) of o - 15
            const int row = o < 15 ? o : (o - 15) / 30;
            const double* x = o < 15 ? raw : raw + 15 + (o - 15) % 30;
            const int stride = o < 15 ? 1 : 30;
            double v = 0;
            for (int m = 0; m < 15; ++m) v += W[row + 15 * m] * x[stride * m];
            raw[465 + o] = v;
            if (!isfinite(v)) atomicOr(&bad, 1);
            if (o < 15) cost += 0.5 * v * v;
        }
    }
    __syncthreads();
    if (!trial) {
        for (long long t = threadIdx.x; t < 930ll * wd.nImu; t += blockDim.x) {
            const int i = (int)(t / 930), e = (int)(t % 930);
            const int k = B.imuKf[wd.imu0 + i] - wd.kf0;
            const double* r = scratch + 930ll * i + 465;
            const double* J = r + 15;
            const int a = e < 900 ? e / 30 : e - 900, b = e % 30;
            double v = 0;
            if (e < 900) {
                for (int m = 0; m < 15; ++m) v += J[30 * m + a] * J[30 * m + b];
                atomicAdd(&H[(long long)(15 * k + a) * Nr + 15 * k + b], v);
            } else {
                for (int m = 0; m < 15; ++m) v += J[30 * m + a] * r[m];
                atomicAdd(&g[15 * k + a], v);
            }
        }
        __syncthreads();
    }
    if (wd.priorRank > 0) {
        const int rank = wd.priorRank, cols = wd.priorCols;  // cols <= kPriorMaxCols (host check)
        double* ps = B.priorScratch + wd.priorScratch0;
        double* delta = ps;           // cols
        double* D = delta + cols;     // cols x 6
        double* r = D + 6ll * cols;   // rank
        double* J = r + rank;         // rank x cols
        // per prior column: its retained column (-1: none) and its block's first column,
        // negated minus one for a block whose tangent is its ambient (speed/bias, td)
        __shared__ int pcol[kPriorMaxCols], poff[kPriorMaxCols];
        for (int b = threadIdx.x; b < wd.priorBlocks; b += blockDim.x) {
            const int pb = wd.priorBlk0 + b;
            const int kind = B.priorKind[pb], off = B.priorOff[pb];
            const int width = kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 6, col = B.priorCol[pb];
            const bool chart = kind == CGMLI_PRIOR_POSE || kind == CGMLI_PRIOR_EXTRINSIC;
            for (int c = 0; c < width; ++c) {
                pcol[off + c] = col < 0 ? -1 : col + c;
                poff[off + c] = chart ? off : -1 - off;
            }
            const double* x = blockValue(B, buf, kind, B.priorIndex[pb], wdx);
            // reference offset: ambient sizes accumulate in block order
            int aoff = 0;
            for (int q = wd.priorBlk0; q < pb; ++q) {
                const int kq = B.priorKind[q];
                aoff += kq == CGMLI_PRIOR_SPEED_BIAS ? 9 : kq == CGMLI_PRIOR_TIME_OFFSET ? 1 : 7;
            }
            const double* ref = B.priorRef + wd.priorRef0 + aoff;
            if (kind == CGMLI_PRIOR_POSE || kind == CGMLI_PRIOR_EXTRINSIC) {
                poseMinus(x, ref, delta + off);
                if (!trial) se3LeftJacobianInverse(delta + off, D + 6ll * off);
            } else {
                const int t = kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : 1;
                for (int i = 0; i < t; ++i) delta[off + i] = x[i] - ref[i];
            }
        }
        __syncthreads();
        const double* A = B.priorA + wd.priorA0;
        const double* r0 = B.priorR0 + wd.priorR00;
        for (int i = threadIdx.x; i < rank; i += blockDim.x) {
            double v = r0[i];
            for (int c = 0; c < cols; ++c) v += A[(long long)i * cols + c] * delta[c];
            r[i] = v;
            if (!isfinite(v)) atomicOr(&bad, 1);
            cost += 0.5 * v * v;
        }
        if (!trial) {
            // J = A * blockdiag(D)
            for (long long e = threadIdx.x; e < (long long)rank * cols; e += blockDim.x) {
                const int i = (int)(e / cols), c = (int)(e % cols), po = poff[c];
                double v;
                if (po >= 0) {
                    v = 0;
                    for (int j = 0; j < 6; ++j) v += A[(long long)i * cols + po + j] * D[6ll * (po + j) + (c - po)];
                } else {
                    v = A[(long long)i * cols + c];
                }
                J[e] = v;
            }
            __syncthreads();
            // J^T J on the upper triangle, written to both halves, and J^T r
            for (long long e = threadIdx.x; e < (long long)cols * (cols + 1); e += blockDim.x) {
                const int p = (int)(e / cols), q = (int)(e % cols);
                if (p < cols) {
                    const int rp = pcol[p], rq = pcol[q];
                    if (p > q || rp < 0 || rq < 0) continue;
                    double v = 0;
                    for (int i = 0; i < rank; ++i) v += J[(long long)i * cols + p] * J[(long long)i * cols + q];
                    H[(long long)rp * Nr + rq] += v;
                    if (p != q) H[(long long)rq * Nr + rp] += v;
                } else {
                    const int rq = pcol[q];
                    if (rq < 0) continue;
                    double v = 0;
                    for (int i = 0; i < rank; ++i) v += J[(long long)i * cols + q] * r[i];
                    g[rq] += v;
                }
            }
        }
    }
    cost = blockSum(cost, red);
    if (threadIdx.x == 0) {
        if (trial) { B.trialRet[wdx] = cost; B.retValid[wdx] = bad ? 0 : 1; }
        else { B.costRet[wdx] = cost; B.retValid[wdx] = bad ? 0 : 1; }
    }
}

// ---------------------------------------------------------------------------------------
// Damped reduced system, FP64 Cholesky and solve (prepareStateSolve + potrf +
// potrs + clampStateStep + statePrediction, VisualCudaBatch.cu:163-189,564-580).
//   S = H_ret + S_visual + lambda * max(diag(H_total), 1e-6),  rhs = -(g_r - B_v)

// Blocked right-looking Cholesky of one window per CTA.  The damped system is
// assembled into the window's slot of Sglob (n x n column-major, lower
// triangle; L2-resident), factored panel by panel: a panel of kPanel columns
// is staged in shared memory and factored there, then the trailing lower
// triangle is updated with 4x4 register tiles (A22 -= L21 L21^T).  The
// triangular solves proceed by the same panels, with each 16x16 diagonal
// block in shared memory.
constexpr int kPanel = 16;

// Entry (i, j) of the damped (or undamped) reduced system, reading the
// symmetric H_ret along the column j so that consecutive i are coalesced.
__device__ __forceinline__ double assembleEntryCol(const DevBatch& B, const WinDesc& wd, int i, int j, double lambda, bool damp) {
    const int Nr = wd.Nr, Npc = wd.Npc, K = wd.K;
    const double* JJ = B.acc + wd.acc0;
    const double* sch = B.sch + wd.sch0;
    double v = B.Hret[wd.dense0 + (long long)j * Nr + i];
    const int pi = pcOfRetained(i, K), pj = pcOfRetained(j, K);
    if (pi >= 0 && pj >= 0) {
        const long long e = pi <= pj ? upIdx(pi, pj, Npc) : upIdx(pj, pi, Npc);
        v += JJ[e] - sch[e];
    }
    if (damp && i == j) {
        double h = B.Hret[wd.dense0 + (long long)i * Nr + i];
        if (pi >= 0) h += JJ[upIdx(pi, pi, Npc)];
        v += lambda * fmax(h, 1e-6);
    }
    return v;
}

// (a, b) with b <= a from the column-by-column enumeration of the lower
// triangle of an m x m tile grid (index of (a, b) = b m - b (b - 1) / 2 + a - b).
__device__ __forceinline__ void lowerTile(int t, int m, int& a, int& b) {
    b = (int)((2.0f * m + 1 - sqrtf((2.0f * m + 1) * (2.0f * m + 1) - 8.0f * t)) * 0.5f);
    if (b < 0) b = 0;
    while (b > 0 && b * m - b * (b - 1) / 2 > t) --b;
    while ((b + 1) * m - (b + 1) * b / 2 <= t) ++b;
    a = b + (t - (b * m - b * (b - 1) / 2));
}

// Solves L y = v (forward) then L^T z = y (backward) in place; L lower,
// column-major with leading dimension n, in global memory.
__device__ void blockedSolve(const double* L, int n, double* v, double* blk) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    for (int k0 = 0; k0 < n; k0 += kPanel) {
        const int bw = min(kPanel, n - k0);
        for (int t = tid; t < bw * bw; t += blockDim.x) {
            const int c = t / bw, r = t % bw;
            blk[r + c * kPanel] = r >= c ? L[(k0 + r) + (long long)(k0 + c) * n] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            for (int c = 0; c < bw; ++c) {
                const double yc = v[k0 + c] / blk[c + c * kPanel];
                __syncwarp();
                if (lane == 0) v[k0 + c] = yc;
                if (lane > c && lane < bw) v[k0 + lane] -= blk[lane + c * kPanel] * yc;
                __syncwarp();
            }
        }
        __syncthreads();
        for (int r = k0 + bw + tid; r < n; r += blockDim.x) {
            double s0 = 0, s1 = 0;
            int c = 0;
            for (; c + 2 <= bw; c += 2) {
                s0 += L[r + (long long)(k0 + c) * n] * v[k0 + c];
                s1 += L[r + (long long)(k0 + c + 1) * n] * v[k0 + c + 1];
            }
            if (c < bw) s0 += L[r + (long long)(k0 + c) * n] * v[k0 + c];
            v[r] -= s0 + s1;
        }
        __syncthreads();
    }
    for (int k0 = ((n - 1) / kPanel) * kPanel; k0 >= 0; k0 -= kPanel) {
        const int bw = min(kPanel, n - k0);
        // v[k0 + c] -= sum_{r >= k0 + bw} L[r, k0 + c] v[r]
        for (int c = warp; c < bw; c += nw) {
            double s0 = 0, s1 = 0;
            int r = k0 + bw + lane;
            for (; r + 32 < n; r += 64) {
                s0 += L[r + (long long)(k0 + c) * n] * v[r];
                s1 += L[r + 32 + (long long)(k0 + c) * n] * v[r + 32];
            }
            if (r < n) s0 += L[r + (long long)(k0 + c) * n] * v[r];
            const double s = warpSum(s0 + s1);
            if (lane == 0) v[k0 + c] -= s;
        }
        for (int t = tid; t < bw * bw; t += blockDim.x) {
            const int c = t / bw, r = t % bw;
            blk[r + c * kPanel] = r >= c ? L[(k0 + r) + (long long)(k0 + c) * n] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            for (int c = bw - 1; c >= 0; --c) {
                double s = (lane > c && lane < bw) ? blk[lane + c * kPanel] * v[k0 + lane] : 0.0;
                s = warpSum(s);
                if (lane == 0) v[k0 + c] = (v[k0 + c] - s) / blk[c + c * kPanel];
                __syncwarp();
            }
        }
        __syncthreads();
    }
}

// Factorization panels of kFacPanel columns: the panel (rows k0.. of its
// columns, padded to a multiple of 32 rows) is staged in shared memory and
// factored left-looking by the whole CTA (column c of every row is reduced by
// one dot product against the panel's earlier columns, then scaled), together
// with the forward substitution of the right-hand side over the panel's
// diagonal block.
// The trailing lower triangle is then updated from the staged panel with the
// 32 x 32 register tiles of dense_tiles.cuh (all warps), and the right-hand
// side below the panel by a GEMV.  The backward substitution runs over the
// same panels.  The undamped assembled system is kept in the strict upper
// triangle of the window's slot (the factor uses the lower one) and its
// diagonal in shared memory, for the prediction (and refinement) products.
constexpr int kFacPanel = 32;

// a[0..32) of every lane -> the warp's sum of a[lane] in lane `lane`, by recursive
// halving: at offset o each lane keeps the half of its entries its bit o selects and
// adds its partner's copy of that half (31 shuffles for 32 sums instead of 160).
__device__ __forceinline__ double transposeSum(double (&a)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const bool hi = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < o; ++k) {
            const double send = hi ? a[k] : a[k + o];
            const double keep = hi ? a[k + o] : a[k];
            a[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return a[0];
}

// h = S_undamped v from the stored upper triangle (A[p + q n], p < q) and diagonal hd:
// a thread per row for the columns right of the diagonal (consecutive rows coalesce,
// four independent sums keep four loads in flight), a warp per column for the rows
// above it.  The form for the narrow windows of a batch (many CTAs per GPU).
__device__ void undampedProduct(const double* A, const double* hd, int n, const double* v, double* h) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    for (int i = tid; i < n; i += blockDim.x) {
        double s0 = hd[i] * v[i], s1 = 0, s2 = 0, s3 = 0;
        int j = i + 1;
        for (; j + 4 <= n; j += 4) {
            s0 += A[i + (long long)j * n] * v[j];
            s1 += A[i + (long long)(j + 1) * n] * v[j + 1];
            s2 += A[i + (long long)(j + 2) * n] * v[j + 2];
            s3 += A[i + (long long)(j + 3) * n] * v[j + 3];
        }
        for (; j < n; ++j) s0 += A[i + (long long)j * n] * v[j];
        h[i] = (s0 + s1) + (s2 + s3);
    }
    __syncthreads();
    for (int i = warp; i < n; i += nw) {
        double s0 = 0, s1 = 0;
        int j = lane;
        for (; j + 32 < i; j += 64) {
            s0 += A[j + (long long)i * n] * v[j];
            s1 += A[j + 32 + (long long)i * n] * v[j + 32];
        }
        if (j < i) s0 += A[j + (long long)i * n] * v[j];
        const double s = warpSum(s0 + s1);
        if (lane == 0) h[i] += s;
    }
    __syncthreads();
}

// The same product for a lone wide window (one CTA over a large system), by blocks of
// 32 columns: every warp owns a fixed set of 32-row chunks, its lanes
// read their rows' 32 entries of the block (one coalesced load per column, 32 in
// flight), add the row part to h and accumulate the column part, which is folded
// across the warp (transposeSum) and across warps in shared memory.
__device__ void undampedProductBlocks(const double* A, const double* hd, int n, const double* v, double* h) {
    constexpr int kWarps = kFactorThreads / 32;
    __shared__ double colPart[kWarps * 32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < n; i += blockDim.x) h[i] = hd[i] * v[i];
    __syncthreads();
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int jw = min(32, n - j0);
        double acc[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) acc[c] = 0.0;
        for (int i0 = warp * 32; i0 < j0 + jw; i0 += kWarps * 32) {  // rows above the block's columns
            const int i = i0 + lane;
            const double vi = i < n ? v[i] : 0.0;
            double row = 0;
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                if (c < jw && i < j0 + c) {  // strict upper: row i, column j0 + c
                    const double a = A[i + (long long)(j0 + c) * n];
                    acc[c] += a * vi;
                    row += a * v[j0 + c];
                }
            }
            if (i < n) h[i] += row;  // row i belongs to this warp in every block
        }
        colPart[warp * 32 + lane] = transposeSum(acc);
        __syncthreads();
        if (tid < jw) {
            double t = 0;
            for (int w = 0; w < kWarps; ++w) t += colPart[w * 32 + tid];
            h[j0 + tid] += t;
        }
        __syncthreads();
    }
}

// Solve-time charts of one window's reduced system (kCol* per retained column),
// the reference's constant blocks, bias-frozen speed/bias and rotation-only rig
// extrinsic of a single solve (BackendOptimizer.cpp:44-66,83-91,783-795).  On
// entry A holds the assembled system (lower triangle damped, strict upper
// undamped), hd its undamped diagonal and x the right-hand side; dmp[i] is the
// damping of column i.  A rotation-only extrinsic's tangent theta moves the full
// left SE(3) tangent along [rho; theta] = [[p]x; I] theta, so the system is
// restricted to those directions: its rho columns are folded into its theta
// columns (columns, then rows, then the right-hand side), and the damping of a
// theta column is lambda max(m^T H m, 1e-6) with m that direction and H the
// undamped total information (retained + J^T J) of the block, as the damping of
// a restricted tangent column is in the reference.  Fixed and folded columns
// then become identity rows and columns with a zero right-hand side, so their
// increments are exactly zero.  On exit A is the restricted damped system in the
// same storage, hd its undamped diagonal (0 at fixed columns).
__device__ void chartSystem(const DevBatch& B, const WinDesc& wd, double lambda, int n, double* A, double* x, double* hd,
                            double* dmp) {
    const signed char* cc = B.colChart + wd.vec0;
    const int tid = threadIdx.x, K = wd.K, Npc = wd.Npc;
    const double* acc = B.acc + wd.acc0;
    for (int i = tid; i < n; i += blockDim.x) A[i + (long long)i * n] = hd[i];
    __syncthreads();
    for (int e = 0; wd.estExt && e < wd.E; ++e) {
        const int c0 = 15 * K + 6 * e;
        if (cc[c0] != kColRotRho) continue;  // uniform over the CTA
        const double* pt = B.ext[0] + 7ll * (wd.ext0 + e);
        const double P[9] = {0, -pt[2], pt[1], pt[2], 0, -pt[0], -pt[1], pt[0], 0};  // [p]x, row-major
        if (tid < 3) {
            const int k = tid;
            double m[6];
            for (int a = 0; a < 3; ++a) { m[a] = P[3 * a + k]; m[3 + a] = a == k ? 1.0 : 0.0; }
            double v = 0;
            for (int a = 0; a < 6; ++a)
                for (int b = 0; b < 6; ++b) {
                    const int pa = 6 * K + 6 * e + a, pb = 6 * K + 6 * e + b;
                    const double h = B.Hret[wd.dense0 + (long long)(c0 + a) * n + c0 + b] + acc[pa <= pb ? upIdx(pa, pb, Npc) : upIdx(pb, pa, Npc)];
                    v += m[a] * m[b] * h;
                }
            dmp[c0 + 3 + k] = lambda * fmax(v, 1e-6);
        }
        for (int r = tid; r < n; r += blockDim.x) {
            const double a0 = A[r + (long long)c0 * n], a1 = A[r + (long long)(c0 + 1) * n], a2 = A[r + (long long)(c0 + 2) * n];
            for (int k = 0; k < 3; ++k) A[r + (long long)(c0 + 3 + k) * n] += a0 * P[k] + a1 * P[3 + k] + a2 * P[6 + k];
        }
        __syncthreads();
        for (int j = tid; j < n; j += blockDim.x) {
            const double a0 = A[c0 + (long long)j * n], a1 = A[c0 + 1 + (long long)j * n], a2 = A[c0 + 2 + (long long)j * n];
            for (int k = 0; k < 3; ++k) A[c0 + 3 + k + (long long)j * n] += a0 * P[k] + a1 * P[3 + k] + a2 * P[6 + k];
        }
        if (tid == 0)
            for (int k = 0; k < 3; ++k) x[c0 + 3 + k] += x[c0] * P[k] + x[c0 + 1] * P[3 + k] + x[c0 + 2] * P[6 + k];
        __syncthreads();
    }
    for (long long t = tid; t < (long long)n * n; t += blockDim.x) {
        const int r = (int)(t % n), c = (int)(t / n);
        const bool fr = cc[r] == kColFixed || cc[r] == kColRotRho, fc = cc[c] == kColFixed || cc[c] == kColRotRho;
        if (fr || fc) A[t] = r == c ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) {
        if (cc[i] == kColFixed || cc[i] == kColRotRho) {
            x[i] = 0.0; dmp[i] = 0.0; hd[i] = 0.0;
        } else {
            hd[i] = A[i + (long long)i * n];
            A[i + (long long)i * n] += dmp[i];
        }
    }
    __syncthreads();
}
__device__ __forceinline__ bool chartFixed(const DevBatch& B, const WinDesc& wd, int i) {
    const signed char c = B.colChart[wd.vec0 + i];
    return c == kColFixed || c == kColRotRho;
}

// Damping lambda max(diag(H_total)_i, 1e-6) of retained column i.
__device__ __forceinline__ double dampingOf(const DevBatch& B, const WinDesc& wd, int i, double lambda) {
    double h = B.Hret[wd.dense0 + (long long)i * wd.Nr + i];
    const int pi = pcOfRetained(i, wd.K);
    if (pi >= 0) h += B.acc[wd.acc0 + upIdx(pi, pi, wd.Npc)];
    return lambda * fmax(h, 1e-6);
}

// Right-hand side -(g_r - B_v) of retained column i.
__device__ __forceinline__ double rhsOf(const DevBatch& B, const WinDesc& wd, int i) {
    const long long nS = (long long)wd.Npc * (wd.Npc + 1) / 2;
    const double* acc = B.acc + wd.acc0;
    double g = B.gret[wd.vec0 + i];
    const int p = pcOfRetained(i, wd.K);
    if (p >= 0) g += acc[nS + wd.Npc + p] - acc[nS + 2ll * wd.Npc + p];
    return -g;
}

// Left-looking factorization of one staged panel: P holds rows [0, m) of the
// panel's bw columns (column-major, leading dimension mp); column c of every
// row r >= c is reduced by one dot product against the panel's earlier columns,
// then scaled by the root of its pivot.  The diagonal stays unscaled in P (its
// root goes to A).  xp[0, bw) is forward-substituted on the way.  Returns false
// (uniform over the CTA) when a pivot is not positive and finite.
__device__ bool factorPanel(double* P, int mp, int m, int bw, double* xp, int* failed) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    for (int c = 0; c < bw; ++c) {
        for (int r = c + tid; r < m; r += blockDim.x) {
            double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
            int k = 0;
            for (; k + 4 <= c; k += 4) {
                s0 += P[r + k * mp] * P[c + k * mp];
                s1 += P[r + (k + 1) * mp] * P[c + (k + 1) * mp];
                s2 += P[r + (k + 2) * mp] * P[c + (k + 2) * mp];
                s3 += P[r + (k + 3) * mp] * P[c + (k + 3) * mp];
            }
            for (; k < c; ++k) s0 += P[r + k * mp] * P[c + k * mp];
            P[r + c * mp] -= (s0 + s1) + (s2 + s3);
        }
        if (warp == nw - 1) {  // forward substitution: x_c - sum_{k<c} L[c][k] y_k
            double t = lane < c ? P[c + lane * mp] * xp[lane] : 0.0;
            t = warpSum(t);
            if (lane == 0) xp[c] -= t;
        }
        __syncthreads();
        const double d = P[c + c * mp];
        if (!(d > 0) || !isfinite(d)) {
            if (tid == 0) *failed = 1;
            return false;  // uniform: every thread read the same d
        }
        const double l = sqrt(d);
        for (int r = c + 1 + tid; r < m; r += blockDim.x) P[r + c * mp] /= l;
        if (tid == 0) xp[c] /= l;
        __syncthreads();
    }
    return true;
}

// The factored panel into A: L's columns (rows k0 + c.., the diagonal as its root).
__device__ __forceinline__ void storePanel(const double* P, int mp, int m, int bw, double* A, int n, int k0) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int c = warp; c < bw; c += nw)
        for (int r = c + lane; r < m; r += 32) A[(k0 + r) + (long long)(k0 + c) * n] = r == c ? sqrt(P[r + c * mp]) : P[r + c * mp];
}

// One 32 x 32 lower tile (row block rb >= column block cb) of the trailing update
// A22 -= L21 L21^T after the panel at k0 (bw columns, m2 trailing rows), on the
// FP64 tensor path.  V is L21 by panel column: V + k ldv is column k's rows.
__device__ __forceinline__ void trailingTile(const double* V, long long ldv, int rb, int cb, int bw, int m2, double* A, int n, int k0) {
    const int lane = threadIdx.x & 31;
    double tacc[4][8];
    zeroTile(tacc);
    rankUpdateMma<false>(tacc, V, rb * 32, cb * 32, 0, bw, 1, (int)ldv);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = tileRowMma(rb, lane, r);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int j = tileCol(cb, lane, c);
            if (i < m2 && j < m2 && i >= j) A[(k0 + bw + i) + (long long)(k0 + bw + j) * n] -= tacc[r][c];
        }
    }
}

// After the factorization (x = y = L^-1 rhs): the backward substitution, the
// refinement steps against the assembled FP64 system and the predicted
// reduction of the state part; writes dr, predState and solveStatus.  x, hd,
// h (scratch), blk and dmp are the CTA's shared vectors.
template <bool kBlocks>
__device__ void factorTail(const DevBatch& B, const WinDesc& wd, int wdx, double lambda, int refinement, const double* A, double* x,
                           const double* hd, double* h, double* blk, const double* dmp, double* red, bool solveOnly = false) {
    auto product = [&](const double* v, double* out) {
        if constexpr (kBlocks) undampedProductBlocks(A, hd, wd.Nr, v, out);
        else undampedProduct(A, hd, wd.Nr, v, out);
    };
    const int n = wd.Nr, Npc = wd.Npc, K = wd.K;
    const bool charts = wd.charts != 0;
    const double* acc = B.acc + wd.acc0;
    const long long nS = (long long)Npc * (Npc + 1) / 2;
    const double* rhsOut = B.rhs + wd.vec0;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    __shared__ double colPart[kFactorThreads];  // per warp, 32 column sums of the backward substitution
    // ---- backward substitution L^T x = y by panels (L lower in A)
    for (int k0 = ((n - 1) / kFacPanel) * kFacPanel; k0 >= 0; k0 -= kFacPanel) {
        const int bw = min(kFacPanel, n - k0);
        if (!kBlocks) {  // x[k0 + c] -= sum over the rows below of L[r][k0 + c] x[r]: a warp per column
            for (int c = warp; c < bw; c += nw) {
                double s0 = 0, s1 = 0;
                int r = k0 + bw + lane;
                for (; r + 32 < n; r += 64) {
                    s0 += A[r + (long long)(k0 + c) * n] * x[r];
                    s1 += A[r + 32 + (long long)(k0 + c) * n] * x[r + 32];
                }
                if (r < n) s0 += A[r + (long long)(k0 + c) * n] * x[r];
                const double s = warpSum(s0 + s1);
                if (lane == 0) x[k0 + c] -= s;
            }
        } else if (k0 + bw < n) {  // the same by row chunks: lanes own rows, 32 column sums folded per warp
            double acc[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) acc[c] = 0.0;
            for (int r0 = k0 + bw + warp * 32; r0 < n; r0 += nw * 32) {
                const int r = r0 + lane;
                const double xr = r < n ? x[r] : 0.0;
#pragma unroll
                for (int c = 0; c < 32; ++c)
                    if (c < bw && r < n) acc[c] += A[r + (long long)(k0 + c) * n] * xr;
            }
            colPart[warp * 32 + lane] = transposeSum(acc);
            __syncthreads();
            if (tid < bw) {
                double t = 0;
                for (int w = 0; w < nw; ++w) t += colPart[w * 32 + tid];
                x[k0 + tid] -= t;
            }
        }
        if constexpr (kBlocks) {  // warp 0: lane r holds y_r and column r of the block (32 loads in flight)
            __syncthreads();
            if (warp == 0) {
                double col[kFacPanel];
#pragma unroll
                for (int c = 0; c < kFacPanel; ++c) col[c] = (lane < c && c < bw) ? A[(k0 + c) + (long long)(k0 + lane) * n] : 0.0;
                const double inv = lane < bw ? 1.0 / A[(k0 + lane) + (long long)(k0 + lane) * n] : 0.0;
                double y = lane < bw ? x[k0 + lane] : 0.0;
#pragma unroll
                for (int c = kFacPanel - 1; c >= 0; --c) {
                    if (c < bw) {
                        const double xc = __shfl_sync(0xffffffffu, y, c) * __shfl_sync(0xffffffffu, inv, c);
                        if (lane < c) y -= col[c] * xc;
                        if (lane == c) y = xc;
                    }
                }
                if (lane < bw) x[k0 + lane] = y;
            }
            __syncthreads();
        } else {
            for (int t = tid; t < bw * bw; t += blockDim.x) {
                const int c = t / bw, r = t % bw;
                blk[r + c * kFacPanel] = r >= c ? A[(k0 + r) + (long long)(k0 + c) * n] : 0.0;
            }
            __syncthreads();
            if (warp == 0) {  // lane r holds y_r; column sweep x_c = y_c / L_cc, y_r -= L[c][r] x_c (r < c)
                double y = lane < bw ? x[k0 + lane] : 0.0;
                for (int c = bw - 1; c >= 0; --c) {
                    const double xc = __shfl_sync(0xffffffffu, y, c) / blk[c + c * kFacPanel];
                    if (lane < c) y -= blk[c + lane * kFacPanel] * xc;
                    if (lane == c) y = xc;
                }
                if (lane < bw) x[k0 + lane] = y;
            }
            __syncthreads();
        }
    }
    double* dr = B.dr + wd.vec0;
    for (int i = tid; i < n; i += blockDim.x) dr[i] = x[i];
    __syncthreads();
    if (solveOnly) return;  // the product and the prediction follow in other kernels
    // ---- iterative refinement against the assembled FP64 system
    for (int it = 0; it < refinement; ++it) {
        if (charts) {
            product(dr, h);
            for (int i = tid; i < n; i += blockDim.x) x[i] = chartFixed(B, wd, i) ? 0.0 : rhsOut[i] - (h[i] + dmp[i] * dr[i]);
            __syncthreads();
            blockedSolve(A, n, x, blk);
            for (int i = tid; i < n; i += blockDim.x) dr[i] += x[i];
            __syncthreads();
            continue;
        }
        for (int i = tid; i < n; i += blockDim.x) x[i] = dampingOf(B, wd, i, lambda);  // damping of row i, kept in x for this pass
        __syncthreads();
        product(dr, h);
        for (int i = tid; i < n; i += blockDim.x) x[i] = rhsOf(B, wd, i) - (h[i] + x[i] * dr[i]);
        __syncthreads();
        blockedSolve(A, n, x, blk);
        for (int i = tid; i < n; i += blockDim.x) dr[i] += x[i];
        __syncthreads();
    }
    // predicted reduction of the state part with the undamped (S_visual + H_ret):
    //   -dx^T (g_r + 0.5 (S_v + H_ret) dx); the landmark terms are added per landmark.
    product(dr, h);
    auto gradient = [&](int i) {  // g_r + G_v of column i (the full gradient, without the Schur term)
        double g = B.gret[wd.vec0 + i];
        const int p = pcOfRetained(i, K);
        if (p >= 0) g += acc[nS + Npc + p];
        return g;
    };
    double pred = 0;
    for (int i = tid; i < n; i += blockDim.x) {
        double g = gradient(i);
        if (charts) {
            if (chartFixed(B, wd, i)) continue;
            if (B.colChart[wd.vec0 + i] == kColRotTheta) {  // restricted gradient m^T g of a rotation-only column
                const int e = (i - 15 * K) / 6, c0 = 15 * K + 6 * e, k = i - c0 - 3;
                const double* pt = B.ext[0] + 7ll * (wd.ext0 + e);
                const double P[9] = {0, -pt[2], pt[1], pt[2], 0, -pt[0], -pt[1], pt[0], 0};
                g += gradient(c0) * P[k] + gradient(c0 + 1) * P[3 + k] + gradient(c0 + 2) * P[6 + k];
            }
        }
        pred += -dr[i] * (g + 0.5 * h[i]);
    }
    pred = blockSum(pred, red);
    if (charts && wd.estExt) {
        // full tangent of the rotation-only extrinsics for the back-substitution: rho = [p]x theta
        for (int e = tid; e < wd.E; e += blockDim.x) {
            const int c0 = 15 * K + 6 * e;
            if (B.colChart[wd.vec0 + c0] != kColRotRho) continue;
            const double* pt = B.ext[0] + 7ll * (wd.ext0 + e);
            const double P[9] = {0, -pt[2], pt[1], pt[2], 0, -pt[0], -pt[1], pt[0], 0};
            for (int a = 0; a < 3; ++a) dr[c0 + a] = P[3 * a] * dr[c0 + 3] + P[3 * a + 1] * dr[c0 + 4] + P[3 * a + 2] * dr[c0 + 5];
        }
    }
    if (tid == 0) { B.predState[wdx] = pred; B.solveStatus[wdx] = CGMLI_OK; }
}

// The damped system as it is factored (lower triangle), stored symmetric and row-major.
__device__ __forceinline__ void storeSdebug(const double* A, int n, double* out) {
    for (long long t = threadIdx.x; t < (long long)n * n; t += blockDim.x) {
        const int r = (int)(t / n), c = (int)(t % n);
        out[t] = r >= c ? A[r + (long long)c * n] : A[c + (long long)r * n];
    }
}

__global__ void __launch_bounds__(kFactorThreads, 2) k_factor(DevBatch B, int refinement, double* Sdebug) {
    const int wdx = B.bigFirst[blockIdx.x];
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const int n = wd.Nr;
    if (isWideWindow(n)) return;  // factored by the wide sequence (k_wide_*)
    const double lambda = B.lm[wdx].lambda;
    extern __shared__ __align__(16) double smem[];
    const int npad = ((n + 31) & ~31) + kFacPanel;
    double* P = smem;                        // npad x kFacPanel, column-major (leading dimension mp <= npad)
    double* x = P + (size_t)npad * kFacPanel;  // n: right-hand side -> y -> increment
    double* hd = x + n;                      // n: undamped diagonal
    double* da = hd + n;                     // n: damping added to the diagonal; then the product h
    double* blk = da + n;                    // kFacPanel x kFacPanel diagonal block (solves)
    double* dmp = blk + kFacPanel * kFacPanel;  // n: damping of each column (solve-time charts only)
    const bool charts = wd.charts != 0;
    __shared__ int failed;
    __shared__ double red[32];
    double* A = B.Sglob + wd.dense0;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int nw = kFactorThreads / 32;
    if (tid == 0) failed = 0;
    for (int i = tid; i < n; i += blockDim.x) da[i] = dampingOf(B, wd, i, lambda);
    __syncthreads();
    // assembly: damped lower triangle (factored in place), undamped strict upper copy
    for (int j = warp; j < n; j += nw)
#pragma unroll 2
    for (int i = j + lane; i < n; i += 32) {
        const double v = assembleEntryCol(B, wd, i, j, lambda, false);
        if (i == j) {
            hd[i] = v;
            A[i + (long long)j * n] = v + da[i];
        } else {
            A[i + (long long)j * n] = v;
            A[j + (long long)i * n] = v;
        }
    }
    double* rhsOut = B.rhs + wd.vec0;
    for (int i = tid; i < n; i += blockDim.x) {
        const double r = rhsOf(B, wd, i);
        x[i] = r;
        rhsOut[i] = r;
        if (charts) dmp[i] = da[i];
    }
    __syncthreads();
    if (charts) {
        chartSystem(B, wd, lambda, n, A, x, hd, dmp);
        for (int i = tid; i < n; i += blockDim.x) rhsOut[i] = x[i];  // the restricted right-hand side
        __syncthreads();
    }
    if (Sdebug) storeSdebug(A, n, Sdebug + wd.dense0);
    // ---- factorization with the forward substitution
    for (int k0 = 0; k0 < n; k0 += kFacPanel) {
        // rows padded so that the trailing rows [bw, mp) are whole 32-row tiles
        const int bw = min(kFacPanel, n - k0), m = n - k0, mp = bw + ((m - bw + 31) & ~31);
        for (int t = tid; t < mp * kFacPanel; t += blockDim.x) {
            const int c = t / mp, r = t % mp;
            P[r + c * mp] = (c < bw && r < m && r >= c) ? A[(k0 + r) + (long long)(k0 + c) * n] : 0.0;
        }
        __syncthreads();
        if (!factorPanel(P, mp, m, bw, x + k0, &failed)) break;
        __syncthreads();
        storePanel(P, mp, m, bw, A, n, k0);
        const int m2 = m - bw;
        if (m2 > 0) {
            const int nb2 = (m2 + 31) >> 5, tiles = nb2 * (nb2 + 1) / 2;
            for (int t = warp; t < tiles; t += nw) {
                int cb, rb;
                tileOf(t, nb2, cb, rb);  // upper enumeration (cb <= rb): rows rb, columns cb
                trailingTile(P + bw, mp, rb, cb, bw, m2, A, n, k0);
            }
            // right-hand side below the panel: y2 -= L21 y1
            for (int i = tid; i < m2; i += blockDim.x) {
                double s = 0;
                for (int c = 0; c < bw; ++c) s += P[bw + i + c * mp] * x[k0 + c];
                x[k0 + bw + i] -= s;
            }
        }
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) B.solveStatus[wdx] = CGMLI_E_NOT_PD;
        return;
    }
    factorTail<false>(B, wd, wdx, lambda, refinement, A, x, hd, da, blk, dmp, red);
}

// ---- wide windows -----------------------------------------------------------------------
// A window whose reduced system has kWideCols columns or more (configuration 3's
// single large window) is factored by a launch sequence that spreads the work over
// the GPU instead of one CTA (k_factor skips it).  The damped system is assembled
// by column blocks (k_wide_assemble); the solve-time charts and the debug copy run
// in one CTA (k_wide_prepare).  The first diagonal block is factored by one CTA
// (k_wide_diag; wideDiagBlock: right-looking over the CTA, one barrier per column,
// the forward substitution of the right-hand side over the block on the way).  Then
// one launch per panel of kFacPanel columns (k_wide_update): every warp owns a
// 32 x 32 tile of the trailing update A22 -= L21 L21^T on the FP64 tensor path and
// first solves the row blocks of L21 it needs against the panel's diagonal block
// (one lane per row, the row in registers); the warps of the diagonal tiles keep
// L21 in a panel buffer and apply y2 -= L21 y1; the first CTA holds tile (0, 0)
// alone and factors the next diagonal block as soon as it is written.  The
// backward substitution, the refinement steps and the prediction follow
// (k_wide_finish, the tail k_factor uses).  Per-window vectors between the kernels:
// B.facVec + 3 vec0 holds x (n), the undamped diagonal (n) and the damping (n).
// A wide window without solve-time charts or refinement steps finishes in three
// kernels (k_wide_finish's solve, k_wide_product, k_wide_predict); otherwise
// k_wide_finish runs the whole tail in one CTA.
__device__ __forceinline__ bool wideSplitTail(const WinDesc& wd, int refinement) { return refinement == 0 && wd.charts == 0; }

__global__ void __launch_bounds__(256) k_wide_assemble(DevBatch B) {
    const int wdx = B.wideList[blockIdx.x];
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const int n = wd.Nr, j0 = 32 * blockIdx.y;
    if (j0 >= n) return;
    const double lambda = B.lm[wdx].lambda;
    double* A = B.Sglob + wd.dense0;
    double* x = B.facVec + 3ll * wd.vec0;
    double* hd = x + n;
    double* dmp = hd + n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    // the rows of each column are split over gridDim.z CTAs (32-row strips, strided)
    for (int j = j0 + warp; j < min(n, j0 + 32); j += nw)
        for (int i = j + lane + 32 * (int)blockIdx.z; i < n; i += 32 * (int)gridDim.z) {
            const double v = assembleEntryCol(B, wd, i, j, lambda, false);
            if (i == j) {
                hd[i] = v;
                A[i + (long long)j * n] = v + dampingOf(B, wd, i, lambda);
            } else {
                A[i + (long long)j * n] = v;
                A[j + (long long)i * n] = v;
            }
        }
    if (blockIdx.y == 0 && blockIdx.z == 0) {
        double* rhsOut = B.rhs + wd.vec0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const double r = rhsOf(B, wd, i);
            x[i] = r;
            rhsOut[i] = r;
            dmp[i] = dampingOf(B, wd, i, lambda);
        }
        if (threadIdx.x == 0) B.facFailed[wdx] = 0;
    }
}

__global__ void __launch_bounds__(kFactorThreads) k_wide_prepare(DevBatch B, double* Sdebug) {
    const int wdx = B.wideList[blockIdx.x];
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const int n = wd.Nr;
    double* A = B.Sglob + wd.dense0;
    if (wd.charts) {
        double* x = B.facVec + 3ll * wd.vec0;
        chartSystem(B, wd, B.lm[wdx].lambda, n, A, x, x + n, x + 2 * n);
        double* rhsOut = B.rhs + wd.vec0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) rhsOut[i] = x[i];  // the restricted right-hand side
        __syncthreads();
    }
    if (Sdebug) storeSdebug(A, n, Sdebug + wd.dense0);
}

// Cholesky of the diagonal block at k0 of window w by the whole CTA, with the forward
// substitution of x over the block; the block is written back as L11 (its diagonal
// the roots).  Right-looking on the unscaled columns: for pivot c every thread
// updates its entries (i, j), c < j <= i, by T[i][c] T[j][c] / d_c (four entries of
// the 32 x 32 block per thread, one barrier per column), and x_i -= T[i][c] x_c / d_c;
// the columns are scaled by 1 / sqrt(d_c) at the end.  A single warp doing the same
// sweep in registers took about 20 k cycles (in-order issue of ~120 dependent
// instructions per column); the CTA takes one update and one barrier per column.
// Returns false (uniform over the CTA) on a pivot that is not positive and finite.
constexpr int kDiagStride = kFacPanel + 1;
__device__ bool wideDiagBlock(const DevBatch& B, const WinDesc& wd, int k0) {
    static_assert(kFacPanel * kFacPanel == 4 * kFactorThreads, "four block entries per thread");
    __shared__ double T[kFacPanel * kDiagStride], xs[kFacPanel];
    const int tid = threadIdx.x, n = wd.Nr, bw = min(kFacPanel, n - k0);
    double* A = B.Sglob + wd.dense0;
    double* x = B.facVec + 3ll * wd.vec0;
    int ei[4], ej[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {  // entry (i, j), by columns: consecutive threads read consecutive rows
        const int q = tid + u * kFactorThreads;
        ei[u] = q % kFacPanel;
        ej[u] = q / kFacPanel;
        if (ei[u] < bw && ej[u] <= ei[u]) T[ei[u] * kDiagStride + ej[u]] = A[(k0 + ei[u]) + (long long)(k0 + ej[u]) * n];
    }
    if (tid < bw) xs[tid] = x[k0 + tid];
    __syncthreads();
    for (int c = 0; c < bw; ++c) {
        const double d = T[c * kDiagStride + c];
        if (!(d > 0) || !isfinite(d)) return false;  // every thread read the same d
        const double invd = 1.0 / d;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = ei[u], j = ej[u];
            if (j > c && i >= j && i < bw) T[i * kDiagStride + j] -= T[i * kDiagStride + c] * T[j * kDiagStride + c] * invd;
        }
        if (tid > c && tid < bw) xs[tid] -= T[tid * kDiagStride + c] * xs[c] * invd;
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int i = ei[u], j = ej[u];
        if (i < bw && j <= i) {
            const double l = sqrt(T[j * kDiagStride + j]);
            A[(k0 + i) + (long long)(k0 + j) * n] = i == j ? l : T[i * kDiagStride + j] / l;
        }
    }
    if (tid < bw) x[k0 + tid] = xs[tid] / sqrt(T[tid * kDiagStride + tid]);
    return true;
}

// The first panel's diagonal block (the later ones are factored by k_wide_trailing).
__global__ void __launch_bounds__(kFactorThreads) k_wide_diag(DevBatch B) {
    const int wdx = B.wideList[blockIdx.x];
    if (B.lm[wdx].mode == kModeDone) return;
    if (!wideDiagBlock(B, B.win[wdx], 0) && threadIdx.x == 0) B.facFailed[wdx] = 1;
}

// One panel's update in one launch: every warp owns a 32 x 32 tile (rb >= cb) of
// A22 -= L21 L21^T and first solves the two row blocks of L21 it needs against the
// panel's factored diagonal block (the same forward substitution as k_wide_trsm, one
// lane per row, so the same values; a block is solved by every warp that needs it,
// which keeps the row solves off the chain of launches).  A22 and the unsolved A21
// are both read during the launch, so L21 goes to a per-panel buffer (two, by panel
// parity) and reaches A in the next panel's launch or in k_wide_finish; the warp of
// a diagonal tile writes its block there and updates the right-hand side y2 -= L21 y1
// of its rows.  The first CTA holds tile (0, 0) alone and then factors the next
// diagonal block.
constexpr int kUpdStride = 2 * kFacPanel + 1;  // per warp: k-major rows of the two blocks (odd stride)
size_t wideUpdateSmemBytes() {
    return sizeof(double) * (kFacPanel * kDiagStride + 2 * kFacPanel + (size_t)(kFactorThreads / 32) * kFacPanel * kUpdStride);
}
__device__ __forceinline__ double* wideL21(const DevBatch& B, int slot, int panel, int wideCols) {
    return B.wideL21 + ((size_t)slot * 2 + (panel & 1)) * kFacPanel * wideCols;
}
// The L21 block of panel `panel` (rows below it, k-major: row r - (k0 + 32) at entry
// k * wideCols) into A's columns of that panel.
__device__ void wideStoreL21(const DevBatch& B, const WinDesc& wd, int slot, int panel, int wideCols, int tid, int threads) {
    const int n = wd.Nr, k0 = panel * kFacPanel, rows = n - k0 - kFacPanel;
    const double* Ls = wideL21(B, slot, panel, wideCols);
    double* A = B.Sglob + wd.dense0;
    for (long long e = tid; e < (long long)rows * kFacPanel; e += threads) {
        const int c = (int)(e / rows), r = (int)(e % rows);
        A[(k0 + kFacPanel + r) + (long long)(k0 + c) * n] = Ls[(size_t)c * wideCols + r];
    }
}
__global__ void __launch_bounds__(kFactorThreads) k_wide_update(DevBatch B, int k0, int wideCols) {
    const int wdx = B.wideList[blockIdx.x];
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const int n = wd.Nr, panel = k0 / kFacPanel;
    if (B.facFailed[wdx]) return;
    // the previous panel's L21 into the factor, off the first CTA's chain: by the other
    // CTAs when there are any (after their tiles), else by the first after its work
    const bool storeHere = panel > 0 && k0 < n && (gridDim.y == 1 || blockIdx.y > 0);
    auto storePrevious = [&]() {
        if (!storeHere) return;
        const int helpers = gridDim.y == 1 ? 1 : gridDim.y - 1, rank = gridDim.y == 1 ? 0 : blockIdx.y - 1;
        wideStoreL21(B, wd, blockIdx.x, panel - 1, wideCols, rank * blockDim.x + threadIdx.x, helpers * blockDim.x);
    };
    if (k0 + kFacPanel >= n) {  // uniform over the CTA
        storePrevious();
        return;
    }
    const int m2 = n - k0 - kFacPanel, nb2 = (m2 + 31) >> 5, tiles = nb2 * (nb2 + 1) / 2;
    // the first CTA holds tile (0, 0) alone, so that the next diagonal block waits for
    // that tile only; the other CTAs hold eight tiles each
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.y == 0 ? (warp == 0 ? 0 : tiles) : 1 + (blockIdx.y - 1) * (kFactorThreads / 32) + warp;
    if (blockIdx.y > 0 && 1 + (blockIdx.y - 1) * (kFactorThreads / 32) >= tiles) {  // uniform over the CTA
        storePrevious();
        return;
    }
    // the tile's current entries, loaded now so that their latency hides behind the
    // staging and the row solves
    int rb = 0, cb = 0;
    if (t < tiles) tileOf(t, nb2, cb, rb);
    double old[4][8];
    if (t < tiles) {
#pragma unroll
        for (int rr = 0; rr < 4; ++rr) {
            const int i = tileRowMma(rb, lane, rr);
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int j = tileCol(cb, lane, c);
                old[rr][c] = (i < m2 && j < m2 && i >= j) ? B.Sglob[wd.dense0 + (k0 + kFacPanel + i) + (long long)(k0 + kFacPanel + j) * n] : 0.0;
            }
        }
    }
    extern __shared__ __align__(16) double usm[];
    double* L = usm;                          // the diagonal block, row-major (stride kDiagStride)
    double* inv = L + kFacPanel * kDiagStride;
    double* y1 = inv + kFacPanel;
    double* Vs = y1 + kFacPanel + (size_t)warp * kFacPanel * kUpdStride;
    double* A = B.Sglob + wd.dense0;
    double* x = B.facVec + 3ll * wd.vec0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {  // by columns (coalesced), four loads in flight
        const int q = threadIdx.x + u * kFactorThreads, i = q % kFacPanel, j = q / kFacPanel;
        L[i * kDiagStride + j] = j <= i ? A[(k0 + i) + (long long)(k0 + j) * n] : 0.0;
    }
    if (threadIdx.x < kFacPanel) {
        y1[threadIdx.x] = x[k0 + threadIdx.x];
        inv[threadIdx.x] = 1.0 / A[(k0 + threadIdx.x) + (long long)(k0 + threadIdx.x) * n];
    }
    __syncthreads();
    if (t < tiles) {
        double* Lcur = wideL21(B, blockIdx.x, panel, wideCols);
        for (int h = 0; h < (rb == cb ? 1 : 2); ++h) {  // the row blocks rb, then cb
            const int blk = h == 0 ? rb : cb, rl = blk * 32 + lane, r = k0 + kFacPanel + rl;
            double a[kFacPanel];
#pragma unroll
            for (int c = 0; c < kFacPanel; ++c) a[c] = r < n ? A[r + (long long)(k0 + c) * n] : 0.0;
            // four partial sums per entry, so the chain from one entry to the next is
            // about a quarter of its dot product
            double y = 0;
#pragma unroll
            for (int c = 0; c < kFacPanel; ++c) {
                double s0 = a[c], s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
                for (int k = 0; k < c; k += 4) {
                    s0 -= a[k] * L[c * kDiagStride + k];
                    if (k + 1 < c) s1 -= a[k + 1] * L[c * kDiagStride + k + 1];
                    if (k + 2 < c) s2 -= a[k + 2] * L[c * kDiagStride + k + 2];
                    if (k + 3 < c) s3 -= a[k + 3] * L[c * kDiagStride + k + 3];
                }
                a[c] = ((s0 + s1) + (s2 + s3)) * inv[c];
                y += a[c] * y1[c];
                Vs[c * kUpdStride + 32 * h + lane] = a[c];
            }
            if (rb == cb && r < n) {  // this block's owner: L21 to the panel buffer, y2 -= L21 y1
#pragma unroll
                for (int c = 0; c < kFacPanel; ++c) Lcur[(size_t)c * wideCols + rl] = a[c];
                x[r] -= y;
            }
        }
        __syncwarp();
        // the tile from the staged blocks (trailingTileFull's operands and MMA order)
        const int g = lane >> 2, kr = lane & 3, cOff = rb == cb ? 0 : 32;
        double av[kFacPanel / 4][4], bv[kFacPanel / 4][4];
#pragma unroll
        for (int st = 0; st < kFacPanel / 4; ++st) {
            const double* row = Vs + (4 * st + kr) * kUpdStride;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                av[st][q] = row[8 * q + g];
                bv[st][q] = row[cOff + 8 * q + g];
            }
        }
        double acc[4][8];
        zeroTile(acc);
#pragma unroll
        for (int st = 0; st < kFacPanel / 4; ++st)
#pragma unroll
            for (int I = 0; I < 4; ++I)
#pragma unroll
                for (int J = 0; J < 4; ++J) mmaF64Tile(acc[I][2 * J], acc[I][2 * J + 1], av[st][I], bv[st][J]);
#pragma unroll
        for (int rr = 0; rr < 4; ++rr) {
            const int i = tileRowMma(rb, lane, rr);
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int j = tileCol(cb, lane, c);
                if (i < m2 && j < m2 && i >= j) A[(k0 + kFacPanel + i) + (long long)(k0 + kFacPanel + j) * n] = old[rr][c] - acc[rr][c];
            }
        }
    }
    if (blockIdx.y == 0) {  // tile (0, 0), this CTA's first, is the next panel's diagonal block
        __syncthreads();
        if (!wideDiagBlock(B, wd, k0 + kFacPanel) && threadIdx.x == 0) B.facFailed[wdx] = 1;
    }
    storePrevious();
}

__global__ void __launch_bounds__(kFactorThreads) k_wide_finish(DevBatch B, int refinement, int wideCols) {
    const int wdx = B.wideList[blockIdx.x];
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const int n = wd.Nr;
    if (B.facFailed[wdx]) {
        if (threadIdx.x == 0) B.solveStatus[wdx] = CGMLI_E_NOT_PD;
        return;
    }
    if (n > kFacPanel)  // the last panel's L21 (the earlier ones reached A in the later panels' launches)
        wideStoreL21(B, wd, blockIdx.x, (n - kFacPanel - 1) / kFacPanel, wideCols, threadIdx.x, blockDim.x);
    extern __shared__ __align__(16) double smem[];
    __shared__ double red[32];
    double* x = smem;
    double* hd = x + n;
    double* dmp = hd + n;
    double* h = dmp + n;
    double* blk = h + n;
    const double* src = B.facVec + 3ll * wd.vec0;
#pragma unroll 4
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) x[i] = src[i];
    __syncthreads();
    factorTail<true>(B, wd, wdx, B.lm[wdx].lambda, refinement, B.Sglob + wd.dense0, x, hd, h, blk, dmp, red,
                     wideSplitTail(wd, refinement));
}

// Without charts or refinement steps, the undamped product h = S dr of the
// prediction is spread over the GPU: one CTA per 32-column block of the stored upper
// triangle (A[i + j n], i < j) forms each row's part over the block's columns (rows
// above them, lanes over rows, a coalesced load per column) and the block's column
// sums (folded across the warp and then across the warps in a fixed order); the
// prediction kernel adds them in block order.  h_i = hd_i dr_i + sum over blocks of
// the row parts + the column part of i's own block.
__global__ void __launch_bounds__(kFactorThreads) k_wide_product(DevBatch B, int refinement, int wideCols) {
    const int wdx = B.wideList[blockIdx.x];
    if (B.lm[wdx].mode == kModeDone || B.facFailed[wdx]) return;
    const WinDesc wd = B.win[wdx];
    const int n = wd.Nr, j0 = 32 * blockIdx.y;
    if (!wideSplitTail(wd, refinement) || j0 >= n) return;
    const int nbMax = (wideCols + 31) / 32, jw = min(32, n - j0);
    double* rowPart = B.wideProd + (size_t)blockIdx.x * (nbMax + 1) * wideCols + (size_t)blockIdx.y * wideCols;
    double* colPart = B.wideProd + (size_t)blockIdx.x * (nbMax + 1) * wideCols + (size_t)nbMax * wideCols;
    const double* A = B.Sglob + wd.dense0;
    const double* v = B.dr + wd.vec0;
    constexpr int kWarps = kFactorThreads / 32;
    __shared__ double part[kWarps * 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) acc[c] = 0.0;
    for (int i0 = warp * 32; i0 < j0 + jw; i0 += kWarps * 32) {
        const int i = i0 + lane;
        const double vi = i < n ? v[i] : 0.0;
        double row = 0;
#pragma unroll
        for (int c = 0; c < 32; ++c) {
            if (c < jw && i < j0 + c) {  // strict upper: row i, column j0 + c
                const double a = A[i + (long long)(j0 + c) * n];
                acc[c] += a * vi;
                row += a * v[j0 + c];
            }
        }
        if (i < j0 + jw) rowPart[i] = row;
    }
    part[warp * 32 + lane] = transposeSum(acc);
    __syncthreads();
    if (threadIdx.x < jw) {
        double t = 0;
        for (int w = 0; w < kWarps; ++w) t += part[w * 32 + threadIdx.x];
        colPart[j0 + threadIdx.x] = t;
    }
}

// The prediction of a split tail: -dx^T (g + 0.5 h) with h summed from the parts.
__global__ void __launch_bounds__(kFactorThreads) k_wide_predict(DevBatch B, int refinement, int wideCols) {
    const int wdx = B.wideList[blockIdx.x];
    if (B.lm[wdx].mode == kModeDone || B.facFailed[wdx]) return;
    const WinDesc wd = B.win[wdx];
    if (!wideSplitTail(wd, refinement)) return;
    const int n = wd.Nr, K = wd.K, Npc = wd.Npc, nbMax = (wideCols + 31) / 32, nb = (n + 31) / 32;
    const double* prod = B.wideProd + (size_t)blockIdx.x * (nbMax + 1) * wideCols;
    const double* hd = B.facVec + 3ll * wd.vec0 + n;
    const double* dr = B.dr + wd.vec0;
    const double* acc = B.acc + wd.acc0;
    const long long nS = (long long)Npc * (Npc + 1) / 2;
    __shared__ double red[32];
    double pred = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double h = hd[i] * dr[i];
        for (int b = i / 32; b < nb; ++b) h += prod[(size_t)b * wideCols + i];
        h += prod[(size_t)nbMax * wideCols + i];
        double g = B.gret[wd.vec0 + i];
        const int p = pcOfRetained(i, K);
        if (p >= 0) g += acc[nS + Npc + p];
        pred += -dr[i] * (g + 0.5 * h);
    }
    pred = blockSum(pred, red);
    if (threadIdx.x == 0) { B.predState[wdx] = pred; B.solveStatus[wdx] = CGMLI_OK; }
}

// ---------------------------------------------------------------------------------------
// Candidate states x [+] dx of the retained blocks (residentTrial, VisualCudaBatch.cu:323-340).
__global__ void k_candidate(DevBatch B) {
    const int wdx = blockIdx.x;
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const double* dr = B.dr + wd.vec0;
    __shared__ double red[32];
    double mx = 0;
    int bad = 0;
    for (int i = threadIdx.x; i < wd.Nr; i += blockDim.x) {
        if (!isfinite(dr[i])) bad = 1; else mx = fmax(mx, fabs(dr[i]));
    }
    // solve-time charts: a fixed block is copied; a rotation-only extrinsic keeps its
    // translation (Plus(T, theta) = (Exp(theta) R, p), GpuRetainedFactorMath.hpp:28-37)
    const signed char* cc = wd.charts ? B.colChart + wd.vec0 : nullptr;
    for (int k = threadIdx.x; k < wd.K; k += blockDim.x) {
        const int gk = wd.kf0 + k;
        if (cc && cc[15 * k] == kColFixed)
            for (int j = 0; j < 7; ++j) B.pose[1][7ll * gk + j] = B.pose[0][7ll * gk + j];
        else
            posePlus(B.pose[0] + 7ll * gk, dr + 15 * k, B.pose[1] + 7ll * gk);
        poseRotation(B.pose[1] + 7ll * gk, B.rotKf[1] + 9ll * gk);
        for (int j = 0; j < 9; ++j)
            B.sb[1][9ll * gk + j] = cc && cc[15 * k + 6 + j] == kColFixed ? B.sb[0][9ll * gk + j] : B.sb[0][9ll * gk + j] + dr[15 * k + 6 + j];
    }
    for (int e = threadIdx.x; e < wd.E; e += blockDim.x) {
        const int ge = wd.ext0 + e;
        const int chart = wd.estExt && cc ? cc[15 * wd.K + 6 * e] : kColFree;
        if (wd.estExt && chart == kColFree) posePlus(B.ext[0] + 7ll * ge, dr + 15 * wd.K + 6 * e, B.ext[1] + 7ll * ge);
        else if (wd.estExt && chart == kColRotRho) posePlusRotation(B.ext[0] + 7ll * ge, dr + 15 * wd.K + 6 * e + 3, B.ext[1] + 7ll * ge);
        else for (int j = 0; j < 7; ++j) B.ext[1][7ll * ge + j] = B.ext[0][7ll * ge + j];
        poseRotation(B.ext[1] + 7ll * ge, B.rotExt[1] + 9ll * ge);
    }
    if (threadIdx.x == 0)
        B.td[1][wdx] = B.td[0][wdx] + (wd.estTd ? dr[15 * wd.K + (wd.estExt ? 6 * wd.E : 0)] : 0.0);
    mx = warpMax(mx);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) red[warp] = bad ? -1.0 : mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0;
        bool anyBad = false;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { if (red[i] < 0) anyBad = true; else m = fmax(m, red[i]); }
        B.out[4ll * wdx + 0] = m;
        B.out[4ll * wdx + 1] = anyBad ? 0.0 : 1.0;
    }
}

// ---------------------------------------------------------------------------------------
// Back-substitution of the inverse distances (backSubstitute,
// VisualCudaBatch.cu:191-205): eight lanes per landmark form c_l . dx_r.
__global__ void __launch_bounds__(256) k_backsub(DevBatch B) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = gt >> 3, sub = threadIdx.x & 7;
    const bool inRange = l < B.numLandmarks;
    const int wdx = inRange ? B.lmWin[l] : 0;
    const bool active = inRange && B.lm[wdx].mode != kModeDone;
    double cd = 0;
    int K = 0, s = 0, x = 0, ns = 0, tdCol = 0;
    const WinDesc* wd = B.win + wdx;
    if (active) {
        K = wd->K;
        s = B.lmNs[l];
        x = B.lmNx[l];
        ns = 6 * (s + x) + (wd->estTd ? 1 : 0);
        tdCol = 6 * K + (wd->estExt ? 6 * wd->E : 0);
        const double* c = B.lmC + B.lmC0[l];
        const int* sk = B.supp + B.lmSupp0[l];
        const double* dr = B.dr + wd->vec0;
        for (int i = sub; i < ns; i += 8) cd += c[i] * dr[retainedOfPc(pcOfLocal(i, s, x, sk, K, tdCol), K)];
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) cd += __shfl_xor_sync(0xffffffffu, cd, o);
    if (!active || sub != 0) return;
    const double lambda = B.lm[wdx].lambda;
    const double d = B.lmD[l], g = B.lmG[l];
    const double dt = d + lambda * fmax(d, 1e-6);
    double dl = -(g + cd) / dt;
    const double rho0 = B.rho[0][l], minInv = wd->minInv;
    if (wd->fixedLm && B.lmFixed[l]) {  // held constant: no increment, no landmark term in the prediction
        B.lmDelta[l] = 0.0;
        B.lmPred[l] = 0.0;
        B.lmMaxInc[l] = 0.0;
        B.rho[1][l] = rho0;
        return;
    }
    if (isfinite(dl)) dl = fmax(minInv - rho0, dl);
    B.lmDelta[l] = dl;
    // landmark terms of -dx^T (g + 0.5 H dx): the cross term c.dx_r is
    // split between the state part (via S_v) and this correction
    B.lmPred[l] = -0.5 * cd * cd / dt - dl * (g + cd + 0.5 * d * dl);
    B.lmMaxInc[l] = isfinite(dl) ? fabs(dl) : -1.0;
    B.rho[1][l] = fmax(minInv, rho0 + dl);
}

// Robust cost of the candidate point (launchTrial, VisualCudaBatch.cu:715-721):
// one warp per tile of <= 32 observations, lane = observation; the per-landmark
// sums are segmented scans over the tile's lanes (a landmark's observations are
// consecutive lanes), written by each landmark's last lane.
constexpr int kTrialWarps = 8;  // warps per CTA of the gate
template <int Warps, int MinBlocks>
__global__ void __launch_bounds__(Warps * 32, MinBlocks) k_trial(DevBatch B, const int2* tiles, int numTiles) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * Warps + warp;
    if (t >= numTiles) return;
    const int2 tile = tiles[t];
    const int lb = tile.x, le = tile.y, nl = le - lb;
    const int wdx = B.lmWin[lb];
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const int ob = B.lmObsBegin[lb], oe = B.lmObsBegin[le];
    const int f = ob + lane;
    const bool live = f < oe;
    const int seg = live ? B.obLm[f] - lb : 32 + lane;  // lanes past the tile: segments of their own
    double cost = 0.0;
    int bad = 0;
    if (live) {
        FactorIn in;
        int kfa, kfb, ea, eb;
        gatherFactor(B, wd, wdx, lb + seg, f, 1, in, kfa, kfb, ea, eb);
        FactorOut o;
        if (!evalBearingFactor(in, false, o)) bad = 1;
        else cost = huberCost(wd.huber, o.r[0] * o.r[0] + o.r[1] * o.r[1]);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double c2 = __shfl_up_sync(0xffffffffu, cost, o);
        const int b2 = __shfl_up_sync(0xffffffffu, bad, o), s2 = __shfl_up_sync(0xffffffffu, seg, o);
        if (lane >= o && s2 == seg) { cost += c2; bad |= b2; }
    }
    // landmarks of the tile without observations keep cost 0
    if (lane < nl) {
        B.lmTrial[lb + lane] = 0.0;
        B.lmTrialValid[lb + lane] = B.lmMaxInc[lb + lane] >= 0.0 ? 1 : 0;  // -1 marks a non-finite step
    }
    __syncwarp();
    const int nextSeg = __shfl_down_sync(0xffffffffu, seg, 1);
    if (live && (lane == 31 || f + 1 >= oe || nextSeg != seg)) {
        const int l = lb + seg;
        B.lmTrial[l] = cost;
        B.lmTrialValid[l] = bad ? 0 : (B.lmMaxInc[l] >= 0.0 ? 1 : 0);
    }
}

// ---------------------------------------------------------------------------------------
// Per-window reductions and the LM decision (BackendOptimizer.cpp:232-306).
// probe != 0: record the step's scalars without changing the LM state.
__global__ void __launch_bounds__(256) k_lm_update(DevBatch B, int maxIterations, int probe) {
    const int wdx = blockIdx.x;
    WinLM& st = B.lm[wdx];
    if (st.mode == kModeDone) { if (threadIdx.x == 0) st.acceptNow = 0; return; }
    const WinDesc wd = B.win[wdx];
    __shared__ double red[32];
    double cost = 0, pred = 0, trial = 0, mx = 0;
    int valid = 1, tvalid = 1;
#pragma unroll 4
    for (int i = threadIdx.x; i < wd.L; i += blockDim.x) {  // unrolled: four landmarks' loads in flight
        const int l = wd.lm0 + i;
        cost += B.lmCost[l];
        pred += B.lmPred[l];
        trial += B.lmTrial[l];
        valid &= B.lmValid[l];
        tvalid &= B.lmTrialValid[l];
        const double m = B.lmMaxInc[l];
        if (m < 0) tvalid = 0; else mx = fmax(mx, m);
    }
    cost = blockSum(cost, red);
    pred = blockSum(pred, red);
    trial = blockSum(trial, red);
    mx = warpMax(mx);
    __shared__ double mxs[32];
    __shared__ int vs[32], tvs[32];
    valid = __all_sync(0xffffffffu, valid);
    tvalid = __all_sync(0xffffffffu, tvalid);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { mxs[warp] = mx; vs[warp] = valid; tvs[warp] = tvalid; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { mx = fmax(mx, mxs[i]); valid &= vs[i]; tvalid &= tvs[i]; }
    mx = fmax(mx, B.out[4ll * wdx + 0]);
    tvalid = tvalid && B.out[4ll * wdx + 1] != 0.0 && B.retValid[wdx];
    const double linCost = cost + B.costRet[wdx];
    const double predicted = pred + B.predState[wdx];
    const double trialCost = trial + B.trialRet[wdx];
    if (st.mode == kModeLinearize) {
        st.linCost = linCost;
        if (!valid || !isfinite(linCost)) { st.status = CGMLI_E_NONFINITE; st.mode = kModeDone; st.acceptNow = 0; return; }
        // the first linearization of a pass sets its cost (a refit pass starts
        // from the gated factor set, whose cost differs from the last accepted one)
        if (st.iterations == st.passStart) {
            st.cost = linCost;
            if (st.iterations == 0) st.initialCost = linCost;
        } else if (fabs(linCost - st.cost) > 1e-8 * fmax(1.0, st.cost)) {
            st.status = CGMLI_E_COST_MISMATCH; st.mode = kModeDone; st.acceptNow = 0; return;
        }
    }
    if (B.solveStatus[wdx] != CGMLI_OK) { st.status = B.solveStatus[wdx]; st.mode = kModeDone; st.acceptNow = 0; return; }
    // time budget (BackendOptimizer.cpp:177,242): after a step solved at pass iteration
    // i >= min_iterations with a step already accepted, an elapsed budget ends the
    // solve before this step's acceptance test
    const bool expired = !probe && B.budgetNs > 0 && globalTimerNs() - st.t0 >= (unsigned long long)B.budgetNs;
    if (expired && st.iterations - st.passStart >= B.minIterations && st.accepted > st.passAccepted) {
        st.mode = kModeDone; st.acceptNow = 0; return;
    }
    st.predicted = predicted;
    st.trialCost = trialCost;
    st.trialValid = tvalid;
    st.maxInc = mx;
    if (probe) { st.acceptNow = 0; return; }
    st.iterations += 1;
    st.acceptNow = 0;
    if (tvalid && mx < 1e-10) {
        st.converged = 1; st.mode = kModeDone;
    } else {
        double gain = -1;
        if (tvalid && predicted > 0 && isfinite(predicted)) gain = (st.cost - trialCost) / predicted;
        if (gain > 1e-3) {
            st.acceptNow = 1;
            st.accepted += 1;
            const bool conv = st.cost - trialCost <= 1e-6 * fmax(1.0, st.cost);
            st.cost = trialCost;
            const double t = 2 * gain - 1;
            st.lambda = fmax(1e-12, st.lambda * fmax(1.0 / 3, 1 - t * t * t));
            st.nu = 2;
            st.converged = conv;
            st.mode = conv ? kModeDone : kModeLinearize;
        } else {
            st.lambda *= st.nu;
            st.nu *= 2;
            st.mode = kModeResolve;
        }
    }
    // the pass may use what the finished passes left of the budget
    if (st.iterations - st.passStart + st.charged >= maxIterations && st.mode != kModeDone) st.mode = kModeDone;
    // an elapsed time budget ends the solve before the next iteration i >= max(min_iterations, 1)
    if (expired && st.mode != kModeDone && st.iterations - st.passStart >= B.minIterations) st.mode = kModeDone;
    if (st.mode == kModeDone && st.status == CGMLI_OK && st.accepted == st.passAccepted && !st.converged) st.status = CGMLI_E_NO_STEP;
}

// ---------------------------------------------------------------------------------------
// Whitened pre-loss NIS gate and outlier refits (BackendOptimizer::statisticalGate
// and the refit loop of optimizeImpl, BackendOptimizer.cpp:394-472,1030-1079).
// Visual factors are gated; IMU factors and the prior have an infinite threshold
// there.  A rejected factor's whitening rows (obP) are zeroed, so every later
// linearization, trial and marginalization sees a zero residual and Jacobian,
// which is what leaving it out of the problem gives.

// Rotations of the accepted states (the last iteration may have left the
// candidate's in place) and the per-gate counters of the windows in this pass.
__global__ void k_gate_prepare(DevBatch B, int pass, int pre, double* gateStats, int* gateCounts) {
    const int w = blockIdx.x;
    if (B.lm[w].pass != pass) return;
    const WinDesc& wd = B.win[w];
    for (int k = threadIdx.x; k < wd.K; k += blockDim.x) poseRotation(B.pose[0] + 7ll * (wd.kf0 + k), B.rotKf[0] + 9ll * (wd.kf0 + k));
    for (int e = threadIdx.x; e < wd.E; e += blockDim.x) poseRotation(B.ext[0] + 7ll * (wd.ext0 + e), B.rotExt[0] + 9ll * (wd.ext0 + e));
    if (threadIdx.x == 0) {
        gateStats[2 * w] = 0.0;      // sum of the evaluated energies
        gateStats[2 * w + 1] = 0.0;  // largest energy
        int* c = gateCounts + kGateCounts * w;
        c[0] = 0;             // evaluated
        c[pre ? 4 : 1] = 0;   // rejected by this gate (before the first solve: slot 4)
        c[3] = 0;             // a residual was not finite
    }
}

// One warp per tile, one lane per observation (as k_trial); a tile's landmarks
// belong to one window, so the warp reduces its counters and energies before one
// atomic each.  Slot 2 of a window's counters counts its rejections over all gates.
__global__ void __launch_bounds__(kTrialWarps * 32, 2) k_gate(DevBatch B, const int2* tiles, int numTiles, int pass, int pre,
                                                            double threshold, double* obP, unsigned char* rejected, double* gateStats,
                                                            int* gateCounts) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * kTrialWarps + warp;
    if (t >= numTiles) return;
    const int2 tile = tiles[t];
    const int lb = tile.x;
    const int wdx = B.lmWin[lb];
    const WinLM& st = B.lm[wdx];
    if (st.pass != pass || st.status != CGMLI_OK) return;
    const WinDesc wd = B.win[wdx];
    const int ob = B.lmObsBegin[lb], oe = B.lmObsBegin[tile.y];
    const int f = ob + lane;
    bool evaluated = false, bad = false, reject = false;
    double energy = 0.0;
    if (f < oe && !rejected[f]) {
        FactorIn in;
        int kfa, kfb, ea, eb;
        gatherFactor(B, wd, wdx, B.obLm[f], f, 0, in, kfa, kfb, ea, eb);
        FactorOut o;
        const bool ok = evalBearingFactor(in, false, o);
        energy = o.r[0] * o.r[0] + o.r[1] * o.r[1];
        if (!ok || !isfinite(energy)) {
            bad = true;
            energy = 0.0;
        } else {
            evaluated = true;
            reject = energy > threshold;
        }
    }
    if (reject) {
        rejected[f] = 1;
        for (int k = 0; k < 6; ++k) obP[6ll * f + k] = 0.0;
    }
    const unsigned full = 0xffffffffu;
    const int nEval = __popc(__ballot_sync(full, evaluated)), nRej = __popc(__ballot_sync(full, reject));
    const bool anyBad = __any_sync(full, bad);
    double sum = energy, mx = energy;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(full, sum, o);
        mx = fmax(mx, __shfl_xor_sync(full, mx, o));
    }
    if (lane == 0) {
        int* c = gateCounts + kGateCounts * wdx;
        if (anyBad) atomicOr(&c[3], 1);
        if (nEval) {
            atomicAdd(&c[0], nEval);
            atomicAdd(&gateStats[2 * wdx], sum);
            // energies are >= 0: their IEEE bit patterns order like the values
            atomicMax(reinterpret_cast<unsigned long long*>(&gateStats[2 * wdx + 1]), (unsigned long long)__double_as_longlong(mx));
        }
        if (nRej) {
            atomicAdd(&c[pre ? 4 : 1], nRej);
            atomicAdd(&c[2], nRej);
        }
    }
}

// Decides, after the gate of pass - 1, which windows run pass `pass`: those that
// rejected factors there with iteration budget left, restarted from their
// accepted state with the initial lambda (a fresh solve of the cleaned problem).
// Every finished pass is charged at least one iteration.
__global__ void k_lm_refit(DevBatch B, int pass, double lambda0, int maxIterations, const int* gateCounts) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= B.numWindows) return;
    WinLM& st = B.lm[w];
    if (st.pass != pass - 1) return;  // stopped refitting earlier
    const int* c = gateCounts + kGateCounts * w;
    if (c[3] && st.status == CGMLI_OK) st.status = CGMLI_E_NONFINITE;
    st.charged += max(1, st.iterations - st.passStart);
    st.mode = kModeDone;
    st.acceptNow = 0;
    if (st.status != CGMLI_OK || c[1] == 0 || st.charged >= maxIterations) return;
    st.pass = pass;
    st.mode = kModeLinearize;
    st.lambda = lambda0;
    st.nu = 2;
    st.converged = 0;
    st.trialValid = 0;
    st.passStart = st.iterations;
    st.passAccepted = st.accepted;
}

// Copy the candidate into the accepted state of windows that accepted a step
// (acceptResident, VisualCudaBatch.cu:702).
__global__ void k_accept(DevBatch B) {
    const int wdx = blockIdx.x;
    if (!B.lm[wdx].acceptNow) return;
    const WinDesc wd = B.win[wdx];
    for (int i = threadIdx.x; i < 7 * wd.K; i += blockDim.x) B.pose[0][7ll * wd.kf0 + i] = B.pose[1][7ll * wd.kf0 + i];
    for (int i = threadIdx.x; i < 9 * wd.K; i += blockDim.x) B.sb[0][9ll * wd.kf0 + i] = B.sb[1][9ll * wd.kf0 + i];
    for (int i = threadIdx.x; i < 7 * wd.E; i += blockDim.x) B.ext[0][7ll * wd.ext0 + i] = B.ext[1][7ll * wd.ext0 + i];
    if (threadIdx.x == 0) B.td[0][wdx] = B.td[1][wdx];
    for (int i = threadIdx.x; i < wd.L; i += blockDim.x) B.rho[0][wd.lm0 + i] = B.rho[1][wd.lm0 + i];
}

__global__ void k_lm_init(DevBatch B, double lambda0) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= B.numWindows) return;
    WinLM& st = B.lm[w];
    st.lambda = lambda0; st.nu = 2; st.cost = 0; st.initialCost = 0; st.linCost = 0; st.trialCost = 0; st.predicted = 0;
    st.maxInc = 0; st.mode = kModeLinearize; st.iterations = 0; st.accepted = 0; st.converged = 0; st.status = CGMLI_OK;
    st.acceptNow = 0; st.trialValid = 0;
    st.passStart = 0; st.passAccepted = 0; st.charged = 0; st.pass = 0; st.pad = 0;
    st.t0 = globalTimerNs();
}

// ---------------------------------------------------------------------------------------
// Per-factor evaluation at the accepted states (VisualCudaBatch::evaluate,
// VisualCudaBatch.cu:11-21,404-431): one thread per observation writes the
// whitened residual and, with derivatives, the 2 x 26 tangent Jacobian (anchor
// pose, observer pose, anchor extrinsic, observer extrinsic, td, rho; before the
// robust loss).  The accepted rotations are refreshed first by k_rotations.
__global__ void k_rotations(DevBatch B) {
    const WinDesc& wd = B.win[blockIdx.x];
    for (int k = threadIdx.x; k < wd.K; k += blockDim.x) poseRotation(B.pose[0] + 7ll * (wd.kf0 + k), B.rotKf[0] + 9ll * (wd.kf0 + k));
    for (int e = threadIdx.x; e < wd.E; e += blockDim.x) poseRotation(B.ext[0] + 7ll * (wd.ext0 + e), B.rotExt[0] + 9ll * (wd.ext0 + e));
}
constexpr int kFactorRecord = 2 + CGMLI_FACTOR_JACOBIAN;  // residual, then the Jacobian rows
__global__ void __launch_bounds__(128) k_evaluate(DevBatch B, int derivatives, double* out, int* valid) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= B.numObs) return;
    const int l = B.obLm[f], wdx = B.lmWin[l];
    const WinDesc wd = B.win[wdx];
    FactorIn in;
    int kfa, kfb, ea, eb;
    gatherFactor(B, wd, wdx, l, f, 0, in, kfa, kfb, ea, eb);
    FactorOut o;
    const bool ok = evalBearingFactor(in, derivatives != 0, o);
    double* dst = out + (long long)kFactorRecord * f;
    dst[0] = ok ? o.r[0] : 0.0;
    dst[1] = ok ? o.r[1] : 0.0;
    valid[f] = ok ? 1 : 0;
    if (!derivatives) return;
    for (int r = 0; r < 2; ++r) {
        double* J = dst + 2 + 26 * r;
        for (int c = 0; c < 6; ++c) {
            J[c] = ok ? o.Ja[6 * r + c] : 0.0;
            J[6 + c] = ok ? o.Jb[6 * r + c] : 0.0;
            J[12 + c] = ok ? o.Jea[6 * r + c] : 0.0;
            J[18 + c] = ok ? o.Jeb[6 * r + c] : 0.0;
        }
        J[24] = ok ? o.Jtd[r] : 0.0;
        J[25] = ok ? o.Jrho[r] : 0.0;
    }
}

// Caller-evaluated factors (solveOnline's retainedH / retainedG and the host
// trial cost, BackendOptimizer.cpp:210-225,276-279): adds the host's normal
// equations and cost to the retained system of each flagged window at a new
// linearization point, or the host's trial cost to the trial.
__global__ void k_add_host(DevBatch B, const double* hostH, const double* hostG, const double* hostCost, const unsigned char* flag,
                           int trial) {
    const int w = blockIdx.x;
    if (!flag[w]) return;
    const int mode = B.lm[w].mode;
    if (mode == kModeDone || (!trial && mode != kModeLinearize)) return;
    const WinDesc& wd = B.win[w];
    if (trial) {
        if (threadIdx.x == 0) B.trialRet[w] += hostCost[w];
        return;
    }
    const long long nn = (long long)wd.Nr * wd.Nr;
    for (long long i = threadIdx.x; i < nn; i += blockDim.x) B.Hret[wd.dense0 + i] += hostH[wd.dense0 + i];
    for (int i = threadIdx.x; i < wd.Nr; i += blockDim.x) B.gret[wd.vec0 + i] += hostG[wd.vec0 + i];
    if (threadIdx.x == 0) B.costRet[w] += hostCost[w];
}

// Observation payload (bearing 3, information square root 6, bearing velocity 3,
// time 1) from each window's caller order into device order: obOrig is the
// caller's index within the window, the window's obs0 its base.  One thread per
// observation; the source runs are contiguous within a landmark.
__global__ void k_gather_obs(const DevBatch B, const int* __restrict__ obOrig, const double* __restrict__ srcBearing,
                             const double* __restrict__ srcP, const double* __restrict__ srcVel, const double* __restrict__ srcTime,
                             double* __restrict__ bearing, double* __restrict__ P, double* __restrict__ vel, double* __restrict__ time) {
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < B.numObs; o += gridDim.x * blockDim.x) {
        const long long f = (long long)B.win[B.lmWin[B.obLm[o]]].obs0 + obOrig[o];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            bearing[3ll * o + k] = srcBearing[3 * f + k];
            vel[3ll * o + k] = srcVel[3 * f + k];
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) P[6ll * o + k] = srcP[6 * f + k];
        time[o] = srcTime[f];
    }
}

// ---------------------------------------------------------------------------------------
// host-side launchers (called by backend_host.cu)
void launchGatherObservations(const DevBatch& B, const int* obOrig, const double* const src[4], double* const dst[4],
                              cudaStream_t s) {
    if (B.numObs <= 0) return;
    const int blocks = (int)std::min<long long>((B.numObs + 255) / 256, 148ll * 8);
    k_gather_obs<<<blocks, 256, 0, s>>>(B, obOrig, src[0], src[1], src[2], src[3], dst[0], dst[1], dst[2], dst[3]);
}
void launchEvaluate(const DevBatch& B, int derivatives, double* out, int* valid, cudaStream_t s) {
    k_rotations<<<B.numWindows, 64, 0, s>>>(B);
    if (B.numObs > 0) k_evaluate<<<(B.numObs + 127) / 128, 128, 0, s>>>(B, derivatives, out, valid);
}
void launchAddHost(const DevBatch& B, const double* hostH, const double* hostG, const double* hostCost, const unsigned char* flag,
                   int trial, cudaStream_t s) {
    k_add_host<<<B.numWindows, 256, 0, s>>>(B, hostH, hostG, hostCost, flag, trial);
}
size_t linearizeSmemBytes(int maxNs, bool mixed) {  // the widest shape's
    size_t m = 0;
    for (const KernelShape& k : kLinShapeTable) m = std::max(m, (size_t)k.warps * landmarkWarpBytes(maxNs, mixed));
    return m;
}
size_t schurSmemBytes() { return kSchurSmemDoubles * sizeof(double); }
size_t wideFinishSmemBytes(int maxNr) { return (4 * (size_t)maxNr + kFacPanel * kFacPanel) * sizeof(double); }
size_t factorSmemBytes(int maxNr) {
    // one panel of kFacPanel columns over the padded rows, four n-vectors, the diagonal block
    const size_t npad = (((size_t)maxNr + 31) & ~(size_t)31) + kFacPanel;
    return (npad * kFacPanel + 4 * (size_t)maxNr + kFacPanel * kFacPanel) * sizeof(double);
}

// The dynamic shared-memory cap is a per-function attribute shared by every
// solver in the process, so it is raised once to the device's opt-in maximum
// (each launch still requests only what its batch needs).
cudaError_t configureKernels(size_t linSmem, size_t facSmem, size_t wideSmem) {
    int device = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes la, lm, fa, sa, sd, pa, pm;
    if ((e = cudaFuncGetAttributes(&la, k_lin_landmark<false, 6, 2>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&lm, k_lin_landmark<true, 6, 2>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&pa, k_lin_pairs<false, false>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&pm, k_lin_pairs<true, false>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, k_factor)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&sa, k_lin_schur)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&sd, k_lin_schur_det)) != cudaSuccess) return e;
    cudaFuncAttributes wf;
    if ((e = cudaFuncGetAttributes(&wf, k_wide_finish)) != cudaSuccess) return e;
    const size_t wideMax = (size_t)optin - wf.sharedSizeBytes;
    if (wideSmem > wideMax) return cudaErrorInvalidValue;
    if ((e = cudaFuncSetAttribute(k_wide_finish, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wideMax)) != cudaSuccess) return e;
    cudaFuncAttributes wu;
    if ((e = cudaFuncGetAttributes(&wu, k_wide_update)) != cudaSuccess) return e;
    if (wideUpdateSmemBytes() > (size_t)optin - wu.sharedSizeBytes) return cudaErrorInvalidValue;
    if ((e = cudaFuncSetAttribute(k_wide_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wideUpdateSmemBytes())) != cudaSuccess)
        return e;
    const size_t linMax = (size_t)optin - std::max(la.sharedSizeBytes, lm.sharedSizeBytes), facMax = (size_t)optin - fa.sharedSizeBytes;
    const size_t schMax = (size_t)optin - std::max(sa.sharedSizeBytes, sd.sharedSizeBytes);
    const size_t pairMax = (size_t)optin - std::max(pa.sharedSizeBytes, pm.sharedSizeBytes);
    if (linSmem > linMax || facSmem > facMax || schurSmemBytes() > schMax || pairCtaBytes() > pairMax) return cudaErrorInvalidValue;
    for (auto k : {k_lin_pairs<false, false>, k_lin_pairs<true, false>, k_lin_pairs<false, true>, k_lin_pairs<true, true>})
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pairCtaBytes())) != cudaSuccess) return e;
    for (auto k : {k_lin_landmark<false, 6, 2>, k_lin_landmark<true, 6, 2>, k_lin_landmark<false, 8, 1>, k_lin_landmark<true, 8, 1>,
                   k_lin_landmark<false, 4, 3>, k_lin_landmark<true, 4, 3>, k_lin_landmark<false, 6, 1>, k_lin_landmark<true, 6, 1>})
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)linMax)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_lin_schur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)schMax)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_lin_schur_det, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)schMax)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)facMax);
}

// The landmark and trial passes in the kernel shape the plan names.
template <bool Mixed, int Warps, int MinBlocks>
void linLandmarkShape(const DevBatch& B, const LaunchPlan& P, cudaStream_t s) {
    const int blocks = (B.numRuns + Warps - 1) / Warps;
    k_lin_landmark<Mixed, Warps, MinBlocks><<<blocks, Warps * 32, Warps * landmarkWarpBytes(P.maxNs, Mixed), s>>>(B, P.runs, P.tiles,
                                                                                                                P.maxNs);
}
template <bool Mixed>
void linLandmarkMixed(const DevBatch& B, const LaunchPlan& P, cudaStream_t s) {
    switch (P.linShape) {
        case 1: linLandmarkShape<Mixed, 8, 1>(B, P, s); break;
        case 2: linLandmarkShape<Mixed, 4, 3>(B, P, s); break;
        case 3: linLandmarkShape<Mixed, 6, 1>(B, P, s); break;
        default: linLandmarkShape<Mixed, 6, 2>(B, P, s); break;
    }
}
static_assert(kLinShapes == 4 && kLinShapeTable[1].warps == 8 && kLinShapeTable[2].minBlocks == 3, "shape table and dispatch");
void launchLinLandmark(const DevBatch& B, const LaunchPlan& P, cudaStream_t s) {
    if (B.mixed) linLandmarkMixed<true>(B, P, s);
    else linLandmarkMixed<false>(B, P, s);
}
template <int Warps, int MinBlocks>
void trialShape(const DevBatch& B, const LaunchPlan& P, cudaStream_t s) {
    k_trial<Warps, MinBlocks><<<(P.numTiles + Warps - 1) / Warps, Warps * 32, 0, s>>>(B, P.tiles, P.numTiles);
}
static_assert(kTrialShapes == 3 && kTrialShapeTable[1].minBlocks == 1 && kTrialShapeTable[2].warps == 4, "shape table and dispatch");
void launchTrial(const DevBatch& B, const LaunchPlan& P, cudaStream_t s) {
    switch (P.trialShape) {
        case 1: trialShape<8, 1>(B, P, s); break;
        case 2: trialShape<4, 4>(B, P, s); break;
        default: trialShape<8, 2>(B, P, s); break;
    }
}

// One LM iteration in three parts (kIterLinearize: the linearization up to the
// retained system; kIterStep: factorization, candidate, back-substitution and
// trial costs; kIterDecide: the LM decision and acceptance), so that a
// host-driven loop can add caller-evaluated factors between them.
int launchIterationParts(const DevBatch& B, const LaunchPlan& P, int refinement, int maxIterations, int probe, double* Sdebug,
                         cudaStream_t s, LaunchHook hook, void* ctx, int parts) {
    const int W = B.numWindows;
    int n = 0;
    auto run = [&](int kind, auto&& launch) {
        if (hook) hook(ctx, kind, 0);
        launch();
        if (hook) hook(ctx, kind, 1);
        ++n;
    };
    if (parts & kIterLinearize) {
    run(CGMLI_KERNEL_ZERO, [&] { k_zero_acc<<<W, 256, 0, s>>>(B); });
    if (B.numRuns > 0) run(CGMLI_KERNEL_LINEARIZE, [&] { launchLinLandmark(B, P, s); });
    const bool det = B.detSlots != nullptr;
    if (P.numPairChunks > 0)
        run(CGMLI_KERNEL_LIN_PAIRS, [&] {
            const int4* units = det ? P.detPairs : P.pairChunks;
            const int n = det ? P.numDetPairs : P.numPairChunks, blocks = (n + kPairWarps - 1) / kPairWarps;
            const size_t smem = pairCtaBytes();
            if (B.mixed && det) k_lin_pairs<true, true><<<blocks, kPairWarps * 32, smem, s>>>(B, units, n);
            else if (B.mixed) k_lin_pairs<true, false><<<blocks, kPairWarps * 32, smem, s>>>(B, units, n);
            else if (det) k_lin_pairs<false, true><<<blocks, kPairWarps * 32, smem, s>>>(B, units, n);
            else k_lin_pairs<false, false><<<blocks, kPairWarps * 32, smem, s>>>(B, units, n);
        });
    if (P.numSchurChunks > 0)
        run(CGMLI_KERNEL_LIN_SCHUR, [&] {
            if (det) k_lin_schur_det<<<P.numDetSchur, kSchurThreads, schurSmemBytes(), s>>>(B, P.schurChunks, P.detSchur);
            else k_lin_schur<<<P.numSchurChunks, kSchurThreads, schurSmemBytes(), s>>>(B, P.schurChunks);
        });
    if (det && (P.numPairChunks > 0 || P.numSchurChunks > 0))
        run(CGMLI_KERNEL_LIN_SCHUR, [&] { k_det_reduce<<<dim3(W, 4), 256, 0, s>>>(B); });
    run(CGMLI_KERNEL_RETAINED, [&] { k_retained<<<W, 256, 0, s>>>(B, 0); });
    }
    if (parts & kIterStep) {
    run(CGMLI_KERNEL_FACTOR, [&] { k_factor<<<W, kFactorThreads, P.facSmem, s>>>(B, refinement, Sdebug); });
    if (P.numWide > 0) {  // the wide sequence (windows of at least kWideCols columns)
        run(CGMLI_KERNEL_FACTOR, [&] { k_wide_assemble<<<dim3(P.numWide, (P.wideCols + 31) / 32, 4), 256, 0, s>>>(B); });
        if (P.wideCharts || Sdebug) run(CGMLI_KERNEL_FACTOR, [&] { k_wide_prepare<<<P.numWide, kFactorThreads, 0, s>>>(B, Sdebug); });
        run(CGMLI_KERNEL_FACTOR, [&] { k_wide_diag<<<P.numWide, kFactorThreads, 0, s>>>(B); });
        for (int k0 = 0; k0 + kFacPanel < P.wideCols; k0 += kFacPanel) {
            const int m2 = P.wideCols - k0 - kFacPanel, nb2 = (m2 + 31) >> 5, tiles = nb2 * (nb2 + 1) / 2;
            const dim3 grid(P.numWide, 1 + (tiles - 1 + kFactorThreads / 32 - 1) / (kFactorThreads / 32));
            run(CGMLI_KERNEL_FACTOR, [&] { k_wide_update<<<grid, kFactorThreads, wideUpdateSmemBytes(), s>>>(B, k0, P.wideCols); });
        }
        run(CGMLI_KERNEL_FACTOR, [&] { k_wide_finish<<<P.numWide, kFactorThreads, P.wideFinishSmem, s>>>(B, refinement, P.wideCols); });
        if (refinement == 0) {  // windows without charts: the product over the GPU, then the prediction
            const dim3 blocks(P.numWide, (P.wideCols + 31) / 32);
            run(CGMLI_KERNEL_FACTOR, [&] { k_wide_product<<<blocks, kFactorThreads, 0, s>>>(B, refinement, P.wideCols); });
            run(CGMLI_KERNEL_FACTOR, [&] { k_wide_predict<<<P.numWide, kFactorThreads, 0, s>>>(B, refinement, P.wideCols); });
        }
    }
    run(CGMLI_KERNEL_CANDIDATE, [&] { k_candidate<<<W, 128, 0, s>>>(B); });
    if (B.numLandmarks > 0) {
        run(CGMLI_KERNEL_BACKSUB_TRIAL, [&] { k_backsub<<<(B.numLandmarks * 8 + 255) / 256, 256, 0, s>>>(B); });
        run(CGMLI_KERNEL_BACKSUB_TRIAL, [&] { launchTrial(B, P, s); });
    }
    run(CGMLI_KERNEL_RETAINED_TRIAL, [&] { k_retained<<<W, 256, 0, s>>>(B, 1); });
    }
    if (parts & kIterDecide) {
    run(CGMLI_KERNEL_LM_UPDATE, [&] { k_lm_update<<<W, 256, 0, s>>>(B, maxIterations, probe); });
    if (!probe) run(CGMLI_KERNEL_ACCEPT, [&] { k_accept<<<W, 256, 0, s>>>(B); });
    }
    return n;
}
int launchIteration(const DevBatch& B, const LaunchPlan& P, int refinement, int maxIterations, int probe, double* Sdebug,
                    cudaStream_t s, LaunchHook hook, void* ctx) {
    return launchIterationParts(B, P, refinement, maxIterations, probe, Sdebug, s, hook, ctx, kIterLinearize | kIterStep | kIterDecide);
}
int launchGate(const DevBatch& B, const LaunchPlan& P, int pass, int pre, double threshold, double* obP, unsigned char* rejected,
               double* gateStats, int* gateCounts, cudaStream_t s) {
    k_gate_prepare<<<B.numWindows, 128, 0, s>>>(B, pass, pre, gateStats, gateCounts);
    if (P.numTiles > 0)
        k_gate<<<(P.numTiles + kTrialWarps - 1) / kTrialWarps, kTrialWarps * 32, 0, s>>>(B, P.tiles, P.numTiles, pass, pre, threshold,
                                                                                         obP, rejected, gateStats, gateCounts);
    return P.numTiles > 0 ? 2 : 1;
}
int launchRefit(const DevBatch& B, int pass, double lambda0, int maxIterations, const int* gateCounts, cudaStream_t s) {
    k_lm_refit<<<(B.numWindows + 127) / 128, 128, 0, s>>>(B, pass, lambda0, maxIterations, gateCounts);
    return 1;
}
int launchLmInit(const DevBatch& B, double lambda0, cudaStream_t s) {
    k_lm_init<<<(B.numWindows + 127) / 128, 128, 0, s>>>(B, lambda0);
    return 1;
}

}  // namespace cgmli
