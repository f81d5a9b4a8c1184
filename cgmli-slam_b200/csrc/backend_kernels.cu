// sm_100a kernels of the sliding-window backend hot path.
//
// One LM iteration over a batch of windows is the launch sequence
//   zero_acc -> linearize -> retained -> factor -> candidate -> backsub_trial
//   -> retained_trial -> lm_update -> accept
// with every decision of the damped LM loop (BackendOptimizer.cpp:167-307)
// taken on the device from per-window state (WinLM), so that a whole solve
// runs without a host round trip and can be captured in a CUDA graph.
#include <cuda_runtime.h>

#include "../../include/cgmli_backend.h"
#include "backend_internal.h"
#include "device_math.cuh"
#include "factor_eval.cuh"

namespace cgmli {

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
// zero the visual accumulators of windows that will be (re)linearized
__global__ void k_zero_acc(DevBatch B) {
    const int w = blockIdx.x;
    if (B.lm[w].mode == kModeDone) return;
    const WinDesc& wd = B.win[w];
    const long long n = (long long)wd.Npc * (wd.Npc + 1) / 2 + 3ll * wd.Npc;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) B.acc[wd.acc0 + i] = 0.0;
}

// ---------------------------------------------------------------------------------------
// Linearization of the bearing factors fused with the per-landmark Schur
// complement at the window's current lambda.  Per landmark l (scalar inverse
// distance) with observations f:
//   d_l = sum J_rho^T J_rho,  g_l = sum J_rho^T r,  c_l = sum J_x^T J_rho
//   S  += sum_f J_f^T J_f - c_l c_l^T / (d_l + lambda max(d_l, 1e-6))
//   rhs correction += c_l g_l / (d_l + lambda max(d_l, 1e-6))
// (accumulateVisualPairs + subtractPointSchur, VisualCudaBatch.cu:74-96,149-161).
//
// Work unit: a run = consecutive landmarks of one window, sorted by their
// keyframe support, processed by one warp in tiles of <= 32 observations
// (lane = observation for the evaluation).  The weighted Jacobians of a tile
// are staged in shared memory; each landmark's dense local block over its
// support (6 columns per keyframe slot + the calibration columns) is formed
// with lanes over distinct entries and added to a warp-private FP64 group
// buffer.  Landmarks with the same support share the buffer; it is flushed to
// the window accumulator with global FP64 reductions when the support changes.
constexpr int kLinWarps = 6;
constexpr int kStage = 56;          // doubles staged per observation
constexpr int kGroupMaxNs = 64;     // largest support width that is buffered
constexpr int kGroupBuf = kGroupMaxNs * (kGroupMaxNs + 1) / 2 + 3 * kGroupMaxNs;
constexpr int kMaxNs = 6 * (kMaxSupport + 8) + 1;
constexpr int kCompact = 25;        // anchor pose 6 | observer pose 6 | ext_a 6 | ext_b 6 | td 1
constexpr int kPairs = kCompact * (kCompact + 1) / 2;
struct LinWarpSmem {
    double stage[32][kStage];  // compact weighted row pair: row0 at [0,25), row1 at [25,50), Jrho 50,51 | r 52,53 | cost 54
    short map[32][kCompact];        // local column of each compact column, -1 if absent
    int flags[32];                  // 1 valid
    double c[kMaxNs];
    double gbuf[kGroupBuf];
};
__constant__ unsigned char kPairA[kPairs], kPairB[kPairs];

// Local column -> visual column for a support (s keyframe slots, x extrinsic slots, td).
__device__ __forceinline__ int pcOfLocal(int i, int s, int x, const int* sk, int K, int tdCol) {
    if (i < 6 * s) return 6 * sk[i / 6] + i % 6;
    if (i < 6 * (s + x)) return 6 * K + 6 * sk[s + (i - 6 * s) / 6] + i % 6;
    return tdCol;
}

// Adds a group buffer (local coordinates of a support) into the window accumulator.
__device__ void flushGroup(const double* gbuf, int ns, int s, int x, const int* sk, int K, int tdCol, int Npc, double* acc,
                           int lane) {
    const int ntri = ns * (ns + 1) / 2;
    const long long nS = (long long)Npc * (Npc + 1) / 2;
    int i = 0, j = lane;
    while (j >= ns && i < ns) { ++i; j = j - ns + i; }
    for (int e = lane; e < ntri; e += 32) {
        const double v = gbuf[e];
        if (v != 0.0) {
            const int pi = pcOfLocal(i, s, x, sk, K, tdCol), pj = pcOfLocal(j, s, x, sk, K, tdCol);
            atomicAdd(&acc[pi <= pj ? upIdx(pi, pj, Npc) : upIdx(pj, pi, Npc)], v);
        }
        j += 32;
        while (j >= ns && i < ns) { ++i; j = j - ns + i; }
    }
    for (int t = lane; t < 3 * ns; t += 32) {
        const double v = gbuf[ntri + t];
        if (v != 0.0) atomicAdd(&acc[nS + (long long)(t / ns) * Npc + pcOfLocal(t % ns, s, x, sk, K, tdCol)], v);
    }
}

__device__ __forceinline__ int localUp(int i, int j, int ns) { return i * ns - i * (i - 1) / 2 + (j - i); }

__global__ void __launch_bounds__(kLinWarps * 32) k_linearize(DevBatch B, const int4* runs, const int2* tiles) {
    extern __shared__ double smemRaw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int runIdx = blockIdx.x * kLinWarps + warp;
    if (runIdx >= B.numRuns) return;
    const int4 run = runs[runIdx];  // {window, tile begin, tile end, -}
    const int wdx = run.x;
    if (B.lm[wdx].mode == kModeDone) return;
    LinWarpSmem& sm = reinterpret_cast<LinWarpSmem*>(smemRaw)[warp];
    const WinDesc wd = B.win[wdx];
    const double lambda = B.lm[wdx].lambda;
    const int K = wd.K, Npc = wd.Npc;
    const int tdCol = 6 * K + (wd.estExt ? 6 * wd.E : 0);
    double* acc = B.acc + wd.acc0;
    const long long nS = (long long)Npc * (Npc + 1) / 2;
    int curGroup = -1, curNs = 0, curS = 0, curX = 0;
    const int* curSk = nullptr;
    bool buffered = false;
    for (int t = run.y; t < run.z; ++t) {
        const int2 tile = tiles[t];
        const int lb = tile.x, le = tile.y;
        const int ob = B.lmObsBegin[lb], oe = B.lmObsBegin[le];
        // ---- evaluation: lane = observation; stage the weighted compact rows
        const int f = ob + lane;
        if (f < oe) {
            int q = 0;
            while (B.lmObsBegin[lb + q + 1] <= f) ++q;
            const int l = lb + q;
            FactorIn in;
            int kfa, kfb, ea, eb;
            gatherFactor(B, wd, wdx, l, f, 0, in, kfa, kfb, ea, eb);
            FactorOut o;
            double* st = sm.stage[lane];
            short* mp = sm.map[lane];
            const bool ok = evalBearingFactor(in, true, o);
            const int s = B.lmNs[l], x = B.lmNx[l];
            const bool same = in.sameKf && !in.splitExt;
            const int obSlot = B.obSlot[f], obX = B.obXslot[f];
            for (int c = 0; c < 6; ++c) {
                mp[c] = in.sameKf ? -1 : c;
                mp[6 + c] = in.sameKf ? -1 : 6 * obSlot + c;
                mp[12 + c] = (wd.estExt && !same) ? 6 * s + c : -1;  // anchor camera's extrinsic = ext slot 0
                mp[18 + c] = (wd.estExt && in.splitExt) ? 6 * (s + obX) + c : -1;
            }
            mp[24] = wd.estTd ? 6 * (s + x) : -1;
            sm.flags[lane] = ok ? 1 : 0;
            if (ok) {
                const double sq = o.r[0] * o.r[0] + o.r[1] * o.r[1];
                const double w = huberWeight(wd.huber, sq);
#pragma unroll
                for (int r = 0; r < 2; ++r) {
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        st[25 * r + c] = w * o.Ja[6 * r + c];
                        st[25 * r + 6 + c] = w * o.Jb[6 * r + c];
                        st[25 * r + 12 + c] = w * o.Jea[6 * r + c];
                        st[25 * r + 18 + c] = w * o.Jeb[6 * r + c];
                    }
                    st[25 * r + 24] = w * o.Jtd[r];
                }
                st[50] = w * o.Jrho[0]; st[51] = w * o.Jrho[1];
                st[52] = w * o.r[0]; st[53] = w * o.r[1];
                st[54] = huberCost(wd.huber, sq);
            } else {
                for (int k = 0; k < kStage; ++k) st[k] = 0.0;
            }
        }
        __syncwarp();
        // ---- per landmark of the tile
        for (int l = lb; l < le; ++l) {
            const int fb = B.lmObsBegin[l] - ob, fe = B.lmObsBegin[l + 1] - ob;
            const int s = B.lmNs[l], x = B.lmNx[l], ns = 6 * (s + x) + (wd.estTd ? 1 : 0);
            const int* sk = B.supp + B.lmSupp0[l];
            const int group = B.lmGroup[l];
            if (group != curGroup) {
                if (buffered) { __syncwarp(); flushGroup(sm.gbuf, curNs, curS, curX, curSk, K, tdCol, Npc, acc, lane); }
                curGroup = group; curNs = ns; curS = s; curX = x; curSk = sk;
                buffered = ns <= kGroupMaxNs;
                __syncwarp();
                if (buffered) {
                    const int n = ns * (ns + 1) / 2 + 3 * ns;
                    for (int e = lane; e < n; e += 32) sm.gbuf[e] = 0.0;
                }
                __syncwarp();
            }
            const int ntri = ns * (ns + 1) / 2;
            // scalars: d, g, cost, validity
            double d = 0, g = 0, cost = 0;
            int valid = 1;
            for (int k = fb + lane; k < fe; k += 32) {
                const double* st = sm.stage[k];
                d += st[50] * st[50] + st[51] * st[51];
                g += st[50] * st[52] + st[51] * st[53];
                cost += st[54];
                valid &= sm.flags[k];
            }
            d = warpSum(d); g = warpSum(g); cost = warpSum(cost);
            valid = __all_sync(0xffffffffu, valid);
            const double inv = 1.0 / (d + lambda * fmax(d, 1e-6));
            for (int i = lane; i < ns; i += 32) sm.c[i] = 0.0;
            __syncwarp();
            // per observation: cross vector, diag(H) and gradient over the compact columns
            for (int k = fb; k < fe; ++k) {
                const double* st = sm.stage[k];
                const short* mp = sm.map[k];
                if (lane < kCompact) {
                    const int li = mp[lane];
                    if (li >= 0) {
                        const double a0 = st[lane], a1 = st[25 + lane];
                        sm.c[li] += a0 * st[50] + a1 * st[51];
                        const double hd = a0 * a0 + a1 * a1, gr = a0 * st[52] + a1 * st[53];
                        if (buffered) { sm.gbuf[ntri + li] += hd; sm.gbuf[ntri + ns + li] += gr; }
                        else {
                            const int p = pcOfLocal(li, s, x, sk, K, tdCol);
                            atomicAdd(&acc[nS + p], hd);
                            atomicAdd(&acc[nS + Npc + p], gr);
                        }
                    }
                }
                __syncwarp();
                // J^T J over the compact pairs
                for (int pidx = lane; pidx < kPairs; pidx += 32) {
                    const int a = kPairA[pidx], b = kPairB[pidx];
                    const int la = mp[a], lb2 = mp[b];
                    if (la < 0 || lb2 < 0) continue;
                    const double v = st[a] * st[b] + st[25 + a] * st[25 + b];
                    if (v == 0.0) continue;
                    const int i = la < lb2 ? la : lb2, j = la < lb2 ? lb2 : la;
                    if (buffered) sm.gbuf[localUp(i, j, ns)] += v;
                    else {
                        const int pi = pcOfLocal(i, s, x, sk, K, tdCol), pj = pcOfLocal(j, s, x, sk, K, tdCol);
                        atomicAdd(&acc[pi <= pj ? upIdx(pi, pj, Npc) : upIdx(pj, pi, Npc)], v);
                    }
                }
                __syncwarp();
            }
            // Schur complement of the inverse distance and the rhs correction
            const long long c0 = B.lmC0[l];
            for (int i = lane; i < ns; i += 32) {
                const double ci = sm.c[i];
                B.lmC[c0 + i] = ci;
                const double bc = inv * ci * g;
                if (buffered) sm.gbuf[ntri + 2 * ns + i] += bc;
                else if (bc != 0.0) atomicAdd(&acc[nS + 2ll * Npc + pcOfLocal(i, s, x, sk, K, tdCol)], bc);
            }
            {
                int i = 0, j = lane;
                while (j >= ns && i < ns) { ++i; j = j - ns + i; }
                for (int e = lane; e < ntri; e += 32) {
                    const double v = -inv * sm.c[i] * sm.c[j];
                    if (buffered) sm.gbuf[e] += v;
                    else if (v != 0.0) {
                        const int pi = pcOfLocal(i, s, x, sk, K, tdCol), pj = pcOfLocal(j, s, x, sk, K, tdCol);
                        atomicAdd(&acc[pi <= pj ? upIdx(pi, pj, Npc) : upIdx(pj, pi, Npc)], v);
                    }
                    j += 32;
                    while (j >= ns && i < ns) { ++i; j = j - ns + i; }
                }
            }
            if (lane == 0) { B.lmD[l] = d; B.lmG[l] = g; B.lmCost[l] = cost; B.lmValid[l] = valid; }
            __syncwarp();
        }
    }
    if (buffered) { __syncwarp(); flushGroup(sm.gbuf, curNs, curS, curX, curSk, K, tdCol, Npc, acc, lane); }
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
__global__ void __launch_bounds__(256) k_retained(DevBatch B, int trial) {
    const int wdx = blockIdx.x;
    const int mode = B.lm[wdx].mode;
    if (mode == kModeDone || (!trial && mode != kModeLinearize)) return;
    const WinDesc wd = B.win[wdx];
    const int Nr = wd.Nr, buf = trial ? 1 : 0;
    __shared__ double red[32];
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    double* H = B.Hret + wd.dense0;
    double* g = B.gret + wd.vec0;
    if (!trial) {
        for (long long i = threadIdx.x; i < (long long)Nr * Nr; i += blockDim.x) H[i] = 0.0;
        for (int i = threadIdx.x; i < Nr; i += blockDim.x) g[i] = 0.0;
    }
    __syncthreads();
    double cost = 0;
    const cgmli_frozen_imu* imus = reinterpret_cast<const cgmli_frozen_imu*>(B.imu);
    double* scratch = B.imuScratch + wd.imuScratch0;
    for (int i = threadIdx.x; i < wd.nImu; i += blockDim.x) {
        const int gi = wd.imu0 + i;
        const int k = B.imuKf[gi];
        double* r = scratch + 465ll * i;
        const bool ok = evalImu(imus[gi], B.pose[buf] + 7ll * k, B.sb[buf] + 9ll * k, B.pose[buf] + 7ll * (k + 1),
                                B.sb[buf] + 9ll * (k + 1), r, trial ? nullptr : r + 15);
        if (!ok) atomicOr(&bad, 1);
        else for (int m = 0; m < 15; ++m) cost += 0.5 * r[m] * r[m];
    }
    __syncthreads();
    if (!trial) {
        for (int i = 0; i < wd.nImu; ++i) {
            const int k = B.imuKf[wd.imu0 + i] - wd.kf0;
            const double* r = scratch + 465ll * i;
            const double* J = r + 15;
            for (int e = threadIdx.x; e < 930; e += blockDim.x) {
                const int a = e < 900 ? e / 30 : e - 900, b = e % 30;
                if (e < 900) {
                    double v = 0;
                    for (int m = 0; m < 15; ++m) v += J[30 * m + a] * J[30 * m + b];
                    H[(long long)(15 * k + a) * Nr + 15 * k + b] += v;
                } else {
                    double v = 0;
                    for (int m = 0; m < 15; ++m) v += J[30 * m + a] * r[m];
                    g[15 * k + a] += v;
                }
            }
            __syncthreads();
        }
    }
    if (wd.priorRank > 0) {
        const int rank = wd.priorRank, cols = wd.priorCols;
        double* ps = B.priorScratch + wd.priorScratch0;
        double* delta = ps;           // cols
        double* D = delta + cols;     // cols x 6
        double* r = D + 6ll * cols;   // rank
        double* J = r + rank;         // rank x cols
        for (int b = threadIdx.x; b < wd.priorBlocks; b += blockDim.x) {
            const int pb = wd.priorBlk0 + b;
            const int kind = B.priorKind[pb], off = B.priorOff[pb];
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
                const int i = (int)(e / cols), c = (int)(e % cols);
                // block of column c
                int pb = wd.priorBlk0;
                while (pb + 1 < wd.priorBlk0 + wd.priorBlocks && B.priorOff[pb + 1] <= c) ++pb;
                const int kind = B.priorKind[pb], off = B.priorOff[pb];
                double v;
                if (kind == CGMLI_PRIOR_POSE || kind == CGMLI_PRIOR_EXTRINSIC) {
                    v = 0;
                    for (int j = 0; j < 6; ++j) v += A[(long long)i * cols + off + j] * D[6ll * (off + j) + (c - off)];
                } else {
                    v = A[(long long)i * cols + c];
                }
                J[e] = v;
            }
            __syncthreads();
            for (long long e = threadIdx.x; e < (long long)cols * (cols + 1); e += blockDim.x) {
                const int p = (int)(e / cols), q = (int)(e % cols);
                int bp = wd.priorBlk0, bq = wd.priorBlk0;
                const int pp = p < cols ? p : q;
                while (bp + 1 < wd.priorBlk0 + wd.priorBlocks && B.priorOff[bp + 1] <= pp) ++bp;
                while (bq + 1 < wd.priorBlk0 + wd.priorBlocks && B.priorOff[bq + 1] <= q) ++bq;
                const int colP = B.priorCol[bp], colQ = B.priorCol[bq];
                if (p < cols) {
                    if (colP < 0 || colQ < 0) continue;
                    double v = 0;
                    for (int i = 0; i < rank; ++i) v += J[(long long)i * cols + p] * J[(long long)i * cols + q];
                    H[(long long)(colP + p - B.priorOff[bp]) * Nr + colQ + q - B.priorOff[bq]] += v;
                } else {
                    if (colQ < 0) continue;
                    double v = 0;
                    for (int i = 0; i < rank; ++i) v += J[(long long)i * cols + q] * r[i];
                    g[colQ + q - B.priorOff[bq]] += v;
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
// The factor is kept packed lower/column-major in shared memory when it fits.
__device__ __forceinline__ double assembleEntry(const DevBatch& B, const WinDesc& wd, int i, int j, double lambda, bool damp) {
    const int Nr = wd.Nr, Npc = wd.Npc, K = wd.K;
    const double* H = B.Hret + wd.dense0;
    const double* acc = B.acc + wd.acc0;
    double v = H[(long long)i * Nr + j];
    const int pi = pcOfRetained(i, K), pj = pcOfRetained(j, K);
    if (pi >= 0 && pj >= 0) v += acc[pi <= pj ? upIdx(pi, pj, Npc) : upIdx(pj, pi, Npc)];
    if (damp && i == j) {
        double h = H[(long long)i * Nr + i];
        if (pi >= 0) h += acc[(long long)Npc * (Npc + 1) / 2 + pi];
        v += lambda * fmax(h, 1e-6);
    }
    return v;
}

__global__ void __launch_bounds__(kFactorThreads) k_factor(DevBatch B, int refinement, double* Sdebug) {
    const int wdx = blockIdx.x;
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const int Nr = wd.Nr, Npc = wd.Npc, K = wd.K;
    const double lambda = B.lm[wdx].lambda;
    extern __shared__ double smem[];
    __shared__ int failed;
    __shared__ double red[32];
    const bool inSmem = Nr <= kSmemPackedMax;
    double* L = inSmem ? smem : B.Sglob + wd.dense0;
    double* x = (inSmem ? smem : B.Sglob + wd.dense0) + (long long)Nr * (Nr + 1) / 2;  // working vector
    const double* acc = B.acc + wd.acc0;
    const long long nS = (long long)Npc * (Npc + 1) / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) failed = 0;
    for (int j = warp; j < Nr; j += nw)
        for (int i = j + lane; i < Nr; i += 32) {
            const double v = assembleEntry(B, wd, i, j, lambda, true);
            L[loIdx(i, j, Nr)] = v;
            if (Sdebug) { Sdebug[wd.dense0 + (long long)i * Nr + j] = v; Sdebug[wd.dense0 + (long long)j * Nr + i] = v; }
        }
    double* rhsOut = B.rhs + wd.vec0;
    for (int i = threadIdx.x; i < Nr; i += blockDim.x) {
        double g = B.gret[wd.vec0 + i];
        const int p = pcOfRetained(i, K);
        if (p >= 0) g += acc[nS + Npc + p] - acc[nS + 2ll * Npc + p];
        x[i] = -g;
        rhsOut[i] = -g;
    }
    __syncthreads();
    for (int k = 0; k < Nr; ++k) {
        if (threadIdx.x == 0) {
            const double v = L[loIdx(k, k, Nr)];
            if (!(v > 0) || !isfinite(v)) failed = 1;
            else L[loIdx(k, k, Nr)] = sqrt(v);
        }
        __syncthreads();
        if (failed) break;
        const double lkk = L[loIdx(k, k, Nr)];
        for (int i = k + 1 + threadIdx.x; i < Nr; i += blockDim.x) L[loIdx(i, k, Nr)] /= lkk;
        __syncthreads();
        for (int j = k + 1 + warp; j < Nr; j += nw) {
            const double ljk = L[loIdx(j, k, Nr)];
            for (int i = j + lane; i < Nr; i += 32) L[loIdx(i, j, Nr)] -= L[loIdx(i, k, Nr)] * ljk;
        }
        __syncthreads();
    }
    if (failed) {
        if (threadIdx.x == 0) B.solveStatus[wdx] = CGMLI_E_NOT_PD;
        return;
    }
    // solves with one warp: L y = x (column-oriented), L^T z = y (row-oriented)
    auto solveInPlace = [&](double* v) {
        if (warp == 0) {
            for (int k = 0; k < Nr; ++k) {
                const double yk = v[k] / L[loIdx(k, k, Nr)];
                __syncwarp();
                if (lane == 0) v[k] = yk;
                for (int i = k + 1 + lane; i < Nr; i += 32) v[i] -= L[loIdx(i, k, Nr)] * yk;
                __syncwarp();
            }
            for (int k = Nr - 1; k >= 0; --k) {
                double s = 0;
                for (int i = k + 1 + lane; i < Nr; i += 32) s += L[loIdx(i, k, Nr)] * v[i];
                s = warpSum(s);
                if (lane == 0) v[k] = (v[k] - s) / L[loIdx(k, k, Nr)];
                __syncwarp();
            }
        }
        __syncthreads();
    };
    solveInPlace(x);
    double* dr = B.dr + wd.vec0;
    for (int i = threadIdx.x; i < Nr; i += blockDim.x) dr[i] = x[i];
    __syncthreads();
    // iterative refinement against the assembled FP64 system
    for (int it = 0; it < refinement; ++it) {
        for (int i = threadIdx.x; i < Nr; i += blockDim.x) {
            double g = B.gret[wd.vec0 + i];
            const int p = pcOfRetained(i, K);
            if (p >= 0) g += acc[nS + Npc + p] - acc[nS + 2ll * Npc + p];
            double v = -g;
            for (int j = 0; j < Nr; ++j) v -= assembleEntry(B, wd, i, j, lambda, true) * dr[j];
            x[i] = v;
        }
        __syncthreads();
        solveInPlace(x);
        for (int i = threadIdx.x; i < Nr; i += blockDim.x) dr[i] += x[i];
        __syncthreads();
    }
    // predicted reduction of the state part with the undamped (S_visual + H_ret):
    //   -dx^T (g_r + 0.5 (S_v + H_ret) dx); the landmark terms are added per landmark.
    double pred = 0;
    for (int i = threadIdx.x; i < Nr; i += blockDim.x) {
        double hd = 0;
        for (int j = 0; j < Nr; ++j) hd += assembleEntry(B, wd, i, j, lambda, false) * dr[j];
        double g = B.gret[wd.vec0 + i];
        const int p = pcOfRetained(i, K);
        if (p >= 0) g += acc[nS + Npc + p];
        pred += -dr[i] * (g + 0.5 * hd);
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
    for (int k = threadIdx.x; k < wd.K; k += blockDim.x) {
        const int gk = wd.kf0 + k;
        posePlus(B.pose[0] + 7ll * gk, dr + 15 * k, B.pose[1] + 7ll * gk);
        for (int j = 0; j < 9; ++j) B.sb[1][9ll * gk + j] = B.sb[0][9ll * gk + j] + dr[15 * k + 6 + j];
    }
    for (int e = threadIdx.x; e < wd.E; e += blockDim.x) {
        const int ge = wd.ext0 + e;
        if (wd.estExt) posePlus(B.ext[0] + 7ll * ge, dr + 15 * wd.K + 6 * e, B.ext[1] + 7ll * ge);
        else for (int j = 0; j < 7; ++j) B.ext[1][7ll * ge + j] = B.ext[0][7ll * ge + j];
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
// VisualCudaBatch.cu:191-205) and the robust cost of the candidate point.
// Warp per tile; lane = landmark for the back-substitution, lane =
// observation for the trial residuals.
__global__ void __launch_bounds__(kLinWarps * 32) k_backsub_trial(DevBatch B, const int4* runs, const int2* tiles) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ double tcost[kLinWarps][32];
    __shared__ int tvalid[kLinWarps][32];
    const int runIdx = blockIdx.x * kLinWarps + warp;
    if (runIdx >= B.numRuns) return;
    const int4 run = runs[runIdx];
    const int wdx = run.x;
    if (B.lm[wdx].mode == kModeDone) return;
    const WinDesc wd = B.win[wdx];
    const double lambda = B.lm[wdx].lambda;
    const int K = wd.K;
    const double* dr = B.dr + wd.vec0;
    for (int t = run.y; t < run.z; ++t) {
        const int2 tile = tiles[t];
        const int lb = tile.x, le = tile.y, nl = le - lb;
        if (lane < nl) {
            const int l = lb + lane;
            const int s = B.lmNs[l], x = B.lmNx[l], ns = 6 * (s + x) + (wd.estTd ? 1 : 0);
            const double* c = B.lmC + B.lmC0[l];
            const int* sk = B.supp + B.lmSupp0[l];
            const int tdCol = 6 * K + (wd.estExt ? 6 * wd.E : 0);
            double cd = 0;
            for (int i = 0; i < ns; ++i) cd += c[i] * dr[retainedOfPc(pcOfLocal(i, s, x, sk, K, tdCol), K)];
            const double d = B.lmD[l], g = B.lmG[l];
            const double dt = d + lambda * fmax(d, 1e-6);
            double dl = -(g + cd) / dt;
            const double rho0 = B.rho[0][l];
            if (isfinite(dl)) dl = fmax(wd.minInv - rho0, dl);
            B.lmDelta[l] = dl;
            // landmark terms of -dx^T (g + 0.5 H dx): the cross term c.dx_r is
            // split between the state part (via S_v) and this correction
            B.lmPred[l] = -0.5 * cd * cd / dt - dl * (g + cd + 0.5 * d * dl);
            B.lmMaxInc[l] = isfinite(dl) ? fabs(dl) : -1.0;
            B.rho[1][l] = fmax(wd.minInv, rho0 + dl);
            tcost[warp][lane] = 0;
            tvalid[warp][lane] = isfinite(dl) ? 1 : 0;
        }
        __syncwarp();
        const int ob = B.lmObsBegin[lb], oe = B.lmObsBegin[le];
        const int f = ob + lane;
        if (f < oe) {
            int q = 0;
            while (B.lmObsBegin[lb + q + 1] <= f) ++q;
            const int l = lb + q;
            FactorIn in;
            int kfa, kfb, ea, eb;
            gatherFactor(B, wd, wdx, l, f, 1, in, kfa, kfb, ea, eb);
            FactorOut o;
            if (!evalBearingFactor(in, false, o)) tvalid[warp][q] = 0;
            else atomicAdd(&tcost[warp][q], huberCost(wd.huber, o.r[0] * o.r[0] + o.r[1] * o.r[1]));
        }
        __syncwarp();
        if (lane < nl) {
            B.lmTrial[lb + lane] = tcost[warp][lane];
            B.lmTrialValid[lb + lane] = tvalid[warp][lane];
        }
        __syncwarp();
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
    for (int i = threadIdx.x; i < wd.L; i += blockDim.x) {
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
        if (st.iterations == 0) st.cost = st.initialCost = linCost;
        else if (fabs(linCost - st.cost) > 1e-8 * fmax(1.0, st.cost)) {
            st.status = CGMLI_E_COST_MISMATCH; st.mode = kModeDone; st.acceptNow = 0; return;
        }
    }
    st.predicted = predicted;
    st.trialCost = trialCost;
    st.trialValid = tvalid;
    st.maxInc = mx;
    if (B.solveStatus[wdx] != CGMLI_OK) { st.status = B.solveStatus[wdx]; st.mode = kModeDone; st.acceptNow = 0; return; }
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
    if (st.iterations >= maxIterations && st.mode != kModeDone) st.mode = kModeDone;
    if (st.mode == kModeDone && st.status == CGMLI_OK && !st.accepted && !st.converged) st.status = CGMLI_E_NO_STEP;
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
}

// ---------------------------------------------------------------------------------------
// host-side launchers (called by backend_host.cu)
size_t linearizeSmemBytes() { return kLinWarps * sizeof(LinWarpSmem); }
size_t factorSmemBytes(int maxNr) {
    // windows with Nr <= kSmemPackedMax factor in shared memory; larger ones in global memory
    const size_t n = (size_t)(maxNr < kSmemPackedMax ? maxNr : kSmemPackedMax);
    return (n * (n + 1) / 2 + n) * sizeof(double);
}

// The dynamic shared-memory cap is a per-function attribute shared by every
// solver in the process, so it is raised once to the device's opt-in maximum
// (each launch still requests only what its batch needs).
cudaError_t configureKernels(size_t linSmem, size_t facSmem) {
    int device = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes la, fa;
    if ((e = cudaFuncGetAttributes(&la, k_linearize)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, k_factor)) != cudaSuccess) return e;
    const size_t linMax = (size_t)optin - la.sharedSizeBytes, facMax = (size_t)optin - fa.sharedSizeBytes;
    if (linSmem > linMax || facSmem > facMax) return cudaErrorInvalidValue;
    unsigned char pa[kPairs], pb[kPairs];
    int n = 0;
    for (int a = 0; a < kCompact; ++a)
        for (int b = a; b < kCompact; ++b) { pa[n] = (unsigned char)a; pb[n] = (unsigned char)b; ++n; }
    if ((e = cudaMemcpyToSymbol(kPairA, pa, sizeof pa)) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(kPairB, pb, sizeof pb)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_linearize, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)linMax)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)facMax);
}

int launchIteration(const DevBatch& B, const int4* runs, const int2* tiles, size_t linSmem, size_t facSmem,
                    int refinement, int maxIterations, int probe, double* Sdebug, cudaStream_t s, LaunchHook hook, void* ctx) {
    const int W = B.numWindows;
    int n = 0;
    auto run = [&](int kind, auto&& launch) {
        if (hook) hook(ctx, kind, 0);
        launch();
        if (hook) hook(ctx, kind, 1);
        ++n;
    };
    run(CGMLI_KERNEL_ZERO, [&] { k_zero_acc<<<W, 256, 0, s>>>(B); });
    const int runBlocks = (B.numRuns + kLinWarps - 1) / kLinWarps;
    if (B.numRuns > 0)
        run(CGMLI_KERNEL_LINEARIZE, [&] { k_linearize<<<runBlocks, kLinWarps * 32, linSmem, s>>>(B, runs, tiles); });
    run(CGMLI_KERNEL_RETAINED, [&] { k_retained<<<W, 256, 0, s>>>(B, 0); });
    run(CGMLI_KERNEL_FACTOR, [&] { k_factor<<<W, kFactorThreads, facSmem, s>>>(B, refinement, Sdebug); });
    run(CGMLI_KERNEL_CANDIDATE, [&] { k_candidate<<<W, 128, 0, s>>>(B); });
    if (B.numRuns > 0)
        run(CGMLI_KERNEL_BACKSUB_TRIAL, [&] { k_backsub_trial<<<runBlocks, kLinWarps * 32, 0, s>>>(B, runs, tiles); });
    run(CGMLI_KERNEL_RETAINED_TRIAL, [&] { k_retained<<<W, 256, 0, s>>>(B, 1); });
    run(CGMLI_KERNEL_LM_UPDATE, [&] { k_lm_update<<<W, 256, 0, s>>>(B, maxIterations, probe); });
    if (!probe) run(CGMLI_KERNEL_ACCEPT, [&] { k_accept<<<W, 256, 0, s>>>(B); });
    return n;
}
int launchLmInit(const DevBatch& B, double lambda0, cudaStream_t s) {
    k_lm_init<<<(B.numWindows + 127) / 128, 128, 0, s>>>(B, lambda0);
    return 1;
}

}  // namespace cgmli
