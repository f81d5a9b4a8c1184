// sm_100a kernels of the Schur-complement marginalization prior
// (Marginalizer::compute, src/backend/Marginalizer.cpp:284-474) and of the
// dense helpers of MarginalCudaWorkspace (src/backend/VisualCudaBatch.cu:898-957).
//
// Per window the consumed factors (all observations of the eliminated inverse
// distances, the IMU factors touching the victim keyframe, the previous prior)
// are linearized at the accepted states, with the Huber loss and with frozen
// calibration blocks differentiated too, into an FP64 system over
// [victim pose+speed/bias | separator]:
//   k_marg_eval      the eliminated landmarks' factors: largest information
//                    d of each window (the scalar cutoff max(1e-12, 1e-9 max d)
//                    of psdSolve) and the staged weighted rows
//   k_marg_rows      dense-row accumulation per run of a window's eliminated
//                    landmarks: factor rows and Schur rows c / sqrt(d) of the
//                    scalar eliminations, register-tiled rank updates
//   k_marg_visual    windows above kRowsMaxN visual columns: one CTA per
//                    eliminated landmark, its factors' normal blocks and its
//                    own scalar Schur term -c c^T / d summed in shared memory
//   k_marg_retained  IMU factors of the victim and the previous prior
//   k_marg_victim    victim block removed by the eigen-based PSD solve
//   k_marg_eigen     Jacobi eigendecomposition of the separator information,
//                    rank cutoff, A = sqrt(lambda) u^T, r0 = u^T b / sqrt(lambda)
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "../../include/cgmli_backend.h"
#include "backend_internal.h"
#include "device_math.cuh"
#include "dense_tiles.cuh"
#include "factor_eval.cuh"

namespace cgmli {

namespace {
__device__ __forceinline__ double mWarpSum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// block-wide sum; every thread gets the result
__device__ double mBlockSum(double v, double* red) {
    v = mWarpSum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0;
    for (int i = 0; i < nw; ++i) t += red[i];
    __syncthreads();
    return t;
}
__device__ double mBlockMax(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = red[0];
    for (int i = 1; i < nw; ++i) t = fmax(t, red[i]);
    __syncthreads();
    return t;
}
// non-negative doubles order like their bit patterns
__device__ __forceinline__ void atomicMaxNonNegative(double* a, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(a), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ int packedUp(int i, int j, int n) { return i * n - i * (i - 1) / 2 + (j - i); }
// symmetric entry of an upper-stored row-major matrix
__device__ __forceinline__ double symAt(const double* H, int i, int j, int m) {
    return i <= j ? H[(long long)i * m + j] : H[(long long)j * m + i];
}

// Weighted factor of observation f of eliminated landmark l, with the
// marginalization's derivative set (extrinsics always, td whenever the window
// has one).  Returns false on an invalid linearization point.
__device__ bool margFactor(const DevBatch& B, const WinDesc& wd, int w, int l, int f, FactorIn& in, FactorOut& o, double& wgt,
                           double& sq, int& kfa, int& kfb, int& ea, int& eb) {
    gatherFactor(B, wd, w, l, f, 0, in, kfa, kfb, ea, eb);
    in.wantExt = true;
    in.wantTd = wd.hasTd != 0;
    if (!(in.rho > 0) || !isfinite(in.rho) || !isfinite(in.td)) return false;
    if (!evalBearingFactor(in, true, o)) return false;
    sq = o.r[0] * o.r[0] + o.r[1] * o.r[1];
    wgt = huberWeight(wd.huber, sq);
    return true;
}
}  // namespace

// ---------------------------------------------------------------------------------------
// One warp per eliminated landmark, one lane per observation: the landmark's
// information d (for the window's cutoff) and, for windows on the dense-row
// path, the staged record of each observation:
//   [0, 25)  weighted row 0 over the observation's columns in block order
//            (anchor pose, observer pose, anchor extrinsic, observer extrinsic, td)
//   [25, 50) weighted row 1
//   50..53   weighted r0, r1, d r0 / d rho, d r1 / d rho
//   54       robust cost
//   55       the four block starts as visual columns (int16, -1 absent)
__global__ void k_marg_eval(DevBatch B, MargBatch M) {
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (e >= M.numElim) return;
    const MargElim me = M.elim[e];
    const WinDesc wd = B.win[me.win];
    const bool stage = M.win[me.win].rowsPath != 0;
    const int ob = B.lmObsBegin[me.lm], oe = B.lmObsBegin[me.lm + 1];
    double d = 0;
    for (int f = ob + lane; f < oe; f += 32) {
        FactorIn in;
        FactorOut o;
        double wgt, sq;
        int kfa, kfb, ea, eb;
        double* rec = M.rows + (long long)kMargRecord * (me.obs0 + (f - ob));
        if (!margFactor(B, wd, me.win, me.lm, f, in, o, wgt, sq, kfa, kfb, ea, eb)) {
            atomicExch(&M.status[me.win], CGMLI_E_NONFINITE);
            if (stage) {
                // no block: only a td column can map, to slot 0 of each row
                rec[0] = rec[25] = 0.0;
                for (int k = 50; k < 55; ++k) rec[k] = 0.0;
                rec[55] = __longlong_as_double(-1ll);
            }
            continue;
        }
        d += wgt * wgt * (o.Jrho[0] * o.Jrho[0] + o.Jrho[1] * o.Jrho[1]);
        if (!stage) continue;
        int n = 0;
        auto push = [&](const double* Jb, int width) {
            for (int c = 0; c < width; ++c, ++n) {
                rec[n] = wgt * Jb[c];
                rec[25 + n] = wgt * Jb[width + c];
            }
        };
        const bool same = in.sameKf && !in.splitExt;
        int st[4] = {-1, -1, -1, -1};
        if (!in.sameKf) { push(o.Ja, 6); push(o.Jb, 6); st[0] = M.visPose[kfa]; st[1] = M.visPose[kfb]; }
        if (!same) { push(o.Jea, 6); st[2] = M.visExt[ea]; }
        if (in.splitExt) { push(o.Jeb, 6); st[3] = M.visExt[eb]; }
        if (in.wantTd) push(o.Jtd, 1);
        rec[50] = wgt * o.r[0];
        rec[51] = wgt * o.r[1];
        rec[52] = wgt * o.Jrho[0];
        rec[53] = wgt * o.Jrho[1];
        rec[54] = huberCost(wd.huber, sq);
        unsigned long long pk = 0;
        for (int b = 0; b < 4; ++b) pk |= (unsigned long long)(unsigned short)(short)st[b] << (16 * b);
        rec[55] = __longlong_as_double((long long)pk);
    }
    d = mWarpSum(d);
    if (lane == 0) atomicMaxNonNegative(&M.maxD[me.win], d);
}

// Dense-row accumulation, one CTA per item (a run of chunks of one window's
// eliminated landmarks).  Per chunk the staged records (prefetched into shared
// memory with cp.async while the previous chunk's rank updates run) become
// dense rows over the window's nv visual columns: two weighted factor rows per
// observation, then per landmark its Schur row c / sqrt(d) (zero below the
// cutoff), with c = sum_k row_k dr_k/drho.  The item's visual information is
//   sum_factor-rows v v^T - sum_Schur-rows s s^T
// (the factor normal blocks minus c c^T / d) and its gradient
//   sum v r - sum s bl / sqrt(d).
// The upper triangle is cut into 32 x 32 tiles, each warp holding one tile's
// FP64 tensor-path accumulators (mma.sync m8n8k4, dense_tiles.cuh) in
// registers.  When the tiles fit the warps, spare warps
// split a tile's rows (k) between them and the blocks are held over the whole
// item; else every warp sums its tiles per chunk.  Either way each block is
// added to the window's H with atomics once per accumulation.
namespace {
__device__ __forceinline__ void flushTile(double (&acc)[4][8], int bi, int bj, int lane, int n, const int* visCol, double* H, int m) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = tileRowMma(bi, lane, r);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int j = tileCol(bj, lane, c);
            const double v = acc[r][c];
            if (i < n && j < n && i <= j && v != 0.0) {
                const int ci = visCol[i], cj = visCol[j];
                atomicAdd(&H[ci <= cj ? (long long)ci * m + cj : (long long)cj * m + ci], v);
            }
        }
    }
}
__device__ __forceinline__ void cpAsync16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// staged records of one chunk into shared memory (16-byte pieces; records are
// kMargRecord doubles, a multiple of 16 bytes, from a 256-byte aligned base)
__device__ __forceinline__ void prefetchRecords(const MargBatch& M, const int4& ch, double* dst) {
    const double* src = M.rows + (long long)kMargRecord * ch.z;
    const int pieces = (ch.w - ch.z) * (kMargRecord / 2);
    for (int i = threadIdx.x; i < pieces; i += blockDim.x) cpAsync16(dst + 2 * i, src + 2 * i);
    cpAsyncCommit();
}
}  // namespace

// rows of a chunk for a window of np (padded) visual columns
__host__ __device__ inline int rowsCapOf(int np) { return np <= 192 ? kRowsCap : 72; }

__global__ void __launch_bounds__(kRowsThreads, 1) k_marg_rows(DevBatch B, MargBatch M) {
    extern __shared__ __align__(16) double smem[];
    const int4 it = M.items[blockIdx.x];
    const int w = it.x;
    const MargWin mw = M.win[w];
    const int n = mw.nv, np = (n + 31) & ~31, nb = np >> 5, ntiles = nb * (nb + 1) / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int nw = kRowsThreads / 32;
    const bool persistent = ntiles <= nw;
    const int wpt = persistent ? nw / ntiles : 1;  // warps per tile (k split)
    double* rec[2];
    rec[0] = smem;                                  // kRowsCap / 2 records each
    rec[1] = rec[0] + (kRowsCap / 2) * kMargRecord;
    double* rv = rec[1] + (kRowsCap / 2) * kMargRecord;  // kRowsCap: residual of each row
    double* jrv = rv + kRowsCap;                    // kRowsCap: rho derivative of each factor row
    double* V = jrv + kRowsCap;                     // rows x np
    __shared__ double red[kRowsThreads / 32];
    const double cutoff = fmax(1e-12, 1e-9 * fmax(0.0, M.maxD[w]));
    const int* visCol = M.visCol + mw.vis0;
    double* H = M.H + mw.H0;
    const int gj = threadIdx.x - (kRowsThreads - np);  // the last np threads own one gradient column each
    double g = 0, cost = 0, rss = 0, reduction = 0;
    double acc[4][8];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;
    prefetchRecords(M, M.chunks[it.y], rec[0]);
    cpAsyncWaitAll();
    __syncthreads();
    for (int ci = it.y; ci < it.z; ++ci) {
        const int4 ch = M.chunks[ci];
        const double* rc = rec[(ci - it.y) & 1];
        const int nobs = ch.w - ch.z, kp = 2 * nobs, K = kp + (ch.y - ch.x);
        // ---- factor rows, one warp per observation
        for (int o = warp; o < nobs; o += nw) {
            const double* r = rc + kMargRecord * o;
            const unsigned long long pk = (unsigned long long)__double_as_longlong(r[55]);
            if (lane == 0) {
                rv[2 * o] = r[50];
                rv[2 * o + 1] = r[51];
                jrv[2 * o] = r[52];
                jrv[2 * o + 1] = r[53];
                cost += r[54];
                rss += r[50] * r[50] + r[51] * r[51];
            }
            double* v0row = V + (long long)(2 * o) * np;
            double* v1row = v0row + np;
            for (int col = lane; col < np; col += 32) {
                int slot = -1, base = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int start = (int)(short)(unsigned short)(pk >> (16 * b));
                    if (start >= 0) {
                        if (col >= start && col < start + 6) slot = base + col - start;
                        base += 6;
                    }
                }
                if (mw.visTd >= 0 && col == mw.visTd) slot = base;
                v0row[col] = slot < 0 ? 0.0 : r[slot];
                v1row[col] = slot < 0 ? 0.0 : r[25 + slot];
            }
        }
        __syncthreads();
        // ---- Schur rows, one warp per landmark
        for (int l = ch.x + warp; l < ch.y; l += nw) {
            const MargElim me = M.elim[l];
            const int nob = B.lmObsBegin[me.lm + 1] - B.lmObsBegin[me.lm];
            const int r0 = 2 * (me.obs0 - ch.z), r1 = r0 + 2 * nob;
            double d = 0, bl = 0;
            for (int k = r0; k < r1; ++k) {
                d += jrv[k] * jrv[k];
                bl += jrv[k] * rv[k];
            }
            const bool eliminate = d > cutoff;
            const double scale = eliminate ? 1.0 / sqrt(d) : 0.0;
            const int sr = kp + (l - ch.x);
            for (int col = lane; col < np; col += 32) {
                double sc = 0;
                for (int k = r0; k < r1; ++k) sc += V[(long long)k * np + col] * jrv[k];
                V[(long long)sr * np + col] = sc * scale;
            }
            if (lane == 0) {
                rv[sr] = bl * scale;
                if (eliminate) reduction += 0.5 * bl * bl / d;
            }
        }
        __syncthreads();
        // ---- next chunk's records in flight; rank updates; gradient columns
        if (ci + 1 < it.z) prefetchRecords(M, M.chunks[ci + 1], rec[(ci + 1 - it.y) & 1]);
        for (int u = warp; u < ntiles * wpt; u += nw) {
            const int t = u / wpt, part = u % wpt;
            int bi, bj;
            tileOf(t, nb, bi, bj);
            if (!persistent) zeroTile(acc);
            rankUpdateMma<false>(acc, V, bi * 32, bj * 32, part, kp, wpt, np);
            rankUpdateMma<true>(acc, V, bi * 32, bj * 32, kp + part, K, wpt, np);
            if (!persistent) flushTile(acc, bi, bj, lane, n, visCol, H, mw.m);
        }
        if (gj >= 0) {
            double s = 0;
            for (int k = 0; k < kp; ++k) s += V[(long long)k * np + gj] * rv[k];
            for (int k = kp; k < K; ++k) s -= V[(long long)k * np + gj] * rv[k];
            g += s;
        }
        cpAsyncWaitAll();
        __syncthreads();
    }
    if (persistent && warp < ntiles * wpt) {
        int bi, bj;
        tileOf(warp / wpt, nb, bi, bj);
        flushTile(acc, bi, bj, lane, n, visCol, H, mw.m);
    }
    if (gj >= 0 && gj < n && g != 0.0) atomicAdd(&M.b[mw.vec0 + visCol[gj]], g);
    cost = mBlockSum(cost, red);
    rss = mBlockSum(rss, red);
    reduction = mBlockSum(reduction, red);
    if (threadIdx.x == 0) {
        atomicAdd(&M.stats[4 * w + 0], cost);
        atomicAdd(&M.stats[4 * w + 1], rss);
        atomicAdd(&M.stats[4 * w + 2], reduction);
    }
}

// One CTA per eliminated landmark of a window above kRowsMaxN visual columns.
// Shared memory: the landmark's local
// information (packed upper, nc x nc), its cross vector c and gradient, then
// the staged weighted rows of its observations.
__global__ void __launch_bounds__(kMargLmThreads) k_marg_visual(DevBatch B, MargBatch M) {
    extern __shared__ double smem[];
    const int e = M.slowElim[blockIdx.x];
    const MargElim me = M.elim[e];
    const int w = me.win, nc = me.nc;
    const MargWin mw = M.win[w];
    const WinDesc wd = B.win[w];
    const int ob = B.lmObsBegin[me.lm], nobs = B.lmObsBegin[me.lm + 1] - ob;
    const int npk = nc * (nc + 1) / 2;
    double* hl = smem;                    // npk
    double* cl = hl + npk;                // nc
    double* gl = cl + nc;                 // nc
    double* jst = gl + nc;                // 32 x 50: weighted rows over the observation's columns
    double* rp = jst + 32 * 50;           // 32 x 4: weighted r0, r1, rho derivative 0, 1
    short* lcol = reinterpret_cast<short*>(rp + 32 * 4);  // 32 x 25 local columns
    int* nn = reinterpret_cast<int*>(lcol + 32 * 25);     // 32 column counts
    __shared__ double red[kMargLmThreads / 32];
    for (int i = threadIdx.x; i < npk + 2 * nc; i += blockDim.x) hl[i] = 0.0;
    double cost = 0, rss = 0;
    if (threadIdx.x < nobs) {
        const int t = threadIdx.x, f = ob + t;
        FactorIn in;
        FactorOut o;
        double wgt, sq;
        int n = 0, kfa, kfb, ea, eb;
        if (margFactor(B, wd, w, me.lm, f, in, o, wgt, sq, kfa, kfb, ea, eb)) {
            cost = huberCost(wd.huber, sq);
            rss = wgt * wgt * sq;
            const int* map = M.obsMap + 5ll * (me.obs0 + t);
            double* J = jst + 50 * t;
            short* lc = lcol + 25 * t;
            auto push = [&](int base, const double* Jb, int width) {
                for (int c = 0; c < width; ++c) {
                    lc[n] = (short)(base + c);
                    J[n] = wgt * Jb[c];
                    J[25 + n] = wgt * Jb[width + c];
                    ++n;
                }
            };
            const bool same = in.sameKf && !in.splitExt;
            if (!in.sameKf) { push(map[0], o.Ja, 6); push(map[1], o.Jb, 6); }
            if (!same) push(map[2], o.Jea, 6);
            if (in.splitExt) push(map[3], o.Jeb, 6);
            if (map[4] >= 0) push(map[4], o.Jtd, 1);
            rp[4 * t + 0] = wgt * o.r[0];
            rp[4 * t + 1] = wgt * o.r[1];
            rp[4 * t + 2] = wgt * o.Jrho[0];
            rp[4 * t + 3] = wgt * o.Jrho[1];
        } else {
            atomicExch(&M.status[w], CGMLI_E_NONFINITE);
            for (int k = 0; k < 4; ++k) rp[4 * t + k] = 0.0;
        }
        nn[t] = n;
    }
    cost = mBlockSum(cost, red);
    rss = mBlockSum(rss, red);
    // factor normal blocks: the columns of one observation are distinct, so
    // the threads of one observation write distinct entries
    for (int t = 0; t < nobs; ++t) {
        const int n = nn[t], pairs = n * (n + 1) / 2;
        const double* J = jst + 50 * t;
        const short* lc = lcol + 25 * t;
        for (int q = threadIdx.x; q < pairs; q += blockDim.x) {
            int i = 0, rem = q;
            while (rem >= n - i) { rem -= n - i; ++i; }
            const int j = i + rem;
            const int a = lc[i], c = lc[j];
            hl[a <= c ? packedUp(a, c, nc) : packedUp(c, a, nc)] += J[i] * J[j] + J[25 + i] * J[25 + j];
        }
        if (threadIdx.x < n) {
            const int i = threadIdx.x, a = lc[i];
            cl[a] += J[i] * rp[4 * t + 2] + J[25 + i] * rp[4 * t + 3];
            gl[a] += J[i] * rp[4 * t + 0] + J[25 + i] * rp[4 * t + 1];
        }
        __syncthreads();
    }
    double d = 0, bl = 0;
    for (int t = 0; t < nobs; ++t) {
        d += rp[4 * t + 2] * rp[4 * t + 2] + rp[4 * t + 3] * rp[4 * t + 3];
        bl += rp[4 * t + 2] * rp[4 * t + 0] + rp[4 * t + 3] * rp[4 * t + 1];
    }
    // scalar elimination with the diagonal PSD rule
    const double cutoff = fmax(1e-12, 1e-9 * fmax(0.0, M.maxD[w]));
    const bool eliminate = d > cutoff;
    const double inv = eliminate ? 1.0 / d : 0.0;
    const int* cols = M.cols + me.col0;
    double* H = M.H + mw.H0;
    double* bw = M.b + mw.vec0;
    for (int q = threadIdx.x; q < npk; q += blockDim.x) {
        int i = 0, rem = q;
        while (rem >= nc - i) { rem -= nc - i; ++i; }
        const int j = i + rem;
        const double v = hl[q] - inv * cl[i] * cl[j];
        if (v == 0.0) continue;
        const int ci = cols[i], cj = cols[j];
        atomicAdd(&H[ci <= cj ? (long long)ci * mw.m + cj : (long long)cj * mw.m + ci], v);
    }
    for (int i = threadIdx.x; i < nc; i += blockDim.x) {
        const double v = gl[i] - inv * cl[i] * bl;
        if (v != 0.0) atomicAdd(&bw[cols[i]], v);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&M.stats[4 * w + 0], cost);
        atomicAdd(&M.stats[4 * w + 1], rss);
        if (eliminate) atomicAdd(&M.stats[4 * w + 2], 0.5 * bl * bl * inv);
    }
}

// IMU factors touching the victim and the previous prior, one CTA per window.
__global__ void __launch_bounds__(256) k_marg_retained(DevBatch B, MargBatch M) {
    const int w = M.bigFirst[blockIdx.x];
    const MargWin mw = M.win[w];
    if (mw.m == 0) return;
    const WinDesc wd = B.win[w];
    const int m = mw.m;
    double* H = M.H + mw.H0;
    double* g = M.b + mw.vec0;
    __shared__ double sc[2 * 465];
    __shared__ double red[8];
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    const cgmli_frozen_imu* imus = reinterpret_cast<const cgmli_frozen_imu*>(B.imu);
    double cost = 0;
    // the consumed IMU factors: the victim's (at most two), or every factor of the
    // window (imuAll); evaluated two at a time into the scratch
    const int nImu = mw.imuAll ? wd.nImu : 2;
    auto factorAt = [&](int q) { return mw.imuAll ? (q < nImu ? wd.imu0 + q : -1) : mw.imu[q]; };
    for (int q0 = 0; q0 < nImu; q0 += 2) {
        // the raw error and Jacobian of each factor by one thread (its Jacobian cleared
        // first by the CTA), then the whitening W [e | U] in place, a thread per column
        // (evalImu's products in its order); a non-finite U shows in those products
        for (int t = threadIdx.x; t < 2 * 450; t += blockDim.x) sc[465 * (t / 450) + 15 + t % 450] = 0.0;
        __syncthreads();
        if (threadIdx.x < 2 && factorAt(q0 + threadIdx.x) >= 0) {
            const int gi = factorAt(q0 + threadIdx.x), k = B.imuKf[gi];
            double* raw = sc + 465 * threadIdx.x;
            if (!evalImuRaw(imus[gi], B.pose[0] + 7ll * k, B.sb[0] + 9ll * k, B.pose[0] + 7ll * (k + 1), B.sb[0] + 9ll * (k + 1), raw,
                            raw + 15, true))
                bad = 1;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < 2 * 31; t += blockDim.x) {
            const int q = t / 31, c = t % 31;
            if (factorAt(q0 + q) < 0) continue;
            const double* W = imus[factorAt(q0 + q)].whitening;  // column-major 15 x 15
            double* f = sc + 465 * q;
            double u[15];
            for (int mm = 0; mm < 15; ++mm) u[mm] = c < 30 ? f[15 + 30 * mm + c] : f[mm];
            for (int i = 0; i < 15; ++i) {
                double v = 0;
                for (int mm = 0; mm < 15; ++mm) v += W[i + 15 * mm] * u[mm];
                if (!isfinite(v)) bad = 1;
                if (c < 30) {
                    f[15 + 30 * i + c] = v;
                } else {
                    f[i] = v;
                    cost += 0.5 * v * v;
                }
            }
        }
        __syncthreads();
        for (int q = 0; q < 2; ++q) {
            if (factorAt(q0 + q) < 0 || bad) continue;
            const int k = B.imuKf[factorAt(q0 + q)];
            const double* r = sc + 465 * q;
            const double* J = r + 15;
            auto colOf = [&](int a) {
                return a < 6 ? M.poseCol[k] + a : a < 15 ? M.sbCol[k] + a - 6 : a < 21 ? M.poseCol[k + 1] + a - 15 : M.sbCol[k + 1] + a - 21;
            };
            for (int e = threadIdx.x; e < 930; e += blockDim.x) {
                if (e < 900) {
                    const int a = e / 30, c = e % 30, ca = colOf(a), cc = colOf(c);
                    if (ca > cc) continue;  // upper triangle: each unordered pair once
                    double v = 0;
                    for (int i = 0; i < 15; ++i) v += J[30 * i + a] * J[30 * i + c];
                    H[(long long)ca * m + cc] += v;
                } else {
                    const int a = e - 900;
                    double v = 0;
                    for (int i = 0; i < 15; ++i) v += J[30 * i + a] * r[i];
                    g[colOf(a)] += v;
                }
            }
            __syncthreads();
        }
        __syncthreads();  // the scratch is rewritten by the next pair
    }
    if (mw.hasPrior && wd.priorRank > 0 && !bad) {
        const int rank = wd.priorRank, cols = wd.priorCols;  // cols <= kPriorMaxCols (host check)
        double* ps = B.priorScratch + wd.priorScratch0;
        double* delta = ps;
        double* D = delta + cols;
        double* r = D + 6ll * cols;
        double* J = r + rank;
        // per prior column: its marginalization column and its block's first column,
        // negated minus one for a block whose tangent is its ambient (speed/bias, td)
        __shared__ int mcol[kPriorMaxCols], poff[kPriorMaxCols];
        for (int bk = threadIdx.x; bk < wd.priorBlocks; bk += blockDim.x) {
            const int pb = wd.priorBlk0 + bk;
            const int kind = B.priorKind[pb], off = B.priorOff[pb], gi = B.priorIndex[pb];
            const int width = kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 6;
            const int base = kind == CGMLI_PRIOR_POSE ? M.poseCol[gi] : kind == CGMLI_PRIOR_SPEED_BIAS ? M.sbCol[gi]
                             : kind == CGMLI_PRIOR_EXTRINSIC ? M.extCol[gi] : mw.tdCol;
            const bool chart = kind == CGMLI_PRIOR_POSE || kind == CGMLI_PRIOR_EXTRINSIC;
            for (int c = 0; c < width; ++c) {
                mcol[off + c] = base + c;
                poff[off + c] = chart ? off : -1 - off;
            }
            int aoff = 0;
            for (int q = wd.priorBlk0; q < pb; ++q) {
                const int kq = B.priorKind[q];
                aoff += kq == CGMLI_PRIOR_SPEED_BIAS ? 9 : kq == CGMLI_PRIOR_TIME_OFFSET ? 1 : 7;
            }
            const double* ref = B.priorRef + wd.priorRef0 + aoff;
            const double* x = blockValue(B, 0, kind, B.priorIndex[pb], w);
            if (kind == CGMLI_PRIOR_POSE || kind == CGMLI_PRIOR_EXTRINSIC) {
                poseMinus(x, ref, delta + off);
                se3LeftJacobianInverse(delta + off, D + 6ll * off);
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
            if (!isfinite(v)) bad = 1;
            cost += 0.5 * v * v;
        }
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
        for (long long e = threadIdx.x; e < (long long)cols * (cols + 1); e += blockDim.x) {
            const int p = (int)(e / cols), q = (int)(e % cols);
            const int cq = mcol[q];
            if (p < cols) {
                const int cp = mcol[p];
                if (cp > cq) continue;
                double v = 0;
                for (int i = 0; i < rank; ++i) v += J[(long long)i * cols + p] * J[(long long)i * cols + q];
                H[(long long)cp * m + cq] += v;
            } else {
                double v = 0;
                for (int i = 0; i < rank; ++i) v += J[(long long)i * cols + q] * r[i];
                g[cq] += v;
            }
        }
    }
    cost = mBlockSum(cost, red);
    if (threadIdx.x == 0) {
        M.stats[4 * w + 0] += cost;
        M.stats[4 * w + 1] += 2 * cost;
        if (bad) M.status[w] = CGMLI_E_NONFINITE;
    }
}

// ---------------------------------------------------------------------------------------
// Cyclic Jacobi eigensolver of a symmetric n x n row-major matrix A (n <= 1024),
// one CTA.  Each round applies n/2 rotations on disjoint index pairs (the
// round-robin ordering), which commute, so a round is one row pass and one
// column pass.  A pair is rotated only while |a_pq| > 1e-15 sqrt|a_pp a_qq|
// and |a_pq| > 1e-16 |A|_F: entries at the rounding level of a rotation are
// left alone (rotating them only makes new noise), so the off-diagonal mass
// left at the end is below n 1e-16 |A|_F; a sweep without rotation ends the
// iteration.  On return the diagonal of A
// holds the eigenvalues and the columns of V the eigenvectors.
__device__ void jacobiEigen(double* A, double* V, int n, int maxSweeps) {
    __shared__ short pairP[512], pairQ[512];
    __shared__ double rc[512], rs[512];
    __shared__ int rotated;
    __shared__ double normRed[32];
    const int np = (n + 1) & ~1;  // even count; index n (if odd) is a dummy
    const int half = np / 2;
    double fro = 0;
    for (long long i = threadIdx.x; i < (long long)n * n; i += blockDim.x) {
        V[i] = (i / n == i % n) ? 1.0 : 0.0;
        fro += A[i] * A[i];
    }
    const double floorAbs = 1e-16 * sqrt(mBlockSum(fro, normRed));
    for (int sweep = 0; sweep < maxSweeps; ++sweep) {
        if (threadIdx.x == 0) rotated = 0;
        __syncthreads();
        for (int round = 0; round < np - 1; ++round) {
            for (int i = threadIdx.x; i < half; i += blockDim.x) {
                const int a = i == 0 ? 0 : 1 + (i - 1 + round) % (np - 1);
                const int b = 1 + (np - 2 - i + round) % (np - 1);
                const int p = a < b ? a : b, q = a < b ? b : a;
                pairP[i] = (short)p;
                pairQ[i] = (short)q;
                double c = 1, s = 0;
                if (q < n) {
                    const double apq = A[(long long)p * n + q], app = A[(long long)p * n + p], aqq = A[(long long)q * n + q];
                    if (fabs(apq) > 1e-15 * sqrt(fabs(app * aqq)) && fabs(apq) > floorAbs) {
                        const double tau = (aqq - app) / (2 * apq);
                        const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1 + tau * tau));
                        c = 1 / sqrt(1 + t * t);
                        s = t * c;
                        rotated = 1;
                    }
                }
                rc[i] = c;
                rs[i] = s;
            }
            __syncthreads();
            // rows p, q of A
            for (int t = threadIdx.x; t < half * n; t += blockDim.x) {
                const int i = t / n, k = t % n;
                if (rs[i] == 0.0) continue;
                const long long p = pairP[i], q = pairQ[i];
                const double c = rc[i], s = rs[i];
                const double apk = A[p * n + k], aqk = A[q * n + k];
                A[p * n + k] = c * apk - s * aqk;
                A[q * n + k] = s * apk + c * aqk;
            }
            __syncthreads();
            // columns p, q of A and V
            for (int t = threadIdx.x; t < half * n; t += blockDim.x) {
                const int k = t / half, i = t % half;
                if (rs[i] == 0.0) continue;
                const int p = pairP[i], q = pairQ[i];
                const double c = rc[i], s = rs[i];
                const long long row = (long long)k * n;
                const double akp = A[row + p], akq = A[row + q];
                A[row + p] = c * akp - s * akq;
                A[row + q] = s * akp + c * akq;
                const double vkp = V[row + p], vkq = V[row + q];
                V[row + p] = c * vkp - s * vkq;
                V[row + q] = s * vkp + c * vkq;
            }
            __syncthreads();
        }
        if (!rotated) break;
        __syncthreads();
    }
}

// The same Jacobi iteration on a symmetric matrix kept as its packed upper
// triangle (row-major, r <= c), typically in shared memory.  Rotations of
// disjoint pairs commute, so one round updates every 2x2 block between pairs
// i <= j once: B' = R_i^T B R_j with R = [[c, s], [-s, c]].  Eigenvectors are
// accumulated as the ROWS of Vt (Vt' = R^T Vt), so their updates are
// contiguous.  On return Ap's diagonal holds the eigenvalues.
__device__ __forceinline__ int pkUp(int r, int c, int n) { return r * n - r * (r - 1) / 2 + (c - r); }
__device__ __forceinline__ int pkSym(int r, int c, int n) { return r <= c ? pkUp(r, c, n) : pkUp(c, r, n); }
// With vCols >= 0 the rotations are applied to the rows (vCols long) of the
// caller's Vt as given, instead of accumulating eigenvectors from the identity:
// Vt ends as U^T Vt.
__device__ void jacobiPacked(double* Ap, double* Vt, int n, int maxSweeps, int vCols = -1) {
    __shared__ short pairP[512], pairQ[512];
    __shared__ double rc[512], rs[512];
    __shared__ int rotated;
    __shared__ double normRed[32];
    const int np = (n + 1) & ~1;
    const int half = np / 2;
    const int blocks = half * (half + 1) / 2;
    if (vCols < 0) {
        vCols = n;
        for (long long i = threadIdx.x; i < (long long)n * n; i += blockDim.x) Vt[i] = (i / n == i % n) ? 1.0 : 0.0;
    }
    double fro = 0;
    for (int r = threadIdx.x; r < n; r += blockDim.x)
        for (int c = r; c < n; ++c) fro += (r == c ? 1.0 : 2.0) * Ap[pkUp(r, c, n)] * Ap[pkUp(r, c, n)];
    const double floorAbs = 1e-16 * sqrt(mBlockSum(fro, normRed));
    // This thread's blocks (i, j) of the pair grid are the same in every round:
    // decode them once (packed i | j << 16).
    constexpr int kMaxBlk = 16;
    const bool cached = blocks <= kMaxBlk * (int)blockDim.x;
    int myBlk[kMaxBlk];
#pragma unroll
    for (int m = 0; m < kMaxBlk; ++m) {
        const int bidx = threadIdx.x + m * blockDim.x;
        myBlk[m] = -1;
        if (cached && bidx < blocks) {
            int i = (int)((2.0f * half + 1 - sqrtf((2.0f * half + 1) * (2.0f * half + 1) - 8.0f * bidx)) * 0.5f);
            if (i < 0) i = 0;
            while (i > 0 && i * half - i * (i - 1) / 2 > bidx) --i;
            while ((i + 1) * half - (i + 1) * i / 2 <= bidx) ++i;
            myBlk[m] = i | (i + (bidx - (i * half - i * (i - 1) / 2))) << 16;
        }
    }
    // eigenvector update: a fixed column k per thread and every step-th pair
    const int vStep = vCols > 0 && vCols <= (int)blockDim.x ? (int)blockDim.x / vCols : 0;
    const int vk = vStep ? (int)threadIdx.x % vCols : 0, vi0 = vStep ? (int)threadIdx.x / vCols : 0;
    const bool vActive = vStep && (int)threadIdx.x < vStep * vCols;
    const bool vGlobal = vCols > 0 && __isGlobal(Vt);
    for (int sweep = 0; sweep < maxSweeps; ++sweep) {
        if (threadIdx.x == 0) rotated = 0;
        __syncthreads();
        for (int round = 0; round < np - 1; ++round) {
            for (int i = threadIdx.x; i < half; i += blockDim.x) {
                const int a = i == 0 ? 0 : 1 + (i - 1 + round) % (np - 1);
                const int b = 1 + (np - 2 - i + round) % (np - 1);
                const int p = a < b ? a : b, q = a < b ? b : a;
                pairP[i] = (short)p;
                pairQ[i] = (short)q;
                double c = 1, s = 0;
                if (q < n) {
                    const double apq = Ap[pkUp(p, q, n)], app = Ap[pkUp(p, p, n)], aqq = Ap[pkUp(q, q, n)];
                    if (apq * apq > 1e-30 * fabs(app * aqq) && fabs(apq) > floorAbs) {
                        // tan of the rotation angle, t = sgn(d) e / (|d| + sqrt(d^2 + e^2)) with
                        // d = a_qq - a_pp, e = 2 a_pq: the smaller root of t^2 + 2 (d / e) t - 1 = 0
                        const double d = aqq - app, e = 2 * apq;
                        const double t = (d >= 0 ? e : -e) / (fabs(d) + sqrt(d * d + e * e));
                        c = rsqrt(1 + t * t);
                        s = t * c;
                        rotated = 1;
                    }
                }
                rc[i] = c;
                rs[i] = s;
            }
            __syncthreads();
            auto rotateBlock = [&](int i, int j) {
                const double si = rs[i], sj = rs[j];
                if (si == 0.0 && sj == 0.0) return;
                const double ci = rc[i], cj = rc[j];
                const int pi = pairP[i], qi = pairQ[i], pj = pairP[j], qj = pairQ[j];
                if (i == j) {
                    const int kpp = pkUp(pi, pi, n), kpq = pkUp(pi, qi, n), kqq = pkUp(qi, qi, n);
                    const double app = Ap[kpp], apq = Ap[kpq], aqq = Ap[kqq];
                    const double t00 = ci * app - si * apq, t01 = si * app + ci * apq;
                    const double t10 = ci * apq - si * aqq, t11 = si * apq + ci * aqq;
                    Ap[kpp] = ci * t00 - si * t10;
                    Ap[kpq] = ci * t01 - si * t11;
                    Ap[kqq] = si * t01 + ci * t11;
                } else {
                    const bool rowQ = qi < n, colQ = qj < n;
                    const int k00 = pkSym(pi, pj, n);
                    const int k01 = colQ ? pkSym(pi, qj, n) : 0;
                    const int k10 = rowQ ? pkSym(qi, pj, n) : 0;
                    const int k11 = rowQ && colQ ? pkSym(qi, qj, n) : 0;
                    const double b00 = Ap[k00], b01 = colQ ? Ap[k01] : 0.0, b10 = rowQ ? Ap[k10] : 0.0,
                                 b11 = rowQ && colQ ? Ap[k11] : 0.0;
                    const double t00 = cj * b00 - sj * b01, t01 = sj * b00 + cj * b01;
                    const double t10 = cj * b10 - sj * b11, t11 = sj * b10 + cj * b11;
                    Ap[k00] = ci * t00 - si * t10;
                    if (colQ) Ap[k01] = ci * t01 - si * t11;
                    if (rowQ) Ap[k10] = si * t00 + ci * t10;
                    if (rowQ && colQ) Ap[k11] = si * t01 + ci * t11;
                }
            };
            if (cached) {
#pragma unroll
                for (int m = 0; m < kMaxBlk; ++m)
                    if (myBlk[m] >= 0) rotateBlock(myBlk[m] & 0xffff, myBlk[m] >> 16);
            } else {
                for (int bidx = threadIdx.x; bidx < blocks; bidx += blockDim.x) {
                    // (i, j), i <= j, from the packed-upper enumeration of a half x half triangle
                    int i = (int)((2.0f * half + 1 - sqrtf((2.0f * half + 1) * (2.0f * half + 1) - 8.0f * bidx)) * 0.5f);
                    if (i < 0) i = 0;
                    while (i > 0 && i * half - i * (i - 1) / 2 > bidx) --i;
                    while ((i + 1) * half - (i + 1) * i / 2 <= bidx) ++i;
                    rotateBlock(i, i + (bidx - (i * half - i * (i - 1) / 2)));
                }
            }
            auto rotateVt = [&](int i, int k) {
                const double s = rs[i];
                if (s == 0.0) return;
                const double c = rc[i];
                const long long p = pairP[i], q = pairQ[i];
                if (q >= n) return;  // the dummy index of an odd n has no row
                const double vp = Vt[p * vCols + k], vq = Vt[q * vCols + k];
                Vt[p * vCols + k] = c * vp - s * vq;
                Vt[q * vCols + k] = s * vp + c * vq;
            };
            if (vStep && !vGlobal) {
                if (vActive)
                    for (int i = vi0; i < half; i += vStep) rotateVt(i, vk);
            } else if (vStep) {
                // a thread's pairs rotate disjoint rows: issue eight pairs' loads
                // before their stores, so that global Vt keeps eight accesses in
                // flight per thread instead of one dependent round trip per pair
                constexpr int kVtBatch = 8;
                if (vActive)
                    for (int i0 = vi0; i0 < half; i0 += kVtBatch * vStep) {
                        double vp[kVtBatch], vq[kVtBatch];
                        bool live[kVtBatch];
#pragma unroll
                        for (int u = 0; u < kVtBatch; ++u) {
                            const int i = i0 + u * vStep;
                            live[u] = i < half && rs[i] != 0.0 && pairQ[i] < n;
                            if (live[u]) {
                                vp[u] = Vt[(long long)pairP[i] * vCols + vk];
                                vq[u] = Vt[(long long)pairQ[i] * vCols + vk];
                            }
                        }
#pragma unroll
                        for (int u = 0; u < kVtBatch; ++u) {
                            if (!live[u]) continue;
                            const int i = i0 + u * vStep;
                            const double c = rc[i], s = rs[i];
                            Vt[(long long)pairP[i] * vCols + vk] = c * vp[u] - s * vq[u];
                            Vt[(long long)pairQ[i] * vCols + vk] = s * vp[u] + c * vq[u];
                        }
                    }
            } else if (vCols > 0) {
                for (int t = threadIdx.x; t < half * vCols; t += blockDim.x) rotateVt(t / vCols, t % vCols);
            }
            __syncthreads();
        }
        if (!rotated) break;
        __syncthreads();
    }
}

// Ascending position of each eigenvalue (ties by index); pos has n entries.
__device__ void ascendingPositions(const double* ev, int n, int* pos) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = ev[i];
        int p = 0;
        for (int j = 0; j < n; ++j) p += ev[j] < v || (ev[j] == v && j < i);
        pos[i] = p;
    }
    __syncthreads();
}

// Victim elimination: X = pinv(Hmm) [Hmr | bm] with the eigen cutoff, then the
// symmetrized separator information Hrr - Hmr^T X and gradient br - Hmr^T y.
__global__ void __launch_bounds__(kMargThreads) k_marg_victim(MargBatch M) {
    const int w = M.bigFirst[blockIdx.x];
    const MargWin mw = M.win[w];
    const int m = mw.m, nm = mw.nm, nr = mw.nr, cols = nr + 1;
    if (m == 0 || nr == 0 || M.status[w] != CGMLI_OK) return;
    const double* H = M.H + mw.H0;
    const double* bw = M.b + mw.vec0;
    double* E = M.sepH + mw.sep0;
    double* bs = M.sepB + mw.vec0;
    __shared__ double Hm[15 * 15], Um[15 * 15], ev[15];
    __shared__ double red[kMargThreads / 32];
    double reduction = 0;
    if (nm > 0) {
        for (int i = threadIdx.x; i < nm * nm; i += blockDim.x) Hm[i] = symAt(H, i / nm, i % nm, m);
        __syncthreads();
        jacobiEigen(Hm, Um, nm, 60);
        double vmax = -INFINITY, vmin = INFINITY;
        for (int i = 0; i < nm; ++i) { vmax = fmax(vmax, Hm[i * nm + i]); vmin = fmin(vmin, Hm[i * nm + i]); }
        const double cutoff = fmax(1e-12, 1e-9 * fmax(0.0, vmax));
        if (vmin < -10 * cutoff || !isfinite(vmin) || !isfinite(vmax)) {
            if (threadIdx.x == 0) M.status[w] = CGMLI_E_INDEFINITE;
            return;
        }
        if (threadIdx.x < nm) ev[threadIdx.x] = Hm[threadIdx.x * nm + threadIdx.x];
        __syncthreads();
        double* P = M.X + mw.x0;              // nm x cols: U^T rhs / lambda
        double* X = P + (long long)nm * cols; // nm x cols
        for (int t = threadIdx.x; t < nm * cols; t += blockDim.x) {
            const int i = t / cols, c = t % cols;
            double v = 0;
            for (int k = 0; k < nm; ++k) v += Um[k * nm + i] * (c < nr ? H[(long long)k * m + nm + c] : bw[k]);
            P[t] = ev[i] > cutoff ? v / ev[i] : 0.0;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nm * cols; t += blockDim.x) {
            const int i = t / cols, c = t % cols;
            double v = 0;
            for (int k = 0; k < nm; ++k) v += Um[i * nm + k] * P[(long long)k * cols + c];
            X[t] = v;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nm; i += blockDim.x) reduction += 0.5 * bw[i] * X[(long long)i * cols + nr];
        for (long long t = threadIdx.x; t < (long long)nr * nr; t += blockDim.x) {
            const int i = (int)(t / nr), j = (int)(t % nr);
            double v1 = symAt(H, nm + i, nm + j, m), v2 = v1;
            for (int k = 0; k < nm; ++k) {
                v1 -= H[(long long)k * m + nm + i] * X[(long long)k * cols + j];
                v2 -= H[(long long)k * m + nm + j] * X[(long long)k * cols + i];
            }
            E[t] = 0.5 * (v1 + v2);
        }
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            double v = bw[nm + i];
            for (int k = 0; k < nm; ++k) v -= H[(long long)k * m + nm + i] * X[(long long)k * cols + nr];
            bs[i] = v;
        }
    } else {
        for (long long t = threadIdx.x; t < (long long)nr * nr; t += blockDim.x)
            E[t] = symAt(H, (int)(t / nr), (int)(t % nr), m);
        for (int i = threadIdx.x; i < nr; i += blockDim.x) bs[i] = bw[i];
    }
    reduction = mBlockSum(reduction, red);
    if (threadIdx.x == 0) M.stats[4 * w + 2] += reduction;
}

// ---------------------------------------------------------------------------------------
// Fast path, one CTA per window with the separator information E in shared
// memory (n <= kFastMaxN) or, for wider separators, in the window's eigenvector
// scratch in global memory (the eigen path re-initializes it when this path
// declines), for spectra with a clean gap at the cutoff
// max(1e-12, 1e-9 lambda_max): nf eigenvalues within |lambda| < 1e-6 cutoff,
// the other k = n - nf above twice the cutoff.  The eigen path then keeps
// exactly the k large eigenpairs, and its prior (A = sqrt(lambda) u^T,
// r0 = u^T b / sqrt(lambda)) is characterised by A^T A = E_k (E without its
// negligible part) and A^T r0 = P b, P the orthogonal projector onto
// range(E_k).  Here instead:
//   - a Householder tridiagonalization T of E gives the spectral facts by
//     Sturm counts (eigenvalues of T below x = negative pivots of T - x I):
//     lambda_max and the smallest kept eigenvalue by multisection, the gap by
//     three counts;
//   - a diagonally pivoted Cholesky stopped after k pivots gives E ~ L L^T
//     and A = L^T (k x n, in pivot order);
//   - b is projected off null(A) explicitly: with N a basis of null(A) (one
//     back substitution per free column), P b = b - N (N^T N)^{-1} N^T b,
//     and r0 solves A^T r0 = P b by forward substitution over the pivots.
// Accepted when every pivot exceeds cutoff / 10 and the uneliminated
// remainder R satisfies |R|_F <= 1e-10 lambda_kept_min: by the sin-theta
// bound null(A) is then within 1e-10 of the negligible eigenspace, so A^T A
// and A^T r0 agree with the eigen path's far below its own rounding.  Other
// windows are left to the eigen path (k_marg_tridiag), which takes over this
// path's tridiagonal form: the reflectors in the window's prior slot, d, e and
// tau in its victim scratch (fast[w] = 2).
constexpr int kFastMaxN = 160;        // E in shared memory up to this width
constexpr int kFastPackedMaxN = 220;  // above it, the tridiagonalization still runs in shared memory on the packed lower triangle
constexpr int kFastMaxFree = 32;      // null directions handled by the projection
__host__ __device__ constexpr size_t fastVecBytes(int n) { return sizeof(double) * 5 * (size_t)n + sizeof(int) * 3 * (size_t)n; }
__host__ __device__ constexpr size_t fastSmemBytes(int n) {
    return n <= kFastMaxN ? sizeof(double) * (size_t)n * n + fastVecBytes(n) : fastVecBytes(n);
}
// the vectors (rounded to whole doubles), then the packed lower triangle of E
__host__ __device__ constexpr size_t fastPackedOffset(int n) { return (fastVecBytes(n) + sizeof(double) - 1) / sizeof(double); }
__host__ __device__ constexpr size_t fastPackedBytes(int n) {
    return sizeof(double) * (fastPackedOffset(n) + (size_t)n * (n + 1) / 2);
}
__device__ __forceinline__ int packedRow(int r) { return r * (r + 1) / 2; }  // row r of a packed lower triangle

// Number of eigenvalues of the symmetric tridiagonal (d, e) below x, e[i]
// coupling i and i + 1.
__device__ int sturmCount(const double* d, const double* e, int n, double x, double pivmin) {
    int c = 0;
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0) ++c;
    for (int i = 1; i < n; ++i) {
        q = d[i] - x - e[i - 1] * e[i - 1] / q;
        if (fabs(q) < pivmin) q = -pivmin;
        if (q < 0) ++c;
    }
    return c;
}

// Householder tridiagonalization of the symmetric E held as its packed lower triangle
// Pk (row r at packedRow(r)) by the CTA: the same reflectors and the same tau as the
// full-square loop of k_marg_fast (d, e, tau and the reflectors saved alike), with
// the trailing update on the lower triangle only.  Row r of the trailing block reads
// its entries left of the diagonal along its packed row and those right of it down
// the packed column.  d[n - 2], e[n - 2] and d[n - 1] are set at the end (thread 0).
__device__ void fastTridiagonalPacked(double* Pk, int n, double* v, double* p, double* wv, double* d, double* e, double* reflectors,
                                      double* saved, double* sc) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        if (warp == 0) {
            double sigma = 0;
            for (int i = lane; i < m; i += 32) {
                const double x = Pk[packedRow(k + 1 + i) + k];
                v[i] = x;
                sigma += x * x;
            }
            sigma = mWarpSum(sigma);
            __syncwarp();
            if (lane == 0) {
                d[k] = Pk[packedRow(k) + k];
                if (sigma == 0.0) {
                    e[k] = 0.0;
                    sc[0] = 0.0;
                } else {
                    const double x0 = v[0];
                    const double alpha = x0 >= 0 ? -sqrt(sigma) : sqrt(sigma);
                    e[k] = alpha;
                    v[0] = x0 - alpha;
                    sc[0] = 1.0 / (sigma - x0 * alpha);
                }
                saved[2 * n + k] = sc[0];
            }
        }
        __syncthreads();
        const double tau = sc[0];
        if (tau == 0.0) {
            __syncthreads();  // every warp has read sc before warp 0 writes the next column's
            continue;
        }
        for (int i = warp; i < m; i += nw) {  // p = tau S v over the trailing block
            const int r = k + 1 + i;
            const double* row = Pk + packedRow(r);
            double sum = 0;
            for (int j = lane; j < m; j += 32) {
                const int c = k + 1 + j;
                sum += (c <= r ? row[c] : Pk[packedRow(c) + r]) * v[j];
            }
            sum = mWarpSum(sum);
            if (lane == 0) p[i] = tau * sum;
        }
        __syncthreads();
        if (warp == 0) {
            double pv = 0;
            for (int i = lane; i < m; i += 32) pv += p[i] * v[i];
            const double K = 0.5 * tau * mWarpSum(pv);
            for (int i = lane; i < m; i += 32) wv[i] = p[i] - K * v[i];
        }
        __syncthreads();
        for (int i = warp; i < m; i += nw) {  // lower triangle of the trailing block
            double* row = Pk + packedRow(k + 1 + i) + (k + 1);
            const double vi = v[i], wi = wv[i];
            for (int j = lane; j <= i; j += 32) row[j] -= vi * wv[j] + wi * v[j];
        }
        for (int i = tid; i < m; i += blockDim.x) reflectors[k * n + (k + 1 + i)] = v[i];  // row k, right of the diagonal
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            d[n - 2] = Pk[packedRow(n - 2) + (n - 2)];
            e[n - 2] = Pk[packedRow(n - 1) + (n - 2)];
        }
        d[n - 1] = Pk[packedRow(n - 1) + (n - 1)];
    }
}

__global__ void __launch_bounds__(kMargThreads) k_marg_fast(MargBatch M) {
    const int w = M.bigFirst[blockIdx.x];
    const MargWin mw = M.win[w];
    const int n = mw.nr;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    if (tid == 0) M.fast[w] = 0;
    if (mw.m == 0 || n == 0 || n > kMargMaxSep || M.status[w] != CGMLI_OK) return;
    extern __shared__ double fsm[];
    const bool inShared = n <= kFastMaxN;
    double* S = inShared ? fsm : M.sepV + mw.sep0;  // n x n row-major
    double* v = inShared ? fsm + n * n : fsm;
    double* p = v + n;
    double* wv = p + n;
    double* d = wv + n;
    double* e = d + n;
    int* piv = reinterpret_cast<int*>(e + n);  // pivot of each Cholesky step
    int* stepOf = piv + n;                     // step at which an index was pivoted (n: never)
    int* rem = stepOf + n;                     // indices not yet pivoted
    __shared__ double sc[8];
    __shared__ int isc[2];
    // the tridiagonal form for the eigen path, should this path decline the window:
    // each reflector in its row of the prior's slot (row-major, right of the
    // diagonal), d, e and tau in the victim solve's scratch
    double* reflectors = M.A + mw.sep0;
    double* saved = M.X + mw.x0;
    __shared__ double G[kFastMaxFree * kFastMaxFree], h[kFastMaxFree];
    const double* E = M.sepH + mw.sep0;
    // windows above kFastMaxN: the tridiagonalization on the packed lower triangle in
    // shared memory when it fits the launch (the rest of this path stays in global memory)
    const bool packed = !inShared && n <= kFastPackedMaxN && (long long)fastPackedBytes(n) <= M.fastSmem;
    if (packed) {
        double* Pk = fsm + fastPackedOffset(n);
        for (int r = warp; r < n; r += nw)
            for (int c = lane; c <= r; c += 32) Pk[packedRow(r) + c] = E[(size_t)r * n + c];
        __syncthreads();
        fastTridiagonalPacked(Pk, n, v, p, wv, d, e, reflectors, saved, sc);
    } else {
    for (int t = tid; t < n * n; t += blockDim.x) S[t] = E[t];
    __syncthreads();
    // Householder tridiagonalization (eigenvalues only)
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        if (warp == 0) {
            double sigma = 0;
            for (int i = lane; i < m; i += 32) {
                const double x = S[(k + 1 + i) * n + k];
                v[i] = x;
                sigma += x * x;
            }
            sigma = mWarpSum(sigma);
            __syncwarp();
            if (lane == 0) {
                d[k] = S[k * n + k];
                if (sigma == 0.0) {
                    e[k] = 0.0;
                    sc[0] = 0.0;
                } else {
                    const double x0 = v[0];
                    const double alpha = x0 >= 0 ? -sqrt(sigma) : sqrt(sigma);
                    e[k] = alpha;
                    v[0] = x0 - alpha;
                    sc[0] = 1.0 / (sigma - x0 * alpha);
                }
                saved[2 * n + k] = sc[0];
            }
        }
        __syncthreads();
        const double tau = sc[0];
        if (tau == 0.0) {
            __syncthreads();  // every warp has read sc before warp 0 writes the next column's
            continue;
        }
        for (int i = warp; i < m; i += nw) {
            const double* row = S + (k + 1 + i) * n + (k + 1);
            double sum = 0;
            for (int j = lane; j < m; j += 32) sum += row[j] * v[j];
            sum = mWarpSum(sum);
            if (lane == 0) p[i] = tau * sum;
        }
        __syncthreads();
        if (warp == 0) {
            double pv = 0;
            for (int i = lane; i < m; i += 32) pv += p[i] * v[i];
            const double K = 0.5 * tau * mWarpSum(pv);
            for (int i = lane; i < m; i += 32) wv[i] = p[i] - K * v[i];
        }
        __syncthreads();
        for (int i = warp; i < m; i += nw) {
            double* row = S + (k + 1 + i) * n + (k + 1);
            const double vi = v[i], wi = wv[i];
            for (int j = lane; j < m; j += 32) row[j] -= vi * wv[j] + wi * v[j];
        }
        for (int i = tid; i < m; i += blockDim.x) reflectors[k * n + (k + 1 + i)] = v[i];  // row k, right of the diagonal
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            d[n - 2] = S[(n - 2) * n + (n - 2)];
            e[n - 2] = S[(n - 1) * n + (n - 2)];
        }
        d[n - 1] = S[(n - 1) * n + (n - 1)];
    }
    }  // packed
    __syncthreads();
    if (tid == 0) {
        e[n - 1] = 0.0;
        double lo = INFINITY, hi = -INFINITY, emax = 0;
        for (int i = 0; i < n; ++i) {
            const double r = fabs(e[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0);
            lo = fmin(lo, d[i] - r);
            hi = fmax(hi, d[i] + r);
            emax = fmax(emax, e[i] * e[i]);
        }
        sc[0] = lo;
        sc[1] = hi;
        sc[2] = fmax(1e-300, 1e-30 * emax);  // pivot guard of the Sturm counts
        for (int k = (n >= 2 ? n - 2 : 0); k < n; ++k) saved[2 * n + k] = 0.0;
        M.fast[w] = 2;  // the tridiagonal form is saved; 1 replaces it if this path forms the prior
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) {
        saved[i] = d[i];
        saved[n + i] = e[i];
    }
    // lambda_max: the point where the Sturm count reaches n, by multisection
    double lo = sc[0], hi = sc[1];
    const double pivmin = sc[2];
    const int T = blockDim.x;
    for (int round = 0; round < 8 && hi - lo > 1e-15 * fmax(fabs(hi), fabs(lo)); ++round) {
        const double x = lo + (hi - lo) * (tid + 1) / (T + 1);
        const int below = __syncthreads_count(sturmCount(d, e, n, x, pivmin) < n);  // points still below lambda_max
        const double nlo = below > 0 ? lo + (hi - lo) * below / (T + 1) : lo;
        const double nhi = below < T ? lo + (hi - lo) * (below + 1) / (T + 1) : hi;
        lo = nlo;
        hi = nhi;
    }
    const double lmax = hi;
    const double cutoff = fmax(1e-12, 1e-9 * fmax(0.0, lmax));
    const double small = 1e-6 * cutoff;
    if (tid == 0) {
        const int c2 = sturmCount(d, e, n, 2.0 * cutoff, pivmin);
        const bool gap = sturmCount(d, e, n, small, pivmin) == c2 && sturmCount(d, e, n, -small, pivmin) == 0 && c2 < n &&
                         c2 <= kFastMaxFree;
        isc[0] = gap ? c2 : -1;
    }
    __syncthreads();
    const int nf = isc[0];
    if (nf < 0) return;  // eigenvalues near the cutoff (or too many below it): eigen path
    const int k = n - nf;
    // smallest kept eigenvalue: the point where the Sturm count passes nf
    double keptMin = 2.0 * cutoff;
    if (nf > 0) {
        double klo = 2.0 * cutoff, khi = lmax;
        for (int round = 0; round < 8 && khi - klo > 1e-3 * klo; ++round) {
            const double x = klo + (khi - klo) * (tid + 1) / (T + 1);
            const int below = __syncthreads_count(sturmCount(d, e, n, x, pivmin) <= nf);
            const double nlo = below > 0 ? klo + (khi - klo) * below / (T + 1) : klo;
            const double nhi = below < T ? klo + (khi - klo) * (below + 1) / (T + 1) : khi;
            klo = nlo;
            khi = nhi;
        }
        keptMin = klo;
    }
    // pivoted Cholesky on the full symmetric E: step s takes the largest
    // remaining diagonal p, stores the column l (over the remaining indices)
    // in column p of S and updates the remaining block by - l l^T
    for (int t = tid; t < n * n; t += blockDim.x) S[t] = E[t];
    for (int x = tid; x < n; x += blockDim.x) {
        rem[x] = x;
        stepOf[x] = n;
    }
    __syncthreads();
    int size = n;
    for (int st = 0; st < k; ++st) {
        if (warp == 0) {
            double best = -INFINITY;
            int bq = 0;
            for (int q = lane; q < size; q += 32) {
                const double x = S[rem[q] * n + rem[q]];
                if (x > best) { best = x; bq = q; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oq = __shfl_xor_sync(0xffffffffu, bq, o);
                if (ob > best || (ob == best && oq < bq)) { best = ob; bq = oq; }
            }
            if (lane == 0) {
                const int pv = rem[bq];
                sc[4] = best;
                isc[1] = pv;
                rem[bq] = rem[size - 1];
                stepOf[pv] = st;
                piv[st] = pv;
            }
        }
        __syncthreads();
        const double dpp = sc[4];
        const int pv = isc[1];
        --size;
        if (!(dpp > 0.1 * cutoff)) return;  // a weak pivot among the kept ones: eigen path (uniform)
        const double lkk = sqrt(dpp);
        for (int q = tid; q < size; q += blockDim.x) {
            const int i = rem[q];
            const double l = S[i * n + pv] / lkk;
            v[q] = l;
            S[i * n + pv] = l;
        }
        if (tid == 0) S[pv * n + pv] = lkk;
        __syncthreads();
        for (int qi = warp; qi < size; qi += nw) {
            const double li = v[qi];
            double* row = S + rem[qi] * n;
            for (int qj = lane; qj < size; qj += 32) row[rem[qj]] -= li * v[qj];
        }
        __syncthreads();
    }
    const double* bs = M.sepB + mw.vec0;
    if (nf > 0) {
        // the remainder must be negligible against the kept spectrum
        if (warp == 0) {
            double f2 = 0;
            for (int t = lane; t < nf * nf; t += 32) {
                const double x = S[rem[t / nf] * n + rem[t % nf]];
                f2 += x * x;
            }
            f2 = mWarpSum(f2);
            if (lane == 0) sc[5] = sqrt(f2);
        }
        __syncthreads();
        if (!(sc[5] <= 1e-10 * keptMin)) return;  // eigen path (uniform)
        // null(A): for free index f, N_f = e_f + sum_s alpha_s e_{p_s} with
        // A N_f = 0, by back substitution over the pivots; alpha_s is kept in
        // S[p_s][f] (row p_s of a non-pivot column holds no factor entry)
        for (int fq = warp; fq < nf; fq += nw) {
            const int f = rem[fq];
            for (int st = k - 1; st >= 0; --st) {
                const int ps = piv[st];
                double sum = 0;
                for (int t = st + 1 + lane; t < k; t += 32) sum += S[piv[t] * n + ps] * S[piv[t] * n + f];
                sum = mWarpSum(sum);
                const double alpha = -(S[f * n + ps] + sum) / S[ps * n + ps];
                if (lane == 0) S[ps * n + f] = alpha;
                __syncwarp();
            }
        }
        __syncthreads();
        // G = N^T N, h = N^T b
        for (int t = warp; t < nf * (nf + 1); t += nw) {
            const int a = t / (nf + 1), c = t % (nf + 1);
            const int fa = rem[a];
            double sum = 0;
            if (c < nf) {
                const int fc = rem[c];
                for (int st = lane; st < k; st += 32) sum += S[piv[st] * n + fa] * S[piv[st] * n + fc];
            } else {
                for (int st = lane; st < k; st += 32) sum += S[piv[st] * n + fa] * bs[piv[st]];
            }
            sum = mWarpSum(sum);
            if (lane == 0) {
                if (c < nf) G[a * nf + c] = sum + (a == c ? 1.0 : 0.0);
                else h[a] = sum + bs[fa];
            }
        }
        __syncthreads();
        if (tid == 0) {  // G y = h (G >= I), y into h
            for (int j = 0; j < nf; ++j) {
                double djj = G[j * nf + j];
                for (int q = 0; q < j; ++q) djj -= G[j * nf + q] * G[j * nf + q];
                djj = sqrt(djj);
                G[j * nf + j] = djj;
                for (int i = j + 1; i < nf; ++i) {
                    double x = G[i * nf + j];
                    for (int q = 0; q < j; ++q) x -= G[i * nf + q] * G[j * nf + q];
                    G[i * nf + j] = x / djj;
                }
            }
            for (int i = 0; i < nf; ++i) {
                double x = h[i];
                for (int q = 0; q < i; ++q) x -= G[i * nf + q] * h[q];
                h[i] = x / G[i * nf + i];
            }
            for (int i = nf - 1; i >= 0; --i) {
                double x = h[i];
                for (int q = i + 1; q < nf; ++q) x -= G[q * nf + i] * h[q];
                h[i] = x / G[i * nf + i];
            }
        }
        __syncthreads();
    }
    // P b at the pivots (N's entries there are the alphas), in pivot order
    for (int st = tid; st < k; st += blockDim.x) {
        const int ps = piv[st];
        double x = bs[ps];
        for (int q = 0; q < nf; ++q) x -= h[q] * S[ps * n + rem[q]];
        p[st] = x;
    }
    __syncthreads();
    // r0: A^T r0 = P b over the pivot rows, A[s][p_t] = S[p_t][p_s] (t >= s)
    if (warp == 0) {
        for (int st = 0; st < k; ++st) {
            const int ps = piv[st];
            const double r = p[st] / S[ps * n + ps];
            __syncwarp();
            if (lane == 0) p[st] = r;
            for (int t = st + 1 + lane; t < k; t += 32) p[t] -= S[piv[t] * n + ps] * r;
            __syncwarp();
        }
    }
    __syncthreads();
    double* A = M.A + mw.sep0;
    double* r0 = M.r0 + mw.vec0;
    for (int st = warp; st < k; st += nw) {
        const int ps = piv[st];
        for (int x = lane; x < n; x += 32) A[(long long)st * n + x] = stepOf[x] >= st ? S[x * n + ps] : 0.0;
    }
    for (int st = tid; st < k; st += blockDim.x) r0[st] = p[st];
    if (tid == 0) {
        M.rank[w] = k;
        M.stats[4 * w + 3] = cutoff;
        M.fast[w] = 1;
    }
}

// Eigendecomposition of the separator information and the square-root prior,
// rows in ascending eigenvalue order.
// ---------------------------------------------------------------------------------------
// Eigen path by the tridiagonal form, one CTA per window the fast path left:
//   1. Householder tridiagonalization E = Q T Q^T, keeping each reflector
//      H_k = I - tau_k v_k v_k^T (v_k in column k below the subdiagonal);
//   2. implicit QL iterations with Wilkinson shifts on T (the QL algorithm of
//      Bowdler, Martin, Reinsch and Wilkinson, Handbook for Automatic
//      Computation vol. II, 1971).  QL converges fastest when T grows toward
//      its bottom; a separator's tridiagonal form usually ends in its near-null
//      directions, so T is flipped (T' = P T P, P the reversal) when its top
//      diagonal entry is the larger end, as LAPACK's steqr picks QL or QR.  An
//      off-diagonal e_i is negligible when e_i^2 <= eps^2 |T| (|d_i| + |d_i+1|),
//      between the absolute test (eps |T|) and the relative one (eps |d|):
//      eigenvalues keep an absolute error of order eps |T|, as the reference's
//      own solver does, and the near-null cluster deflates in a few sweeps
//      (under the relative test alone it took up to 60 iterations for one
//      eigenvalue).  Warp 0 runs the iterations: a ballot over 32 indices finds
//      the block, lane 0 chases the bulge and logs its plane rotations into one
//      of two buffers; meanwhile the other warps apply the previous iteration's
//      rotations to the rows of V (thread per component, the running row in a
//      register, the next rows loaded ahead), so a chase and the application of
//      its predecessor overlap.  V stays orthogonal to rounding by construction;
//   3. U = Q V by the reflectors in reverse order (warp per eigenvector).
// Eigenvectors are kept as the rows of Vt (Vt[j n + r] = component r of
// eigenvector j), so both the rotations (thread per component) and the
// reflectors (lanes over components) touch consecutive addresses.  The prior
// is then formed from (lambda, U) exactly as the Jacobi path does.
// S and Vt live in shared memory up to kTriSmemN columns (when the launch's
// shared memory holds them), else in the window's eigenvector scratch (S) and
// in its separator information (Vt; E is copied into S first).  A window whose
// QL does not converge within 60 iterations per eigenvalue (NaN entries never
// converge) is left to the Jacobi kernel (fast[w] stays 0) when E is still
// intact (shared memory), and fails with CGMLI_E_NONFINITE otherwise.
constexpr int kTriSmemN = 110;
constexpr int kQlMaxIterations = 60;
constexpr int kTriReflBlock = 8;        // reflectors staged together in the back-transformation
constexpr int kTriStageMaxRows = 64;    // eigenvector rows staged together (global-memory case)
__host__ __device__ constexpr size_t triVecBytes(int n) { return sizeof(double) * 7 * (size_t)n; }  // d, e, tau, 2 x (cos, sin)
// the shared-memory case also stages the reflector block after S and V
__host__ __device__ constexpr size_t triSmemBytes(int n) {
    return (n <= kTriSmemN ? sizeof(double) * 2 * (size_t)n * n : 0) + triVecBytes(n) + sizeof(double) * kTriReflBlock * (size_t)n;
}
// global-memory case: the vectors, R staged eigenvector rows and the reflector block
__host__ __device__ constexpr size_t triStageBytes(int n, int rows) {
    return triVecBytes(n) + sizeof(double) * ((size_t)rows + kTriReflBlock) * (size_t)n;
}
// rows of V the global-memory case stages with `bytes` of dynamic shared memory (>= 1)
__host__ __device__ inline int triStageRows(int n, long long bytes) {
    const long long rows = (bytes / (long long)sizeof(double) - 7ll * n - (long long)kTriReflBlock * n) / n;
    return (int)(rows < 1 ? 1 : rows > kTriStageMaxRows ? kTriStageMaxRows : rows);
}
__global__ void __launch_bounds__(kEigenThreads) k_marg_tridiag(MargBatch M) {
    const int w = M.bigFirst[blockIdx.x];
    const MargWin mw = M.win[w];
    const int n = mw.nr;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    // fast[w] == 2: the fast path declined the window after its tridiagonalization,
    // which is this kernel's step 1 operation for operation, and saved it
    const bool saved = M.fast[w] == 2;
    if ((M.fast[w] && !saved) || mw.m == 0 || n == 0 || n > kMargMaxSep || M.status[w] != CGMLI_OK) return;
    extern __shared__ double tsm[];
    const bool inShared = n <= kTriSmemN && (long long)triSmemBytes(n) <= M.triSmem;
    double* S = inShared ? tsm : saved ? M.A + mw.sep0 : M.sepV + mw.sep0;  // n x n row-major
    double* Vt = inShared ? tsm + (size_t)n * n : M.sepH + mw.sep0;
    double* d = inShared ? tsm + 2 * (size_t)n * n : tsm;
    double* e = d + n;
    double* tau = e + n;
    double* rc = tau + n;  // rotations of a QL chase (cos, sin; two buffers), also the reflector scratch
    double* rs = rc + 2 * n;
    __shared__ double sc[4];
    __shared__ int isc[4];
    __shared__ int qlMid[2], qlCount[2];  // per rotation buffer: the chase's block end m and its rotation count
    __shared__ double red[kEigenThreads / 32];
    __shared__ int pos[kMargMaxSep];
    const double* E = M.sepH + mw.sep0;
    if (saved) {  // the reflectors from the prior's slot, d, e and tau from the victim scratch
        if (inShared)
            for (long long t = tid; t < (long long)n * n; t += blockDim.x) S[t] = M.A[mw.sep0 + t];
        const double* sv = M.X + mw.x0;
        for (int i = tid; i < 3 * n; i += blockDim.x) d[i] = sv[i];  // d, e, tau are consecutive
    } else {
        for (long long t = tid; t < (long long)n * n; t += blockDim.x) S[t] = E[t];
    }
    __syncthreads();
    // 1. tridiagonalization; the trailing block is updated on both triangles
    for (int k = 0; !saved && k + 2 < n; ++k) {
        const int m = n - k - 1;
        double* v = rc;  // the reflector of this column
        double* p = rs;
        if (warp == 0) {
            double sigma = 0;
            for (int i = lane; i < m; i += 32) {
                const double x = S[(size_t)(k + 1 + i) * n + k];
                v[i] = x;
                sigma += x * x;
            }
            sigma = mWarpSum(sigma);
            __syncwarp();
            if (lane == 0) {
                d[k] = S[(size_t)k * n + k];
                if (sigma == 0.0) {
                    e[k] = 0.0;
                    sc[0] = 0.0;
                } else {
                    const double x0 = v[0];
                    const double alpha = x0 >= 0 ? -sqrt(sigma) : sqrt(sigma);
                    e[k] = alpha;
                    v[0] = x0 - alpha;
                    sc[0] = 1.0 / (sigma - x0 * alpha);
                }
                tau[k] = sc[0];
            }
        }
        __syncthreads();
        const double tk = sc[0];
        if (tk == 0.0) {
            __syncthreads();  // every warp has read sc before warp 0 writes the next column's
            continue;
        }
        for (int i = warp; i < m; i += nw) {  // p = tau S v over the trailing block
            const double* row = S + (size_t)(k + 1 + i) * n + (k + 1);
            double sum = 0;
            for (int j = lane; j < m; j += 32) sum += row[j] * v[j];
            sum = mWarpSum(sum);
            if (lane == 0) p[i] = tk * sum;
        }
        __syncthreads();
        if (warp == 0) {  // w = p - (tau p^T v / 2) v, kept in p
            double pv = 0;
            for (int i = lane; i < m; i += 32) pv += p[i] * v[i];
            const double K = 0.5 * tk * mWarpSum(pv);
            __syncwarp();
            for (int i = lane; i < m; i += 32) p[i] -= K * v[i];
        }
        __syncthreads();
        for (int i = warp; i < m; i += nw) {
            double* row = S + (size_t)(k + 1 + i) * n + (k + 1);
            const double vi = v[i], wi = p[i];
            for (int j = lane; j < m; j += 32) row[j] -= vi * p[j] + wi * v[j];
        }
        __syncthreads();
        // keep the reflector in row k right of the diagonal (contiguous; no later step reads there)
        for (int i = tid; i < m; i += blockDim.x) S[(size_t)k * n + (k + 1 + i)] = v[i];
        __syncthreads();
    }
    if (tid == 0) {
        if (!saved) {
            if (n >= 2) {
                d[n - 2] = S[(size_t)(n - 2) * n + (n - 2)];
                e[n - 2] = S[(size_t)(n - 1) * n + (n - 2)];
                tau[n - 2] = 0.0;
            }
            d[n - 1] = S[(size_t)(n - 1) * n + (n - 1)];
            e[n - 1] = 0.0;
            tau[n - 1] = 0.0;
        }
        double norm = 0;
        for (int i = 0; i < n; ++i) norm = fmax(norm, fmax(fabs(d[i]), fabs(e[i])));
        sc[1] = norm;
        isc[3] = fabs(d[0]) > fabs(d[n - 1]) ? 1 : 0;
    }
    __syncthreads();
    const bool flipped = isc[3] != 0;
    const double deflation = DBL_EPSILON * DBL_EPSILON * sc[1];
    if (flipped) {  // T' = P T P: d reversed, e reversed over its n - 1 couplings
        for (int i = tid; i < n / 2; i += blockDim.x) {
            const double t = d[i];
            d[i] = d[n - 1 - i];
            d[n - 1 - i] = t;
        }
        for (int i = tid; i < (n - 1) / 2; i += blockDim.x) {
            const double t = e[i];
            e[i] = e[n - 2 - i];
            e[n - 2 - i] = t;
        }
    }
    // V starts as the identity in T's coordinates: P itself when T was flipped
    for (long long t = tid; t < (long long)n * n; t += blockDim.x) {
        const int j = (int)(t / n), r = (int)(t % n);
        Vt[t] = (flipped ? j + r == n - 1 : j == r) ? 1.0 : 0.0;
    }
    __syncthreads();
    // 2. implicit QL; e[i] couples i and i + 1.  Step s: warp 0 runs one iteration into
    // buffer s & 1 while the other warps apply the rotations of step s - 1.
    int l = 0, iter = 0;  // warp 0's position (uniform over the warp)
    int qlEnd = 0;        // -1: converged, -2: an eigenvalue did not converge
    for (int step = 0;; ++step) {
        const int b = step & 1;
        if (warp == 0) {
            int m = l, count = -1;
            while (l < n) {  // the first negligible coupling at or after l (n - 1: none)
                for (int base = l;; base += 32) {
                    const int i = base + lane;
                    bool negligible = i >= n - 1;
                    if (!negligible) {
                        const double ei = e[i];
                        negligible = fabs(ei) < DBL_MIN || ei * ei <= deflation * (fabs(d[i]) + fabs(d[i + 1]));
                    }
                    const unsigned hit = __ballot_sync(0xffffffffu, negligible);
                    if (hit) {
                        m = base + __ffs(hit) - 1;
                        break;
                    }
                }
                if (m != l) break;
                ++l;  // d[l] is an eigenvalue
                iter = 0;
            }
            if (l < n) {
                if (iter >= kQlMaxIterations) {
                    count = -2;
                } else {
                    if (lane == 0) {  // chase the bulge from m up to l, logging each rotation
                        double* cb = rc + b * n;
                        double* sb = rs + b * n;
                        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                        double r = hypot(g, 1.0);
                        g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
                        double s = 1.0, c = 1.0, p = 0.0;
                        bool split = false;
                        count = 0;
                        // d[i], d[i + 1] and e[i] of a step are not yet written by this chase: they
                        // are carried in registers and the next step's are loaded ahead
                        double ei = e[m - 1], di = d[m - 1], dip1 = d[m];
                        for (int i = m - 1; i >= l; --i) {
                            const double en = i > l ? e[i - 1] : 0.0, dn = i > l ? d[i - 1] : 0.0;
                            const double f = s * ei, bq = c * ei;
                            const double q = f * f + g * g;
                            if (q > 1e-280 && q < 1e280) {  // one reciprocal square root for r, c and s
                                const double rq = rsqrt(q);
                                r = q * rq;
                                s = f * rq;
                                c = g * rq;
                            } else {
                                r = hypot(f, g);
                                if (r != 0.0) {
                                    s = f / r;
                                    c = g / r;
                                }
                            }
                            e[i + 1] = r;
                            if (r == 0.0) {  // the bulge vanished: deflate and restart the chase
                                d[i + 1] = dip1 - p;
                                e[m] = 0.0;
                                split = true;
                                break;
                            }
                            g = dip1 - p;
                            r = (di - g) * s + 2.0 * c * bq;
                            p = s * r;
                            d[i + 1] = g + p;
                            g = c * r - bq;
                            cb[count] = c;
                            sb[count] = s;
                            ++count;
                            dip1 = di;
                            di = dn;
                            ei = en;
                        }
                        if (!split) {
                            d[l] -= p;
                            e[l] = g;
                            e[m] = 0.0;
                        }
                    }
                    count = __shfl_sync(0xffffffffu, count, 0);
                    ++iter;
                    __syncwarp();  // lane 0's d, e before the next scan
                }
            }
            if (lane == 0) {
                qlMid[b] = m;
                qlCount[b] = count;
            }
        } else if (step > 0) {
            // rotation q of the previous chase acts on rows (m - 1 - q, m - q) of V
            const int pb = b ^ 1, m = qlMid[pb], count = qlCount[pb];
            const double* cb = rc + pb * n;
            const double* sb = rs + pb * n;
            for (int r = tid - 32; count > 0 && r < n; r += blockDim.x - 32) {
                double carry = Vt[(size_t)m * n + r];
                int q = 0;
                for (; q + 8 <= count; q += 8) {
                    double a[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) a[u] = Vt[(size_t)(m - 1 - q - u) * n + r];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const double c = cb[q + u], s = sb[q + u];
                        Vt[(size_t)(m - q - u) * n + r] = s * a[u] + c * carry;
                        carry = c * a[u] - s * carry;
                    }
                }
                for (; q < count; ++q) {
                    const double a = Vt[(size_t)(m - 1 - q) * n + r];
                    const double c = cb[q], s = sb[q];
                    Vt[(size_t)(m - q) * n + r] = s * a + c * carry;
                    carry = c * a - s * carry;
                }
                Vt[(size_t)(m - count) * n + r] = carry;
            }
        }
        __syncthreads();
        // the buffer written in this step is rewritten two steps on, after another barrier
        if (qlCount[b] < 0) {
            qlEnd = qlCount[b];
            break;
        }
    }
    if (qlEnd == -2) {  // not converged (uniform): the Jacobi kernel takes the window while E is intact
        if (tid == 0) {
            if (inShared) M.fast[w] = 0;
            else { M.status[w] = CGMLI_E_NONFINITE; M.rank[w] = 0; M.fast[w] = 3; }
        }
        return;
    }
    // 3. U = Q V: H_k acts on components k + 1.. of every eigenvector, for k = n - 3 down to 0.
    // With V in global memory, batches of R eigenvector rows are staged in shared memory
    // and every reflector is applied to a batch while it is there; the reflectors come
    // kTriReflBlock at a time (one round of coalesced loads per block).
    const int R = inShared ? n : triStageRows(n, M.triSmem);
    double* Bt = inShared ? Vt : rs + 2 * n;                       // R x n rows of V
    double* rb = inShared ? rs + 2 * n : Bt + (size_t)R * n;         // kTriReflBlock reflectors, n apart
    for (int j0 = 0; j0 < n; j0 += R) {
        const int rows = min(R, n - j0);
        if (!inShared) {
            for (long long t = tid; t < (long long)rows * n; t += blockDim.x) Bt[t] = Vt[(size_t)j0 * n + t];
            __syncthreads();
        }
        for (int kb = n - 3; kb >= 0; kb -= kTriReflBlock) {
            const int nk = min(kTriReflBlock, kb + 1);  // reflectors kb, kb - 1, .., kb - nk + 1
            for (int q = 0; q < nk; ++q) {
                const int k = kb - q, m = n - k - 1;
                for (int i = tid; i < m; i += blockDim.x) rb[(size_t)q * n + i] = S[(size_t)k * n + (k + 1 + i)];
            }
            __syncthreads();
            for (int q = 0; q < nk; ++q) {
                const int k = kb - q, m = n - k - 1;
                const double tk = tau[k];
                if (tk == 0.0) continue;  // uniform
                const double* v = rb + (size_t)q * n;
                // eight threads per eigenvector row (a reduction of three shuffles), four rows per
                // warp; the loop bound is uniform over the warp, so every lane reaches the shuffles
                const int g = tid & 7;
                for (int j0 = warp * 4; j0 < rows; j0 += nw * 4) {
                    const int j = j0 + ((tid >> 3) & 3);
                    const bool active = j < rows;
                    double* u = Bt + (size_t)j * n + (k + 1);
                    double z = 0;
                    if (active)
                        for (int i = g; i < m; i += 8) z += v[i] * u[i];
                    z += __shfl_xor_sync(0xffffffffu, z, 4);
                    z += __shfl_xor_sync(0xffffffffu, z, 2);
                    z += __shfl_xor_sync(0xffffffffu, z, 1);
                    z *= tk;
                    if (active)
                        for (int i = g; i < m; i += 8) u[i] -= z * v[i];
                }
                __syncthreads();
            }
        }
        if (!inShared) {
            for (long long t = tid; t < (long long)rows * n; t += blockDim.x) Vt[(size_t)j0 * n + t] = Bt[t];
            __syncthreads();
        }
    }
    // the prior from (lambda, U) as the Jacobi path forms it; eigenvector i is column i of V
    double* ev = M.evals + mw.vec0;
    const double* bs = M.sepB + mw.vec0;
    for (int i = tid; i < n; i += blockDim.x) ev[i] = d[i];
    __syncthreads();
    double vmax = -INFINITY, vmin = INFINITY;
    bool finite = true;
    for (int i = tid; i < n; i += blockDim.x) {
        vmax = fmax(vmax, ev[i]);
        vmin = fmin(vmin, ev[i]);
        finite = finite && isfinite(ev[i]);
    }
    vmax = mBlockMax(vmax, red);
    vmin = -mBlockMax(-vmin, red);
    const double nonFinite = mBlockMax(finite ? 0.0 : 1.0, red);
    const double cutoff = fmax(1e-12, 1e-9 * fmax(0.0, vmax));
    if (nonFinite > 0 || vmin < -10 * cutoff) {
        if (tid == 0) { M.status[w] = nonFinite > 0 ? CGMLI_E_NONFINITE : CGMLI_E_INDEFINITE; M.rank[w] = 0; M.fast[w] = 3; }
        return;
    }
    ascendingPositions(ev, n, pos);
    double low = 0;
    for (int i = tid; i < n; i += blockDim.x) low += ev[i] > cutoff ? 0.0 : 1.0;
    const int nLow = (int)mBlockSum(low, red);
    double* A = M.A + mw.sep0;
    double* r0 = M.r0 + mw.vec0;
    for (long long t = tid; t < (long long)n * n; t += blockDim.x) {
        const int i = (int)(t / n), k = (int)(t % n);  // eigenpair i, component k
        if (!(ev[i] > cutoff)) continue;
        A[(long long)(pos[i] - nLow) * n + k] = sqrt(ev[i]) * Vt[t];
    }
    for (int i = warp; i < n; i += nw) {
        if (!(ev[i] > cutoff)) continue;  // uniform over the warp
        double ub = 0;
        for (int k = lane; k < n; k += 32) ub += Vt[(size_t)i * n + k] * bs[k];
        ub = mWarpSum(ub);
        if (lane == 0) r0[pos[i] - nLow] = ub / sqrt(ev[i]);
    }
    if (tid == 0) {
        M.rank[w] = n - nLow;
        M.stats[4 * w + 3] = cutoff;
        M.fast[w] = 3;  // formed here: the Jacobi kernel skips the window
    }
}

__global__ void __launch_bounds__(kEigenThreads) k_marg_eigen(MargBatch M) {
    const int w = M.bigFirst[blockIdx.x];
    const MargWin mw = M.win[w];
    const int nr = mw.nr;
    if (M.fast[w]) return;  // prior formed by k_marg_fast or k_marg_tridiag
    if (mw.m == 0 || nr == 0 || M.status[w] != CGMLI_OK) {
        if (threadIdx.x == 0) M.rank[w] = 0;
        return;
    }
    extern __shared__ double eigSmem[];
    double* E = M.sepH + mw.sep0;
    double* ev = M.evals + mw.vec0;
    const double* bs = M.sepB + mw.vec0;
    __shared__ int pos[kMargMaxSep];
    __shared__ double red[kEigenThreads / 32];
    // component k of eigenvector i is Vv[i * si + k * sk]
    const double* Vv;
    long long si, sk;
    const long long packed = (long long)nr * (nr + 1) / 2;
    if (packed * 8 <= M.eigenSmem) {
        double* Ap = eigSmem;
        double* Vt = (packed + (long long)nr * nr) * 8 <= M.eigenSmem ? eigSmem + packed : M.sepV + mw.sep0;
        for (long long t = threadIdx.x; t < (long long)nr * nr; t += blockDim.x) {
            const int i = (int)(t / nr), j = (int)(t % nr);
            if (i <= j) Ap[pkUp(i, j, nr)] = E[t];
        }
        __syncthreads();
        jacobiPacked(Ap, Vt, nr, 60);
        for (int i = threadIdx.x; i < nr; i += blockDim.x) ev[i] = Ap[pkUp(i, i, nr)];
        Vv = Vt; si = nr; sk = 1;
    } else {
        double* V = M.sepV + mw.sep0;
        jacobiEigen(E, V, nr, 60);
        for (int i = threadIdx.x; i < nr; i += blockDim.x) ev[i] = E[(long long)i * nr + i];
        Vv = V; si = 1; sk = nr;
    }
    __syncthreads();
    double vmax = -INFINITY, vmin = INFINITY;
    bool finite = true;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        vmax = fmax(vmax, ev[i]);
        vmin = fmin(vmin, ev[i]);
        finite = finite && isfinite(ev[i]);
    }
    vmax = mBlockMax(vmax, red);
    vmin = -mBlockMax(-vmin, red);
    const double nonFinite = mBlockMax(finite ? 0.0 : 1.0, red);
    const double cutoff = fmax(1e-12, 1e-9 * fmax(0.0, vmax));
    if (nonFinite > 0 || vmin < -10 * cutoff) {
        if (threadIdx.x == 0) { M.status[w] = nonFinite > 0 ? CGMLI_E_NONFINITE : CGMLI_E_INDEFINITE; M.rank[w] = 0; }
        return;
    }
    ascendingPositions(ev, nr, pos);
    double low = 0;
    for (int i = threadIdx.x; i < nr; i += blockDim.x) low += ev[i] > cutoff ? 0.0 : 1.0;
    const int nLow = (int)mBlockSum(low, red);
    double* A = M.A + mw.sep0;
    double* r0 = M.r0 + mw.vec0;
    for (long long t = threadIdx.x; t < (long long)nr * nr; t += blockDim.x) {
        const int i = (int)(t / nr), k = (int)(t % nr);  // eigenpair i, component k
        if (!(ev[i] > cutoff)) continue;
        A[(long long)(pos[i] - nLow) * nr + k] = sqrt(ev[i]) * Vv[i * si + k * sk];
    }
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        if (!(ev[i] > cutoff)) continue;
        double ub = 0;
        for (int k = 0; k < nr; ++k) ub += Vv[i * si + k * sk] * bs[k];
        r0[pos[i] - nLow] = ub / sqrt(ev[i]);
    }
    if (threadIdx.x == 0) {
        M.rank[w] = nr - nLow;
        M.stats[4 * w + 3] = cutoff;
    }
}

// ---------------------------------------------------------------------------------------
// Conditional information of the calibration blocks given every other state of
// the window (BackendOptimizer::calibrationInformation,
// BackendOptimizer.cpp:1084-1170), one CTA per window.  The formation kernels
// have left H over [nuisance (poses, speed/biases) | calibration (extrinsics, td)]
// with every landmark range eliminated; here
//   C = Hcc - Hxc^T pinv(Hxx) Hxc,   pinv with the cutoff max(1e-12, 1e-9 lambda_max)
// (Marginalizer::psdSolve; significantly negative eigenvalues are an error),
// reported per extrinsic block as [theta, p] (the left-SE(3) tangent [rho, theta]
// reordered, then dp = rho - [p]x dtheta: C' = B^T C B with B(p rows, theta cols)
// = [p]x), td last; symmetrized, eigen-decomposed, negative round-off clamped.
// work holds per window 2 nx^2 + 2 nx nc + 4 nc^2 doubles from work0[w].  The
// nuisance block's Jacobi runs on its packed upper triangle in dynamic shared
// memory when it fits in packedSmem bytes (eigenvectors as rows in global
// memory), in global memory otherwise.
constexpr int kCalibMaxCols = 64;
__global__ void __launch_bounds__(kMargThreads) k_calib_conditional(DevBatch B, MargBatch M, double* work, const long long* work0,
                                                                  double* cond, double* evals, long long packedSmem) {
    extern __shared__ double calibSmem[];
    const int w = M.bigFirst[blockIdx.x];
    const MargWin mw = M.win[w];
    const int m = mw.m, nx = mw.nm, nc = mw.nr;
    if (m == 0 || M.status[w] != CGMLI_OK) return;
    if (nc == 0 || nc > kCalibMaxCols) {
        if (threadIdx.x == 0) M.status[w] = nc == 0 ? CGMLI_E_INVALID : CGMLI_E_LIMIT;
        return;
    }
    const WinDesc wd = B.win[w];
    const double* H = M.H + mw.H0;
    double* A = work + work0[w];
    double* V = A + (long long)nx * nx;
    double* P = V + (long long)nx * nx;  // nx x nc
    double* X = P + (long long)nx * nc;  // nx x nc
    double* Cr = X + (long long)nx * nc; // nc x nc
    double* V2 = Cr + nc * nc;           // nc x nc
    double* Cs = V2 + nc * nc;           // nc x nc
    double* Bt = Cs + nc * nc;           // nc x nc
    __shared__ double red[kMargThreads / 32];
    __shared__ int report[kCalibMaxCols], extOf[kCalibMaxCols], blockStart[kCalibMaxCols], pos[kCalibMaxCols];
    // separator layout: extrinsic blocks in index order, then td
    if (threadIdx.x == 0) {
        for (int j = 0; j < nc; ++j) { extOf[j] = -1; blockStart[j] = j; report[j] = j; }
        for (int e = 0; e < wd.E; ++e) {
            const int c = M.extCol[wd.ext0 + e];
            if (c < nx) continue;
            const int s0 = c - nx;
            for (int t = 0; t < 6; ++t) {
                extOf[s0 + t] = wd.ext0 + e;
                blockStart[s0 + t] = s0;
                report[s0 + t] = s0 + (t < 3 ? 3 + t : t - 3);  // [rho, theta] -> [theta, rho]
            }
        }
    }
    // 1. eigen-decomposition of the nuisance block.  In shared memory the
    // rotations act on Hxc's rows directly (Y = U^T Hxc, nc wide), so that
    // C = Hcc - sum over lambda_i > cut of y_i y_i^T / lambda_i needs no U;
    // otherwise U is accumulated in global memory and C = Hcc - Hxc^T U P.
    const bool inShared = nx > 0 && (long long)nx * (nx + 1) / 2 * 8 <= packedSmem;
    double* Ap = calibSmem;
    if (inShared) {
        for (long long t = threadIdx.x; t < (long long)nx * nx; t += blockDim.x) {
            const int i = (int)(t / nx), j = (int)(t % nx);
            if (i <= j) Ap[pkUp(i, j, nx)] = H[(long long)i * m + j];
        }
        for (long long t = threadIdx.x; t < (long long)nx * nc; t += blockDim.x)
            P[t] = symAt(H, (int)(t / nc), nx + (int)(t % nc), m);
        __syncthreads();
        jacobiPacked(Ap, P, nx, 60, nc);
    } else {
        for (long long t = threadIdx.x; t < (long long)nx * nx; t += blockDim.x) A[t] = symAt(H, (int)(t / nx), (int)(t % nx), m);
        __syncthreads();
        if (nx > 0) jacobiEigen(A, V, nx, 60);
    }
    __syncthreads();
    auto lam = [&](int i) { return inShared ? Ap[pkUp(i, i, nx)] : A[(long long)i * nx + i]; };
    double vmax = -INFINITY, vmin = INFINITY;
    bool finite = true;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const double v = lam(i);
        vmax = fmax(vmax, v);
        vmin = fmin(vmin, v);
        finite = finite && isfinite(v);
    }
    vmax = mBlockMax(vmax, red);
    vmin = -mBlockMax(-vmin, red);
    const double bad = mBlockMax(finite ? 0.0 : 1.0, red);
    const double cut = fmax(1e-12, 1e-9 * fmax(0.0, vmax));
    if (bad > 0 || (nx > 0 && vmin < -10 * cut)) {
        if (threadIdx.x == 0) M.status[w] = bad > 0 ? CGMLI_E_NONFINITE : CGMLI_E_INDEFINITE;
        return;
    }
    if (inShared) {
        // 2. C = Hcc - sum y_i y_i^T / lambda_i, in report order
        for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {
            const int a = t / nc, c = t % nc;
            double v = symAt(H, nx + a, nx + c, m);
            for (int i = 0; i < nx; ++i) {
                const double li = lam(i);
                if (li > cut) v -= P[(long long)i * nc + a] * P[(long long)i * nc + c] / li;
            }
            Cs[report[a] * nc + report[c]] = v;
        }
    } else {
        // 2. X = U diag(1/lambda) U^T Hxc, C = Hcc - Hxc^T X, in report order
        for (long long t = threadIdx.x; t < (long long)nx * nc; t += blockDim.x) {
            const int i = (int)(t / nc), c = (int)(t % nc);
            const double li = lam(i);
            double v = 0;
            if (li > cut) {
                for (int k = 0; k < nx; ++k) v += V[(long long)k * nx + i] * symAt(H, k, nx + c, m);
                v /= li;
            }
            P[t] = v;
        }
        __syncthreads();
        for (long long t = threadIdx.x; t < (long long)nx * nc; t += blockDim.x) {
            const int k = (int)(t / nc), c = (int)(t % nc);
            double v = 0;
            for (int i = 0; i < nx; ++i) v += V[(long long)k * nx + i] * P[(long long)i * nc + c];
            X[t] = v;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {
            const int a = t / nc, c = t % nc;
            double v = symAt(H, nx + a, nx + c, m);
            for (int k = 0; k < nx; ++k) v -= symAt(H, k, nx + a, m) * X[(long long)k * nc + c];
            Cs[report[a] * nc + report[c]] = v;
        }
    }
    __syncthreads();
    // 3. C' = B^T C B, B = I except [p]x in (p rows, theta cols) of each extrinsic block
    auto basis = [&](int r, int c) -> double {  // B(r, c), report order
        if (r == c) return 1.0;
        const int e = extOf[r];
        if (e < 0 || extOf[c] != e) return 0.0;
        const int s0 = blockStart[r], i = r - s0, j = c - s0;
        if (i < 3 || j >= 3) return 0.0;
        const double* p = B.ext[0] + 7ll * e;  // [p]x (i - 3, j)
        const int a = i - 3;
        if (a == j) return 0.0;
        const double pk = p[3 - a - j];
        return (a + 1) % 3 == j ? -pk : pk;
    };
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {  // Bt = B^T C
        const int r = t / nc, c = t % nc;
        double v = 0;
        for (int k = 0; k < nc; ++k) v += basis(k, r) * Cs[k * nc + c];
        Bt[t] = v;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {  // Cr = Bt B
        const int r = t / nc, c = t % nc;
        double v = 0;
        for (int k = 0; k < nc; ++k) v += Bt[r * nc + k] * basis(k, c);
        Cr[t] = v;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {  // symmetrize
        const int r = t / nc, c = t % nc;
        Cs[t] = 0.5 * Cr[t] + 0.5 * Cr[c * nc + r];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) Cr[t] = Cs[t];
    __syncthreads();
    // 4. eigen-decomposition, clamp, recompose
    jacobiEigen(Cr, V2, nc, 60);
    __syncthreads();
    double emax = -INFINITY, emin = INFINITY;
    finite = true;
    for (int i = threadIdx.x; i < nc; i += blockDim.x) {
        const double v = Cr[i * nc + i];
        emax = fmax(emax, v);
        emin = fmin(emin, v);
        finite = finite && isfinite(v);
    }
    emax = mBlockMax(emax, red);
    emin = -mBlockMax(-emin, red);
    const double bad2 = mBlockMax(finite ? 0.0 : 1.0, red);
    const double cut2 = fmax(1e-12, 1e-9 * fmax(0.0, emax));
    if (bad2 > 0 || emin < -10 * cut2) {
        if (threadIdx.x == 0) M.status[w] = bad2 > 0 ? CGMLI_E_NONFINITE : CGMLI_E_INDEFINITE;
        return;
    }
    double* ev = evals + 2 * mw.vec0;  // 2 m per window: sorted, then the unsorted copy
    for (int i = threadIdx.x; i < nc; i += blockDim.x) ev[nc + i] = fmax(Cr[i * nc + i], 0.0);
    __syncthreads();
    ascendingPositions(ev + nc, nc, pos);
    for (int i = threadIdx.x; i < nc; i += blockDim.x) ev[pos[i]] = ev[nc + i];
    double* out = cond + mw.sep0;  // upper triangle computed, mirrored: exactly symmetric
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) {
        const int r = t / nc, c = t % nc;
        if (r > c) continue;
        double v = 0;
        for (int i = 0; i < nc; ++i) v += V2[r * nc + i] * ev[nc + i] * V2[c * nc + i];
        out[t] = v;
        out[c * nc + r] = v;
    }
}

// ---------------------------------------------------------------------------------------
// Dense helpers (one CTA).  H, rhs, solution column-major; H is read from its
// lower triangle like cusolverDnDsyevd with CUBLAS_FILL_MODE_LOWER.
__global__ void __launch_bounds__(kMargThreads) k_dense_eigen(const double* H, int n, double* work, double* evals, double* evecs,
                                                              int* status) {
    double* A = work;
    double* V = work + (long long)n * n;
    __shared__ int pos[kMargMaxSep];
    for (long long t = threadIdx.x; t < (long long)n * n; t += blockDim.x) {
        const int i = (int)(t / n), j = (int)(t % n);
        A[t] = i >= j ? H[i + (long long)j * n] : H[j + (long long)i * n];
    }
    __syncthreads();
    jacobiEigen(A, V, n, 60);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        evals[n + i] = A[(long long)i * n + i];  // unsorted copy in the upper half of evals
        if (!isfinite(evals[n + i])) *status = CGMLI_E_NONFINITE;
    }
    __syncthreads();
    ascendingPositions(evals + n, n, pos);
    for (int i = threadIdx.x; i < n; i += blockDim.x) evals[pos[i]] = evals[n + i];
    for (long long t = threadIdx.x; t < (long long)n * n; t += blockDim.x) {
        const int k = (int)(t / n), i = (int)(t % n);  // row k of V, eigenpair i
        evecs[k + (long long)pos[i] * n] = V[t];
    }
}
// projected = U^T rhs with the cutoff (eigenvalues ascending, U column-major).
__global__ void k_dense_psd_project(const double* evals, const double* U, const double* rhs, int n, int columns, double absCut,
                                    double relCut, double* projected, int* status) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * columns) return;
    const int i = (int)(t % n), c = (int)(t / n);
    const double cutoff = fmax(absCut, relCut * fmax(0.0, evals[n - 1])), v = evals[i];
    if (v < -10 * cutoff || !isfinite(v)) *status = CGMLI_E_INDEFINITE;
    double s = 0;
    for (int k = 0; k < n; ++k) s += U[k + (long long)i * n] * rhs[k + (long long)c * n];
    projected[t] = v > cutoff ? s / v : 0.0;
}
// solution = U projected
__global__ void k_dense_psd_expand(const double* U, const double* projected, int n, int columns, double* solution) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * columns) return;
    const int i = (int)(t % n), c = (int)(t / n);
    double s = 0;
    for (int k = 0; k < n; ++k) s += U[i + (long long)k * n] * projected[k + (long long)c * n];
    solution[t] = s;
}
// [H | g] -= coupling^T solution; coupling nm x nr, solution nm x (nr + 1).
__global__ void k_dense_subtract(const double* coupling, const double* solution, int nm, int nr, double* Hg) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nr * (nr + 1)) return;
    const int i = (int)(t % nr), c = (int)(t / nr);
    double s = 0;
    for (int k = 0; k < nm; ++k) s += coupling[k + (long long)i * nm] * solution[k + (long long)c * nm];
    Hg[t] -= s;
}

// ---------------------------------------------------------------------------------------
size_t margVisualSmemBytes(int maxNc) {
    return sizeof(double) * ((size_t)maxNc * (maxNc + 1) / 2 + 2 * maxNc + 32 * 50 + 32 * 4) + sizeof(short) * 32 * 25 +
           sizeof(int) * 32;
}
// Sets the dynamic shared memory limits of the marginalization kernels for a
// batch whose largest separator has maxNr columns; returns the eigen CTA's
// dynamic shared memory in eigenSmem.
size_t margRowsSmemBytes(int maxNv) {
    const int np = (maxNv + 31) & ~31;
    size_t v = 0;  // widest rows x np over the padded widths up to np
    for (int p = 32; p <= np; p += 32) v = std::max(v, (size_t)rowsCapOf(p) * p);
    return sizeof(double) * ((size_t)kRowsCap * kMargRecord + 2 * kRowsCap + v);
}
int margRowsCap(int nv) { return rowsCapOf((nv + 31) & ~31); }
cudaError_t configureMarginalization(size_t visualSmem, size_t rowsSmem, int maxNr, int maxFastNr, long long* eigenSmem,
                                     long long* fastSmem, long long* triSmem) {
    cudaError_t e = cudaFuncSetAttribute(k_marg_visual, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)visualSmem);
    if (e != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_marg_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rowsSmem)) != cudaSuccess)
        return e;
    // the widest shared-memory window, the widest packed one, the widest window's vectors
    *fastSmem = maxFastNr > 0 ? (long long)std::max({fastSmemBytes(maxFastNr < kFastMaxN ? maxFastNr : kFastMaxN),
                                                    maxFastNr > kFastMaxN ? fastPackedBytes(std::min(maxFastNr, kFastPackedMaxN)) : (size_t)0,
                                                    fastSmemBytes(maxFastNr < kMargMaxSep ? maxFastNr : kMargMaxSep)})
                              : 0;
    if ((e = cudaFuncSetAttribute(k_marg_fast, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)std::max(fastSmemBytes(kFastMaxN), fastPackedBytes(kFastPackedMaxN)))) != cudaSuccess)
        return e;
    int dev = 0, optin = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, k_marg_eigen)) != cudaSuccess) return e;
    const long long avail = (long long)optin - (long long)fa.sharedSizeBytes;
    // eigenvectors in shared memory too when they fit
    const long long n = maxNr, want = 8 * (n * (n + 1) / 2 + n * n), packedOnly = 8 * (n * (n + 1) / 2);
    long long use = want <= avail ? want : (packedOnly <= avail ? packedOnly : 0);
    if (use < 0) use = 0;
    *eigenSmem = use;
    if ((e = cudaFuncSetAttribute(k_marg_eigen, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)use)) != cudaSuccess) return e;
    cudaFuncAttributes ta;
    if ((e = cudaFuncGetAttributes(&ta, k_marg_tridiag)) != cudaSuccess) return e;
    // windows up to kTriSmemN columns in shared memory, the vectors of the widest one
    const int triN = maxNr < 1 ? 1 : (maxNr > kMargMaxSep ? kMargMaxSep : maxNr);
    // the largest shared-memory window, or the widest window's vectors with its staged rows
    // (as many as fit under 200 KB, at most kTriStageMaxRows, at least one)
    const int stageRows = std::max(1, std::min(kTriStageMaxRows, (int)((200ll * 1024 / sizeof(double) - 7ll * triN - (long long)kTriReflBlock * triN) / std::max(triN, 1))));
    *triSmem = (long long)std::max(triSmemBytes(triN < kTriSmemN ? triN : kTriSmemN), triStageBytes(triN, stageRows));
    if (*triSmem > (long long)optin - (long long)ta.sharedSizeBytes) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(k_marg_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<long long>(*triSmem, 1));
}
// Returns the number of launches.
// Rotations of the accepted state (the factors' inputs), one thread per keyframe or extrinsic.
__global__ void k_marg_rotations(DevBatch B) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < B.numKf) poseRotation(B.pose[0] + 7ll * t, B.rotKf[0] + 9ll * t);
    else if (t < B.numKf + B.numExt) poseRotation(B.ext[0] + 7ll * (t - B.numKf), B.rotExt[0] + 9ll * (t - B.numKf));
}
int launchMarginalization(const DevBatch& B, const MargBatch& M, size_t visualSmem, cudaStream_t s) {
    int n = 1;
    k_marg_rotations<<<(B.numKf + B.numExt + 255) / 256, 256, 0, s>>>(B);
    if (M.numElim > 0) {
        const int warps = 8;
        k_marg_eval<<<(M.numElim + warps - 1) / warps, 32 * warps, 0, s>>>(B, M);
        ++n;
    }
    if (M.numItems > 0) {
        k_marg_rows<<<M.numItems, kRowsThreads, (size_t)M.rowsSmem, s>>>(B, M);
        ++n;
    }
    if (M.numSlowElim > 0) {
        k_marg_visual<<<M.numSlowElim, kMargLmThreads, visualSmem, s>>>(B, M);
        ++n;
    }
    k_marg_retained<<<M.numWindows, 256, 0, s>>>(B, M);
    k_marg_victim<<<M.numWindows, kMargThreads, 0, s>>>(M);
    k_marg_fast<<<M.numWindows, kMargThreads, (size_t)M.fastSmem, s>>>(M);
    k_marg_tridiag<<<M.numWindows, kEigenThreads, (size_t)M.triSmem, s>>>(M);
    k_marg_eigen<<<M.numWindows, kEigenThreads, (size_t)M.eigenSmem, s>>>(M);
    return n + 5;
}

int launchCalibration(const DevBatch& B, const MargBatch& M, size_t visualSmem, double* work, const long long* work0, double* cond,
                      double* evals, int maxNuisance, cudaStream_t s) {
    int n = 1;
    k_marg_rotations<<<(B.numKf + B.numExt + 255) / 256, 256, 0, s>>>(B);
    if (M.numElim > 0) {
        const int warps = 8;
        k_marg_eval<<<(M.numElim + warps - 1) / warps, 32 * warps, 0, s>>>(B, M);
        ++n;
    }
    if (M.numItems > 0) {
        k_marg_rows<<<M.numItems, kRowsThreads, (size_t)M.rowsSmem, s>>>(B, M);
        ++n;
    }
    if (M.numSlowElim > 0) {
        k_marg_visual<<<M.numSlowElim, kMargLmThreads, visualSmem, s>>>(B, M);
        ++n;
    }
    k_marg_retained<<<M.numWindows, 256, 0, s>>>(B, M);
    // the packed nuisance block in shared memory when the widest one fits
    long long use = 0;
    int dev = 0, optin = 0;
    cudaFuncAttributes fa;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
        cudaFuncGetAttributes(&fa, k_calib_conditional) == cudaSuccess) {
        const long long want = 8ll * maxNuisance * (maxNuisance + 1) / 2, avail = (long long)optin - (long long)fa.sharedSizeBytes;
        use = want <= avail ? want : 0;
        if (cudaFuncSetAttribute(k_calib_conditional, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)use) != cudaSuccess) use = 0;
    }
    k_calib_conditional<<<M.numWindows, kMargThreads, (size_t)use, s>>>(B, M, work, work0, cond, evals, use);
    return n + 2;
}
void launchDenseEigen(const double* H, int n, double* work, double* evals, double* evecs, int* status, cudaStream_t s) {
    k_dense_eigen<<<1, kMargThreads, 0, s>>>(H, n, work, evals, evecs, status);
}
void launchDensePsd(const double* evals, const double* U, const double* rhs, int n, int columns, double absCut, double relCut,
                    double* projected, double* solution, int* status, cudaStream_t s) {
    const long long count = (long long)n * columns;
    const int blocks = (int)((count + 127) / 128);
    k_dense_psd_project<<<blocks, 128, 0, s>>>(evals, U, rhs, n, columns, absCut, relCut, projected, status);
    k_dense_psd_expand<<<blocks, 128, 0, s>>>(U, projected, n, columns, solution);
}
void launchDenseSubtract(const double* coupling, const double* solution, int nm, int nr, double* Hg, cudaStream_t s) {
    const long long count = (long long)nr * (nr + 1);
    k_dense_subtract<<<(int)((count + 127) / 128), 128, 0, s>>>(coupling, solution, nm, nr, Hg);
}

}  // namespace cgmli
