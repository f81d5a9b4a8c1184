// Batched IMU preintegration on the device: the frozen IMU factor of every
// keyframe interval in one launch, one warp per interval.
//
// Reference (host, one factor at a time):
//   ImuError::redoPreintegration   src/factor/ImuError.cpp:254-462
//   PseudoInverse::symmSqrtU       src/factor/PseudoInverse.hpp:117-145
//   validImuInterval, gyroAt,
//   BodyImuCost construction       src/factor/BodyImuFactor.cpp:10-38,136-166
//
// Work of one interval:
//   1. checks of the sample range (finite readings, increasing times, gaps,
//      bracketing of [t0, t1]) and the first / last integration step, by
//      ballots over the range;
//   2. per chunk of 32 steps, every lane prepares one step independently of the
//      others: its dt (with the interpolated start / end readings of the first
//      and last step), the half-angle rotation increment dq, the right Jacobian
//      of omega*dt, the rotation of dq^-1, the bias-corrected acceleration and the
//      saturation factors;
//   3. the steps of the chunk are applied in order.  The 3x3 state (rotation
//      integrals, cross-term accumulator, bias Jacobians) is spread over lanes
//      0..8, one matrix entry per lane; the quaternion and the vector integrals
//      are kept in every lane.  The 15x15 covariance follows
//      P <- F P F^T + Q with F = I + E, where E is nonzero only in rows 0..8 and
//      columns 3..14, so F P touches rows 0..8 and (F P) F^T columns 0..8:
//      about 2.2k FMAs per step instead of the dense 6.75k per matrix.
//      The reference propagates the four derivatives dP/dsigma_j^2 and forms
//      P = sum_j sigma_j^2 dP_j at the end; by linearity one covariance with the
//      weighted noise sum_j sigma_j^2 K_j per step is the same matrix;
//   4. symmetrize, eigen-decompose by a parallel-ordered two-sided Jacobi (8
//      disjoint rotations per round, round-robin over the 16-padded index set,
//      a rotation skipped when |a_pq| <= 1e-14 sqrt(a_pp a_qq), which keeps the
//      small eigenvalues of the graded covariance accurate relative to
//      themselves), and write W = diag(1/sqrt(lambda)) U^T with eigenvalues in
//      ascending order and those at or below max(eps, 15 eps lambda_max)
//      raised to it.
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cgmli_backend.h"
#include "device_math.cuh"
#include "imu_preintegration.h"

namespace cgmli {
int setLastError(int code, const char* message);
}

namespace {
using namespace cgmli;

constexpr int kImuWarps = 4;     // intervals per CTA
constexpr int kStepFields = 28;  // dt, dq(4), Jr(9), R(dq^-1)(9), acc(3), gyro / acc saturation
constexpr int kJacobiStride = 17;
constexpr int kJacobiMaxSweeps = 40;

struct ImuWarpSmem {
    double P[2][225];                 // covariance, row-major, double buffer
    double T[135];                    // rows 0..8 of F P
    double E[9 * 12];                 // rows 0..8, columns 3..14 of F - I
    double step[kStepFields * 32];    // prepared steps of the chunk [field][lane]; Jacobi A / V afterwards
};
static_assert(2 * 16 * kJacobiStride <= kStepFields * 32, "Jacobi matrices must fit the step area");

enum { kDt = 0, kDq = 1, kJr = 5, kRinv = 14, kAcc = 23, kGsat = 26, kAsat = 27 };

// Duration::toSec of a signed nanosecond count (whole seconds + 1e-9 * remainder)
__device__ __forceinline__ double nsToSec(long long ns) {
    long long sec = ns / 1000000000LL, rem = ns % 1000000000LL;
    if (rem < 0) { rem += 1000000000LL; sec -= 1; }
    return (double)sec + 1e-9 * (double)rem;
}
// ode::sinc (src/factor/ode.hpp:15-27)
__device__ __forceinline__ double odeSinc(double x) {
    if (fabs(x) > 1e-6) return sin(x) / x;
    const double x2 = x * x, x4 = x2 * x2, x6 = x2 * x2 * x2;
    return 1.0 - x2 / 6.0 + x4 / 120.0 - x6 / 5040.0;
}

// The five row (or column) pairs a warp's two half-warps handle together;
// pairs share their E column range.  Pair 4 is row 5 in both halves.
__device__ __forceinline__ int pairRow(int pair, int half) {
    // pairs (0,1) (2,6) (7,8) (3,4) (5,5), one nibble per pair
    return ((half ? 0x54861 : 0x53720) >> (4 * pair)) & 15;
}

__device__ __forceinline__ d3 rowSel(const m3& M, int r) {
    return r == 0 ? mk(M.a[0], M.a[1], M.a[2]) : r == 1 ? mk(M.a[3], M.a[4], M.a[5]) : mk(M.a[6], M.a[7], M.a[8]);
}
__device__ __forceinline__ double compSel(d3 v, int c) { return c == 0 ? v.x : c == 1 ? v.y : v.z; }
// entry (r, c) of the cross-product matrix [v]x
__device__ __forceinline__ double skewSel(d3 v, int r, int c) {
    if (r == c) return 0.0;
    const double vk = compSel(v, 3 - r - c);
    return (r + 1) % 3 == c ? -vk : vk;
}

// Diagonal of sum_j sigma_j^2 K_j (ImuError.cpp:411-421): gs / as are the
// saturation factors of the step.
__device__ __forceinline__ double noiseDiag(int c, double dt, double gs, double as, double sg2, double sa2, double sgw2, double saw2) {
    if (c < 3) return sa2 * (0.5 * dt * dt * dt * as * as * as);
    if (c < 6) return sg2 * (gs * dt);
    if (c < 9) return sa2 * (as * dt);
    if (c < 12) return sgw2 * dt;
    return saw2 * dt;
}
// Pair m (0..7) of Jacobi round r (0..14): round-robin over the indices 0..15
// with 15 fixed; over the 15 rounds every pair p < q meets once.
__device__ __forceinline__ void jacobiPair(int round, int m, int& p, int& q) {
    if (m == 0) { p = round; q = 15; return; }
    const int a = (round + m) % 15, b = (round - m + 15) % 15;
    p = min(a, b);
    q = max(a, b);
}

__global__ void __launch_bounds__(kImuWarps * 32) k_imu_preintegrate(const ImuLaunch L, int count) {
    extern __shared__ __align__(16) unsigned char smemRaw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int iv = blockIdx.x * kImuWarps + warp;
    if (iv >= count) return;
    ImuWarpSmem& S = reinterpret_cast<ImuWarpSmem*>(smemRaw)[warp];
    const unsigned full = 0xffffffffu;
    const cgmli_imu_parameters& prm = L.prm;
    int* status = L.status;

    // linearization bias; a refresh first checks the drift from the factor's reference
    const bool refresh = L.biases == nullptr;
    d3 bg, ba;
    if (!refresh) {
        bg = ld3(L.biases + 6 * iv);
        ba = ld3(L.biases + 6 * iv + 3);
    } else {
        if (L.ranges[2 * iv] == L.ranges[2 * iv + 1]) {  // a factor without samples keeps its value
            if (lane == 0) { status[iv] = CGMLI_OK; L.refreshed[iv] = 0; }
            return;
        }
        const double* x = L.sb + 9ll * L.kf[iv];
        bg = ld3(x + 3);
        ba = ld3(x + 6);
        if (!L.force) {
            const double* ref = L.out[iv].reference_bias;
            const bool drift = norm(bg - ld3(ref)) > L.gyroThreshold || norm(ba - ld3(ref + 3)) > L.accelThreshold;
            if (!drift) {
                if (lane == 0) { status[iv] = CGMLI_OK; L.refreshed[iv] = 0; }
                return;
            }
        }
    }
    const bool viaScratch = refresh && !L.force;

    const int b = L.ranges[2 * iv] - L.sampleOffset, n = L.ranges[2 * iv + 1] - L.ranges[2 * iv];
    const long long* ts = L.times + b;
    const double* rd = L.readings + 6 * (size_t)b;
    const long long t0 = L.t0s[iv], t1 = L.t1s[iv];

    // ---- 1. sample checks (validImuInterval) and step bounds -------------------------
    bool bad = false;
    int nLE0 = 0, nLT0 = 0, nLT1 = 0;
    for (int base = 0; base < n; base += 32) {
        const int j = base + lane;
        bool ok = true, le0 = false, lt0 = false, lt1 = false;
        if (j < n) {
            const long long t = ts[j];
            for (int k = 0; k < 6; ++k) ok = ok && isfinite(rd[6 * j + k]);
            if (j > 0) {
                const long long tp = ts[j - 1];
                ok = ok && t > tp;
                if (tp < t1 && t > t0 && nsToSec(t - tp) > prm.max_sample_gap + 1e-9) ok = false;
            }
            le0 = t <= t0; lt0 = t < t0; lt1 = t < t1;
        }
        bad |= __any_sync(full, !ok);
        nLE0 += __popc(__ballot_sync(full, le0));
        nLT0 += __popc(__ballot_sync(full, lt0));
        nLT1 += __popc(__ballot_sync(full, lt1));
    }
    const bool gapOk = isfinite(prm.max_sample_gap) && prm.max_sample_gap > 0;
    if (bad || !gapOk || n < 2 || t1 <= t0 || ts[0] > t0 || ts[n - 1] < t1) {
        if (lane == 0) {
            status[iv] = CGMLI_E_INVALID;
            if (refresh) L.refreshed[iv] = 0;
        }
        return;
    }
    const int first = nLE0 - 1, last = nLT1 - 1;  // steps (sample pairs) [first, last]

    const double sg2 = prm.sigma_g_c * prm.sigma_g_c, sa2 = prm.sigma_a_c * prm.sigma_a_c;
    const double sgw2 = prm.sigma_gw_c * prm.sigma_gw_c, saw2 = prm.sigma_aw_c * prm.sigma_aw_c;

    for (int e = lane; e < 225; e += 32) S.P[0][e] = 0.0;
    for (int e = lane; e < 9 * 12; e += 32) S.E[e] = 0.0;  // structural zeros stay zero
    int cur = 0;

    // lane-distributed 3x3 state: entry (r, c) of each matrix
    const int el = lane < 9 ? lane : lane % 9, er = el / 3, ec = el % 3;
    double Cint = 0, Cdint = 0, crossAcc = 0, dAlpha = 0, dVel = 0, dPos = 0;
    d3 accInt = mk(0, 0, 0), accDint = mk(0, 0, 0);
    qd Dq = {0, 0, 0, 1};
    m3 C = eye3();

    for (int chunk = first; chunk <= last; chunk += 32) {
        // ---- 2. prepare the chunk's steps, one per lane --------------------------------
        __syncwarp();
        {
            const int it = chunk + lane;
            double* st = S.step;
            if (it <= last) {
                d3 w0 = ld3(rd + 6 * it), a0 = ld3(rd + 6 * it + 3), w1 = ld3(rd + 6 * it + 6), a1 = ld3(rd + 6 * it + 9);
                const long long ti = ts[it], tn = ts[it + 1];
                const long long time = it == first ? t0 : ti;
                long long next = tn;
                double dt = nsToSec(next - time);
                if (t1 < next) {
                    const double interval = nsToSec(next - ti);
                    next = t1;
                    dt = nsToSec(next - time);
                    const double r = dt / interval;
                    w1 = (1.0 - r) * w0 + r * w1;
                    a1 = (1.0 - r) * a0 + r * a1;
                }
                if (it == first) {
                    const double r = dt / nsToSec(next - ti);
                    w0 = r * w0 + (1.0 - r) * w1;
                    a0 = r * a0 + (1.0 - r) * a1;
                }
                const bool gsat = fabs(w0.x) > prm.g_max || fabs(w0.y) > prm.g_max || fabs(w0.z) > prm.g_max ||
                                  fabs(w1.x) > prm.g_max || fabs(w1.y) > prm.g_max || fabs(w1.z) > prm.g_max;
                const bool asat = fabs(a0.x) > prm.a_max || fabs(a0.y) > prm.a_max || fabs(a0.z) > prm.a_max ||
                                  fabs(a1.x) > prm.a_max || fabs(a1.y) > prm.a_max || fabs(a1.z) > prm.a_max;
                const d3 omega = 0.5 * (w0 + w1) - bg;
                const double half = norm(omega) * 0.5 * dt;
                const double sc = odeSinc(half);
                const qd dq = {sc * omega.x * 0.5 * dt, sc * omega.y * 0.5 * dt, sc * omega.z * 0.5 * dt, cos(half)};
                // right Jacobian of phi = omega dt (src/kinematics/Transformation.hpp:47-62)
                const d3 phi = dt * omega;
                const double a = norm(phi);
                const m3 W = skew(phi), W2 = mul(W, W);
                double c1, c2;
                if (a < 1e-4) { c1 = -0.5; c2 = 1.0 / 6.0; }
                else { c1 = -(1.0 - cos(a)) / (a * a); c2 = (a - sin(a)) / (a * a * a); }
                const m3 Jr = madd(eye3(), madd(mscl(c1, W), mscl(c2, W2)));
                const m3 Rinv = qrot(qconj(dq));
                const d3 acc = 0.5 * (a0 + a1) - ba;
                st[kDt * 32 + lane] = dt;
                st[(kDq + 0) * 32 + lane] = dq.x; st[(kDq + 1) * 32 + lane] = dq.y;
                st[(kDq + 2) * 32 + lane] = dq.z; st[(kDq + 3) * 32 + lane] = dq.w;
                for (int k = 0; k < 9; ++k) { st[(kJr + k) * 32 + lane] = Jr.a[k]; st[(kRinv + k) * 32 + lane] = Rinv.a[k]; }
                st[(kAcc + 0) * 32 + lane] = acc.x; st[(kAcc + 1) * 32 + lane] = acc.y; st[(kAcc + 2) * 32 + lane] = acc.z;
                st[kGsat * 32 + lane] = gsat ? 100.0 : 1.0;
                st[kAsat * 32 + lane] = asat ? 100.0 : 1.0;
            }
        }
        __syncwarp();
        const int steps = min(32, last - chunk + 1);
        for (int j = 0; j < steps; ++j) {
            // ---- 3a. the 3x3 state and E (rows 0..8 of F - I) -------------------------
            const double* st = S.step;
            const double dt = st[kDt * 32 + j];
            const qd dq = {st[(kDq + 0) * 32 + j], st[(kDq + 1) * 32 + j], st[(kDq + 2) * 32 + j], st[(kDq + 3) * 32 + j]};
            const d3 acc = mk(st[(kAcc + 0) * 32 + j], st[(kAcc + 1) * 32 + j], st[(kAcc + 2) * 32 + j]);
            const qd Dq1 = qmul(Dq, dq);
            const m3 C1 = qrot(Dq1);
            const m3 CC = madd(C, C1);
            const d3 CCa = mv(CC, acc);
            const double dt2 = dt * dt;
            // this lane's rows of C, C1 (selected, not indexed: keeps them in registers)
            const d3 cRow = rowSel(C, er), c1Row = rowSel(C1, er);
            const double c1El = compSel(c1Row, ec);
            const double ccEl = compSel(cRow, ec) + c1El;
            const double Cint1 = Cint + dt * (0.5 * ccEl);
            const d3 accInt1 = accInt + dt * (0.5 * CCa);
            const double CintOld = Cint;
            Cdint = Cdint + (dt * Cint + dt2 * (0.25 * ccEl));
            const d3 accIntOld = accInt;
            accDint = accDint + (dt * accInt + dt2 * (0.25 * CCa));
            // dalpha/dbg += dt C1 Jr
            double c1jr = 0;
            c1jr += c1Row.x * st[(kJr + ec) * 32 + j];
            c1jr += c1Row.y * st[(kJr + 3 + ec) * 32 + j];
            c1jr += c1Row.z * st[(kJr + 6 + ec) * 32 + j];
            dAlpha += dt * c1jr;
            // cross1 = R(dq^-1) cross + dt Jr
            double crk[3], cr1k[3];
            for (int k = 0; k < 3; ++k) crk[k] = __shfl_sync(full, crossAcc, 3 * k + ec);
            double cross1 = dt * st[(kJr + 3 * er + ec) * 32 + j];
            {
                double s = 0;
                for (int k = 0; k < 3; ++k) s += st[(kRinv + 3 * er + k) * 32 + j] * crk[k];
                cross1 += s;
            }
            for (int k = 0; k < 3; ++k) cr1k[k] = __shfl_sync(full, cross1, 3 * k + ec);
            // row er of C [acc]x and C1 [acc]x
            const double cax[3] = {cRow.y * acc.z - cRow.z * acc.y, cRow.z * acc.x - cRow.x * acc.z, cRow.x * acc.y - cRow.y * acc.x};
            const double c1ax[3] = {c1Row.y * acc.z - c1Row.z * acc.y, c1Row.z * acc.x - c1Row.x * acc.z,
                                    c1Row.x * acc.y - c1Row.y * acc.x};
            double both = 0;
            for (int k = 0; k < 3; ++k) both += cax[k] * crk[k];
            {
                double s = 0;
                for (int k = 0; k < 3; ++k) s += c1ax[k] * cr1k[k];
                both += s;
            }
            const double dVelOld = dVel;
            const double dVel1 = dVel + 0.5 * dt * both;
            dPos = dPos + (dt * dVel + 0.25 * dt2 * both);
            if (lane < 9) {
                // -[v]x entry (r, c): 0 on the diagonal, -v_k / +v_k off it
                const d3 v03 = dt * accIntOld + dt2 * (0.25 * CCa);
                const d3 v63 = dt * (0.5 * CCa);
                double* E = S.E;  // column k stored at k - 3
                E[12 * er + ec] = -skewSel(v03, er, ec);
                E[12 * er + 3 + ec] = er == ec ? dt : 0.0;
                E[12 * er + 6 + ec] = dt * dVelOld + 0.25 * dt2 * both;
                E[12 * er + 9 + ec] = -dt * CintOld + dt2 * (0.25 * ccEl);
                E[12 * (3 + er) + 6 + ec] = -dt * c1El;
                E[12 * (6 + er) + ec] = -skewSel(v63, er, ec);
                E[12 * (6 + er) + 6 + ec] = 0.5 * dt * both;
                E[12 * (6 + er) + 9 + ec] = -dt * (0.5 * ccEl);
            }
            // weighted noise sum_j sigma_j^2 K_j (diagonal)
            const double gs = st[kGsat * 32 + j], as = st[kAsat * 32 + j];
            __syncwarp();
            // ---- 3b. T = F P (rows 0..8) ---------------------------------------------
            // pairs 0..2 read E columns 3..14, pairs 3..4 columns 9..11: fixed trip
            // counts, so every shared load has an immediate offset
            const double* P = S.P[cur];
            double* Pn = S.P[cur ^ 1];
            {
                const int half = lane >> 4, c = lane & 15;
                if (c < 15) {
                    const double* Pc = P + c;
#pragma unroll
                    for (int pr = 0; pr < 3; ++pr) {
                        const int r = pairRow(pr, half);
                        const double* Er = S.E + 12 * r;
                        double s = Pc[15 * r];
#pragma unroll
                        for (int k = 3; k < 15; ++k) s += Er[k - 3] * Pc[15 * k];
                        S.T[15 * r + c] = s;
                    }
#pragma unroll
                    for (int pr = 3; pr < 5; ++pr) {
                        const int r = pairRow(pr, half);
                        const double* Er = S.E + 12 * r;
                        double s = Pc[15 * r];
#pragma unroll
                        for (int k = 9; k < 12; ++k) s += Er[k - 3] * Pc[15 * k];
                        S.T[15 * r + c] = s;
                    }
                }
            }
            __syncwarp();
            // ---- 3c. N = T F^T + Q: columns 0..8 through E, columns 9..14 copied -------
            {
                const int half = lane >> 4, r = lane & 15;
                if (r < 15) {
                    const double* Tr = r < 9 ? S.T + 15 * r : P + 15 * r;  // rows 9..14 of F P are those of P
#pragma unroll
                    for (int pc = 0; pc < 3; ++pc) {
                        const int c = pairRow(pc, half);
                        const double* Ec = S.E + 12 * c;
                        double s = Tr[c];
#pragma unroll
                        for (int k = 3; k < 15; ++k) s += Ec[k - 3] * Tr[k];
                        if (r == c) s += noiseDiag(c, dt, gs, as, sg2, sa2, sgw2, saw2);
                        Pn[15 * r + c] = s;
                    }
#pragma unroll
                    for (int pc = 3; pc < 5; ++pc) {
                        const int c = pairRow(pc, half);
                        const double* Ec = S.E + 12 * c;
                        double s = Tr[c];
#pragma unroll
                        for (int k = 9; k < 12; ++k) s += Ec[k - 3] * Tr[k];
                        if (r == c) s += noiseDiag(c, dt, gs, as, sg2, sa2, sgw2, saw2);
                        Pn[15 * r + c] = s;
                    }
                }
                for (int e = lane; e < 90; e += 32) {
                    const int rr = e / 6, cc = 9 + e % 6;
                    double v = rr < 9 ? S.T[15 * rr + cc] : P[15 * rr + cc];
                    if (rr == cc) v += noiseDiag(cc, dt, gs, as, sg2, sa2, sgw2, saw2);
                    Pn[15 * rr + cc] = v;
                }
            }
            __syncwarp();
            cur ^= 1;
            // state shift
            Dq = Dq1; C = C1; Cint = Cint1; accInt = accInt1; crossAcc = cross1; dVel = dVel1;
        }
    }

    // ---- 4. symmetrize, Jacobi eigen-decomposition, whitening ---------------------------
    __syncwarp();
    double* A = S.step;                       // 16 x 16, row stride 17 (conflict-free columns)
    double* V = S.step + 16 * kJacobiStride;  // eigenvectors as columns
    {
        const double* P = S.P[cur];
        for (int e = lane; e < 256; e += 32) {
            const int r = e >> 4, c = e & 15;
            A[kJacobiStride * r + c] = (r < 15 && c < 15) ? 0.5 * P[15 * r + c] + 0.5 * P[15 * c + r] : 0.0;
            V[kJacobiStride * r + c] = r == c ? 1.0 : 0.0;
        }
    }
    __syncwarp();
    for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
        bool rotated = false;
        for (int round = 0; round < 15; ++round) {
            double c = 1.0, s = 0.0;
            bool rot = false;
            if (lane < 8) {
                int p, q;
                jacobiPair(round, lane, p, q);
                const double apq = A[kJacobiStride * p + q];
                const double app = A[kJacobiStride * p + p], aqq = A[kJacobiStride * q + q];
                if (apq != 0.0 && fabs(apq) > 1e-14 * sqrt(fabs(app * aqq))) {
                    const double tau = (aqq - app) / (2.0 * apq);
                    const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                    c = 1.0 / sqrt(1.0 + t * t);
                    s = t * c;
                    rot = true;
                }
            }
            rotated |= __any_sync(full, rot);
            // A <- A J and V <- V J (columns p, q of every pair), then A <- J^T A (rows)
            double cs[4], sn[4];
            int pp[4], qq[4], kk[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int task = lane + 32 * i, m = task >> 4;
                cs[i] = __shfl_sync(full, c, m);
                sn[i] = __shfl_sync(full, s, m);
                jacobiPair(round, m, pp[i], qq[i]);
                kk[i] = task & 15;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (sn[i] == 0.0) continue;
                const int k = kk[i];
                double* ak = A + kJacobiStride * k;
                const double akp = ak[pp[i]], akq = ak[qq[i]];
                ak[pp[i]] = cs[i] * akp - sn[i] * akq;
                ak[qq[i]] = sn[i] * akp + cs[i] * akq;
                double* vk = V + kJacobiStride * k;
                const double vkp = vk[pp[i]], vkq = vk[qq[i]];
                vk[pp[i]] = cs[i] * vkp - sn[i] * vkq;
                vk[qq[i]] = sn[i] * vkp + cs[i] * vkq;
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (sn[i] == 0.0) continue;
                const int k = kk[i];
                double* ap = A + kJacobiStride * pp[i];
                double* aq = A + kJacobiStride * qq[i];
                const double apk = ap[k], aqk = aq[k];
                ap[k] = cs[i] * apk - sn[i] * aqk;
                aq[k] = sn[i] * apk + cs[i] * aqk;
            }
            __syncwarp();
        }
        if (!rotated) break;
    }

    cgmli_frozen_imu& o = viaScratch ? L.scratch[iv] : L.out[iv];
    bool finiteOut = true;
    {
        double lmax = A[0];
        for (int i = 1; i < 15; ++i) lmax = fmax(lmax, A[kJacobiStride * i + i]);
        const double tol = fmax(DBL_EPSILON, DBL_EPSILON * 15 * lmax);
        if (lane < 15) {
            const double li = A[kJacobiStride * lane + lane];
            int rank = 0;
            for (int j = 0; j < 15; ++j) {
                const double lj = A[kJacobiStride * j + j];
                rank += (lj < li || (lj == li && j < lane)) ? 1 : 0;
            }
            const double sc = sqrt(li > tol ? 1.0 / li : 1.0 / tol);
            for (int c = 0; c < 15; ++c) {
                const double w = sc * V[kJacobiStride * c + lane];
                o.whitening[rank + 15 * c] = w;
                finiteOut = finiteOut && isfinite(w);
            }
        }
    }
    if (lane < 9) {
        const int cm = er + 3 * ec;  // column-major
        o.rotation_gyro[cm] = dAlpha;
        o.velocity_gyro[cm] = dVel;
        o.position_gyro[cm] = dPos;
        o.velocity_accel[cm] = Cint;
        o.position_accel[cm] = Cdint;
        finiteOut = finiteOut && isfinite(dAlpha) && isfinite(dVel) && isfinite(dPos) && isfinite(Cint) && isfinite(Cdint);
    }
    if (lane == 0) {
        o.duration = nsToSec(t1 - t0);
        o.gravity = prm.g;
        o.delta_quaternion[0] = Dq.x; o.delta_quaternion[1] = Dq.y; o.delta_quaternion[2] = Dq.z; o.delta_quaternion[3] = Dq.w;
        o.delta_velocity[0] = accInt.x; o.delta_velocity[1] = accInt.y; o.delta_velocity[2] = accInt.z;
        o.delta_position[0] = accDint.x; o.delta_position[1] = accDint.y; o.delta_position[2] = accDint.z;
        for (int k = 0; k < 3; ++k) o.sensor_position[k] = prm.sensor_position[k];
        for (int k = 0; k < 4; ++k) o.sensor_quaternion[k] = prm.sensor_quaternion[k];
        finiteOut = finiteOut && isfinite(qn2(Dq)) && finite3(accInt) && finite3(accDint);
    }
    if (lane < 6) o.reference_bias[lane] = lane < 3 ? compSel(bg, lane) : compSel(ba, lane - 3);
    if (lane < 6) {
        // gyroAt (src/factor/BodyImuFactor.cpp:29-38) at t0 (lanes 0..2) and t1 (lanes 3..5)
        const int end = lane / 3, axis = lane % 3;
        const int k = end ? nLT1 : nLT0;  // first sample not before the epoch
        const long long epoch = end ? t1 : t0;
        double g;
        if (k == 0) g = rd[axis];
        else if (k == n) g = rd[6 * (n - 1) + axis];
        else {
            const double alpha = nsToSec(epoch - ts[k - 1]) / nsToSec(ts[k] - ts[k - 1]);
            g = (1 - alpha) * rd[6 * (k - 1) + axis] + alpha * rd[6 * k + axis];
        }
        o.gyros[3 * end + axis] = g;
        finiteOut = finiteOut && isfinite(g);
    }
    const bool anyBad = __any_sync(full, !finiteOut);
    if (viaScratch) {
        // replace the factor only with a finite result
        __syncwarp();
        if (!anyBad) {
            const double* src = reinterpret_cast<const double*>(&L.scratch[iv]);
            double* dst = reinterpret_cast<double*>(&L.out[iv]);
            for (int k = lane; k < (int)(sizeof(cgmli_frozen_imu) / sizeof(double)); k += 32) dst[k] = src[k];
        }
        if (lane == 0) L.refreshed[iv] = anyBad ? 0 : 1;
    } else if (refresh && lane == 0) {
        L.refreshed[iv] = anyBad ? 0 : 1;
    }
    if (lane == 0) status[iv] = anyBad ? CGMLI_E_NONFINITE : CGMLI_OK;
}

// ---- host side ------------------------------------------------------------------------
template <class T>
struct GrowBuffer {
    T* p = nullptr;
    size_t cap = 0;
    cudaError_t reserve(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(std::max(n, cap + cap / 2), 1);
        const cudaError_t e = cudaMalloc(&p, want * sizeof(T));
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

struct ImuWorkspace {
    std::mutex mu;
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double lastKernelMs = 0;
    GrowBuffer<long long> times, t0, t1;
    GrowBuffer<double> readings, bias;
    GrowBuffer<int> ranges, status;
    GrowBuffer<cgmli_frozen_imu> out;
    std::vector<int> hostStatus;
} g_imu;

size_t imuSmemBytes() { return sizeof(ImuWarpSmem) * kImuWarps; }

int cudaFailure(cudaError_t e, const char* what) {
    return setLastError(CGMLI_E_CUDA, (std::string("imu_preintegrate: ") + what + ": " + cudaGetErrorString(e)).c_str());
}
}  // namespace

namespace cgmli {
// Launches the preintegration of count intervals whose arrays are already on the device.
cudaError_t launchImuPreintegration(const ImuLaunch& L, int count, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    // the shared-memory attribute is set once per device; callers on several
    // threads (the solver path and cgmli_imu_preintegrate) may race to do it
    static std::atomic<int> configured[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !configured[dev].load(std::memory_order_acquire)) {
        e = cudaFuncSetAttribute(k_imu_preintegrate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)imuSmemBytes());
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) configured[dev].store(1, std::memory_order_release);
    }
    const int blocks = (count + kImuWarps - 1) / kImuWarps;
    k_imu_preintegrate<<<blocks, kImuWarps * 32, imuSmemBytes(), s>>>(L, count);
    return cudaGetLastError();
}
}  // namespace cgmli

extern "C" {

int cgmli_imu_preintegrate(const cgmli_imu_parameters* params, const long long* sample_time_ns, const double* sample_readings,
                           int num_samples, const int* range, const long long* t0_ns, const long long* t1_ns, const double* bias,
                           int count, cgmli_frozen_imu* frozen) {
    if (!params || count < 0) return setLastError(CGMLI_E_INVALID, "imu_preintegrate: null parameters or negative count");
    if (count == 0) return CGMLI_OK;
    if (!sample_time_ns || !sample_readings || !range || !t0_ns || !t1_ns || !bias || !frozen || num_samples < 2)
        return setLastError(CGMLI_E_INVALID, "imu_preintegrate: null buffers or fewer than 2 samples");
    int lo = num_samples, hi = 0;
    for (int i = 0; i < count; ++i) {
        const int b = range[2 * i], e = range[2 * i + 1];
        if (b < 0 || e > num_samples || e - b < 2) {
            const std::string msg = "imu_preintegrate: interval " + std::to_string(i) + ": sample range [" + std::to_string(b) + ", " +
                                    std::to_string(e) + ") outside the samples or shorter than 2";
            return setLastError(CGMLI_E_INVALID, msg.c_str());
        }
        lo = std::min(lo, b);
        hi = std::max(hi, e);
    }
    std::lock_guard<std::mutex> lock(g_imu.mu);
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return cudaFailure(ce, "cudaGetDevice");
    if (g_imu.device != dev) {
        if (g_imu.device >= 0) {
            // buffers, stream and events of the previous device: released with that device current
            if ((ce = cudaSetDevice(g_imu.device)) != cudaSuccess) return cudaFailure(ce, "cudaSetDevice (previous device)");
            if (g_imu.stream) cudaStreamSynchronize(g_imu.stream);
            g_imu.times.release(); g_imu.t0.release(); g_imu.t1.release(); g_imu.readings.release(); g_imu.bias.release();
            g_imu.ranges.release(); g_imu.status.release(); g_imu.out.release();
            if (g_imu.stream) cudaStreamDestroy(g_imu.stream);
            if (g_imu.ev0) cudaEventDestroy(g_imu.ev0);
            if (g_imu.ev1) cudaEventDestroy(g_imu.ev1);
            g_imu.stream = nullptr;
            g_imu.ev0 = g_imu.ev1 = nullptr;
            g_imu.device = -1;
            if ((ce = cudaSetDevice(dev)) != cudaSuccess) return cudaFailure(ce, "cudaSetDevice");
        }
        if ((ce = cudaStreamCreateWithFlags(&g_imu.stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cudaFailure(ce, "cudaStreamCreate");
        if ((ce = cudaEventCreate(&g_imu.ev0)) != cudaSuccess || (ce = cudaEventCreate(&g_imu.ev1)) != cudaSuccess)
            return cudaFailure(ce, "cudaEventCreate");
        g_imu.device = dev;
    }
    const size_t span = (size_t)(hi - lo);
    cudaStream_t s = g_imu.stream;
#define IMU_CK(call)                                              \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cudaFailure(e_, #call);    \
    } while (0)
    IMU_CK(g_imu.times.reserve(span));
    IMU_CK(g_imu.readings.reserve(6 * span));
    IMU_CK(g_imu.ranges.reserve(2 * (size_t)count));
    IMU_CK(g_imu.t0.reserve(count));
    IMU_CK(g_imu.t1.reserve(count));
    IMU_CK(g_imu.bias.reserve(6 * (size_t)count));
    IMU_CK(g_imu.out.reserve(count));
    IMU_CK(g_imu.status.reserve(count));
    IMU_CK(cudaMemcpyAsync(g_imu.times.p, sample_time_ns + lo, span * sizeof(long long), cudaMemcpyHostToDevice, s));
    IMU_CK(cudaMemcpyAsync(g_imu.readings.p, sample_readings + 6 * (size_t)lo, 6 * span * sizeof(double), cudaMemcpyHostToDevice, s));
    IMU_CK(cudaMemcpyAsync(g_imu.ranges.p, range, 2 * (size_t)count * sizeof(int), cudaMemcpyHostToDevice, s));
    IMU_CK(cudaMemcpyAsync(g_imu.t0.p, t0_ns, count * sizeof(long long), cudaMemcpyHostToDevice, s));
    IMU_CK(cudaMemcpyAsync(g_imu.t1.p, t1_ns, count * sizeof(long long), cudaMemcpyHostToDevice, s));
    IMU_CK(cudaMemcpyAsync(g_imu.bias.p, bias, 6 * (size_t)count * sizeof(double), cudaMemcpyHostToDevice, s));
    IMU_CK(cudaEventRecord(g_imu.ev0, s));
    ImuLaunch L{};
    L.prm = *params;
    L.times = g_imu.times.p; L.readings = g_imu.readings.p; L.sampleOffset = lo;
    L.ranges = g_imu.ranges.p; L.t0s = g_imu.t0.p; L.t1s = g_imu.t1.p;
    L.out = g_imu.out.p; L.status = g_imu.status.p; L.biases = g_imu.bias.p;
    IMU_CK(launchImuPreintegration(L, count, s));
    IMU_CK(cudaEventRecord(g_imu.ev1, s));
    g_imu.hostStatus.resize(count);
    IMU_CK(cudaMemcpyAsync(frozen, g_imu.out.p, count * sizeof(cgmli_frozen_imu), cudaMemcpyDeviceToHost, s));
    IMU_CK(cudaMemcpyAsync(g_imu.hostStatus.data(), g_imu.status.p, count * sizeof(int), cudaMemcpyDeviceToHost, s));
    IMU_CK(cudaStreamSynchronize(s));
    float kernelMs = 0;
    IMU_CK(cudaEventElapsedTime(&kernelMs, g_imu.ev0, g_imu.ev1));
#undef IMU_CK
    for (int i = 0; i < count; ++i) {
        const int st = g_imu.hostStatus[i];
        if (st == CGMLI_OK) continue;
        const std::string what = st == CGMLI_E_INVALID
                                     ? ": samples not finite, not increasing, gapped beyond max_sample_gap or not bracketing [t0, t1]"
                                     : ": result not finite";
        return setLastError(st, ("imu_preintegrate: interval " + std::to_string(i) + what).c_str());
    }
    g_imu.lastKernelMs = kernelMs;
    return CGMLI_OK;
}

int cgmli_imu_last_timing(double* kernel_ms) {
    if (!kernel_ms) return setLastError(CGMLI_E_INVALID, "imu_last_timing: null pointer");
    std::lock_guard<std::mutex> lock(g_imu.mu);
    *kernel_ms = g_imu.lastKernelMs;
    return CGMLI_OK;
}

}  // extern "C"
