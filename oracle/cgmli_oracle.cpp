// FP64 CPU ORACLE of the CGMLI-SLAM sliding-window backend hot path.
//
// TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
// baseline arm of bench.py load this library, and only to check or time the
// CUDA path; the product never links or calls it.
//
// It restates, in plain C++17 with no Eigen/Ceres (neither exists here), the
// reference's algorithm for the path:
//   * S^2 inverse-distance bearing factor  src/backend/VisualSphereBatchMath.hpp:29-174,
//     src/backend/WindowVisualFactor.cpp:411-577 (analytic) and :411-430,578-611 (numeric)
//   * frozen IMU factor                     src/backend/GpuRetainedFactorMath.hpp:14-140
//   * marginalization prior factor          src/backend/MarginalizationPrior.cpp:20-66,
//                                           src/backend/VisualCudaBatch.cu:216-268
//   * Huber weight and cost                 src/backend/VisualCudaBatch.cu:54-59,125-136
//   * Schur step at fixed lambda            src/backend/VisualCudaBatch.cu:138-205,530-604
//   * resident LM loop                      src/backend/BackendOptimizer.cpp:167-307,
//                                           src/backend/VisualCudaBatch.cu:291-340
//   * marginalization                       src/backend/Marginalizer.cpp:240-474,
//                                           src/backend/SlidingWindowManager.cpp:627-652
//   * IMU preintegration                    src/factor/ImuError.cpp:254-462,
//                                           src/factor/BodyImuFactor.cpp:10-38,136-166,
//                                           src/factor/PseudoInverse.hpp:117-145
// Parity is pinned by the reference's own known-answer tests
// (src/backend/tests/ManagedWindowRegression.cpp:119-329), restated in tests/.
#include "../include/cgmli_backend.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>

namespace orc {
using V3 = std::array<double, 3>;
using M3 = std::array<double, 9>;  // row-major
struct Q { double x, y, z, w; };   // Eigen coefficient order

static inline V3 add(const V3& a, const V3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
static inline V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
static inline V3 scl(double s, const V3& a) { return {s * a[0], s * a[1], s * a[2]}; }
static inline double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline double nrm(const V3& a) { return std::sqrt(dot(a, a)); }
static inline V3 cross(const V3& a, const V3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
static inline V3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
static inline M3 eye() { return {1, 0, 0, 0, 1, 0, 0, 0, 1}; }
static inline M3 skew(const V3& v) { return {0, -v[2], v[1], v[2], 0, -v[0], -v[1], v[0], 0}; }
static inline M3 mul(const M3& a, const M3& b) {
    M3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
    return r;
}
static inline V3 mv(const M3& a, const V3& v) {
    return {a[0] * v[0] + a[1] * v[1] + a[2] * v[2], a[3] * v[0] + a[4] * v[1] + a[5] * v[2],
            a[6] * v[0] + a[7] * v[1] + a[8] * v[2]};
}
static inline M3 tr(const M3& a) { return {a[0], a[3], a[6], a[1], a[4], a[7], a[2], a[5], a[8]}; }
static inline M3 madd(const M3& a, const M3& b) { M3 r; for (int i = 0; i < 9; ++i) r[i] = a[i] + b[i]; return r; }
static inline M3 msub(const M3& a, const M3& b) { M3 r; for (int i = 0; i < 9; ++i) r[i] = a[i] - b[i]; return r; }
static inline M3 mscl(double s, const M3& a) { M3 r; for (int i = 0; i < 9; ++i) r[i] = s * a[i]; return r; }
static inline M3 outer(const V3& a, const V3& b) {
    return {a[0] * b[0], a[0] * b[1], a[0] * b[2], a[1] * b[0], a[1] * b[1], a[1] * b[2], a[2] * b[0], a[2] * b[1], a[2] * b[2]};
}
static inline M3 colmajor(const double* p) { return {p[0], p[3], p[6], p[1], p[4], p[7], p[2], p[5], p[8]}; }

static inline Q qload(const double* p) { return {p[0], p[1], p[2], p[3]}; }
static inline double qnorm2(const Q& q) { return q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w; }
static inline Q qnormalized(const Q& q) { double n = std::sqrt(qnorm2(q)); return {q.x / n, q.y / n, q.z / n, q.w / n}; }
static inline Q qconj(const Q& q) { return {-q.x, -q.y, -q.z, q.w}; }
static inline Q qmul(const Q& a, const Q& b) {
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
            a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
static inline V3 qvec(const Q& q) { return {q.x, q.y, q.z}; }
static inline M3 qrot(const Q& q) {  // rotation matrix of a (unit) quaternion
    const double tx = 2 * q.x, ty = 2 * q.y, tz = 2 * q.z, twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
    const double txx = tx * q.x, txy = ty * q.x, txz = tz * q.x, tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
    return {1 - (tyy + tzz), txy - twz, txz + twy, txy + twz, 1 - (txx + tzz), tyz - twx, txz - twy, tyz + twx, 1 - (txx + tyy)};
}
static inline V3 qapply(const Q& q, const V3& v) {  // q * v for a unit quaternion
    V3 uv = cross(qvec(q), v);
    uv = scl(2, uv);
    return add(add(v, scl(q.w, uv)), cross(qvec(q), uv));
}
static inline bool fin(double v) { return std::isfinite(v); }
static inline bool fin3(const V3& v) { return fin(v[0]) && fin(v[1]) && fin(v[2]); }

// ---- left SE(3) chart of the resident device path (GpuRetainedFactorMath.hpp:14-51)
static Q rotationExp(const V3& angle) {
    const double a = nrm(angle);
    const double s = a < 1e-8 ? 0.5 - a * a / 48.0 : std::sin(0.5 * a) / a;
    return {s * angle[0], s * angle[1], s * angle[2], std::cos(0.5 * a)};
}
static M3 rotationJacobian(const V3& angle) {
    const double a2 = dot(angle, angle), a = std::sqrt(a2);
    const M3 w = skew(angle);
    const double c1 = a2 < 1e-10 ? 0.5 - a2 / 24 : (1 - std::cos(a)) / a2;
    const double c2 = a2 < 1e-10 ? 1.0 / 6 - a2 / 120 : (a - std::sin(a)) / (a2 * a);
    return madd(madd(eye(), mscl(c1, w)), mscl(c2, mul(w, w)));
}
static void posePlus(const double* x, const double* d, double* y, bool rotationOnly = false) {
    const V3 angle = ld3(d + (rotationOnly ? 0 : 3));
    const Q q = rotationExp(angle);
    V3 p = ld3(x);
    if (!rotationOnly) p = add(qapply(q, p), mv(rotationJacobian(angle), ld3(d)));
    const Q out = qnormalized(qmul(q, qload(x + 3)));
    y[0] = p[0]; y[1] = p[1]; y[2] = p[2];
    y[3] = out.x; y[4] = out.y; y[5] = out.z; y[6] = out.w;
}
static void poseMinus(const double* x, const double* ref, double* d) {
    Q q = qnormalized(qmul(qload(x + 3), qconj(qload(ref + 3))));
    if (q.w < 0) q = {-q.x, -q.y, -q.z, -q.w};
    const double s = nrm(qvec(q));
    const V3 theta = scl(s < 1e-10 ? 2.0 : 2.0 * std::atan2(s, q.w) / s, qvec(q));
    const double a2 = dot(theta, theta), a = std::sqrt(a2);
    const M3 w = skew(theta);
    const double c = a2 < 1e-10 ? 1.0 / 12 + a2 / 720 : (1 - 0.5 * a / std::tan(0.5 * a)) / a2;
    const V3 p = mv(madd(msub(eye(), mscl(0.5, w)), mscl(c, mul(w, w))), sub(ld3(x), qapply(q, ld3(ref))));
    d[0] = p[0]; d[1] = p[1]; d[2] = p[2]; d[3] = theta[0]; d[4] = theta[1]; d[5] = theta[2];
}
// Inverse of the SE(3) left Jacobian at xi = [rho, theta]: derivative of
// poseMinus(Exp(delta)*x, ref) with respect to delta at delta = 0.  The
// reference differentiates the same map by central differences with h = 1e-7
// (VisualCudaBatch.cu:234-245); the analytic form uses the published SE(3)
// Jacobian (Barfoot, State Estimation for Robotics, 2017, eqs. 7.85-7.86).
static void se3LeftJacobianInverse(const double* xi, double* D /*6x6 row-major*/) {
    const V3 rho = ld3(xi), th = ld3(xi + 3);
    const double t2 = dot(th, th), t = std::sqrt(t2);
    const M3 W = skew(th), R = skew(rho), WW = mul(W, W);
    double c1, c2, c3, cj;
    if (t < 0.1) {
        c1 = 1.0 / 6 - t2 / 120 + t2 * t2 / 5040 - t2 * t2 * t2 / 362880;
        c2 = 1.0 / 24 - t2 / 720 + t2 * t2 / 40320 - t2 * t2 * t2 / 3628800;
        c3 = 0.5 * (c2 - 3 * (1.0 / 120 - t2 / 5040 + t2 * t2 / 362880 - t2 * t2 * t2 / 39916800));
    } else {
        const double s = std::sin(t), c = std::cos(t);
        c1 = (t - s) / (t2 * t);
        c2 = (t2 / 2 + c - 1) / (t2 * t2);
        c3 = 0.5 * (c2 + 3 * (t - s - t2 * t / 6) / (t2 * t2 * t));
    }
    cj = t2 < 1e-10 ? 1.0 / 12 + t2 / 720 : (1 - 0.5 * t / std::tan(0.5 * t)) / t2;
    const M3 WR = mul(W, R), RW = mul(R, W), WRW = mul(WR, W);
    M3 Qm = mscl(0.5, R);
    Qm = madd(Qm, mscl(c1, madd(madd(WR, RW), WRW)));
    Qm = madd(Qm, mscl(c2, msub(madd(mul(WW, R), mul(R, WW)), mscl(3, WRW))));
    Qm = madd(Qm, mscl(c3, madd(mul(WRW, W), mul(W, WRW))));
    const M3 Ji = madd(msub(eye(), mscl(0.5, W)), mscl(cj, WW));
    const M3 top = mscl(-1, mul(mul(Ji, Qm), Ji));
    for (int i = 0; i < 36; ++i) D[i] = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            D[6 * i + j] = Ji[3 * i + j];
            D[6 * i + 3 + j] = top[3 * i + j];
            D[6 * (i + 3) + 3 + j] = Ji[3 * i + j];
        }
}
// Reference chart derivative (VisualCudaBatch.cu:234-245): central differences, h = 1e-7.
static void chartDerivativeFD(const double* x, const double* ref, double* D) {
    constexpr double h = 1e-7;
    double step[6]{}, plus[7], minus[7], dp[6], dm[6];
    for (int c = 0; c < 6; ++c) {
        step[c] = h; posePlus(x, step, plus);
        step[c] = -h; posePlus(x, step, minus);
        step[c] = 0;
        poseMinus(plus, ref, dp); poseMinus(minus, ref, dm);
        for (int r = 0; r < 6; ++r) D[6 * r + c] = (dp[r] - dm[r]) / (2 * h);
    }
}

// ---- window layout -------------------------------------------------------
struct Layout {
    int K, E, L, Nr, ext0, tdc;
    bool estExt, estTd;
    explicit Layout(const cgmli_window& w)
        : K(w.num_keyframes), E(w.num_extrinsics), L(w.num_landmarks), estExt(w.estimate_extrinsics != 0),
          estTd(w.estimate_td != 0 && w.td) {
        ext0 = 15 * K;
        tdc = ext0 + (estExt ? 6 * E : 0);
        Nr = tdc + (estTd ? 1 : 0);
    }
    int pose(int k) const { return 15 * k; }
    int sb(int k) const { return 15 * k + 6; }
    int ext(int e) const { return estExt ? ext0 + 6 * e : -1; }
    int td() const { return estTd ? tdc : -1; }
};

// ---- S^2 bearing factor ----------------------------------------------------
struct Fac {
    double r[2];
    double Ja[12], Jb[12], Jea[12], Jeb[12], Jtd[2], Jrho[2];  // 2x6 row-major tangent blocks
    int a, b, ea, eb;
    bool same;   // same-epoch with a shared extrinsic: pose/extrinsic columns exactly zero
    bool split;  // anchor and observer cameras use different extrinsic blocks
};

// timeBearing of VisualSphereBatchMath.hpp:29-49
static V3 timeBearing(const double* raw, const double* vel, double dt, bool differentiate, V3& derivative) {
    const V3 bearing = ld3(raw), v = ld3(vel);
    if (!differentiate) {
        const V3 u = scl(dt, v);
        const double angle = nrm(u);
        if (angle < 1e-8) { V3 s = add(bearing, u); return scl(1 / nrm(s), s); }
        return add(scl(std::cos(angle), bearing), scl(std::sin(angle) / angle, u));
    }
    const double speed = nrm(v), angle = speed * dt;
    if (std::fabs(angle) < 1e-8) {
        const V3 direction = add(bearing, scl(dt, v));
        const double length = nrm(direction);
        const V3 unit = scl(1 / length, direction);
        derivative = scl(-1 / length, mv(msub(eye(), outer(unit, unit)), v));
        return unit;
    }
    const double sine = std::sin(angle), cosine = std::cos(angle);
    derivative = sub(scl(speed * sine, bearing), scl(cosine, v));
    return add(scl(cosine, bearing), scl(sine / speed, v));
}

static bool validPose(const double* x) {
    for (int i = 0; i < 7; ++i) if (!fin(x[i])) return false;
    return x[3] * x[3] + x[4] * x[4] + x[5] * x[5] + x[6] * x[6] > 1e-16;
}

// writePose + PlusJacobian lift of the reference (VisualSphereBatchMath.hpp:51-63,
// LeftSE3Manifold.cpp:288-298, VisualCudaBatch.cu:60-71): ambient 2x7, then 2x6 tangent.
static bool liftPose(const double* x, const double tr2[6], const double rot2[6], double* J) {
    const Q q = qload(x + 3);
    if (!(fin(q.x) && fin(q.y) && fin(q.z) && fin(q.w)) || std::fabs(qnorm2(q) - 1) > 1e-6) return false;
    double lift[12];  // 3x4
    const M3 top = mscl(2, madd(mscl(q.w, eye()), skew(qvec(q))));
    for (int r = 0; r < 3; ++r) { for (int c = 0; c < 3; ++c) lift[4 * r + c] = top[3 * r + c]; }
    lift[3] = -2 * q.x; lift[7] = -2 * q.y; lift[11] = -2 * q.z;
    double amb[14];
    for (int r = 0; r < 2; ++r) {
        for (int c = 0; c < 3; ++c) amb[7 * r + c] = tr2[3 * r + c];
        for (int c = 0; c < 4; ++c) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += rot2[3 * r + k] * lift[4 * k + c];
            amb[7 * r + 3 + c] = s;
        }
    }
    double plus[42] = {0};  // 7x6
    plus[0] = plus[7] = plus[14] = 1;
    const M3 ms = skew(ld3(x));
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) plus[6 * r + 3 + c] = -ms[3 * r + c];
    const M3 ql = mscl(0.5, msub(mscl(q.w, eye()), skew(qvec(q))));
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) plus[6 * (3 + r) + 3 + c] = ql[3 * r + c];
    plus[6 * 6 + 3] = -0.5 * q.x; plus[6 * 6 + 4] = -0.5 * q.y; plus[6 * 6 + 5] = -0.5 * q.z;
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 6; ++c) {
            double s = 0;
            for (int k = 0; k < 7; ++k) s += amb[7 * r + k] * plus[6 * k + c];
            J[6 * r + c] = s;
        }
    for (int i = 0; i < 12; ++i) if (!fin(J[i])) return false;
    return true;
}
static void mul23x33(const double* A, const M3& B, double* out) {  // (2x3)(3x3)
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c) out[3 * r + c] = A[3 * r] * B[c] + A[3 * r + 1] * B[3 + c] + A[3 * r + 2] * B[6 + c];
}
static void tangentDirect(const double* D, const M3& Rt, const V3& lever, double sign, double* J) {
    // J = sign*[D*Rt, -D*Rt*skew(lever)] (2x6)
    double DR[6], DRs[6];
    mul23x33(D, Rt, DR);
    mul23x33(DR, skew(lever), DRs);
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c) { J[6 * r + c] = sign * DR[3 * r + c]; J[6 * r + 3 + c] = -sign * DRs[3 * r + c]; }
}

// Analytic factor: sphere_batch::evaluate (VisualSphereBatchMath.hpp:67-174) with
// the tangent lift of projectVisualRows (VisualCudaBatch.cu:60-71).
static bool visualFactor(const cgmli_window& w, int l, int f, bool derivatives, Fac& o, bool forceCalib = false) {
    const Layout lay(w);
    // Marginalization differentiates frozen calibration blocks too
    // (BackendProblem.hpp:75-80 with honorConstant=false).
    const bool extDerivative = lay.estExt || forceCalib;
    const int a = w.lm_anchor_kf[l], b = w.obs_kf[f], ca = w.lm_anchor_cam[l], cb = w.obs_cam[f];
    const int ea = w.cam_ext[ca], eb = w.cam_ext[cb];
    o.a = a; o.b = b; o.ea = ea; o.eb = eb;
    o.split = ea != eb;
    o.same = (a == b) && !o.split;
    const double rho = w.rho[l];
    const double anchorTime = w.lm_anchor_time ? w.lm_anchor_time[l] : 0.0;
    const double measuredTime = w.obs_time ? w.obs_time[f] : 0.0;
    const double td = w.td ? *w.td : anchorTime;
    if (!(rho > 0) || !fin(rho) || !fin(td)) return false;
    const double* xa = w.poses + 7 * a;
    const double* xb = w.poses + 7 * b;
    const double* xea = w.extrinsics + 7 * ea;
    const double* xeb = w.extrinsics + 7 * eb;
    if (!validPose(xa) || !validPose(xb) || !validPose(xea) || !validPose(xeb)) return false;
    const bool timeDerivative = derivatives && (lay.estTd || (forceCalib && w.td));
    static const double zero3[3] = {0, 0, 0};
    const double* va = w.lm_anchor_velocity ? w.lm_anchor_velocity + 3 * l : zero3;
    const double* vb = w.obs_velocity ? w.obs_velocity + 3 * f : zero3;
    const bool movingAnchor = dot(ld3(va), ld3(va)) > 0, movingMeasured = dot(ld3(vb), ld3(vb)) > 0;
    const V3 measured = ld3(w.obs_bearing + 3 * f);
    V3 ba = ld3(w.lm_anchor_bearing + 3 * l), bb = measured, da{0, 0, 0}, db{0, 0, 0};
    ba = scl(1 / nrm(ba), ba);
    bb = scl(1 / nrm(bb), bb);
    if (movingAnchor) ba = timeBearing(w.lm_anchor_bearing + 3 * l, va, anchorTime - td, timeDerivative, da);
    if (movingMeasured) bb = timeBearing(w.obs_bearing + 3 * f, vb, measuredTime - td, timeDerivative, db);
    if (!fin3(ba) || !fin3(bb)) return false;
    const M3 Rca = {w.cam_R[9 * ca + 0], w.cam_R[9 * ca + 1], w.cam_R[9 * ca + 2], w.cam_R[9 * ca + 3], w.cam_R[9 * ca + 4],
                    w.cam_R[9 * ca + 5], w.cam_R[9 * ca + 6], w.cam_R[9 * ca + 7], w.cam_R[9 * ca + 8]};
    const M3 Rcb = {w.cam_R[9 * cb + 0], w.cam_R[9 * cb + 1], w.cam_R[9 * cb + 2], w.cam_R[9 * cb + 3], w.cam_R[9 * cb + 4],
                    w.cam_R[9 * cb + 5], w.cam_R[9 * cb + 6], w.cam_R[9 * cb + 7], w.cam_R[9 * cb + 8]};
    const V3 tca = ld3(w.cam_t + 3 * ca), tcb = ld3(w.cam_t + 3 * cb);
    const V3 local = add(mv(Rca, scl(1 / rho, ba)), tca);
    M3 Ra{}, Rb{}, Rea{}, Reb{}, W{}, cameraRotation{};
    V3 pc, bodyA{}, rotatedBody{}, relative{}, observerBody{}, tea{}, teb{};
    if (o.same) {
        pc = mv(tr(Rcb), sub(local, tcb));
        cameraRotation = mul(tr(Rcb), Rca);
    } else {
        Ra = qrot(qnormalized(qload(xa + 3)));
        Rb = qrot(qnormalized(qload(xb + 3)));
        Rea = qrot(qnormalized(qload(xea + 3)));
        Reb = qrot(qnormalized(qload(xeb + 3)));
        tea = ld3(xea); teb = ld3(xeb);
        W = tr(mul(mul(Rb, Reb), Rcb));
        cameraRotation = mul(W, mul(mul(Ra, Rea), Rca));
        const V3 separation = sub(ld3(xa), ld3(xb));
        if (!o.split) {
            // offset form of the reference (VisualSphereBatchMath.hpp:107-111)
            const V3 offset = mv(W, add(sub(mv(Ra, add(mv(Rea, tca), tea)), mv(Rb, add(mv(Reb, tcb), teb))), separation));
            pc = add(mv(cameraRotation, scl(1 / rho, ba)), offset);
        } else {
            // two extrinsic blocks: explicit camera chain
            bodyA = add(mv(Rea, local), tea);
            const V3 world = add(mv(Ra, bodyA), ld3(xa));
            const V3 ob = mv(tr(Rb), sub(world, ld3(xb)));
            pc = mv(tr(Rcb), sub(mv(tr(Reb), sub(ob, teb)), tcb));
        }
        bodyA = add(mv(Rea, local), tea);
        rotatedBody = mv(Ra, bodyA);
        relative = add(rotatedBody, separation);
        observerBody = mv(tr(Rb), relative);
    }
    const double range = nrm(pc);
    if (!fin3(pc) || !fin(range) || range < 1e-10) return false;
    const V3 n = scl(1 / range, pc);
    const double c = std::fmin(1.0, std::fmax(-1.0, dot(bb, n))), s = nrm(cross(bb, n));
    const double denominator = movingMeasured ? 1 + dot(measured, bb) : 2;
    if (c < -1 + 1e-8 || denominator < 1e-8) return false;
    const V3 u = sub(n, scl(c, bb));
    const double d = 1 - c;
    const bool series = c > 0 && s < 1e-3;
    const double theta = series ? 0 : std::atan2(s, c);
    const double fcoef = s < 1e-8 ? 1.0 : (series ? 1 + d / 3 + 2 * d * d / 15 + 2 * d * d * d / 35 : theta / s);
    const V3 logarithm = scl(fcoef, u);
    const double* meas = w.obs_P + 6 * f;
    double P[6];
    for (int i = 0; i < 6; ++i) P[i] = meas[i];
    M3 K{};
    if (movingMeasured) {
        K = skew(cross(measured, bb));
        const M3 transport = madd(madd(eye(), K), mscl(1 / denominator, mul(K, K)));
        mul23x33(meas, tr(transport), P);
    }
    for (int r = 0; r < 2; ++r) o.r[r] = P[3 * r] * logarithm[0] + P[3 * r + 1] * logarithm[1] + P[3 * r + 2] * logarithm[2];
    if (!fin(o.r[0]) || !fin(o.r[1])) return false;
    for (int i = 0; i < 12; ++i) o.Ja[i] = o.Jb[i] = o.Jea[i] = o.Jeb[i] = 0;
    o.Jtd[0] = o.Jtd[1] = o.Jrho[0] = o.Jrho[1] = 0;
    if (!derivatives) return true;
    const double g = s < 1e-8 ? 0.0 : (series ? (-1.0 / 3.0 - 4 * d / 15.0 - 6 * d * d / 35.0) : (theta * c - s) / (s * s * s));
    double proj[6], red[6];
    for (int r = 0; r < 2; ++r) {
        const double Pu = P[3 * r] * u[0] + P[3 * r + 1] * u[1] + P[3 * r + 2] * u[2];
        const double Pb = P[3 * r] * bb[0] + P[3 * r + 1] * bb[1] + P[3 * r + 2] * bb[2];
        for (int k = 0; k < 3; ++k) proj[3 * r + k] = fcoef * P[3 * r + k] + (g * Pu - fcoef * Pb) * bb[k];
        const double pn = proj[3 * r] * n[0] + proj[3 * r + 1] * n[1] + proj[3 * r + 2] * n[2];
        for (int k = 0; k < 3; ++k) red[3 * r + k] = (proj[3 * r + k] - pn * n[k]) / range;
    }
    if (!o.same) {
        double D[6], tmp[6];
        mul23x33(red, W, D);
        if (!o.split) {
            // reference ambient route, then tangent lift
            double t1[6], r1[6];
            for (int i = 0; i < 6; ++i) t1[i] = D[i];
            mul23x33(D, skew(rotatedBody), tmp);
            for (int i = 0; i < 6; ++i) r1[i] = -tmp[i];
            if (!liftPose(xa, t1, r1, o.Ja)) return false;
            for (int i = 0; i < 6; ++i) t1[i] = -D[i];
            mul23x33(D, skew(relative), r1);
            if (!liftPose(xb, t1, r1, o.Jb)) return false;
            if (a == b) for (int i = 0; i < 12; ++i) { o.Ja[i] += o.Jb[i]; o.Jb[i] = 0; }
            if (extDerivative) {
                mul23x33(D, msub(Ra, Rb), t1);
                double r2[6];
                mul23x33(D, mscl(-1, mul(Ra, skew(sub(bodyA, tea)))), r1);
                mul23x33(D, mul(Rb, skew(sub(observerBody, tea))), r2);
                for (int i = 0; i < 6; ++i) r1[i] += r2[i];
                if (!liftPose(xea, t1, r1, o.Jea)) return false;
            }
        } else {
            // separate anchor and observer extrinsic blocks: each takes the tangent form of its
            // own camera chain (anchor [D R_a, -D R_a [b_a]x], observer [-D R_b, D R_b [o_b]x])
            const V3 world = add(rotatedBody, ld3(xa));
            if (a != b) {
                tangentDirect(D, eye(), world, 1.0, o.Ja);
                tangentDirect(D, eye(), world, -1.0, o.Jb);
            }
            if (extDerivative) {
                tangentDirect(D, Ra, bodyA, 1.0, o.Jea);
                tangentDirect(D, Rb, observerBody, -1.0, o.Jeb);
            }
        }
    }
    {
        double RC[6];
        mul23x33(red, cameraRotation, RC);
        const V3 q = scl(-1 / (rho * rho), ba);
        for (int r = 0; r < 2; ++r) o.Jrho[r] = RC[3 * r] * q[0] + RC[3 * r + 1] * q[1] + RC[3 * r + 2] * q[2];
        if (!fin(o.Jrho[0]) || !fin(o.Jrho[1])) return false;
    }
    if (timeDerivative && (movingAnchor || movingMeasured)) {
        const M3 Jb = madd(mscl(fcoef, msub(mscl(-1, outer(bb, n)), mscl(c, eye()))), mscl(g, outer(u, n)));
        const M3 dK = skew(cross(measured, db));
        const M3 dR = msub(madd(dK, mscl(1 / denominator, madd(mul(dK, K), mul(K, dK)))),
                           mscl(dot(measured, db) / (denominator * denominator), mul(K, K)));
        double RC[6], PJ[6], MdR[6];
        mul23x33(red, cameraRotation, RC);
        mul23x33(P, Jb, PJ);
        mul23x33(meas, tr(dR), MdR);
        const V3 q = scl(1 / rho, da);
        for (int r = 0; r < 2; ++r) {
            o.Jtd[r] = RC[3 * r] * q[0] + RC[3 * r + 1] * q[1] + RC[3 * r + 2] * q[2] + PJ[3 * r] * db[0] + PJ[3 * r + 1] * db[1] +
                       PJ[3 * r + 2] * db[2] + MdR[3 * r] * logarithm[0] + MdR[3 * r + 1] * logarithm[1] + MdR[3 * r + 2] * logarithm[2];
        }
        if (!fin(o.Jtd[0]) || !fin(o.Jtd[1])) return false;
    }
    return true;
}

// Numeric reference residual (WindowVisualFactor.cpp:411-430): explicit camera
// chain and Quaternion::FromTwoVectors transport.
static Q fromTwoVectors(const V3& a, const V3& b) {
    const V3 v0 = scl(1 / nrm(a), a), v1 = scl(1 / nrm(b), b);
    const double c = dot(v1, v0);
    if (c < -1 + 1e-12) {  // antiparallel: not reached in the tests (rejected earlier)
        return {1, 0, 0, 0};
    }
    const V3 axis = cross(v0, v1);
    const double s = std::sqrt((1 + c) * 2), invs = 1 / s;
    return {axis[0] * invs, axis[1] * invs, axis[2] * invs, s * 0.5};
}
static bool visualResidualNumeric(const cgmli_window& w, int l, int f, double* out) {
    const int a = w.lm_anchor_kf[l], b = w.obs_kf[f], ca = w.lm_anchor_cam[l], cb = w.obs_cam[f];
    const int ea = w.cam_ext[ca], eb = w.cam_ext[cb];
    const double rho = w.rho[l];
    const double anchorTime = w.lm_anchor_time ? w.lm_anchor_time[l] : 0.0;
    const double measuredTime = w.obs_time ? w.obs_time[f] : 0.0;
    const double td = w.td ? *w.td : anchorTime;
    if (!fin(rho) || rho <= 0 || !fin(td)) return false;
    static const double zero3[3] = {0, 0, 0};
    const double* va = w.lm_anchor_velocity ? w.lm_anchor_velocity + 3 * l : zero3;
    const double* vb = w.obs_velocity ? w.obs_velocity + 3 * f : zero3;
    V3 dummy;
    const V3 ba = timeBearing(w.lm_anchor_bearing + 3 * l, va, anchorTime - td, false, dummy);
    const V3 bb = timeBearing(w.obs_bearing + 3 * f, vb, measuredTime - td, false, dummy);
    auto camPose = [&](const double* x, const double* e, int cam, M3& R, V3& t) {
        const M3 Rb = qrot(qnormalized(qload(x + 3))), Re = qrot(qnormalized(qload(e + 3)));
        const M3 Rc = {w.cam_R[9 * cam], w.cam_R[9 * cam + 1], w.cam_R[9 * cam + 2], w.cam_R[9 * cam + 3], w.cam_R[9 * cam + 4],
                       w.cam_R[9 * cam + 5], w.cam_R[9 * cam + 6], w.cam_R[9 * cam + 7], w.cam_R[9 * cam + 8]};
        R = mul(mul(Rb, Re), Rc);
        t = add(mv(Rb, add(mv(Re, ld3(w.cam_t + 3 * cam)), ld3(e))), ld3(x));
    };
    M3 RWa, RWb; V3 tWa, tWb;
    camPose(w.poses + 7 * a, w.extrinsics + 7 * ea, ca, RWa, tWa);
    camPose(w.poses + 7 * b, w.extrinsics + 7 * eb, cb, RWb, tWb);
    const V3 pW = add(mv(RWa, scl(1 / rho, ba)), tWa);
    const V3 pC = mv(tr(RWb), sub(pW, tWb));
    if (!fin3(pC) || nrm(pC) < 1e-10 || !fin3(bb)) return false;
    const V3 predicted = scl(1 / nrm(pC), pC);
    const double c = std::clamp(dot(bb, predicted), -1.0, 1.0), s = nrm(cross(bb, predicted));
    const V3 measured = ld3(w.obs_bearing + 3 * f);
    if (c < -1.0 + 1e-8 || dot(measured, bb) < -1.0 + 1e-8) return false;
    const V3 logarithm = s < 1e-8 ? sub(predicted, scl(c, bb)) : scl(std::atan2(s, c) / s, sub(predicted, scl(c, bb)));
    // measurement_ = sqrtInfo * basis^T, so sqrtInfo * (T*basis)^T = measurement_ * T^T
    const M3 T = qrot(fromTwoVectors(measured, bb));
    double P[6];
    mul23x33(w.obs_P + 6 * f, tr(T), P);
    for (int r = 0; r < 2; ++r) out[r] = P[3 * r] * logarithm[0] + P[3 * r + 1] * logarithm[1] + P[3 * r + 2] * logarithm[2];
    return fin(out[0]) && fin(out[1]);
}

// Huber loss of the reference (VisualCudaBatch.cu:54-59,131-133)
static inline double huberWeight(double scale, double squared) {
    return scale > 0 && squared > scale * scale ? std::sqrt(scale / std::sqrt(squared)) : 1.0;
}
static inline double huberCost(double scale, double squared) {
    return scale > 0 && squared > scale * scale ? scale * (std::sqrt(squared) - 0.5 * scale) : 0.5 * squared;
}

// ---- frozen IMU factor (GpuRetainedFactorMath.hpp:53-140) -------------------
struct Sensor { V3 p, v, arm, lever; Q q; };
static Sensor sensorState(const cgmli_frozen_imu& imu, const double* pose, const double* sb, int end) {
    const Q q = qnormalized(qload(pose + 3));
    Sensor s;
    s.q = qnormalized(qmul(q, qload(imu.sensor_quaternion)));
    s.arm = qapply(q, ld3(imu.sensor_position));
    s.lever = cross(qapply(s.q, sub(ld3(imu.gyros + 3 * end), ld3(sb + 3))), s.arm);
    s.p = add(ld3(pose), s.arm);
    s.v = add(ld3(sb), s.lever);
    return s;
}
// r: 15 whitened residual; J: 15 x 30 row-major over [pose_i(6), sb_i(9), pose_j(6), sb_j(9)]
static bool imuFactor(const cgmli_frozen_imu& imu, const double* p0, const double* sb0, const double* p1, const double* sb1,
                      double* r, double* J) {
    const Sensor s0 = sensorState(imu, p0, sb0, 0), s1 = sensorState(imu, p1, sb1, 1);
    const M3 A = colmajor(imu.rotation_gyro), V = colmajor(imu.velocity_gyro), P = colmajor(imu.position_gyro),
             Va = colmajor(imu.velocity_accel), Pa = colmajor(imu.position_accel);
    const M3 R = qrot(qconj(s0.q));
    const double dt = imu.duration;
    const V3 gravity{0, 0, imu.gravity};
    const V3 bg = sub(ld3(sb0 + 3), ld3(imu.reference_bias)), ba = sub(ld3(sb0 + 6), ld3(imu.reference_bias + 3));
    const V3 dp = sub(add(sub(s0.p, s1.p), scl(dt, s0.v)), scl(0.5 * dt * dt, gravity));
    const V3 dv = sub(sub(s0.v, s1.v), scl(dt, gravity));
    const V3 phi = scl(-1, mv(A, bg));
    const Q correction = rotationExp(phi), dq = qmul(correction, qload(imu.delta_quaternion));
    const Q tail = qmul(qmul(qload(imu.delta_quaternion), qconj(s1.q)), s0.q);
    double e[15];
    const V3 e0 = sub(add(add(mv(R, dp), ld3(imu.delta_position)), mv(P, bg)), mv(Pa, ba));
    const V3 e1 = scl(2, qvec(qmul(dq, qmul(qconj(s1.q), s0.q))));
    const V3 e2 = sub(add(add(mv(R, dv), ld3(imu.delta_velocity)), mv(V, bg)), mv(Va, ba));
    for (int i = 0; i < 3; ++i) { e[i] = e0[i]; e[3 + i] = e1[i]; e[6 + i] = e2[i]; }
    for (int i = 0; i < 6; ++i) e[9 + i] = sb0[3 + i] - sb1[3 + i];
    for (int i = 0; i < 15; ++i) {
        double v = 0;
        for (int k = 0; k < 15; ++k) v += imu.whitening[i + 15 * k] * e[k];
        r[i] = v;
        if (!fin(v)) return false;
    }
    if (!J) return true;
    const M3 gyroAngle = mscl(-1, mul(rotationJacobian(scl(-1, phi)), A));
    M3 Jrot{}, Jbias{};
    for (int j = 0; j < 3; ++j) {
        const Q ax{j == 0 ? 1.0 : 0.0, j == 1 ? 1.0 : 0.0, j == 2 ? 1.0 : 0.0, 0};
        const Q db{gyroAngle[j], gyroAngle[3 + j], gyroAngle[6 + j], 0};
        const V3 c1 = qvec(qmul(qmul(qmul(dq, qconj(s1.q)), ax), s0.q));
        const V3 c2 = qvec(qmul(qmul(correction, db), tail));
        for (int i = 0; i < 3; ++i) { Jrot[3 * i + j] = c1[i]; Jbias[3 * i + j] = c2[i]; }
    }
    for (int i = 0; i < 15 * 30; ++i) J[i] = 0;
    const int width[4] = {6, 9, 6, 9}, col0[4] = {0, 6, 15, 21};
    for (int k = 0; k < 4; ++k) {
        const bool first = k < 2;
        const double sign = first ? 1 : -1;
        const Sensor& s = first ? s0 : s1;
        double Jk[15 * 9] = {0};
        auto put = [&](int r0, int c0, const M3& m, bool accumulate) {
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double& t = Jk[9 * (r0 + i) + c0 + j];
                    t = accumulate ? t + m[3 * i + j] : m[3 * i + j];
                }
        };
        if (k % 2 == 0) {
            put(0, 0, mscl(sign, R), false);
            put(0, 3, mscl(-sign, mul(R, skew(s.p))), false);
            put(3, 3, mscl(sign, Jrot), false);
            put(6, 3, mscl(-sign, mul(R, skew(s.lever))), false);
            if (first) {
                put(0, 3, mul(R, msub(skew(dp), mscl(dt, skew(s.lever)))), true);
                put(6, 3, mul(R, skew(dv)), true);
            }
        } else {
            const M3 leverBias = mul(skew(s.arm), qrot(s.q));
            put(6, 0, mscl(sign, R), false);
            put(6, 3, mscl(sign, mul(R, leverBias)), false);
            put(9, 3, mscl(sign, eye()), false);
            put(12, 6, mscl(sign, eye()), false);
            if (first) {
                put(0, 0, mscl(dt, R), false);
                put(0, 3, madd(mscl(dt, mul(R, leverBias)), P), false);
                put(0, 6, mscl(-1, Pa), false);
                put(3, 3, Jbias, false);
                put(6, 3, V, true);
                put(6, 6, mscl(-1, Va), false);
            }
        }
        for (int j = 0; j < width[k]; ++j)
            for (int i = 0; i < 15; ++i) {
                double v = 0;
                for (int m = 0; m < 15; ++m) v += imu.whitening[i + 15 * m] * Jk[9 * m + j];
                if (!fin(v)) return false;
                J[30 * i + col0[k] + j] = v;
            }
    }
    return true;
}

// ---- IMU preintegration ------------------------------------------------------
// Duration::toSec (src/utils/Duration.h:62-64) of a signed nanosecond count:
// whole seconds (floor) plus 1e-9 * the non-negative remainder.
static double nsToSec(long long ns) {
    long long sec = ns / 1000000000LL, rem = ns % 1000000000LL;
    if (rem < 0) { rem += 1000000000LL; sec -= 1; }
    return (double)sec + 1e-9 * (double)rem;
}
// ode::sinc (src/factor/ode.hpp:15-27)
static double odeSinc(double x) {
    if (std::fabs(x) > 1e-6) return std::sin(x) / x;
    const double x2 = x * x, x4 = x2 * x2, x6 = x2 * x2 * x2;
    return 1.0 - x2 / 6.0 + x4 / 120.0 - x6 / 5040.0;
}
// kinematics::rightJacobian (src/kinematics/Transformation.hpp:47-62)
static M3 rightJacobianSO3(const V3& phi) {
    const double a = nrm(phi);
    const M3 W = skew(phi), W2 = mul(W, W);
    if (a < 1e-4) return madd(eye(), madd(mscl(-0.5, W), mscl(1.0 / 6.0, W2)));
    return madd(eye(), madd(mscl(-(1.0 - std::cos(a)) / (a * a), W), mscl((a - std::sin(a)) / (a * a * a), W2)));
}
// validImuInterval (src/factor/BodyImuFactor.cpp:10-28) over samples [0, n)
static bool imuIntervalValid(const long long* t, const double* m, int n, long long t0, long long t1, double maxGap) {
    if (!std::isfinite(maxGap) || maxGap <= 0) return false;
    if (n < 2 || t1 <= t0 || t[0] > t0 || t[n - 1] < t1) return false;
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < 6; ++k) if (!fin(m[6 * i + k])) return false;
        if (i && t[i] <= t[i - 1]) return false;
        if (i && t[i - 1] < t1 && t[i] > t0 && nsToSec(t[i] - t[i - 1]) > maxGap + 1e-9) return false;
    }
    return true;
}
// gyroAt (src/factor/BodyImuFactor.cpp:29-38): gyro reading interpolated at time e
static V3 gyroReadingAt(const long long* t, const double* m, int n, long long e) {
    int k = 0;
    while (k < n && t[k] < e) ++k;  // first sample not before e
    if (k == 0) return ld3(m);
    if (k == n) return ld3(m + 6 * (n - 1));
    const double alpha = nsToSec(e - t[k - 1]) / nsToSec(t[k] - t[k - 1]);
    return add(scl(1 - alpha, ld3(m + 6 * (k - 1))), scl(alpha, ld3(m + 6 * k)));
}
// Cyclic Jacobi with a relative skip test |a_pq| <= 1e-14 sqrt(a_pp a_qq), so
// that a graded positive definite matrix (the IMU covariance spans ~12 decades)
// keeps its small eigenvalues and their eigenvectors accurate relative to
// themselves; sweeps until one applies no rotation.  Row-major in, eigenvalues
// ascending, eigenvectors as columns of V.
static bool jacobiGraded(int n, const double* Ain, double* evals, double* V) {
    std::vector<double> A(Ain, Ain + (size_t)n * n);
    for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) V[(size_t)i * n + j] = i == j;
    for (int sweep = 0; sweep < 40; ++sweep) {
        bool rotated = false;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                if (apq == 0 || std::fabs(apq) <= 1e-14 * std::sqrt(std::fabs(app * aqq))) continue;
                rotated = true;
                const double tau = (aqq - app) / (2 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1 + tau * tau));
                const double c = 1 / std::sqrt(1 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - s * akq;
                    A[(size_t)k * n + q] = s * akp + c * akq;
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = c * vkp - s * vkq;
                    V[(size_t)k * n + q] = s * vkp + c * vkq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - s * aqk;
                    A[(size_t)q * n + k] = s * apk + c * aqk;
                }
            }
        if (!rotated) break;
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return A[(size_t)x * n + x] < A[(size_t)y * n + y]; });
    std::vector<double> Vs((size_t)n * n);
    for (int j = 0; j < n; ++j) {
        evals[j] = A[(size_t)order[j] * n + order[j]];
        for (int i = 0; i < n; ++i) Vs[(size_t)i * n + j] = V[(size_t)i * n + order[j]];
    }
    std::copy(Vs.begin(), Vs.end(), V);
    for (int i = 0; i < n; ++i) if (!fin(evals[i])) return false;
    return true;
}
// 15x15 row-major helpers
static void mat15Mul(const double* A, const double* B, double* C) {
    for (int r = 0; r < 15; ++r)
        for (int c = 0; c < 15; ++c) {
            double s = 0;
            for (int k = 0; k < 15; ++k) s += A[15 * r + k] * B[15 * k + c];
            C[15 * r + c] = s;
        }
}
static void setBlock15(double* F, int r0, int c0, const M3& b) {
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) F[15 * (r0 + i) + c0 + j] = b[3 * i + j];
}
// ImuError::redoPreintegration (src/factor/ImuError.cpp:254-462) over samples
// [0, n) from t0 to t1 at bias [b_g, b_a], with the four covariance
// derivatives dP/dsigma^2 propagated separately and summed at the end as the
// reference does, then PseudoInverse::symmSqrtU (src/factor/PseudoInverse.hpp:117-145).
static bool preintegrateInterval(const cgmli_imu_parameters& prm, const long long* ts, const double* m, int n, long long t0,
                                 long long t1, const double* bias, cgmli_frozen_imu& out, double* covariance) {
    Q Dq{0, 0, 0, 1};
    M3 Cint{}, Cdint{}, crossAcc{}, dAlphaDbg{}, dVelDbg{}, dPosDbg{};
    V3 accInt{0, 0, 0}, accDint{0, 0, 0};
    std::vector<double> dPdSigma(4 * 225, 0.0);
    const V3 bg = ld3(bias), ba = ld3(bias + 3);
    long long time = t0;
    bool started = false;
    int steps = 0;
    for (int it = 0; it + 1 < n; ++it) {
        V3 w0 = ld3(m + 6 * it), a0 = ld3(m + 6 * it + 3), w1 = ld3(m + 6 * it + 6), a1 = ld3(m + 6 * it + 9);
        long long next = ts[it + 1];
        double dt = nsToSec(next - time);
        if (t1 < next) {  // the interval ends inside this sample pair: interpolate its end
            const double interval = nsToSec(next - ts[it]);
            next = t1;
            dt = nsToSec(next - time);
            const double r = dt / interval;
            w1 = add(scl(1.0 - r, w0), scl(r, w1));
            a1 = add(scl(1.0 - r, a0), scl(r, a1));
        }
        if (dt <= 0.0) continue;
        if (!started) {  // first pair: move its start reading to t0
            started = true;
            const double r = dt / nsToSec(next - ts[it]);
            w0 = add(scl(r, w0), scl(1.0 - r, w1));
            a0 = add(scl(r, a0), scl(1.0 - r, a1));
        }
        double gyroSat = 1.0, accSat = 1.0;
        for (int k = 0; k < 3; ++k) {
            if (std::fabs(w0[k]) > prm.g_max || std::fabs(w1[k]) > prm.g_max) gyroSat = 100.0;
            if (std::fabs(a0[k]) > prm.a_max || std::fabs(a1[k]) > prm.a_max) accSat = 100.0;
        }
        // orientation increment
        const V3 omega = sub(scl(0.5, add(w0, w1)), bg);
        const double halfAngle = nrm(omega) * 0.5 * dt;
        const double sincHalf = odeSinc(halfAngle);
        const Q dq{sincHalf * omega[0] * 0.5 * dt, sincHalf * omega[1] * 0.5 * dt, sincHalf * omega[2] * 0.5 * dt, std::cos(halfAngle)};
        const Q Dq1 = qmul(Dq, dq);
        const M3 C = qrot(Dq), C1 = qrot(Dq1), CC = madd(C, C1);
        const V3 acc = sub(scl(0.5, add(a0, a1)), ba);
        // rotation integrals
        const M3 Cint1 = madd(Cint, mscl(dt, mscl(0.5, CC)));
        const V3 accInt1 = add(accInt, scl(dt, mv(mscl(0.5, CC), acc)));
        Cdint = madd(Cdint, madd(mscl(dt, Cint), mscl(dt * dt, mscl(0.25, CC))));
        accDint = add(accDint, add(scl(dt, accInt), scl(dt * dt, mv(mscl(0.25, CC), acc))));
        // bias Jacobians
        const M3 Jr = rightJacobianSO3(scl(dt, omega));
        dAlphaDbg = madd(dAlphaDbg, mscl(dt, mul(C1, Jr)));
        const Q dqInv{-dq.x, -dq.y, -dq.z, dq.w};
        const M3 cross1 = madd(mul(qrot(dqInv), crossAcc), mscl(dt, Jr));
        const M3 ax = skew(acc);
        const M3 both = madd(mul(mul(C, ax), crossAcc), mul(mul(C1, ax), cross1));
        const M3 dVel1 = madd(dVelDbg, mscl(0.5 * dt, both));
        dPosDbg = madd(dPosDbg, madd(mscl(dt, dVelDbg), mscl(0.25 * dt * dt, both)));
        // transition of the 15-dimensional increment error
        double F[225];
        for (int i = 0; i < 225; ++i) F[i] = (i / 15 == i % 15) ? 1.0 : 0.0;
        setBlock15(F, 0, 3, mscl(-1.0, skew(add(scl(dt, accInt), scl(dt * dt, mv(mscl(0.25, CC), acc))))));
        setBlock15(F, 0, 6, mscl(dt, eye()));
        setBlock15(F, 0, 9, madd(mscl(dt, dVelDbg), mscl(0.25 * dt * dt, both)));
        setBlock15(F, 0, 12, madd(mscl(-dt, Cint), mscl(dt * dt, mscl(0.25, CC))));
        setBlock15(F, 3, 9, mscl(-dt, C1));
        setBlock15(F, 6, 3, mscl(-1.0, skew(scl(dt, mv(mscl(0.5, CC), acc)))));
        setBlock15(F, 6, 9, mscl(0.5 * dt, both));
        setBlock15(F, 6, 12, mscl(-dt, mscl(0.5, CC)));
        double Ft[225];
        for (int r = 0; r < 15; ++r) for (int c = 0; c < 15; ++c) Ft[15 * c + r] = F[15 * r + c];
        // noise of each sigma^2 (K0 .. K3)
        double noise[4][15] = {};
        for (int i = 3; i < 6; ++i) noise[0][i] = gyroSat * dt;
        for (int i = 0; i < 3; ++i) noise[1][i] = 0.5 * dt * dt * dt * accSat * accSat * accSat;
        for (int i = 6; i < 9; ++i) noise[1][i] = accSat * dt;
        for (int i = 9; i < 12; ++i) noise[2][i] = dt;
        for (int i = 12; i < 15; ++i) noise[3][i] = dt;
        for (int j = 0; j < 4; ++j) {
            double T[225];
            double* D = &dPdSigma[225 * j];
            mat15Mul(F, D, T);
            mat15Mul(T, Ft, D);
            for (int i = 0; i < 15; ++i) D[16 * i] += noise[j][i];
        }
        Dq = Dq1; Cint = Cint1; accInt = accInt1; crossAcc = cross1; dVelDbg = dVel1;
        time = next;
        ++steps;
        if (next == t1) break;
    }
    if (steps <= 0) return false;
    // symmetrize each derivative, weight by the noise densities
    const double s2[4] = {prm.sigma_g_c * prm.sigma_g_c, prm.sigma_a_c * prm.sigma_a_c, prm.sigma_gw_c * prm.sigma_gw_c,
                          prm.sigma_aw_c * prm.sigma_aw_c};
    double P[225] = {};
    for (int j = 0; j < 4; ++j)
        for (int r = 0; r < 15; ++r)
            for (int c = 0; c < 15; ++c)
                P[15 * r + c] += (0.5 * dPdSigma[225 * j + 15 * r + c] + 0.5 * dPdSigma[225 * j + 15 * c + r]) * s2[j];
    if (covariance) std::copy(P, P + 225, covariance);
    // W = diag(sqrt(1/lambda)) U^T with eigenvalues at or below the tolerance raised to it.
    // The reference's Eigen::SelfAdjointEigenSolver is accurate to eps * lambda_max in
    // every eigenvalue; the graded Jacobi is accurate relative to each one.
    double lam[15], U[225];
    if (!jacobiGraded(15, P, lam, U)) return false;
    const double eps = std::numeric_limits<double>::epsilon();
    double lmax = lam[0];
    for (int i = 1; i < 15; ++i) lmax = std::max(lmax, lam[i]);
    const double tol = std::max(eps, eps * 15 * lmax);
    for (int r = 0; r < 15; ++r) {
        const double s = std::sqrt(lam[r] > tol ? 1.0 / lam[r] : 1.0 / tol);
        for (int c = 0; c < 15; ++c) out.whitening[r + 15 * c] = s * U[15 * c + r];
    }
    auto toColumnMajor = [](const M3& a, double* dst) {
        for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) dst[r + 3 * c] = a[3 * r + c];
    };
    out.delta_quaternion[0] = Dq.x; out.delta_quaternion[1] = Dq.y; out.delta_quaternion[2] = Dq.z; out.delta_quaternion[3] = Dq.w;
    for (int i = 0; i < 3; ++i) { out.delta_velocity[i] = accInt[i]; out.delta_position[i] = accDint[i]; }
    for (int i = 0; i < 6; ++i) out.reference_bias[i] = bias[i];
    toColumnMajor(dAlphaDbg, out.rotation_gyro);
    toColumnMajor(dVelDbg, out.velocity_gyro);
    toColumnMajor(dPosDbg, out.position_gyro);
    toColumnMajor(Cint, out.velocity_accel);
    toColumnMajor(Cdint, out.position_accel);
    out.duration = nsToSec(t1 - t0);
    out.gravity = prm.g;
    for (int i = 0; i < 3; ++i) out.sensor_position[i] = prm.sensor_position[i];
    for (int i = 0; i < 4; ++i) out.sensor_quaternion[i] = prm.sensor_quaternion[i];
    const V3 g0 = gyroReadingAt(ts, m, n, t0), g1 = gyroReadingAt(ts, m, n, t1);
    for (int i = 0; i < 3; ++i) { out.gyros[i] = g0[i]; out.gyros[3 + i] = g1[i]; }
    const double* all = &out.duration;
    for (size_t i = 0; i < sizeof(cgmli_frozen_imu) / sizeof(double); ++i)
        if (!fin(all[i])) return false;
    return true;
}

// ---- marginalization prior factor -------------------------------------------
static int blockTangent(int kind) { return kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 6; }
static int blockAmbient(int kind) { return kind == CGMLI_PRIOR_SPEED_BIAS ? 9 : kind == CGMLI_PRIOR_TIME_OFFSET ? 1 : 7; }
static const double* blockValue(const cgmli_window& w, int kind, int index) {
    switch (kind) {
        case CGMLI_PRIOR_POSE: return w.poses + 7 * index;
        case CGMLI_PRIOR_SPEED_BIAS: return w.speed_bias + 9 * index;
        case CGMLI_PRIOR_EXTRINSIC: return w.extrinsics + 7 * index;
        default: return w.td;
    }
}
static int blockColumn(const Layout& lay, int kind, int index) {
    switch (kind) {
        case CGMLI_PRIOR_POSE: return lay.pose(index);
        case CGMLI_PRIOR_SPEED_BIAS: return lay.sb(index);
        case CGMLI_PRIOR_EXTRINSIC: return lay.ext(index);
        default: return lay.td();
    }
}
// r = r0 + A*(x [-] ref); Jt = A*D (tangent, rank x cols); fdChart selects the
// reference's finite-difference chart derivative instead of the analytic one.
static bool priorFactor(const cgmli_window& w, std::vector<double>& r, std::vector<double>* Jt, bool fdChart = false) {
    const int rank = w.prior_rank;
    int cols = 0;
    for (int b = 0; b < w.prior_num_blocks; ++b) cols += blockTangent(w.prior_block_kind[b]);
    std::vector<double> delta(cols), D(cols * 6, 0.0);
    int off = 0, aoff = 0;
    std::vector<int> offs(w.prior_num_blocks);
    for (int b = 0; b < w.prior_num_blocks; ++b) {
        const int kind = w.prior_block_kind[b], t = blockTangent(kind), a = blockAmbient(kind);
        const double* x = blockValue(w, kind, w.prior_block_index[b]);
        const double* ref = w.prior_ref + aoff;
        if (!x) return false;
        for (int i = 0; i < a; ++i) if (!fin(x[i])) return false;
        offs[b] = off;
        if (kind == CGMLI_PRIOR_POSE || kind == CGMLI_PRIOR_EXTRINSIC) {
            poseMinus(x, ref, delta.data() + off);
            if (Jt) {
                double Dm[36];
                if (fdChart) chartDerivativeFD(x, ref, Dm); else se3LeftJacobianInverse(delta.data() + off, Dm);
                std::copy(Dm, Dm + 36, D.begin() + 6 * off);
            }
        } else {
            for (int i = 0; i < t; ++i) delta[off + i] = x[i] - ref[i];
        }
        off += t; aoff += a;
    }
    r.assign(rank, 0.0);
    for (int i = 0; i < rank; ++i) {
        double v = w.prior_r0[i];
        for (int c = 0; c < cols; ++c) v += w.prior_A[(size_t)i * cols + c] * delta[c];
        r[i] = v;
        if (!fin(v)) return false;
    }
    if (!Jt) return true;
    Jt->assign((size_t)rank * cols, 0.0);
    for (int b = 0; b < w.prior_num_blocks; ++b) {
        const int kind = w.prior_block_kind[b], t = blockTangent(kind), o = offs[b];
        const bool se3 = kind == CGMLI_PRIOR_POSE || kind == CGMLI_PRIOR_EXTRINSIC;
        for (int i = 0; i < rank; ++i)
            for (int c = 0; c < t; ++c) {
                double v = 0;
                if (se3) for (int j = 0; j < 6; ++j) v += w.prior_A[(size_t)i * cols + o + j] * D[6 * (o + j) + c];
                else v = w.prior_A[(size_t)i * cols + o + c];
                (*Jt)[(size_t)i * cols + o + c] = v;
            }
    }
    return true;
}

// ---- dense linear algebra ---------------------------------------------------
static bool cholesky(std::vector<double>& A, int n) {  // in place, lower, row-major
    for (int j = 0; j < n; ++j) {
        double s = A[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) s -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        if (!(s > 0) || !fin(s)) return false;
        const double d = std::sqrt(s);
        A[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double v = A[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) v -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = v / d;
        }
    }
    return true;
}
static void cholSolve(const std::vector<double>& L, int n, std::vector<double>& x) {
    for (int i = 0; i < n; ++i) {
        double v = x[i];
        for (int k = 0; k < i; ++k) v -= L[(size_t)i * n + k] * x[k];
        x[i] = v / L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double v = x[i];
        for (int k = i + 1; k < n; ++k) v -= L[(size_t)k * n + i] * x[k];
        x[i] = v / L[(size_t)i * n + i];
    }
}
// Cyclic Jacobi eigensolver for a symmetric matrix (row-major in, eigenvalues
// ascending, eigenvectors as columns of V row-major).  Stands in for
// Eigen::SelfAdjointEigenSolver (Marginalizer.cpp:270,436).
static bool eigenSym(int n, const double* Ain, double* evals, double* V) {
    std::vector<double> A(Ain, Ain + (size_t)n * n);
    for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) V[(size_t)i * n + j] = i == j;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, total = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const double v = A[(size_t)i * n + j] * A[(size_t)i * n + j];
                total += v;
                if (i != j) off += v;
            }
        if (off <= 1e-32 * total || off == 0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                if (apq == 0) continue;
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                const double tau = (aqq - app) / (2 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1 + tau * tau));
                const double c = 1 / std::sqrt(1 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - s * akq;
                    A[(size_t)k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - s * aqk;
                    A[(size_t)q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = c * vkp - s * vkq;
                    V[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return A[(size_t)x * n + x] < A[(size_t)y * n + y]; });
    std::vector<double> Vs((size_t)n * n);
    for (int j = 0; j < n; ++j) {
        evals[j] = A[(size_t)order[j] * n + order[j]];
        for (int i = 0; i < n; ++i) Vs[(size_t)i * n + j] = V[(size_t)i * n + order[j]];
    }
    std::copy(Vs.begin(), Vs.end(), V);
    for (int i = 0; i < n; ++i) if (!fin(evals[i])) return false;
    return true;
}
// Marginalizer::psdSolve (Marginalizer.cpp:240-283).  H: n x n row-major,
// rhs/x: n x cols row-major.  Returns CGMLI_OK or CGMLI_E_INDEFINITE.
static int psdSolve(int n, const double* H, int cols, const double* rhs, double absCut, double relCut, double* x) {
    if (!n) return CGMLI_OK;
    for (size_t i = 0; i < (size_t)n * n; ++i) if (!fin(H[i])) return CGMLI_E_INVALID;
    bool diagonal = true;
    for (int i = 0; i < n && diagonal; ++i)
        for (int j = 0; j < n; ++j) if (i != j && H[(size_t)i * n + j] != 0.0) { diagonal = false; break; }
    if (diagonal) {
        double maxd = -std::numeric_limits<double>::infinity(), mind = std::numeric_limits<double>::infinity();
        for (int i = 0; i < n; ++i) { maxd = std::max(maxd, H[(size_t)i * n + i]); mind = std::min(mind, H[(size_t)i * n + i]); }
        const double cutoff = std::max(absCut, relCut * std::max(0.0, maxd));
        if (mind < -10.0 * cutoff) return CGMLI_E_INDEFINITE;
        for (int i = 0; i < n; ++i) {
            const double h = H[(size_t)i * n + i];
            for (int c = 0; c < cols; ++c) x[(size_t)i * cols + c] = h > cutoff ? rhs[(size_t)i * cols + c] / h : 0.0;
        }
        return CGMLI_OK;
    }
    std::vector<double> S((size_t)n * n), ev(n), U((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) S[(size_t)i * n + j] = 0.5 * (H[(size_t)i * n + j] + H[(size_t)j * n + i]);
    if (!eigenSym(n, S.data(), ev.data(), U.data())) return CGMLI_E_NONFINITE;
    const double cutoff = std::max(absCut, relCut * std::max(0.0, ev[n - 1]));
    if (ev[0] < -10.0 * cutoff) return CGMLI_E_INDEFINITE;
    std::vector<double> proj((size_t)n * cols, 0.0);
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < cols; ++c) {
            double v = 0;
            for (int k = 0; k < n; ++k) v += U[(size_t)k * n + i] * rhs[(size_t)k * cols + c];
            proj[(size_t)i * cols + c] = ev[i] > cutoff ? v / ev[i] : 0.0;
        }
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < cols; ++c) {
            double v = 0;
            for (int k = 0; k < n; ++k) v += U[(size_t)i * n + k] * proj[(size_t)k * cols + c];
            x[(size_t)i * cols + c] = v;
        }
    return CGMLI_OK;
}

// ---- window linearization -----------------------------------------------------
struct Linear {
    int Nr = 0, L = 0;
    std::vector<double> H;                // Nr x Nr (visual + IMU + prior), full
    std::vector<double> g;                // Nr + L
    std::vector<double> d;                // L
    std::vector<std::vector<int>> sc;     // per landmark: support columns (sorted)
    std::vector<std::vector<double>> sv;  // per landmark: cross values on those columns
    double cost = 0, visualCost = 0, rss = 0;
    bool valid = true;
};

struct ColumnAdder {  // accumulates a factor's rows into H/g (retained block) and cross
    static void addRows(Linear& lin, int nrows, const double* J /*nrows x m*/, const int* cols, int m, const double* r) {
        for (int i = 0; i < m; ++i) {
            if (cols[i] < 0) continue;
            double gi = 0;
            for (int k = 0; k < nrows; ++k) gi += J[k * m + i] * r[k];
            lin.g[cols[i]] += gi;
            for (int j = 0; j < m; ++j) {
                if (cols[j] < 0) continue;
                double h = 0;
                for (int k = 0; k < nrows; ++k) h += J[k * m + i] * J[k * m + j];
                lin.H[(size_t)cols[i] * lin.Nr + cols[j]] += h;
            }
        }
    }
};

static bool linearize(const cgmli_window& w, Linear& lin, bool applyLoss = true) {
    const Layout lay(w);
    lin = Linear();
    lin.Nr = lay.Nr; lin.L = lay.L;
    lin.H.assign((size_t)lay.Nr * lay.Nr, 0.0);
    lin.g.assign(lay.Nr + lay.L, 0.0);
    lin.d.assign(lay.L, 0.0);
    lin.sc.resize(lay.L); lin.sv.resize(lay.L);
    std::vector<double> cross(lay.Nr);
    std::vector<char> touched(lay.Nr);
    for (int l = 0; l < lay.L; ++l) {
        std::vector<int> touchedList;
        for (int f = w.lm_obs_begin[l]; f < w.lm_obs_begin[l + 1]; ++f) {
            Fac o;
            if (!visualFactor(w, l, f, true, o)) { lin.valid = false; return false; }
            const double sq = o.r[0] * o.r[0] + o.r[1] * o.r[1];
            const double wgt = applyLoss ? huberWeight(w.huber_scale, sq) : 1.0;
            lin.visualCost += applyLoss ? huberCost(w.huber_scale, sq) : 0.5 * sq;
            lin.rss += wgt * wgt * sq;
            // columns: anchor 6, observer 6, ext_a 6, ext_b 6, td 1, rho 1
            int cols[26];
            double J[2 * 26];
            const double* blocks[4] = {o.Ja, o.Jb, o.Jea, o.Jeb};
            const int base[4] = {lay.pose(o.a), lay.pose(o.b), lay.ext(o.ea), lay.ext(o.eb)};
            for (int bl = 0; bl < 4; ++bl)
                for (int c = 0; c < 6; ++c) {
                    int col = base[bl] < 0 ? -1 : base[bl] + c;
                    if (bl == 1 && o.a == o.b) col = -1;   // merged into the anchor block
                    if (bl == 3 && !o.split) col = -1;     // shared extrinsic: one block
                    if (o.same && bl != 3) col = bl == 0 || bl == 2 ? -1 : col;
                    cols[6 * bl + c] = col;
                    for (int k = 0; k < 2; ++k) J[26 * k + 6 * bl + c] = wgt * blocks[bl][6 * k + c];
                }
            cols[24] = lay.td();
            cols[25] = -1;
            for (int k = 0; k < 2; ++k) { J[26 * k + 24] = wgt * o.Jtd[k]; J[26 * k + 25] = wgt * o.Jrho[k]; }
            const double rw[2] = {wgt * o.r[0], wgt * o.r[1]};
            ColumnAdder::addRows(lin, 2, J, cols, 26, rw);
            lin.d[l] += J[25] * J[25] + J[26 + 25] * J[26 + 25];
            lin.g[lay.Nr + l] += J[25] * rw[0] + J[26 + 25] * rw[1];
            for (int i = 0; i < 25; ++i) {
                if (cols[i] < 0) continue;
                cross[cols[i]] += J[i] * J[25] + J[26 + i] * J[26 + 25];
                if (!touched[cols[i]]) { touched[cols[i]] = 1; touchedList.push_back(cols[i]); }
            }
        }
        std::sort(touchedList.begin(), touchedList.end());
        lin.sc[l] = touchedList;
        lin.sv[l].resize(touchedList.size());
        for (size_t i = 0; i < touchedList.size(); ++i) {
            lin.sv[l][i] = cross[touchedList[i]];
            cross[touchedList[i]] = 0;
            touched[touchedList[i]] = 0;
        }
    }
    double rcost = 0;
    for (int i = 0; i < w.num_imu; ++i) {
        const int k = w.imu_kf[i];
        double r[15], J[15 * 30];
        if (!imuFactor(w.imu[i], w.poses + 7 * k, w.speed_bias + 9 * k, w.poses + 7 * (k + 1), w.speed_bias + 9 * (k + 1), r, J)) {
            lin.valid = false; return false;
        }
        int cols[30];
        for (int c = 0; c < 30; ++c) cols[c] = 15 * k + c;
        ColumnAdder::addRows(lin, 15, J, cols, 30, r);
        for (int c = 0; c < 15; ++c) { rcost += 0.5 * r[c] * r[c]; lin.rss += r[c] * r[c]; }
    }
    if (w.prior_rank > 0) {
        std::vector<double> r, Jt;
        if (!priorFactor(w, r, &Jt)) { lin.valid = false; return false; }
        std::vector<int> cols;
        for (int b = 0; b < w.prior_num_blocks; ++b) {
            const int kind = w.prior_block_kind[b], col = blockColumn(lay, kind, w.prior_block_index[b]);
            for (int c = 0; c < blockTangent(kind); ++c) cols.push_back(col < 0 ? -1 : col + c);
        }
        ColumnAdder::addRows(lin, w.prior_rank, Jt.data(), cols.data(), (int)cols.size(), r.data());
        for (double v : r) { rcost += 0.5 * v * v; lin.rss += v * v; }
    }
    lin.cost = lin.visualCost + rcost;
    if (!fin(lin.cost)) { lin.valid = false; return false; }
    return true;
}

static double dampedPoint(double d, double lambda) { return d + lambda * std::max(d, 1e-6); }

struct Step {
    std::vector<double> delta, S, rhs;  // delta: Nr + L
    double predicted = 0;
    int status = CGMLI_OK;
};
// solveOnline (VisualCudaBatch.cu:138-205,530-604) at fixed lambda.
// Solve-time charts (the reference's constant blocks and restricted tangents of
// one solve, BackendOptimizer.cpp:44-66,83-91,783-795): the columns of T map the
// restricted tangent into the window's full tangent.  A free column is a unit
// vector; a rotation-only extrinsic's theta_k moves [rho; theta] along
// [[p]x e_k; e_k] (its Plus keeps the translation, GpuRetainedFactorMath.hpp:28-37);
// fixed columns (constant blocks, frozen biases, the folded rho columns) have none.
struct Charts {
    std::vector<int> col;                 // restricted coordinate -> its full column (free or theta)
    std::vector<std::vector<double>> T;   // restricted coordinate -> its full-tangent direction (n)
    std::vector<char> fixed;              // per full column
    bool any = false;
};
static Charts chartsOf(const cgmli_window& w) {
    const Layout lay(w);
    const int n = lay.Nr;
    Charts c;
    c.fixed.assign(n, 0);
    std::vector<char> theta(n, 0);
    if (w.kf_fixed)
        for (int k = 0; k < lay.K; ++k) {
            const int m = w.kf_fixed[k];
            for (int j = 0; j < 6; ++j) if (m & CGMLI_FIX_POSE) c.fixed[lay.pose(k) + j] = 1;
            for (int j = 0; j < 3; ++j) if (m & CGMLI_FIX_VELOCITY) c.fixed[lay.sb(k) + j] = 1;
            for (int j = 3; j < 9; ++j) if (m & CGMLI_FIX_BIAS) c.fixed[lay.sb(k) + j] = 1;
        }
    if (lay.estExt && w.ext_chart)
        for (int e = 0; e < lay.E; ++e) {
            if (w.ext_chart[e] == CGMLI_CHART_FIXED) for (int j = 0; j < 6; ++j) c.fixed[lay.ext(e) + j] = 1;
            if (w.ext_chart[e] == CGMLI_CHART_ROTATION_ONLY) {
                for (int j = 0; j < 3; ++j) { c.fixed[lay.ext(e) + j] = 1; theta[lay.ext(e) + 3 + j] = 1; }
            }
        }
    for (int i = 0; i < n; ++i) {
        if (c.fixed[i]) { c.any = true; continue; }
        std::vector<double> t(n, 0.0);
        t[i] = 1.0;
        if (theta[i]) {
            const int e = (i - lay.ext0) / 6, c0 = lay.ext(e), k = i - c0 - 3;
            const M3 P = skew(ld3(w.extrinsics + 7 * e));
            for (int a = 0; a < 3; ++a) t[c0 + a] = P[3 * a + k];
            c.any = true;
        }
        c.col.push_back(i);
        c.T.push_back(std::move(t));
    }
    return c;
}
static bool landmarkFixed(const cgmli_window& w, int l) { return w.lm_fixed && w.lm_fixed[l]; }

static Step schurStep(const cgmli_window& w, const Linear& lin, double lambda, int refinement = 0) {
    Step st;
    const int n = lin.Nr, L = lin.L;
    const Charts ch = chartsOf(w);
    st.S = lin.H;
    st.rhs.assign(n, 0.0);
    for (int i = 0; i < n; ++i) st.rhs[i] = lin.g[i];
    for (int l = 0; l < L; ++l) {
        if (landmarkFixed(w, l)) continue;  // held constant: not eliminated
        const double inv = 1 / dampedPoint(lin.d[l], lambda);
        const auto& c = lin.sc[l];
        const auto& v = lin.sv[l];
        for (size_t i = 0; i < c.size(); ++i) {
            for (size_t j = 0; j < c.size(); ++j) st.S[(size_t)c[i] * n + c[j]] -= inv * v[i] * v[j];
            st.rhs[c[i]] -= inv * v[i] * lin.g[n + l];
        }
    }
    for (int i = 0; i < n; ++i) st.rhs[i] = -st.rhs[i];
    std::vector<double> x(n, 0.0);
    if (!ch.any) {
        for (int i = 0; i < n; ++i) st.S[(size_t)i * n + i] += lambda * std::max(lin.H[(size_t)i * n + i], 1e-6);
        std::vector<double> Lm = st.S;
        if (!cholesky(Lm, n)) { st.status = CGMLI_E_NOT_PD; return st; }
        x = st.rhs;
        cholSolve(Lm, n, x);
        for (int it = 0; it < refinement; ++it) {
            std::vector<double> res(n);
            for (int i = 0; i < n; ++i) {
                double v = st.rhs[i];
                for (int j = 0; j < n; ++j) v -= st.S[(size_t)i * n + j] * x[j];
                res[i] = v;
            }
            cholSolve(Lm, n, res);
            for (int i = 0; i < n; ++i) x[i] += res[i];
        }
    } else {
        // restricted system S' = T^T S T damped by lambda max(diag(T^T H T), 1e-6), rhs' = T^T rhs;
        // reported embedded in the full columns with identity rows at the fixed ones
        const int m = (int)ch.col.size();
        auto quad = [&](const std::vector<double>& M, const std::vector<double>& a, const std::vector<double>& b) {
            double v = 0;
            for (int i = 0; i < n; ++i) {
                if (a[i] == 0) continue;
                double r = 0;
                for (int j = 0; j < n; ++j) r += M[(size_t)i * n + j] * b[j];
                v += a[i] * r;
            }
            return v;
        };
        std::vector<double> Sr((size_t)m * m), Sd((size_t)m * m), rr(m);
        for (int p = 0; p < m; ++p) {
            for (int q = 0; q < m; ++q) Sr[(size_t)p * m + q] = quad(st.S, ch.T[p], ch.T[q]);
            double v = 0;
            for (int i = 0; i < n; ++i) v += ch.T[p][i] * st.rhs[i];
            rr[p] = v;
        }
        Sd = Sr;
        for (int p = 0; p < m; ++p) Sd[(size_t)p * m + p] += lambda * std::max(quad(lin.H, ch.T[p], ch.T[p]), 1e-6);
        std::vector<double> Lm = Sd, y = rr;
        if (!cholesky(Lm, m)) { st.status = CGMLI_E_NOT_PD; return st; }
        cholSolve(Lm, m, y);
        for (int it = 0; it < refinement; ++it) {
            std::vector<double> res(m);
            for (int p = 0; p < m; ++p) {
                double v = rr[p];
                for (int q = 0; q < m; ++q) v -= Sd[(size_t)p * m + q] * y[q];
                res[p] = v;
            }
            cholSolve(Lm, m, res);
            for (int p = 0; p < m; ++p) y[p] += res[p];
        }
        for (int p = 0; p < m; ++p)
            for (int i = 0; i < n; ++i) x[i] += ch.T[p][i] * y[p];
        std::fill(st.S.begin(), st.S.end(), 0.0);
        std::fill(st.rhs.begin(), st.rhs.end(), 0.0);
        for (int i = 0; i < n; ++i) if (ch.fixed[i]) st.S[(size_t)i * n + i] = 1.0;
        for (int p = 0; p < m; ++p) {
            st.rhs[ch.col[p]] = rr[p];
            for (int q = 0; q < m; ++q) st.S[(size_t)ch.col[p] * n + ch.col[q]] = Sd[(size_t)p * m + q];
        }
    }
    st.delta.assign(n + L, 0.0);
    for (int i = 0; i < n; ++i) st.delta[i] = x[i];  // states are unbounded: clampStateStep is the identity
    double pred = 0;
    for (int i = 0; i < n; ++i) {
        double hd = 0;
        for (int j = 0; j < n; ++j) hd += lin.H[(size_t)i * n + j] * x[j];
        pred += -x[i] * (lin.g[i] + 0.5 * hd);
    }
    for (int l = 0; l < L; ++l) {
        if (landmarkFixed(w, l)) continue;  // no increment, no landmark term
        double c = 0;
        for (size_t i = 0; i < lin.sc[l].size(); ++i) c += lin.sv[l][i] * x[lin.sc[l][i]];
        const double gl = lin.g[n + l];
        double dl = -(gl + c) / dampedPoint(lin.d[l], lambda);
        const double lower = w.min_inverse_distance - w.rho[l];
        if (fin(dl)) dl = std::max(lower, dl);
        st.delta[n + l] = dl;
        pred += -dl * (gl + c + 0.5 * lin.d[l] * dl);
    }
    st.predicted = pred;
    return st;
}

// Candidate state x [+] delta of residentTrial (VisualCudaBatch.cu:323-340).
struct States {
    std::vector<double> poses, sb, ext, rho;
    double td = 0;
};
static States grab(const cgmli_window& w) {
    States s;
    s.poses.assign(w.poses, w.poses + 7 * w.num_keyframes);
    s.sb.assign(w.speed_bias, w.speed_bias + 9 * w.num_keyframes);
    s.ext.assign(w.extrinsics, w.extrinsics + 7 * w.num_extrinsics);
    s.rho.assign(w.rho, w.rho + w.num_landmarks);
    if (w.td) s.td = *w.td;
    return s;
}
static void put(cgmli_window& w, const States& s) {
    std::copy(s.poses.begin(), s.poses.end(), w.poses);
    std::copy(s.sb.begin(), s.sb.end(), w.speed_bias);
    std::copy(s.ext.begin(), s.ext.end(), w.extrinsics);
    std::copy(s.rho.begin(), s.rho.end(), w.rho);
    if (w.td) *w.td = s.td;
}
static bool applyStep(const cgmli_window& w, const std::vector<double>& delta, States& out, double& maxInc) {
    const Layout lay(w);
    out = grab(w);
    maxInc = 0;
    bool ok = true;
    for (int i = 0; i < (int)delta.size(); ++i) {
        if (!fin(delta[i])) ok = false;
        else maxInc = std::max(maxInc, std::fabs(delta[i]));
    }
    if (!ok) return false;
    // solve-time charts: fixed blocks stay as they are; a rotation-only extrinsic keeps its translation
    const unsigned char fixPose = CGMLI_FIX_POSE;
    for (int k = 0; k < lay.K; ++k) {
        const int m = w.kf_fixed ? w.kf_fixed[k] : 0;
        if (!(m & fixPose)) posePlus(w.poses + 7 * k, delta.data() + lay.pose(k), out.poses.data() + 7 * k);
        for (int j = 0; j < 9; ++j) {
            const bool held = j < 3 ? (m & CGMLI_FIX_VELOCITY) != 0 : (m & CGMLI_FIX_BIAS) != 0;
            if (!held) out.sb[9 * k + j] = w.speed_bias[9 * k + j] + delta[lay.sb(k) + j];
        }
    }
    if (lay.estExt)
        for (int e = 0; e < lay.E; ++e) {
            const int chart = w.ext_chart ? w.ext_chart[e] : CGMLI_CHART_FULL;
            if (chart == CGMLI_CHART_FULL) posePlus(w.extrinsics + 7 * e, delta.data() + lay.ext(e), out.ext.data() + 7 * e);
            else if (chart == CGMLI_CHART_ROTATION_ONLY)
                posePlus(w.extrinsics + 7 * e, delta.data() + lay.ext(e) + 3, out.ext.data() + 7 * e, true);
        }
    if (lay.estTd) out.td = *w.td + delta[lay.td()];
    for (int l = 0; l < lay.L; ++l)
        if (!landmarkFixed(w, l)) out.rho[l] = std::max(w.min_inverse_distance, w.rho[l] + delta[lay.Nr + l]);
    for (double v : out.poses) if (!fin(v)) return false;
    for (double v : out.sb) if (!fin(v)) return false;
    for (double v : out.rho) if (!fin(v)) return false;
    return true;
}
// Robust cost of the window at its current states (no derivatives): the trial
// evaluation of launchTrial (VisualCudaBatch.cu:715-721).
static bool windowCost(const cgmli_window& w, double& cost) {
    cost = 0;
    for (int l = 0; l < w.num_landmarks; ++l)
        for (int f = w.lm_obs_begin[l]; f < w.lm_obs_begin[l + 1]; ++f) {
            Fac o;
            if (!visualFactor(w, l, f, false, o)) return false;
            const double sq = o.r[0] * o.r[0] + o.r[1] * o.r[1];
            if (!fin(sq)) return false;
            cost += huberCost(w.huber_scale, sq);
        }
    for (int i = 0; i < w.num_imu; ++i) {
        const int k = w.imu_kf[i];
        double r[15];
        if (!imuFactor(w.imu[i], w.poses + 7 * k, w.speed_bias + 9 * k, w.poses + 7 * (k + 1), w.speed_bias + 9 * (k + 1), r, nullptr))
            return false;
        for (double v : r) cost += 0.5 * v * v;
    }
    if (w.prior_rank > 0) {
        std::vector<double> r;
        if (!priorFactor(w, r, nullptr)) return false;
        for (double v : r) cost += 0.5 * v * v;
    }
    return fin(cost);
}

// Options of the LM loop beyond the iteration budget: the reference's
// minIterations and realtime budget (BackendOptimizer.cpp:177,242; the oracle
// cannot see the device's clock, so the budget is either elapsed from the start
// or never), and caller-evaluated factors (solveOnline's retainedH / retainedG,
// :210-225, and the host trial cost, :276-279) through the C ABI's callback.
struct LmOptions {
    int minIterations = 0;
    bool budgetElapsed = false;
    cgmli_host_factor_fn host = nullptr;
    void* hostCtx = nullptr;
    int hostWindow = 0;
};
static bool hostLinearize(const cgmli_window& w, const LmOptions& o, Linear& lin) {
    if (!o.host) return true;
    const int n = lin.Nr;
    std::vector<double> H((size_t)n * n, 0.0), g(n, 0.0);
    double cost = 0, td = w.td ? *w.td : 0.0;
    if (o.host(o.hostCtx, o.hostWindow, 0, w.poses, w.speed_bias, w.extrinsics, &td, H.data(), g.data(), &cost) != 0 || !fin(cost))
        return false;
    for (size_t i = 0; i < H.size(); ++i) lin.H[i] += H[i];
    for (int i = 0; i < n; ++i) lin.g[i] += g[i];
    lin.cost += cost;
    return true;
}
static bool hostTrialCost(const cgmli_window& w, const LmOptions& o, double& cost) {
    cost = 0;
    if (!o.host) return true;
    double td = w.td ? *w.td : 0.0;
    return o.host(o.hostCtx, o.hostWindow, 1, w.poses, w.speed_bias, w.extrinsics, &td, nullptr, nullptr, &cost) == 0 && fin(cost);
}

// Resident LM loop of solveVisualSchur (BackendOptimizer.cpp:167-307).
static int lmSolve(cgmli_window& w, int maxIterations, cgmli_solve_report* rep, double initialLambda, int refinement,
                   const LmOptions& opt = LmOptions()) {
    cgmli_solve_report report{};
    double lambda = initialLambda, increase = 2, cost = 0;
    int accepted = 0;
    bool newPoint = true, converged = false;
    Linear lin;
    int it = 0, status = CGMLI_OK;
    for (it = 0; it < maxIterations; ++it) {
        if (it >= opt.minIterations && it > 0 && opt.budgetElapsed) break;
        if (newPoint) {
            if (!linearize(w, lin) || !hostLinearize(w, opt, lin)) { status = CGMLI_E_NONFINITE; break; }
            if (it > 0 && std::fabs(lin.cost - cost) > 1e-8 * std::max(1.0, cost)) { status = CGMLI_E_COST_MISMATCH; break; }
            if (it == 0) report.initial_cost = cost = lin.cost;
        }
        Step st = schurStep(w, lin, lambda, refinement);
        if (st.status != CGMLI_OK) { status = st.status; break; }
        if (it >= opt.minIterations && accepted > 0 && opt.budgetElapsed) break;
        States cand;
        double maxInc = 0, trial = 0;
        bool trialValid = applyStep(w, st.delta, cand, maxInc);
        if (trialValid) {
            cgmli_window cw = w;
            cw.poses = cand.poses.data(); cw.speed_bias = cand.sb.data(); cw.extrinsics = cand.ext.data(); cw.rho = cand.rho.data();
            double tdv = cand.td;
            if (w.td) cw.td = &tdv;
            double host = 0;
            trialValid = windowCost(cw, trial);
            if (trialValid) {
                if (hostTrialCost(cw, opt, host)) trial += host;
                else trial = std::numeric_limits<double>::quiet_NaN();  // a failed host evaluation rejects the step
            }
        }
        report.predicted_reduction = st.predicted;
        report.max_increment = maxInc;
        if (trialValid && maxInc < 1e-10) { converged = true; ++it; break; }
        double gain = -1;
        if (trialValid && st.predicted > 0 && fin(st.predicted)) gain = (cost - trial) / st.predicted;
        if (gain > 1e-3) {
            put(w, cand);
            ++accepted;
            converged = cost - trial <= 1e-6 * std::max(1.0, cost);
            cost = trial;
            lambda = std::max(1e-12, lambda * std::max(1.0 / 3, 1 - std::pow(2 * gain - 1, 3)));
            increase = 2; newPoint = true;
            if (converged) { ++it; break; }
        } else {
            lambda *= increase; increase *= 2; newPoint = false;
        }
    }
    if (status == CGMLI_OK && !accepted && !converged) status = CGMLI_E_NO_STEP;
    report.final_cost = cost;
    report.lambda = lambda;
    report.iterations = it;
    report.accepted_steps = accepted;
    report.converged = converged;
    report.status = status;
    if (rep) *rep = report;
    return status;
}

// Whitened pre-loss NIS gate and outlier refits around the LM loop
// (BackendOptimizer::statisticalGate and the refit loop of optimizeImpl,
// BackendOptimizer.cpp:394-472,1030-1079), visual factors only.  A rejected
// factor leaves the problem: its whitening rows are zeroed in a private copy.
struct GateOut {
    int passes = 0, rejectedPre = 0, evaluated = 0, rejectedLast = 0, rejectedTotal = 0;
    double nisSum = 0, nisMax = 0;
};
static int lmSolveGated(cgmli_window& w, int maxIterations, double threshold, int maxRefits, bool preGate, double initialLambda,
                        int refinement, cgmli_solve_report* rep, GateOut& g, unsigned char* rejected) {
    std::vector<double> P(w.obs_P, w.obs_P + 6 * (size_t)w.num_observations);
    const double* callerP = w.obs_P;
    w.obs_P = P.data();
    // one gate at the current states: statistics of the factors still in the
    // problem, rejection of those above the threshold
    auto gate = [&](int& rejectedNow) -> int {
        g.evaluated = 0; g.nisSum = 0; g.nisMax = 0; rejectedNow = 0;
        for (int l = 0; l < w.num_landmarks; ++l)
            for (int f = w.lm_obs_begin[l]; f < w.lm_obs_begin[l + 1]; ++f) {
                if (rejected[f]) continue;
                Fac o;
                const bool ok = visualFactor(w, l, f, false, o);
                const double energy = o.r[0] * o.r[0] + o.r[1] * o.r[1];
                if (!ok || !fin(energy)) return CGMLI_E_NONFINITE;
                ++g.evaluated;
                g.nisSum += energy;
                g.nisMax = std::max(g.nisMax, energy);
                if (energy > threshold) {
                    rejected[f] = 1;
                    for (int k = 0; k < 6; ++k) P[6 * (size_t)f + k] = 0.0;
                    ++rejectedNow;
                    ++g.rejectedTotal;
                }
            }
        return CGMLI_OK;
    };
    cgmli_solve_report total{};
    int charged = 0, status = CGMLI_OK;
    if (preGate) status = gate(g.rejectedPre);
    for (int pass = 0; pass <= maxRefits && status == CGMLI_OK; ++pass) {
        cgmli_solve_report r{};
        status = lmSolve(w, maxIterations - charged, &r, initialLambda, refinement);
        ++g.passes;
        if (pass == 0) total.initial_cost = r.initial_cost;
        total.final_cost = r.final_cost; total.lambda = r.lambda;
        total.predicted_reduction = r.predicted_reduction; total.max_increment = r.max_increment;
        total.iterations += r.iterations; total.accepted_steps += r.accepted_steps;
        total.converged = r.converged; total.status = status;
        charged += std::max(1, r.iterations);  // every pass costs at least one iteration
        if (status != CGMLI_OK) break;
        status = gate(g.rejectedLast);
        total.status = status;
        if (status != CGMLI_OK || !g.rejectedLast || charged >= maxIterations || pass == maxRefits) break;
    }
    w.obs_P = callerP;
    total.status = status;
    if (rep) *rep = total;
    return status;
}

// ---- marginalization --------------------------------------------------------------
struct MargBlock { int kind, index, size, offset; bool eliminate, landmark; };
struct MargOut {
    int status = CGMLI_OK, rank = 0, nr = 0;
    std::vector<double> Hprior, bprior, A, r0;
    double robustCost = 0, rss = 0, eliminatedReduction = 0, cutoff = 0, newReferenceNorm = 0;
};
// Marginalizer::compute (Marginalizer.cpp:333-473) on a linearized system.
static void marginalizeSystem(int n, const std::vector<double>& H, const std::vector<double>& b,
                              const std::vector<MargBlock>& blocks, MargOut& out, double absCut = 1e-12, double relCut = 1e-9) {
    std::vector<int> m, r, ranges, states;
    for (const auto& bl : blocks) {
        auto& idx = bl.eliminate ? m : r;
        for (int j = 0; j < bl.size; ++j) idx.push_back(bl.offset + j);
    }
    for (const auto& bl : blocks)
        if (bl.eliminate)
            for (int j = 0; j < bl.size; ++j) {
                const int idx = (int)(std::find(m.begin(), m.end(), bl.offset + j) - m.begin());
                (bl.landmark && bl.size == 1 ? ranges : states).push_back(idx);
            }
    int nm = (int)m.size();
    const int nr = (int)r.size();
    out.nr = nr;
    if (!nr) return;
    auto at = [&](int i, int j) { return H[(size_t)i * n + j]; };
    std::vector<double> Hmm((size_t)nm * nm), Hmr((size_t)nm * nr), Hrr((size_t)nr * nr), bm(nm), br(nr);
    for (int i = 0; i < nm; ++i) {
        bm[i] = b[m[i]];
        for (int j = 0; j < nm; ++j) Hmm[(size_t)i * nm + j] = at(m[i], m[j]);
        for (int j = 0; j < nr; ++j) Hmr[(size_t)i * nr + j] = at(m[i], r[j]);
    }
    for (int i = 0; i < nr; ++i) {
        br[i] = b[r[i]];
        for (int j = 0; j < nr; ++j) Hrr[(size_t)i * nr + j] = at(r[i], r[j]);
    }
    const int nl = (int)ranges.size(), ns = (int)states.size();
    if (nl) {
        std::vector<double> Hll((size_t)nl * nl);
        bool diagonal = true;
        for (int i = 0; i < nl; ++i)
            for (int j = 0; j < nl; ++j) {
                Hll[(size_t)i * nl + j] = Hmm[(size_t)ranges[i] * nm + ranges[j]];
                if (i != j && Hll[(size_t)i * nl + j] != 0.0) diagonal = false;
            }
        if (diagonal) {
            const int w = ns + nr;
            std::vector<double> coupling((size_t)nl * w), rhsL((size_t)nl * (w + 1)), solvedL((size_t)nl * (w + 1));
            for (int i = 0; i < nl; ++i) {
                for (int j = 0; j < ns; ++j) coupling[(size_t)i * w + j] = Hmm[(size_t)ranges[i] * nm + states[j]];
                for (int j = 0; j < nr; ++j) coupling[(size_t)i * w + ns + j] = Hmr[(size_t)ranges[i] * nr + j];
                for (int j = 0; j < w; ++j) rhsL[(size_t)i * (w + 1) + j] = coupling[(size_t)i * w + j];
                rhsL[(size_t)i * (w + 1) + w] = bm[ranges[i]];
            }
            const int st = psdSolve(nl, Hll.data(), w + 1, rhsL.data(), absCut, relCut, solvedL.data());
            if (st != CGMLI_OK) { out.status = st; return; }
            for (int i = 0; i < nl; ++i) out.eliminatedReduction += 0.5 * bm[ranges[i]] * solvedL[(size_t)i * (w + 1) + w];
            std::vector<double> reduced((size_t)w * w, 0.0), gradient(w);
            for (int i = 0; i < ns; ++i) {
                gradient[i] = bm[states[i]];
                for (int j = 0; j < ns; ++j) reduced[(size_t)i * w + j] = Hmm[(size_t)states[i] * nm + states[j]];
                for (int j = 0; j < nr; ++j) {
                    reduced[(size_t)i * w + ns + j] = Hmr[(size_t)states[i] * nr + j];
                    reduced[(size_t)(ns + j) * w + i] = Hmr[(size_t)states[i] * nr + j];
                }
            }
            for (int i = 0; i < nr; ++i) {
                gradient[ns + i] = br[i];
                for (int j = 0; j < nr; ++j) reduced[(size_t)(ns + i) * w + ns + j] = Hrr[(size_t)i * nr + j];
            }
            for (int i = 0; i < w; ++i) {
                for (int j = 0; j < w; ++j) {
                    double v = 0;
                    for (int k = 0; k < nl; ++k) v += coupling[(size_t)k * w + i] * solvedL[(size_t)k * (w + 1) + j];
                    reduced[(size_t)i * w + j] -= v;
                }
                double v = 0;
                for (int k = 0; k < nl; ++k) v += coupling[(size_t)k * w + i] * solvedL[(size_t)k * (w + 1) + w];
                gradient[i] -= v;
            }
            Hmm.assign((size_t)ns * ns, 0); Hmr.assign((size_t)ns * nr, 0); bm.assign(ns, 0);
            for (int i = 0; i < ns; ++i) {
                bm[i] = gradient[i];
                for (int j = 0; j < ns; ++j) Hmm[(size_t)i * ns + j] = reduced[(size_t)i * w + j];
                for (int j = 0; j < nr; ++j) Hmr[(size_t)i * nr + j] = reduced[(size_t)i * w + ns + j];
            }
            for (int i = 0; i < nr; ++i) {
                br[i] = gradient[ns + i];
                for (int j = 0; j < nr; ++j) Hrr[(size_t)i * nr + j] = reduced[(size_t)(ns + i) * w + ns + j];
            }
            nm = ns;
        }
    }
    std::vector<double> rhs((size_t)nm * (nr + 1)), solved((size_t)nm * (nr + 1));
    for (int i = 0; i < nm; ++i) {
        for (int j = 0; j < nr; ++j) rhs[(size_t)i * (nr + 1) + j] = Hmr[(size_t)i * nr + j];
        rhs[(size_t)i * (nr + 1) + nr] = bm[i];
    }
    const int st = psdSolve(nm, Hmm.data(), nr + 1, rhs.data(), absCut, relCut, solved.data());
    if (st != CGMLI_OK) { out.status = st; return; }
    for (int i = 0; i < nm; ++i) out.eliminatedReduction += 0.5 * bm[i] * solved[(size_t)i * (nr + 1) + nr];
    for (int i = 0; i < nr; ++i) {
        for (int j = 0; j < nr; ++j) {
            double v = 0;
            for (int k = 0; k < nm; ++k) v += Hmr[(size_t)k * nr + i] * solved[(size_t)k * (nr + 1) + j];
            Hrr[(size_t)i * nr + j] -= v;
        }
        double v = 0;
        for (int k = 0; k < nm; ++k) v += Hmr[(size_t)k * nr + i] * solved[(size_t)k * (nr + 1) + nr];
        br[i] -= v;
    }
    out.Hprior.assign((size_t)nr * nr, 0.0);
    for (int i = 0; i < nr; ++i)
        for (int j = 0; j < nr; ++j) out.Hprior[(size_t)i * nr + j] = 0.5 * (Hrr[(size_t)i * nr + j] + Hrr[(size_t)j * nr + i]);
    out.bprior = br;
    std::vector<double> ev(nr), U((size_t)nr * nr);
    if (!eigenSym(nr, out.Hprior.data(), ev.data(), U.data())) { out.status = CGMLI_E_NONFINITE; return; }
    const double cutoff = std::max(absCut, relCut * std::max(0.0, ev[nr - 1]));
    out.cutoff = cutoff;
    if (ev[0] < -10.0 * cutoff) { out.status = CGMLI_E_INDEFINITE; return; }
    for (int i = 0; i < nr; ++i) if (ev[i] > cutoff) ++out.rank;
    out.A.assign((size_t)out.rank * nr, 0.0);
    out.r0.assign(out.rank, 0.0);
    int row = 0;
    for (int i = 0; i < nr; ++i)
        if (ev[i] > cutoff) {
            const double root = std::sqrt(ev[i]);
            double ub = 0;
            for (int k = 0; k < nr; ++k) { out.A[(size_t)row * nr + k] = root * U[(size_t)k * nr + i]; ub += U[(size_t)k * nr + i] * br[k]; }
            out.r0[row] = ub / root;
            ++row;
        }
    double rn = 0;
    for (double v : out.r0) rn += v * v;
    out.newReferenceNorm = std::sqrt(rn);
}

// Elimination set and consumed factors of SlidingWindowManager::marginalize
// (SlidingWindowManager.cpp:627-652, Marginalizer.cpp:293-315), then
// linearization of the consumed factors with the Huber loss and the prior.
struct WindowMarg {
    MargOut out;
    std::vector<int> sepKind, sepIndex;  // separator blocks in column order
    std::vector<double> sepRef;
    // calibration information (calib mode): conditional in report order, eigenvalues ascending
    std::vector<double> conditional, eigenvalues;
};
static void calibrationConditional(const cgmli_window& w, int n, const std::vector<double>& H, const std::vector<MargBlock>& blocks,
                                   WindowMarg& res);
// calib: the formation of BackendOptimizer::calibrationInformation instead of a
// marginalization: every landmark with observations, every IMU factor and (with
// calibPrior) the prior; poses and speed/biases are the nuisance block.
static void marginalizeWindow(const cgmli_window& w, int victim, int policy, WindowMarg& res, bool skipImu = false, bool calib = false,
                              bool calibPrior = false) {
    const Layout lay(w);
    const int L = lay.L;
    std::vector<char> elim(L, 0), consumeObs(w.num_observations, 0);
    for (int l = 0; l < L; ++l) {
        bool e = calib ? w.lm_obs_begin[l + 1] > w.lm_obs_begin[l] : w.lm_anchor_kf[l] == victim;
        if (policy == CGMLI_MARGIN_OLD && !calib)
            for (int f = w.lm_obs_begin[l]; f < w.lm_obs_begin[l + 1]; ++f) e = e || w.obs_kf[f] == victim;
        elim[l] = e;
        if (e) for (int f = w.lm_obs_begin[l]; f < w.lm_obs_begin[l + 1]; ++f) consumeObs[f] = 1;
    }
    // Blocks touched by consumed factors (and the prior), in column order.
    std::vector<char> poseUsed(lay.K, 0), sbUsed(lay.K, 0), extUsed(lay.E, 0);
    bool tdUsed = false;
    for (int l = 0; l < L; ++l)
        for (int f = w.lm_obs_begin[l]; f < w.lm_obs_begin[l + 1]; ++f)
            if (consumeObs[f]) {
                poseUsed[w.lm_anchor_kf[l]] = 1;
                poseUsed[w.obs_kf[f]] = 1;
                extUsed[w.cam_ext[w.lm_anchor_cam[l]]] = 1;
                extUsed[w.cam_ext[w.obs_cam[f]]] = 1;
                tdUsed = true;
            }
    std::vector<int> imuUsed;
    for (int i = 0; i < w.num_imu && !skipImu; ++i)
        if (calib || w.imu_kf[i] == victim || w.imu_kf[i] + 1 == victim) {
            imuUsed.push_back(i);
            const int k = w.imu_kf[i];
            poseUsed[k] = poseUsed[k + 1] = sbUsed[k] = sbUsed[k + 1] = 1;
        }
    const bool withPrior = (!calib || calibPrior) && w.prior_rank > 0;
    for (int b = 0; b < (withPrior ? w.prior_num_blocks : 0); ++b) {
        const int kind = w.prior_block_kind[b], idx = w.prior_block_index[b];
        if (kind == CGMLI_PRIOR_POSE) poseUsed[idx] = 1;
        else if (kind == CGMLI_PRIOR_SPEED_BIAS) sbUsed[idx] = 1;
        else if (kind == CGMLI_PRIOR_EXTRINSIC) extUsed[idx] = 1;
        else tdUsed = true;
    }
    std::vector<MargBlock> blocks;
    int n = 0;
    std::vector<int> poseCol(lay.K, -1), sbCol(lay.K, -1), extCol(lay.E, -1);
    int tdCol = -1;
    auto addBlock = [&](int kind, int index, int size, bool eliminate) {
        blocks.push_back({kind, index, size, n, eliminate, false});
        const int c = n;
        n += size;
        return c;
    };
    for (int k = 0; k < lay.K; ++k) {
        if (poseUsed[k]) poseCol[k] = addBlock(CGMLI_PRIOR_POSE, k, 6, calib || k == victim);
        if (sbUsed[k]) sbCol[k] = addBlock(CGMLI_PRIOR_SPEED_BIAS, k, 9, calib || k == victim);
    }
    for (int e = 0; e < lay.E; ++e) if (extUsed[e]) extCol[e] = addBlock(CGMLI_PRIOR_EXTRINSIC, e, 6, false);
    if (tdUsed && w.td) tdCol = addBlock(CGMLI_PRIOR_TIME_OFFSET, 0, 1, false);
    std::vector<int> lmCol(L, -1);
    for (int l = 0; l < L; ++l)
        if (elim[l]) { blocks.push_back({-1, l, 1, n, true, true}); lmCol[l] = n++; }
    auto colOfBlock = [&](int kind, int index) {
        switch (kind) {
            case CGMLI_PRIOR_POSE: return poseCol[index];
            case CGMLI_PRIOR_SPEED_BIAS: return sbCol[index];
            case CGMLI_PRIOR_EXTRINSIC: return extCol[index];
            default: return tdCol;
        }
    };
    std::vector<double> H((size_t)n * n, 0.0), b(n, 0.0);
    double robust = 0, rss = 0;
    auto addRows = [&](int rows, const double* J, const int* cols, int m, const double* r) {
        for (int i = 0; i < m; ++i) {
            if (cols[i] < 0) continue;
            double gi = 0;
            for (int k = 0; k < rows; ++k) gi += J[k * m + i] * r[k];
            b[cols[i]] += gi;
            for (int j = 0; j < m; ++j) {
                if (cols[j] < 0) continue;
                double h = 0;
                for (int k = 0; k < rows; ++k) h += J[k * m + i] * J[k * m + j];
                H[(size_t)cols[i] * n + cols[j]] += h;
            }
        }
    };
    for (int l = 0; l < L; ++l)
        for (int f = w.lm_obs_begin[l]; f < w.lm_obs_begin[l + 1]; ++f) {
            if (!consumeObs[f]) continue;
            Fac o;
            if (!visualFactor(w, l, f, true, o, true)) { res.out.status = CGMLI_E_NONFINITE; return; }
            const double sq = o.r[0] * o.r[0] + o.r[1] * o.r[1];
            const double wgt = huberWeight(w.huber_scale, sq);
            robust += huberCost(w.huber_scale, sq);
            rss += wgt * wgt * sq;
            int cols[26];
            double J[52];
            const double* bl[4] = {o.Ja, o.Jb, o.Jea, o.Jeb};
            const int base[4] = {poseCol[o.a], poseCol[o.b], extCol[o.ea], extCol[o.eb]};
            for (int q = 0; q < 4; ++q)
                for (int c = 0; c < 6; ++c) {
                    int col = base[q] < 0 ? -1 : base[q] + c;
                    if (q == 1 && o.a == o.b) col = -1;
                    if (q == 3 && !o.split) col = -1;
                    if (o.same && (q == 0 || q == 2)) col = -1;
                    cols[6 * q + c] = col;
                    for (int k = 0; k < 2; ++k) J[26 * k + 6 * q + c] = wgt * bl[q][6 * k + c];
                }
            cols[24] = tdCol;
            cols[25] = lmCol[l];
            for (int k = 0; k < 2; ++k) { J[26 * k + 24] = wgt * o.Jtd[k]; J[26 * k + 25] = wgt * o.Jrho[k]; }
            const double rw[2] = {wgt * o.r[0], wgt * o.r[1]};
            addRows(2, J, cols, 26, rw);
        }
    for (int i : imuUsed) {
        const int k = w.imu_kf[i];
        double r[15], J[450];
        if (!imuFactor(w.imu[i], w.poses + 7 * k, w.speed_bias + 9 * k, w.poses + 7 * (k + 1), w.speed_bias + 9 * (k + 1), r, J)) {
            res.out.status = CGMLI_E_NONFINITE; return;
        }
        int cols[30];
        for (int c = 0; c < 15; ++c) { cols[c] = poseCol[k] < 0 ? -1 : (c < 6 ? poseCol[k] + c : sbCol[k] + c - 6); cols[15 + c] = c < 6 ? poseCol[k + 1] + c : sbCol[k + 1] + c - 6; }
        addRows(15, J, cols, 30, r);
        for (double v : r) { robust += 0.5 * v * v; rss += v * v; }
    }
    if (withPrior) {
        std::vector<double> r, Jt;
        if (!priorFactor(w, r, &Jt)) { res.out.status = CGMLI_E_NONFINITE; return; }
        std::vector<int> cols;
        for (int bb = 0; bb < w.prior_num_blocks; ++bb) {
            const int kind = w.prior_block_kind[bb], col = colOfBlock(kind, w.prior_block_index[bb]);
            for (int c = 0; c < blockTangent(kind); ++c) cols.push_back(col < 0 ? -1 : col + c);
        }
        addRows(w.prior_rank, Jt.data(), cols.data(), (int)cols.size(), r.data());
        for (double v : r) { robust += 0.5 * v * v; rss += v * v; }
    }
    res.out.robustCost = robust;
    res.out.rss = rss;
    if (calib) {
        for (const auto& bl : blocks)
            if (!bl.eliminate) { res.sepKind.push_back(bl.kind); res.sepIndex.push_back(bl.index); }
        calibrationConditional(w, n, H, blocks, res);
        return;
    }
    marginalizeSystem(n, H, b, blocks, res.out);
    for (const auto& bl : blocks)
        if (!bl.eliminate) {
            res.sepKind.push_back(bl.kind);
            res.sepIndex.push_back(bl.index);
            const double* x = blockValue(w, bl.kind, bl.index);
            res.sepRef.insert(res.sepRef.end(), x, x + blockAmbient(bl.kind));
        }
}
}  // namespace orc

namespace orc {
// BackendOptimizer::calibrationInformation (BackendOptimizer.cpp:1084-1170) on
// the window's full normal matrix H (landmark ranges, nuisance, calibration).
static void calibrationConditional(const cgmli_window& w, int n, const std::vector<double>& H, const std::vector<MargBlock>& blocks,
                                   WindowMarg& res) {
    std::vector<int> ranges, nuisance, calib, report;
    std::vector<int> extOfCol;  // extrinsic index of each calibration column, -1 for td
    for (const auto& bl : blocks) {
        if (bl.landmark) { ranges.push_back(bl.offset); continue; }
        if (bl.eliminate) { for (int j = 0; j < bl.size; ++j) nuisance.push_back(bl.offset + j); continue; }
        const int base = (int)calib.size();
        for (int j = 0; j < bl.size; ++j) {
            calib.push_back(bl.offset + j);
            // [rho, theta] -> [theta, rho]; td as is
            report.push_back(bl.kind == CGMLI_PRIOR_EXTRINSIC ? base + (j < 3 ? 3 + j : j - 3) : base + j);
            extOfCol.push_back(bl.kind == CGMLI_PRIOR_EXTRINSIC ? bl.index : -1);
        }
    }
    const int nx = (int)nuisance.size(), nc = (int)calib.size();
    if (!nc) { res.out.status = CGMLI_E_INVALID; return; }
    auto h = [&](int i, int j) { return H[(size_t)i * n + j]; };
    std::vector<double> Hxx((size_t)nx * nx), Hxc((size_t)nx * nc), Hcc((size_t)nc * nc);
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < nx; ++j) Hxx[(size_t)i * nx + j] = h(nuisance[i], nuisance[j]);
        for (int j = 0; j < nc; ++j) Hxc[(size_t)i * nc + j] = h(nuisance[i], calib[j]);
    }
    for (int i = 0; i < nc; ++i) for (int j = 0; j < nc; ++j) Hcc[(size_t)i * nc + j] = h(calib[i], calib[j]);
    // independent scalar ranges: eliminated one by one above the cutoff
    double dmax = 0;
    for (int r : ranges) dmax = std::max(dmax, h(r, r));
    const double cutoff = std::max(1e-12, 1e-9 * dmax);
    std::vector<double> x(nx), c(nc);
    for (int r : ranges) {
        const double d = h(r, r);
        if (d <= cutoff) continue;
        const double scale = 1.0 / std::sqrt(d);
        for (int j = 0; j < nx; ++j) x[j] = scale * h(r, nuisance[j]);
        for (int j = 0; j < nc; ++j) c[j] = scale * h(r, calib[j]);
        for (int i = 0; i < nx; ++i) {
            for (int j = 0; j < nx; ++j) Hxx[(size_t)i * nx + j] -= x[i] * x[j];
            for (int j = 0; j < nc; ++j) Hxc[(size_t)i * nc + j] -= x[i] * c[j];
        }
        for (int i = 0; i < nc; ++i) for (int j = 0; j < nc; ++j) Hcc[(size_t)i * nc + j] -= c[i] * c[j];
    }
    std::vector<double> solved((size_t)nx * nc, 0.0);
    if (nx) {
        const int st = psdSolve(nx, Hxx.data(), nc, Hxc.data(), 1e-12, 1e-9, solved.data());
        if (st != CGMLI_OK) { res.out.status = st; return; }
    }
    std::vector<double> C((size_t)nc * nc);
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            double v = Hcc[(size_t)i * nc + j];
            for (int k = 0; k < nx; ++k) v -= Hxc[(size_t)k * nc + i] * solved[(size_t)k * nc + j];
            C[(size_t)report[i] * nc + report[j]] = v;
        }
    // basis to [theta, p]: dp = rho - [p]x dtheta under the left SE(3) chart
    std::vector<double> B((size_t)nc * nc, 0.0);
    for (int i = 0; i < nc; ++i) B[(size_t)i * nc + i] = 1.0;
    for (int s0 = 0; s0 < nc; ++s0) {
        const int e = extOfCol[s0];
        if (e < 0 || (s0 > 0 && extOfCol[s0 - 1] == e)) continue;  // block starts only
        const M3 px = skew(ld3(w.extrinsics + 7 * e));
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) B[(size_t)(s0 + 3 + i) * nc + s0 + j] = px[3 * i + j];
    }
    std::vector<double> BtC((size_t)nc * nc, 0.0), Cb((size_t)nc * nc, 0.0);
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            double v = 0;
            for (int k = 0; k < nc; ++k) v += B[(size_t)k * nc + i] * C[(size_t)k * nc + j];
            BtC[(size_t)i * nc + j] = v;
        }
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
            double v = 0;
            for (int k = 0; k < nc; ++k) v += BtC[(size_t)i * nc + k] * B[(size_t)k * nc + j];
            Cb[(size_t)i * nc + j] = v;
        }
    std::vector<double> S((size_t)nc * nc);
    for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) S[(size_t)i * nc + j] = 0.5 * Cb[(size_t)i * nc + j] + 0.5 * Cb[(size_t)j * nc + i];
    std::vector<double> ev(nc), V((size_t)nc * nc);
    if (!eigenSym(nc, S.data(), ev.data(), V.data())) { res.out.status = CGMLI_E_NONFINITE; return; }
    const double cut2 = std::max(1e-12, 1e-9 * std::max(0.0, ev[nc - 1]));
    if (ev[0] < -10 * cut2) { res.out.status = CGMLI_E_INDEFINITE; return; }
    for (double& v : ev) v = std::max(v, 0.0);
    res.eigenvalues = ev;
    res.conditional.assign((size_t)nc * nc, 0.0);
    for (int i = 0; i < nc; ++i)
        for (int j = i; j < nc; ++j) {
            double v = 0;
            for (int k = 0; k < nc; ++k) v += V[(size_t)i * nc + k] * ev[k] * V[(size_t)j * nc + k];
            res.conditional[(size_t)i * nc + j] = res.conditional[(size_t)j * nc + i] = v;
        }
}

// SECOND_NEW with the IMU merge (SlidingWindowManager::prepareEviction,
// SlidingWindowManager.cpp:263-310; mergeBodyImuRecords, BodyImuFactor.cpp:306-388).
// Factor q of the window integrates samples [range[2q], range[2q+1]) of one
// stream from t0[q] to t1[q].  The victim's two edges merge when they are its only
// IMU factors and its speed/bias is not in the prior: the merged factor covers
// [t0(left), t1(right)] at the left keyframe's bias, or, above maxInterval, both
// edges are dropped.  skipImu tells the marginalization to leave the edges out.
struct ImuStream {
    const cgmli_imu_parameters* prm;
    const long long* t;
    const double* m;
    int n;
    const int* range;
    const long long* t0;
    const long long* t1;
    double maxInterval;
    int maxSamples;
};
static int planImuMerge(const cgmli_window& w, int victim, const ImuStream& s, int& state, cgmli_frozen_imu& merged, bool& skipImu) {
    state = CGMLI_IMU_MERGE_BRIDGE;
    skipImu = false;
    int left = -1, right = -1, incident = 0;
    for (int i = 0; i < w.num_imu; ++i) {
        if (w.imu_kf[i] + 1 == victim) { left = i; ++incident; }
        else if (w.imu_kf[i] == victim) { right = i; ++incident; }
    }
    bool sbInPrior = false;
    for (int b = 0; b < w.prior_num_blocks; ++b)
        sbInPrior = sbInPrior || (w.prior_block_kind[b] == CGMLI_PRIOR_SPEED_BIAS && w.prior_block_index[b] == victim);
    if (incident != 2 || left < 0 || right < 0 || sbInPrior || !s.t) return CGMLI_OK;
    const int lb = s.range[2 * left], le = s.range[2 * left + 1], rb = s.range[2 * right], re = s.range[2 * right + 1];
    if (s.t1[left] != s.t0[right] || rb < lb || rb > le || re < le) return CGMLI_E_INVALID;
    skipImu = true;
    if (nsToSec(s.t1[right] - s.t0[left]) > s.maxInterval) {
        state = CGMLI_IMU_MERGE_SUPPRESSED;
        return CGMLI_OK;
    }
    if (re - lb > s.maxSamples) return CGMLI_E_LIMIT;
    state = CGMLI_IMU_MERGE_REINTEGRATED;
    const long long* t = s.t + lb;
    const double* m = s.m + 6 * (size_t)lb;
    if (!imuIntervalValid(t, m, re - lb, s.t0[left], s.t1[right], s.prm->max_sample_gap)) return CGMLI_E_INVALID;
    const double* bias = w.speed_bias + 9 * w.imu_kf[left] + 3;
    if (!preintegrateInterval(*s.prm, t, m, re - lb, s.t0[left], s.t1[right], bias, merged, nullptr)) return CGMLI_E_NONFINITE;
    return CGMLI_OK;
}
}  // namespace orc

// ================================ C ABI (tests / CPU baseline) =================
extern "C" {

int oracle_version(void) { return 1; }

// Conditional calibration information of a window (BackendOptimizer::
// calibrationInformation); sizes first (buffers NULL), then the data.
int oracle_calibration_information(const cgmli_window* w, int include_prior, int* size, int* num_blocks, int* block_kind,
                                   int* block_index, double* conditional, double* eigenvalues) {
    orc::WindowMarg res;
    orc::marginalizeWindow(*w, -1, CGMLI_MARGIN_OLD, res, false, true, include_prior != 0);
    if (res.out.status != CGMLI_OK) return res.out.status;
    *size = (int)res.eigenvalues.size();
    *num_blocks = (int)res.sepKind.size();
    if (block_kind) std::copy(res.sepKind.begin(), res.sepKind.end(), block_kind);
    if (block_index) std::copy(res.sepIndex.begin(), res.sepIndex.end(), block_index);
    if (conditional) std::copy(res.conditional.begin(), res.conditional.end(), conditional);
    if (eigenvalues) std::copy(res.eigenvalues.begin(), res.eigenvalues.end(), eigenvalues);
    return CGMLI_OK;
}

// SECOND_NEW window marginalization with the IMU merge: as
// oracle_marginalize_window, plus the merge outcome (CGMLI_IMU_MERGE_*) and the
// merged factor.
int oracle_marginalize_window_merge(const cgmli_window* w, int victim, const cgmli_imu_parameters* prm, const long long* t,
                                    const double* m, int n, const int* range, const long long* t0, const long long* t1,
                                    double max_interval, int max_samples, int* rank, int* cols, int* num_blocks, int* block_kind,
                                    int* block_index, double* reference, double* A, double* r0, int* state, cgmli_frozen_imu* merged) {
    orc::ImuStream s{prm, t, m, n, range, t0, t1, max_interval, max_samples};
    bool skipImu = false;
    const int st = orc::planImuMerge(*w, victim, s, *state, *merged, skipImu);
    if (st != CGMLI_OK) return st;
    orc::WindowMarg res;
    orc::marginalizeWindow(*w, victim, CGMLI_MARGIN_SECOND_NEW, res, skipImu);
    if (res.out.status != CGMLI_OK) return res.out.status;
    *rank = res.out.rank; *cols = res.out.nr; *num_blocks = (int)res.sepKind.size();
    if (block_kind) std::copy(res.sepKind.begin(), res.sepKind.end(), block_kind);
    if (block_index) std::copy(res.sepIndex.begin(), res.sepIndex.end(), block_index);
    if (reference) std::copy(res.sepRef.begin(), res.sepRef.end(), reference);
    if (A) std::copy(res.out.A.begin(), res.out.A.end(), A);
    if (r0) std::copy(res.out.r0.begin(), res.out.r0.end(), r0);
    return CGMLI_OK;
}

// LM solve with the NIS gate and outlier refits; gate: {passes, rejected
// before the first solve, evaluated by the last gate, rejected by it, rejected
// in total}, nis: {sum, max} of the last gate; rejected: num_observations flags.
int oracle_lm_solve_gated(cgmli_window* w, int max_iterations, double threshold, int max_refits, int pre_gate,
                          cgmli_solve_report* report, int* gate, double* nis, unsigned char* rejected) {
    orc::GateOut g;
    std::vector<unsigned char> mask(w->num_observations, 0);
    const int st = orc::lmSolveGated(*w, max_iterations, threshold, max_refits, pre_gate != 0, 1e-4, 0, report, g, mask.data());
    gate[0] = g.passes; gate[1] = g.rejectedPre; gate[2] = g.evaluated; gate[3] = g.rejectedLast; gate[4] = g.rejectedTotal;
    nis[0] = g.nisSum; nis[1] = g.nisMax;
    std::copy(mask.begin(), mask.end(), rejected);
    return st;
}

// Batched IMU preintegration with the semantics of cgmli_imu_preintegrate
// (status 0, CGMLI_E_INVALID for a malformed interval, CGMLI_E_NONFINITE).
int oracle_imu_preintegrate(const cgmli_imu_parameters* prm, const long long* time_ns, const double* readings, int num_samples,
                            const int* range, const long long* t0, const long long* t1, const double* bias, int count,
                            cgmli_frozen_imu* frozen, double* covariance /* count x 225 row-major, or NULL */) {
    for (int i = 0; i < count; ++i) {
        const int b = range[2 * i], e = range[2 * i + 1];
        if (b < 0 || e > num_samples || e - b < 2) return CGMLI_E_INVALID;
        if (!orc::imuIntervalValid(time_ns + b, readings + 6 * (size_t)b, e - b, t0[i], t1[i], prm->max_sample_gap))
            return CGMLI_E_INVALID;
        if (!orc::preintegrateInterval(*prm, time_ns + b, readings + 6 * (size_t)b, e - b, t0[i], t1[i], bias + 6 * i, frozen[i],
                                       covariance ? covariance + 225 * (size_t)i : nullptr))
            return CGMLI_E_NONFINITE;
    }
    return CGMLI_OK;
}

// Per-factor residual and tangent Jacobians (unweighted).  J: 2 x 26 row-major
// columns [anchor pose 6 | observer pose 6 | ext_a 6 | ext_b 6 | td | rho].
int oracle_visual_factor(const cgmli_window* w, int landmark, int obs, int derivatives, double* r, double* J, int* flags) {
    orc::Fac o;
    const bool ok = orc::visualFactor(*w, landmark, obs, derivatives != 0, o);
    if (!ok) return 0;
    r[0] = o.r[0]; r[1] = o.r[1];
    if (J) {
        const double* bl[4] = {o.Ja, o.Jb, o.Jea, o.Jeb};
        for (int k = 0; k < 2; ++k) {
            for (int q = 0; q < 4; ++q) for (int c = 0; c < 6; ++c) J[26 * k + 6 * q + c] = bl[q][6 * k + c];
            J[26 * k + 24] = o.Jtd[k];
            J[26 * k + 25] = o.Jrho[k];
        }
    }
    if (flags) { flags[0] = o.same; flags[1] = o.split; }
    return 1;
}
int oracle_visual_residual_numeric(const cgmli_window* w, int landmark, int obs, double* r) {
    return orc::visualResidualNumeric(*w, landmark, obs, r) ? 1 : 0;
}
int oracle_imu_factor(const cgmli_frozen_imu* imu, const double* p0, const double* sb0, const double* p1, const double* sb1,
                      double* r, double* J) {
    return orc::imuFactor(*imu, p0, sb0, p1, sb1, r, J) ? 1 : 0;
}
void oracle_pose_plus(const double* x, const double* d, double* y) { orc::posePlus(x, d, y); }
void oracle_pose_minus(const double* x, const double* ref, double* d) { orc::poseMinus(x, ref, d); }
void oracle_chart_derivative(const double* x, const double* ref, int finite_difference, double* D) {
    if (finite_difference) orc::chartDerivativeFD(x, ref, D);
    else { double xi[6]; orc::poseMinus(x, ref, xi); orc::se3LeftJacobianInverse(xi, D); }
}
int oracle_prior_factor(const cgmli_window* w, int finite_difference, double* r, double* J) {
    std::vector<double> rr, JJ;
    if (!orc::priorFactor(*w, rr, J ? &JJ : nullptr, finite_difference != 0)) return 0;
    std::copy(rr.begin(), rr.end(), r);
    if (J) std::copy(JJ.begin(), JJ.end(), J);
    return 1;
}

// Linearization products: H (Nr x Nr), g (Nr + L), d (L), C (L x Nr dense
// cross), cost.  Any output pointer may be NULL.
int oracle_linearize(const cgmli_window* w, double* H, double* g, double* d, double* C, double* cost) {
    orc::Linear lin;
    if (!orc::linearize(*w, lin)) return CGMLI_E_NONFINITE;
    const int n = lin.Nr;
    if (H) std::copy(lin.H.begin(), lin.H.end(), H);
    if (g) std::copy(lin.g.begin(), lin.g.end(), g);
    if (d) std::copy(lin.d.begin(), lin.d.end(), d);
    if (C) {
        std::fill(C, C + (size_t)lin.L * n, 0.0);
        for (int l = 0; l < lin.L; ++l)
            for (size_t i = 0; i < lin.sc[l].size(); ++i) C[(size_t)l * n + lin.sc[l][i]] = lin.sv[l][i];
    }
    if (cost) *cost = lin.cost;
    return CGMLI_OK;
}
// One damped Schur step at lambda from the current states: increment
// (Nr + L), reduced S (Nr x Nr, damped) and rhs, predicted reduction, trial
// cost (NaN when the trial is invalid) and max |increment|.
int oracle_step(const cgmli_window* w, double lambda, int refinement, double* delta, double* S, double* rhs, double* cost,
                double* predicted, double* trial_cost, double* max_increment) {
    orc::Linear lin;
    if (!orc::linearize(*w, lin)) return CGMLI_E_NONFINITE;
    orc::Step st = orc::schurStep(*w, lin, lambda, refinement);
    if (S) std::copy(st.S.begin(), st.S.end(), S);
    if (rhs) std::copy(st.rhs.begin(), st.rhs.end(), rhs);
    if (cost) *cost = lin.cost;
    if (st.status != CGMLI_OK) return st.status;
    std::copy(st.delta.begin(), st.delta.end(), delta);
    if (predicted) *predicted = st.predicted;
    orc::States cand;
    double maxInc = 0, trial = std::numeric_limits<double>::quiet_NaN();
    if (orc::applyStep(*w, st.delta, cand, maxInc)) {
        cgmli_window cw = *w;
        cw.poses = cand.poses.data(); cw.speed_bias = cand.sb.data(); cw.extrinsics = cand.ext.data(); cw.rho = cand.rho.data();
        double tdv = cand.td;
        if (w->td) cw.td = &tdv;
        double c = 0;
        if (orc::windowCost(cw, c)) trial = c;
    }
    if (trial_cost) *trial_cost = trial;
    if (max_increment) *max_increment = maxInc;
    return CGMLI_OK;
}
int oracle_window_cost(const cgmli_window* w, double* cost) { return orc::windowCost(*w, *cost) ? CGMLI_OK : CGMLI_E_NONFINITE; }
int oracle_lm_solve(cgmli_window* w, int max_iterations, double initial_lambda, int refinement, cgmli_solve_report* report) {
    return orc::lmSolve(*w, max_iterations, report, initial_lambda, refinement);
}
// The LM loop with the minimum iterations, a budget elapsed from the start (or
// never) and caller-evaluated factors (fn may be NULL).
int oracle_lm_solve_options(cgmli_window* w, int max_iterations, double initial_lambda, int refinement, int min_iterations,
                            int budget_elapsed, cgmli_host_factor_fn fn, void* ctx, int window_index, cgmli_solve_report* report) {
    orc::LmOptions o;
    o.minIterations = min_iterations;
    o.budgetElapsed = budget_elapsed != 0;
    o.host = fn;
    o.hostCtx = ctx;
    o.hostWindow = window_index;
    return orc::lmSolve(*w, max_iterations, report, initial_lambda, refinement, o);
}
// CPU baseline: LM over many windows on `threads` host threads.
int oracle_lm_solve_batch(cgmli_window* windows, int count, int max_iterations, int threads, cgmli_solve_report* reports) {
    threads = std::max(1, threads);
    std::vector<std::thread> pool;
    std::mutex mu;
    int next = 0, worst = CGMLI_OK;
    auto work = [&]() {
        for (;;) {
            int i;
            { std::lock_guard<std::mutex> g(mu); i = next++; }
            if (i >= count) return;
            const int st = orc::lmSolve(windows[i], max_iterations, reports ? reports + i : nullptr, 1e-4, 0);
            if (st != CGMLI_OK) { std::lock_guard<std::mutex> g(mu); worst = st; }
        }
    };
    for (int t = 0; t < threads; ++t) pool.emplace_back(work);
    for (auto& t : pool) t.join();
    return worst;
}

// Robust normal equations of one residual block (rows x cols, row-major J):
// Ceres' Huber corrector scales r and J by sqrt(rho') (rho'' <= 0), as
// Marginalizer::linearize / accumulateNormalEquations consume them
// (Marginalizer.cpp:18-64,185-198).
int oracle_robust_normal(int rows, int cols, const double* J, const double* r, double huber, double* H, double* g, double* cost,
                         double* rss) {
    double s = 0;
    for (int i = 0; i < rows; ++i) s += r[i] * r[i];
    const double w = orc::huberWeight(huber, s);
    *cost = orc::huberCost(huber, s);
    *rss = w * w * s;
    for (int a = 0; a < cols; ++a) {
        double v = 0;
        for (int i = 0; i < rows; ++i) v += J[(size_t)i * cols + a] * r[i];
        g[a] = w * w * v;
        for (int b = 0; b < cols; ++b) {
            double h = 0;
            for (int i = 0; i < rows; ++i) h += J[(size_t)i * cols + a] * J[(size_t)i * cols + b];
            H[(size_t)a * cols + b] = w * w * h;
        }
    }
    return CGMLI_OK;
}

int oracle_eigen_sym(int n, const double* H, double* evals, double* evecs) {
    return orc::eigenSym(n, H, evals, evecs) ? CGMLI_OK : CGMLI_E_NONFINITE;
}
int oracle_psd_solve(int n, const double* H, int cols, const double* rhs, double abs_cut, double rel_cut, double* x) {
    return orc::psdSolve(n, H, cols, rhs, abs_cut, rel_cut, x);
}
// Marginalizer::compute on a given system.  block_desc: per block
// {size, eliminate, landmark}; blocks are consecutive columns.  Outputs the
// retained Schur information (nr x nr), gradient, A (rank x nr), r0 and the
// formation statistics {eliminated reduction, cutoff, new reference norm}.
int oracle_marginalize_system(int n, const double* H, const double* b, int num_blocks, const int* block_desc, int* rank, int* nr,
                              double* Hprior, double* bprior, double* A, double* r0, double* stats) {
    std::vector<orc::MargBlock> blocks;
    int off = 0;
    for (int i = 0; i < num_blocks; ++i) {
        blocks.push_back({0, i, block_desc[3 * i], off, block_desc[3 * i + 1] != 0, block_desc[3 * i + 2] != 0});
        off += block_desc[3 * i];
    }
    if (off != n) return CGMLI_E_INVALID;
    orc::MargOut out;
    orc::marginalizeSystem(n, std::vector<double>(H, H + (size_t)n * n), std::vector<double>(b, b + n), blocks, out);
    if (out.status != CGMLI_OK) return out.status;
    *rank = out.rank; *nr = out.nr;
    if (Hprior) std::copy(out.Hprior.begin(), out.Hprior.end(), Hprior);
    if (bprior) std::copy(out.bprior.begin(), out.bprior.end(), bprior);
    if (A) std::copy(out.A.begin(), out.A.end(), A);
    if (r0) std::copy(out.r0.begin(), out.r0.end(), r0);
    if (stats) { stats[0] = out.eliminatedReduction; stats[1] = out.cutoff; stats[2] = out.newReferenceNorm; }
    return CGMLI_OK;
}
// Window marginalization.  Sizes first (buffers NULL), then data.
int oracle_marginalize_window(const cgmli_window* w, int victim, int policy, int* rank, int* cols, int* num_blocks, int* block_kind,
                              int* block_index, double* reference, double* Hprior, double* bprior, double* A, double* r0, double* formation) {
    orc::WindowMarg res;
    orc::marginalizeWindow(*w, victim, policy, res);
    if (res.out.status != CGMLI_OK) return res.out.status;
    *rank = res.out.rank; *cols = res.out.nr; *num_blocks = (int)res.sepKind.size();
    if (block_kind) std::copy(res.sepKind.begin(), res.sepKind.end(), block_kind);
    if (block_index) std::copy(res.sepIndex.begin(), res.sepIndex.end(), block_index);
    if (reference) std::copy(res.sepRef.begin(), res.sepRef.end(), reference);
    if (Hprior) std::copy(res.out.Hprior.begin(), res.out.Hprior.end(), Hprior);
    if (bprior) std::copy(res.out.bprior.begin(), res.out.bprior.end(), bprior);
    if (A) std::copy(res.out.A.begin(), res.out.A.end(), A);
    if (r0) std::copy(res.out.r0.begin(), res.out.r0.end(), r0);
    if (formation) {
        formation[0] = res.out.robustCost; formation[1] = res.out.rss;
        formation[2] = res.out.eliminatedReduction; formation[3] = res.out.cutoff;
    }
    return CGMLI_OK;
}
}
