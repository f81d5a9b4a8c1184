// Device math of the sliding-window hot path: small fixed-size algebra, the
// left SE(3) chart, the S^2 inverse-distance bearing factor with tangent
// Jacobians, the frozen IMU factor and the square-root prior chart.
//
// The factor formulas follow src/backend/VisualSphereBatchMath.hpp:29-174
// (residual, log-map series, transport, time-offset derivative) and
// src/backend/GpuRetainedFactorMath.hpp:14-140 (IMU, chart).  Jacobians are
// produced directly in the left tangent [rho, theta] instead of the
// reference's ambient 2x7 rows followed by the PlusJacobian lift
// (VisualCudaBatch.cu:60-71); both give the same numbers up to rounding:
//   anchor pose    [ D, -D [p_W]x ]        observer pose  [ -D, D [p_W]x ]
//   anchor T_BR    [ D R_a, -D R_a [b_a]x ] observer T_BR [ -D R_b, D R_b [o_b]x ]
// with D = reduce * W, p_W the world point, b_a = T_BR * local anchor point and
// o_b the point in the observer body frame.  A shared T_BR sums both sides.
#pragma once
#include <cmath>

namespace cgmli {

struct d3 { double x, y, z; };
struct m3 { double a[9]; };  // row-major
struct qd { double x, y, z, w; };

__device__ __forceinline__ d3 mk(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ d3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator*(double s, d3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double norm(d3 a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ d3 cross(d3 a, d3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ bool finite3(d3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

__device__ __forceinline__ m3 eye3() { return {{1, 0, 0, 0, 1, 0, 0, 0, 1}}; }
__device__ __forceinline__ m3 skew(d3 v) { return {{0, -v.z, v.y, v.z, 0, -v.x, -v.y, v.x, 0}}; }
__device__ __forceinline__ m3 ldm3(const double* p) {
    m3 r;
#pragma unroll
    for (int i = 0; i < 9; ++i) r.a[i] = p[i];
    return r;
}
__device__ __forceinline__ m3 colmajor(const double* p) {
    return {{p[0], p[3], p[6], p[1], p[4], p[7], p[2], p[5], p[8]}};
}
__device__ __forceinline__ m3 mul(const m3& A, const m3& B) {
    m3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.a[3 * i + j] = A.a[3 * i] * B.a[j] + A.a[3 * i + 1] * B.a[3 + j] + A.a[3 * i + 2] * B.a[6 + j];
    return r;
}
__device__ __forceinline__ d3 mv(const m3& A, d3 v) {
    return {A.a[0] * v.x + A.a[1] * v.y + A.a[2] * v.z, A.a[3] * v.x + A.a[4] * v.y + A.a[5] * v.z,
            A.a[6] * v.x + A.a[7] * v.y + A.a[8] * v.z};
}
__device__ __forceinline__ d3 mtv(const m3& A, d3 v) {  // A^T v
    return {A.a[0] * v.x + A.a[3] * v.y + A.a[6] * v.z, A.a[1] * v.x + A.a[4] * v.y + A.a[7] * v.z,
            A.a[2] * v.x + A.a[5] * v.y + A.a[8] * v.z};
}
__device__ __forceinline__ m3 tr(const m3& A) { return {{A.a[0], A.a[3], A.a[6], A.a[1], A.a[4], A.a[7], A.a[2], A.a[5], A.a[8]}}; }
__device__ __forceinline__ m3 madd(const m3& A, const m3& B) { m3 r; for (int i = 0; i < 9; ++i) r.a[i] = A.a[i] + B.a[i]; return r; }
__device__ __forceinline__ m3 msub(const m3& A, const m3& B) { m3 r; for (int i = 0; i < 9; ++i) r.a[i] = A.a[i] - B.a[i]; return r; }
__device__ __forceinline__ m3 mscl(double s, const m3& A) { m3 r; for (int i = 0; i < 9; ++i) r.a[i] = s * A.a[i]; return r; }
__device__ __forceinline__ m3 outer(d3 a, d3 b) {
    return {{a.x * b.x, a.x * b.y, a.x * b.z, a.y * b.x, a.y * b.y, a.y * b.z, a.z * b.x, a.z * b.y, a.z * b.z}};
}

__device__ __forceinline__ qd ldq(const double* p) { return {p[0], p[1], p[2], p[3]}; }
__device__ __forceinline__ double qn2(qd q) { return q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w; }
__device__ __forceinline__ qd qnormalized(qd q) { const double n = sqrt(qn2(q)); return {q.x / n, q.y / n, q.z / n, q.w / n}; }
__device__ __forceinline__ qd qconj(qd q) { return {-q.x, -q.y, -q.z, q.w}; }
__device__ __forceinline__ qd qmul(qd a, qd b) {
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
            a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
__device__ __forceinline__ d3 qvec(qd q) { return {q.x, q.y, q.z}; }
__device__ __forceinline__ m3 qrot(qd q) {
    const double tx = 2 * q.x, ty = 2 * q.y, tz = 2 * q.z, twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
    const double txx = tx * q.x, txy = ty * q.x, txz = tz * q.x, tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
    return {{1 - (tyy + tzz), txy - twz, txz + twy, txy + twz, 1 - (txx + tzz), tyz - twx, txz - twy, tyz + twx, 1 - (txx + tyy)}};
}
__device__ __forceinline__ d3 qapply(qd q, d3 v) {  // unit quaternion rotation
    d3 uv = cross(qvec(q), v);
    uv = 2.0 * uv;
    return v + q.w * uv + cross(qvec(q), uv);
}

// ---- left SE(3) chart (GpuRetainedFactorMath.hpp:14-51) -----------------------------
__device__ __forceinline__ qd rotationExp(d3 angle) {
    const double a = norm(angle);
    const double s = a < 1e-8 ? 0.5 - a * a / 48.0 : sin(0.5 * a) / a;
    return {s * angle.x, s * angle.y, s * angle.z, cos(0.5 * a)};
}
__device__ __forceinline__ m3 rotationJacobian(d3 angle) {
    const double a2 = dot(angle, angle), a = sqrt(a2);
    const m3 w = skew(angle);
    const double c1 = a2 < 1e-10 ? 0.5 - a2 / 24 : (1 - cos(a)) / a2;
    const double c2 = a2 < 1e-10 ? 1.0 / 6 - a2 / 120 : (a - sin(a)) / (a2 * a);
    return madd(madd(eye3(), mscl(c1, w)), mscl(c2, mul(w, w)));
}
__device__ __forceinline__ void posePlus(const double* x, const double* d, double* y) {
    const d3 angle = ld3(d + 3);
    const qd q = rotationExp(angle);
    const d3 p = qapply(q, ld3(x)) + mv(rotationJacobian(angle), ld3(d));
    const qd out = qnormalized(qmul(q, ldq(x + 3)));
    y[0] = p.x; y[1] = p.y; y[2] = p.z; y[3] = out.x; y[4] = out.y; y[5] = out.z; y[6] = out.w;
}
// Rotation-only chart of a rig extrinsic: the translation stays, the rotation
// moves on the left (posePlus with rotationOnly, GpuRetainedFactorMath.hpp:28-37).
__device__ __forceinline__ void posePlusRotation(const double* x, const double* theta, double* y) {
    const qd q = rotationExp(ld3(theta));
    const qd out = qnormalized(qmul(q, ldq(x + 3)));
    y[0] = x[0]; y[1] = x[1]; y[2] = x[2]; y[3] = out.x; y[4] = out.y; y[5] = out.z; y[6] = out.w;
}
__device__ __forceinline__ void poseMinus(const double* x, const double* ref, double* d) {
    qd q = qnormalized(qmul(ldq(x + 3), qconj(ldq(ref + 3))));
    if (q.w < 0) q = {-q.x, -q.y, -q.z, -q.w};
    const double s = norm(qvec(q));
    const d3 theta = (s < 1e-10 ? 2.0 : 2.0 * atan2(s, q.w) / s) * qvec(q);
    const double a2 = dot(theta, theta), a = sqrt(a2);
    const m3 w = skew(theta);
    const double c = a2 < 1e-10 ? 1.0 / 12 + a2 / 720 : (1 - 0.5 * a / tan(0.5 * a)) / a2;
    const d3 p = mv(madd(msub(eye3(), mscl(0.5, w)), mscl(c, mul(w, w))), ld3(x) - qapply(q, ld3(ref)));
    d[0] = p.x; d[1] = p.y; d[2] = p.z; d[3] = theta.x; d[4] = theta.y; d[5] = theta.z;
}
// Inverse SE(3) left Jacobian at xi = [rho, theta] (analytic derivative of the
// prior chart; the reference uses central differences, VisualCudaBatch.cu:234-245).
__device__ inline void se3LeftJacobianInverse(const double* xi, double* D) {
    const d3 rho = ld3(xi), th = ld3(xi + 3);
    const double t2 = dot(th, th), t = sqrt(t2);
    const m3 W = skew(th), R = skew(rho), WW = mul(W, W);
    double c1, c2, c3;
    if (t < 0.1) {
        c1 = 1.0 / 6 - t2 / 120 + t2 * t2 / 5040 - t2 * t2 * t2 / 362880;
        c2 = 1.0 / 24 - t2 / 720 + t2 * t2 / 40320 - t2 * t2 * t2 / 3628800;
        c3 = 0.5 * (c2 - 3 * (1.0 / 120 - t2 / 5040 + t2 * t2 / 362880 - t2 * t2 * t2 / 39916800));
    } else {
        const double s = sin(t), c = cos(t);
        c1 = (t - s) / (t2 * t);
        c2 = (t2 / 2 + c - 1) / (t2 * t2);
        c3 = 0.5 * (c2 + 3 * (t - s - t2 * t / 6) / (t2 * t2 * t));
    }
    const double cj = t2 < 1e-10 ? 1.0 / 12 + t2 / 720 : (1 - 0.5 * t / tan(0.5 * t)) / t2;
    const m3 WR = mul(W, R), RW = mul(R, W), WRW = mul(WR, W);
    m3 Qm = mscl(0.5, R);
    Qm = madd(Qm, mscl(c1, madd(madd(WR, RW), WRW)));
    Qm = madd(Qm, mscl(c2, msub(madd(mul(WW, R), mul(R, WW)), mscl(3, WRW))));
    Qm = madd(Qm, mscl(c3, madd(mul(WRW, W), mul(W, WRW))));
    const m3 Ji = madd(msub(eye3(), mscl(0.5, W)), mscl(cj, WW));
    const m3 top = mscl(-1, mul(mul(Ji, Qm), Ji));
    for (int i = 0; i < 36; ++i) D[i] = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            D[6 * i + j] = Ji.a[3 * i + j];
            D[6 * i + 3 + j] = top.a[3 * i + j];
            D[6 * (i + 3) + 3 + j] = Ji.a[3 * i + j];
        }
}

__device__ __forceinline__ bool validPose(const double* x) {
    for (int i = 0; i < 7; ++i) if (!isfinite(x[i])) return false;
    return x[3] * x[3] + x[4] * x[4] + x[5] * x[5] + x[6] * x[6] > 1e-16;
}
__device__ __forceinline__ bool unitPose(const double* x) {
    const double n = x[3] * x[3] + x[4] * x[4] + x[5] * x[5] + x[6] * x[6];
    return fabs(n - 1) <= 1e-6;
}

// Rotation matrix (row-major) of a pose's normalized quaternion; computed once
// per keyframe and extrinsic per state and read by every factor that uses it.
__device__ __forceinline__ void poseRotation(const double* x, double* R) {
    const m3 m = qrot(qnormalized(ldq(x + 3)));
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = m.a[i];
}

// ---- S^2 bearing factor -------------------------------------------------------------
// Inputs of one factor, gathered by the caller.
struct FactorIn {
    const double* xa;   // anchor pose (7)
    const double* xb;   // observer pose
    const double* xea;  // extrinsic of the anchor camera
    const double* xeb;  // extrinsic of the observer camera
    const double* Ra; const double* Rb; const double* Rea; const double* Reb;  // their rotations (poseRotation)
    const double* Rca; const double* tca;  // fixed T_RC of the anchor camera (row-major)
    const double* Rcb; const double* tcb;
    d3 anchor, anchorVel, measured, measuredVel;
    const double* meas;  // 2x3 sqrtInfo * basis^T
    double rho, td, anchorTime, measuredTime;
    bool sameKf, splitExt, wantExt, wantTd;
};
struct FactorOut {
    double r[2];
    double Ja[12], Jb[12], Jea[12], Jeb[12];  // 2x6 tangent blocks, row-major
    double Jtd[2], Jrho[2];
};

__device__ __forceinline__ d3 timeBearing(d3 b, d3 v, double dt, bool differentiate, d3& derivative) {
    if (!differentiate) {
        const d3 u = dt * v;
        const double angle = norm(u);
        if (angle < 1e-8) { const d3 s = b + u; return (1 / norm(s)) * s; }
        return cos(angle) * b + (sin(angle) / angle) * u;
    }
    const double speed = norm(v), angle = speed * dt;
    if (fabs(angle) < 1e-8) {
        const d3 direction = b + dt * v;
        const double length = norm(direction);
        const d3 unit = (1 / length) * direction;
        derivative = (-1 / length) * (v - dot(unit, v) * unit);
        return unit;
    }
    const double sine = sin(angle), cosine = cos(angle);
    derivative = (speed * sine) * b - cosine * v;
    return cosine * b + (sine / speed) * v;
}

__device__ __forceinline__ void rowTimesM(const double* A, const m3& B, double* out) {  // (2x3)(3x3)
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) out[3 * r + c] = A[3 * r] * B.a[c] + A[3 * r + 1] * B.a[3 + c] + A[3 * r + 2] * B.a[6 + c];
}
// J = sign * [M, -M [v]x] for a 2x3 M
__device__ __forceinline__ void poseBlock(const double* M, d3 v, double sign, double* J) {
    double Ms[6];
    rowTimesM(M, skew(v), Ms);
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) { J[6 * r + c] = sign * M[3 * r + c]; J[6 * r + 3 + c] = -sign * Ms[3 * r + c]; }
}


// The bearing factor: residual and Jacobians in FP64, one straight-line routine.
// Returns false for an invalid factor (the reference's valid = 0).
__device__ inline bool evalBearingFactor(const FactorIn& in, bool derivatives, FactorOut& o) {
    const double rho = in.rho;
    if (!(rho > 0) || !isfinite(rho) || !isfinite(in.td)) return false;
    if (!validPose(in.xa) || !validPose(in.xb) || !validPose(in.xea) || !validPose(in.xeb)) return false;
    const bool same = in.sameKf && !in.splitExt;
    const bool timeDerivative = derivatives && in.wantTd;
    const bool movingAnchor = dot(in.anchorVel, in.anchorVel) > 0, movingMeasured = dot(in.measuredVel, in.measuredVel) > 0;
    d3 ba = (1 / norm(in.anchor)) * in.anchor, bb = (1 / norm(in.measured)) * in.measured, da = {0, 0, 0}, db = {0, 0, 0};
    if (movingAnchor) ba = timeBearing(in.anchor, in.anchorVel, in.anchorTime - in.td, timeDerivative, da);
    if (movingMeasured) bb = timeBearing(in.measured, in.measuredVel, in.measuredTime - in.td, timeDerivative, db);
    if (!finite3(ba) || !finite3(bb)) return false;
    const m3 Rca = ldm3(in.Rca), Rcb = ldm3(in.Rcb);
    const d3 tca = ld3(in.tca), tcb = ld3(in.tcb);
    const d3 local = mv(Rca, (1 / rho) * ba) + tca;
    // Ra and Rb, and the points in the body frames that the pose derivatives need, are
    // formed again where the derivatives are taken (the same operations on the same
    // inputs, so the same values), so that they are not held across the residual
    m3 W, cameraRotation;
    d3 pc;
    if (same) {
        pc = mtv(Rcb, local - tcb);
        cameraRotation = mul(tr(Rcb), Rca);
    } else {
        const m3 Ra = ldm3(in.Ra);
        const m3 Rb = ldm3(in.Rb);
        const m3 Rea = ldm3(in.Rea), Reb = ldm3(in.Reb);
        const d3 tea = ld3(in.xea), teb = ld3(in.xeb);
        W = tr(mul(mul(Rb, Reb), Rcb));
        cameraRotation = mul(W, mul(mul(Ra, Rea), Rca));
        if (!in.splitExt) {
            const d3 separation = ld3(in.xa) - ld3(in.xb);
            const d3 offset = mv(W, (mv(Ra, mv(Rea, tca) + tea) - mv(Rb, mv(Reb, tcb) + teb)) + separation);
            pc = mv(cameraRotation, (1 / rho) * ba) + offset;
        } else {
            const d3 bodyA = mv(Rea, local) + tea;
            const d3 wpt = mv(Ra, bodyA) + ld3(in.xa);
            const d3 ob = mtv(Rb, wpt - ld3(in.xb));
            pc = mtv(Rcb, mtv(Reb, ob - teb) - tcb);
        }
    }
    const double range = norm(pc);
    if (!finite3(pc) || !isfinite(range) || range < 1e-10) return false;
    const d3 n = (1 / range) * pc;
    const double c = fmin(1.0, fmax(-1.0, dot(bb, n))), s = norm(cross(bb, n));
    const double denominator = movingMeasured ? 1 + dot(in.measured, bb) : 2;
    if (c < -1 + 1e-8 || denominator < 1e-8) return false;
    const d3 u = n - c * bb;
    const double d = 1 - c;
    const bool series = c > 0 && s < 1e-3;
    const double theta = series ? 0 : atan2(s, c);
    const double f = s < 1e-8 ? 1.0 : (series ? 1 + d / 3 + 2 * d * d / 15 + 2 * d * d * d / 35 : theta / s);
    const d3 logarithm = f * u;
    double P[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) P[i] = in.meas[i];
    if (movingMeasured) {
        const m3 K = skew(cross(in.measured, bb));
        const m3 transport = madd(madd(eye3(), K), mscl(1 / denominator, mul(K, K)));
        rowTimesM(in.meas, tr(transport), P);
    }
    o.r[0] = P[0] * logarithm.x + P[1] * logarithm.y + P[2] * logarithm.z;
    o.r[1] = P[3] * logarithm.x + P[4] * logarithm.y + P[5] * logarithm.z;
    if (!isfinite(o.r[0]) || !isfinite(o.r[1])) return false;
    if (!derivatives) return true;
    const double g = s < 1e-8 ? 0.0 : (series ? (-1.0 / 3.0 - 4 * d / 15.0 - 6 * d * d / 35.0) : (theta * c - s) / (s * s * s));
    double red[6];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const d3 Pr = {P[3 * r], P[3 * r + 1], P[3 * r + 2]};
        const double Pu = dot(Pr, u), Pb = dot(Pr, bb);
        const d3 proj = f * Pr + (g * Pu - f * Pb) * bb;
        const double pn = dot(proj, n);
        red[3 * r] = (proj.x - pn * n.x) / range;
        red[3 * r + 1] = (proj.y - pn * n.y) / range;
        red[3 * r + 2] = (proj.z - pn * n.z) / range;
    }
    // the derivatives through the camera rotation first (depth, and the anchor-side
    // term of the time offset), so that the rotation is not held further
    const bool tdTerm = timeDerivative && (movingAnchor || movingMeasured);
    double jt0 = 0, jt1 = 0;
    {
        double RC[6];
        rowTimesM(red, cameraRotation, RC);
        const d3 q = (-1 / (rho * rho)) * ba;
        o.Jrho[0] = RC[0] * q.x + RC[1] * q.y + RC[2] * q.z;
        o.Jrho[1] = RC[3] * q.x + RC[4] * q.y + RC[5] * q.z;
        if (!isfinite(o.Jrho[0]) || !isfinite(o.Jrho[1])) return false;
        if (tdTerm) {
            const d3 qt = (1 / rho) * da;
            jt0 = RC[0] * qt.x + RC[1] * qt.y + RC[2] * qt.z;
            jt1 = RC[3] * qt.x + RC[4] * qt.y + RC[5] * qt.z;
        }
    }
#pragma unroll
    for (int i = 0; i < 12; ++i) { o.Ja[i] = 0; o.Jb[i] = 0; o.Jea[i] = 0; o.Jeb[i] = 0; }
    if (!same) {
        // reference checks: unit quaternions of differentiated pose blocks (writePose)
        if (!unitPose(in.xa) || !unitPose(in.xb)) return false;
        double D[6];
        rowTimesM(red, W, D);
        const d3 bodyA = mv(ldm3(in.Rea), mv(ldm3(in.Rca), (1 / rho) * ba) + ld3(in.tca)) + ld3(in.xea);
        const d3 rotated = mv(ldm3(in.Ra), bodyA);
        const d3 world = rotated + ld3(in.xa);
        const d3 observerBody = mtv(ldm3(in.Rb), rotated + (ld3(in.xa) - ld3(in.xb)));
        if (!in.sameKf) {
            poseBlock(D, world, 1.0, o.Ja);
            poseBlock(D, world, -1.0, o.Jb);
        }
        if (in.wantExt) {
            if (!unitPose(in.xea) || !unitPose(in.xeb)) return false;
            double DR[6];
            rowTimesM(D, ldm3(in.Ra), DR);
            poseBlock(DR, bodyA, 1.0, o.Jea);
            rowTimesM(D, ldm3(in.Rb), DR);
            poseBlock(DR, observerBody, -1.0, in.splitExt ? o.Jeb : o.Jb);  // temporarily in Jb when shared
            if (!in.splitExt) {
                // shared extrinsic: sum both sides into Jea, restore the observer pose block
#pragma unroll
                for (int i = 0; i < 12; ++i) o.Jea[i] += o.Jb[i];
                if (!in.sameKf) poseBlock(D, world, -1.0, o.Jb);
                else for (int i = 0; i < 12; ++i) o.Jb[i] = 0;
            }
        }
    }
    o.Jtd[0] = o.Jtd[1] = 0;
    if (tdTerm) {
        const m3 Jb = madd(mscl(f, msub(mscl(-1, outer(bb, n)), mscl(c, eye3()))), mscl(g, outer(u, n)));
        double PJ[6];
        rowTimesM(P, Jb, PJ);
        jt0 = jt0 + PJ[0] * db.x + PJ[1] * db.y + PJ[2] * db.z;
        jt1 = jt1 + PJ[3] * db.x + PJ[4] * db.y + PJ[5] * db.z;
        m3 K = {{0, 0, 0, 0, 0, 0, 0, 0, 0}};
        if (movingMeasured) K = skew(cross(in.measured, bb));
        const m3 dK = skew(cross(in.measured, db));
        const m3 dR = msub(madd(dK, mscl(1 / denominator, madd(mul(dK, K), mul(K, dK)))),
                           mscl(dot(in.measured, db) / (denominator * denominator), mul(K, K)));
        double MdR[6];
        rowTimesM(in.meas, tr(dR), MdR);
        o.Jtd[0] = jt0 + MdR[0] * logarithm.x + MdR[1] * logarithm.y + MdR[2] * logarithm.z;
        o.Jtd[1] = jt1 + MdR[3] * logarithm.x + MdR[4] * logarithm.y + MdR[5] * logarithm.z;
        if (!isfinite(o.Jtd[0]) || !isfinite(o.Jtd[1])) return false;
    }
    return true;
}

__device__ __forceinline__ double huberWeight(double scale, double squared) {
    return scale > 0 && squared > scale * scale ? sqrt(scale / sqrt(squared)) : 1.0;
}
__device__ __forceinline__ double huberCost(double scale, double squared) {
    return scale > 0 && squared > scale * scale ? scale * (sqrt(squared) - 0.5 * scale) : 0.5 * squared;
}

}  // namespace cgmli
