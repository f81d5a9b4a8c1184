// Seeded synthetic sliding windows in the cgmli_window layout.
//
// Stands in for the Hilti 2023 robot replay (not available offline): a
// multi-camera pinhole rig on a smooth trajectory, landmarks tracked across
// cameras and keyframes, Gaussian pixel noise with uniform outliers, and IMU
// samples at 200 Hz synthesized from the trajectory's derivatives and
// preintegrated between keyframes.
//
// Measurement model and whitening follow FrameStore::observation
// (src/backend/FrameStore.cpp:102-125) with the pinhole back-projection of
// src/cameras/PinholeCamera.hpp:778-806.  IMU preintegration follows
// ImuError::redoPreintegration (src/factor/ImuError.cpp:254-462), the
// exported data follows FrozenImu::exportData
// (src/factor/BodyImuFactor.cpp:85-94) and the whitening is
// PseudoInverse::symmSqrtU (src/factor/PseudoInverse.hpp:117-145).
#include "../../include/cgmli_backend.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

namespace {
using V3 = std::array<double, 3>;
using M3 = std::array<double, 9>;  // row-major
struct Qt { double x, y, z, w; };

V3 add(const V3& a, const V3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
V3 scl(double s, const V3& a) { return {s * a[0], s * a[1], s * a[2]}; }
double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double nrm(const V3& a) { return std::sqrt(dot(a, a)); }
V3 cross(const V3& a, const V3& b) { return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}; }
M3 eye() { return {1, 0, 0, 0, 1, 0, 0, 0, 1}; }
M3 mul(const M3& a, const M3& b) {
    M3 r{};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
    return r;
}
V3 mv(const M3& a, const V3& v) {
    return {a[0] * v[0] + a[1] * v[1] + a[2] * v[2], a[3] * v[0] + a[4] * v[1] + a[5] * v[2], a[6] * v[0] + a[7] * v[1] + a[8] * v[2]};
}
M3 tr(const M3& a) { return {a[0], a[3], a[6], a[1], a[4], a[7], a[2], a[5], a[8]}; }
M3 madd(const M3& a, const M3& b) { M3 r; for (int i = 0; i < 9; ++i) r[i] = a[i] + b[i]; return r; }
M3 mscl(double s, const M3& a) { M3 r; for (int i = 0; i < 9; ++i) r[i] = s * a[i]; return r; }
M3 skew(const V3& v) { return {0, -v[2], v[1], v[2], 0, -v[0], -v[1], v[0], 0}; }
M3 Rz(double a) { return {std::cos(a), -std::sin(a), 0, std::sin(a), std::cos(a), 0, 0, 0, 1}; }
M3 Ry(double a) { return {std::cos(a), 0, std::sin(a), 0, 1, 0, -std::sin(a), 0, std::cos(a)}; }
M3 Rx(double a) { return {1, 0, 0, 0, std::cos(a), -std::sin(a), 0, std::sin(a), std::cos(a)}; }
M3 expSO3(const V3& w) {
    const double t = nrm(w);
    const M3 W = skew(w);
    const double a = t < 1e-8 ? 1 - t * t / 6 : std::sin(t) / t;
    const double b = t < 1e-8 ? 0.5 - t * t / 24 : (1 - std::cos(t)) / (t * t);
    return madd(madd(eye(), mscl(a, W)), mscl(b, mul(W, W)));
}
V3 logSO3(const M3& R) {
    const double c = std::max(-1.0, std::min(1.0, 0.5 * (R[0] + R[4] + R[8] - 1)));
    const double t = std::acos(c);
    const V3 v{R[7] - R[5], R[2] - R[6], R[3] - R[1]};
    const double s = t < 1e-8 ? 0.5 : t / (2 * std::sin(t));
    return scl(s, v);
}
Qt quatFromR(const M3& R) {
    const double tr3 = R[0] + R[4] + R[8];
    Qt q;
    if (tr3 > 0) {
        const double s = std::sqrt(tr3 + 1.0) * 2;
        q = {(R[7] - R[5]) / s, (R[2] - R[6]) / s, (R[3] - R[1]) / s, 0.25 * s};
    } else if (R[0] > R[4] && R[0] > R[8]) {
        const double s = std::sqrt(1.0 + R[0] - R[4] - R[8]) * 2;
        q = {0.25 * s, (R[1] + R[3]) / s, (R[2] + R[6]) / s, (R[7] - R[5]) / s};
    } else if (R[4] > R[8]) {
        const double s = std::sqrt(1.0 + R[4] - R[0] - R[8]) * 2;
        q = {(R[1] + R[3]) / s, 0.25 * s, (R[5] + R[7]) / s, (R[2] - R[6]) / s};
    } else {
        const double s = std::sqrt(1.0 + R[8] - R[0] - R[4]) * 2;
        q = {(R[2] + R[6]) / s, (R[5] + R[7]) / s, 0.25 * s, (R[3] - R[1]) / s};
    }
    const double n = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (q.w < 0) return {-q.x / n, -q.y / n, -q.z / n, -q.w / n};
    return {q.x / n, q.y / n, q.z / n, q.w / n};
}
Qt qmul(const Qt& a, const Qt& b) {
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z,
            a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
M3 qrot(const Qt& q) {
    const double tx = 2 * q.x, ty = 2 * q.y, tz = 2 * q.z, twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
    const double txx = tx * q.x, txy = ty * q.x, txz = tz * q.x, tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
    return {1 - (tyy + tzz), txy - twz, txz + twy, txy + twz, 1 - (txx + tzz), tyz - twx, txz - twy, tyz + twx, 1 - (txx + tyy)};
}
// Right Jacobian of SO(3) as used by the preintegration (kinematics/Transformation.hpp:47-62).
M3 rightJacobian(const V3& phi) {
    const double t = nrm(phi);
    const M3 W = skew(phi), W2 = mul(W, W);
    if (t < 1e-4) return madd(madd(eye(), mscl(-0.5, W)), mscl(1.0 / 6.0, W2));
    return madd(madd(eye(), mscl(-(1 - std::cos(t)) / (t * t), W)), mscl((t - std::sin(t)) / (t * t * t), W2));
}
double sinc(double x) {  // ode::sinc (src/factor/ode.hpp:15-27)
    if (std::fabs(x) > 1e-6) return std::sin(x) / x;
    const double x2 = x * x;
    return 1.0 - x2 / 6.0 + x2 * x2 / 120.0 - x2 * x2 * x2 / 5040.0;
}

// Symmetric eigen-decomposition by cyclic Jacobi (n small).
void jacobiEigen(int n, std::vector<double> A, std::vector<double>& ev, std::vector<double>& V) {
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0, total = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) { const double v = A[(size_t)i * n + j] * A[(size_t)i * n + j]; total += v; if (i != j) off += v; }
        if (off <= 1e-32 * total || off == 0) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                if (apq == 0) continue;
                const double tau = (A[(size_t)q * n + q] - A[(size_t)p * n + p]) / (2 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1 + tau * tau));
                const double c = 1 / std::sqrt(1 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - s * akq; A[(size_t)k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - s * aqk; A[(size_t)q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = c * vkp - s * vkq; V[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    ev.resize(n);
    for (int i = 0; i < n; ++i) ev[i] = A[(size_t)i * n + i];
}

struct Params {
    int keyframes, landmarks, cameras, track_min, track_max;
    double outlier_fraction, pixel_sigma, huber;
    int with_imu, with_prior, estimate_extrinsics, per_camera_extrinsics, estimate_td, with_velocity;
    double extrinsic_jitter_m, extrinsic_jitter_rad, init_position_sigma, init_rotation_sigma;
};

struct Trajectory {
    double v0, a[3], w[3], ph[3], yawAmp, yawW, yawPh, pitchAmp, rollAmp, attW[2], attPh[2];
    V3 p(double t) const {
        return {v0 * t + a[0] * std::sin(w[0] * t + ph[0]), a[1] * std::sin(w[1] * t + ph[1]), a[2] * std::sin(w[2] * t + ph[2])};
    }
    V3 v(double t) const {
        return {v0 + a[0] * w[0] * std::cos(w[0] * t + ph[0]), a[1] * w[1] * std::cos(w[1] * t + ph[1]),
                a[2] * w[2] * std::cos(w[2] * t + ph[2])};
    }
    V3 acc(double t) const {
        return {-a[0] * w[0] * w[0] * std::sin(w[0] * t + ph[0]), -a[1] * w[1] * w[1] * std::sin(w[1] * t + ph[1]),
                -a[2] * w[2] * w[2] * std::sin(w[2] * t + ph[2])};
    }
    M3 R(double t) const {
        const V3 vel = v(t);
        const double yaw = std::atan2(vel[1], vel[0]) + yawAmp * std::sin(yawW * t + yawPh);
        const double pitch = pitchAmp * std::sin(attW[0] * t + attPh[0]);
        const double roll = rollAmp * std::sin(attW[1] * t + attPh[1]);
        return mul(mul(Rz(yaw), Ry(pitch)), Rx(roll));
    }
    V3 omegaBody(double t) const {  // body angular rate by central difference of R(t)
        const double h = 1e-5;
        return scl(1 / (2 * h), logSO3(mul(tr(R(t - h)), R(t + h))));
    }
};

struct ImuSample { double t; V3 gyro, acc; };

struct Store {
    cgmli_window w{};
    std::vector<double> poses, sb, ext, rho, td;
    std::vector<double> truePoses, trueSb, trueExt, trueRho;
    double trueTd = 0;
    std::vector<double> camR, camT;
    std::vector<int> camExt, lmKf, lmCam, lmBegin, obsKf, obsCam, imuKf, priorKind, priorIndex;
    std::vector<double> lmBearing, lmVel, obsBearing, obsP, obsVel, priorRef, priorA, priorR0;
    std::vector<cgmli_frozen_imu> imu;
    std::vector<int> obsOutlier;
};

struct Camera { double fx = 350, fy = 350, cx = 360, cy = 270; int width = 720, height = 540; };

// FrameStore::observation: bearing and 2x2 whitening of a pixel (sigma px).
bool whiten(const Camera& cam, double u, double v, double sigma, V3& bearing, double P[6]) {
    const V3 ray{(u - cam.cx) / cam.fx, (v - cam.cy) / cam.fy, 1.0};
    const double rn = nrm(ray);
    bearing = scl(1 / rn, ray);
    // J of the back-projection (3x2): d ray / d pixel
    const double J[6] = {1 / cam.fx, 0, 0, 1 / cam.fy, 0, 0};
    double D[6];  // (I - b b^T) J / |ray|
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 2; ++c) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += ((r == k ? 1.0 : 0.0) - bearing[r] * bearing[k]) * J[2 * k + c];
            D[2 * r + c] = s / rn;
        }
    // sphereBasis (WindowVisualFactor.cpp:324-328)
    const V3 axis = std::fabs(bearing[0]) < 0.8 ? V3{1, 0, 0} : V3{0, 1, 0};
    V3 b0 = sub(axis, scl(dot(bearing, axis), bearing));
    b0 = scl(1 / nrm(b0), b0);
    const V3 b1 = cross(bearing, b0);
    double BD[4];
    for (int c = 0; c < 2; ++c) {
        BD[c] = b0[0] * D[c] + b0[1] * D[2 + c] + b0[2] * D[4 + c];
        BD[2 + c] = b1[0] * D[c] + b1[1] * D[2 + c] + b1[2] * D[4 + c];
    }
    const double s2 = sigma * sigma;
    const double c00 = s2 * (BD[0] * BD[0] + BD[1] * BD[1]);
    const double c01 = s2 * (BD[0] * BD[2] + BD[1] * BD[3]);
    const double c11 = s2 * (BD[2] * BD[2] + BD[3] * BD[3]);
    // LLT, then sqrtInformation = L^-1
    if (!(c00 > 0)) return false;
    const double l00 = std::sqrt(c00), l10 = c01 / l00, t = c11 - l10 * l10;
    if (!(t > 0)) return false;
    const double l11 = std::sqrt(t);
    const double i00 = 1 / l00, i11 = 1 / l11, i10 = -l10 / (l00 * l11);
    // measurement = sqrtInfo * basis^T (2x3)
    for (int k = 0; k < 3; ++k) {
        P[k] = i00 * b0[k];
        P[3 + k] = i10 * b0[k] + i11 * b1[k];
    }
    return true;
}

// ImuError::redoPreintegration restated (ImuError.cpp:254-462), T_BS = identity.
bool preintegrate(const std::vector<ImuSample>& m, double t0, double t1, const double sbLin[9], cgmli_frozen_imu& out) {
    const double sgc = 1.7e-4, sac = 2e-3, sgw = 2e-5, saw = 3e-3, g = 9.81, gmax = 7.8, amax = 176.0;
    Qt Dq{0, 0, 0, 1};
    M3 Cint{}, Cdint{}, cross_{}, dalpha{}, dv{}, dp{};
    V3 aint{0, 0, 0}, adint{0, 0, 0};
    std::array<std::vector<double>, 4> dP;
    for (auto& x : dP) x.assign(225, 0.0);
    double time = t0;
    bool started = false;
    const V3 bg{sbLin[3], sbLin[4], sbLin[5]}, ba{sbLin[6], sbLin[7], sbLin[8]};
    for (size_t it = 0; it + 1 < m.size(); ++it) {
        V3 w0 = m[it].gyro, a0 = m[it].acc, w1 = m[it + 1].gyro, a1 = m[it + 1].acc;
        double next = m[it + 1].t;
        if (next <= time) continue;
        double dt = next - time;
        if (t1 < next) {
            const double interval = next - m[it].t;
            next = t1;
            dt = next - time;
            const double r = dt / interval;
            w1 = add(scl(1 - r, w0), scl(r, w1));
            a1 = add(scl(1 - r, a0), scl(r, a1));
        }
        if (dt <= 0) continue;
        if (!started) {
            started = true;
            const double r = dt / (next - m[it].t);
            w0 = add(scl(r, w0), scl(1 - r, w1));
            a0 = add(scl(r, a0), scl(1 - r, a1));
        }
        double gsat = 1, asat = 1;
        for (int k = 0; k < 3; ++k) {
            if (std::fabs(w0[k]) > gmax || std::fabs(w1[k]) > gmax) gsat = 100;
            if (std::fabs(a0[k]) > amax || std::fabs(a1[k]) > amax) asat = 100;
        }
        const V3 wt = sub(scl(0.5, add(w0, w1)), bg);
        const double th = nrm(wt) * 0.5 * dt;
        const double sc = sinc(th);
        const V3 dqv = scl(sc * 0.5 * dt, wt);
        const Qt dq{dqv[0], dqv[1], dqv[2], std::cos(th)};
        const Qt Dq1 = qmul(Dq, dq);
        const M3 C = qrot(Dq), C1 = qrot(Dq1);
        const V3 at = sub(scl(0.5, add(a0, a1)), ba);
        const M3 CC = madd(C, C1);
        const M3 Cint1 = madd(Cint, mscl(0.5 * dt, CC));
        const V3 aint1 = add(aint, scl(0.5 * dt, mv(CC, at)));
        Cdint = madd(Cdint, madd(mscl(dt, Cint), mscl(0.25 * dt * dt, CC)));
        adint = add(adint, add(scl(dt, aint), scl(0.25 * dt * dt, mv(CC, at))));
        const M3 Jr = rightJacobian(scl(dt, wt));
        dalpha = madd(dalpha, mscl(dt, mul(C1, Jr)));
        const Qt dqi{-dq.x, -dq.y, -dq.z, dq.w};
        const M3 cross1 = madd(mul(qrot(dqi), cross_), mscl(dt, Jr));
        const M3 ax = skew(at);
        const M3 term = madd(mul(mul(C, ax), cross_), mul(mul(C1, ax), cross1));
        const M3 dv1 = madd(dv, mscl(0.5 * dt, term));
        dp = madd(dp, madd(mscl(dt, dv), mscl(0.25 * dt * dt, term)));
        double F[225];
        for (int i = 0; i < 225; ++i) F[i] = (i % 16 == 0) ? 1.0 : 0.0;
        auto setF = [&](int r0, int c0, const M3& M) {
            for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) F[15 * (r0 + i) + c0 + j] = M[3 * i + j];
        };
        setF(0, 3, mscl(-1, skew(add(scl(dt, aint), scl(0.25 * dt * dt, mv(CC, at))))));
        setF(0, 6, mscl(dt, eye()));
        setF(0, 9, madd(mscl(dt, dv), mscl(0.25 * dt * dt, term)));
        setF(0, 12, madd(mscl(-dt, Cint), mscl(0.25 * dt * dt, CC)));
        setF(3, 9, mscl(-dt, C1));
        setF(6, 3, mscl(-1, skew(scl(0.5 * dt, mv(CC, at)))));
        setF(6, 9, mscl(0.5 * dt, term));
        setF(6, 12, mscl(-0.5 * dt, CC));
        double Kd[4][15] = {};
        for (int i = 3; i < 6; ++i) Kd[0][i] = gsat * dt;
        for (int i = 0; i < 3; ++i) Kd[1][i] = 0.5 * dt * dt * dt * asat * asat * asat;
        for (int i = 6; i < 9; ++i) Kd[1][i] = asat * dt;
        for (int i = 9; i < 12; ++i) Kd[2][i] = dt;
        for (int i = 12; i < 15; ++i) Kd[3][i] = dt;
        for (int j = 0; j < 4; ++j) {
            double T[225], N[225];
            for (int r = 0; r < 15; ++r)
                for (int c = 0; c < 15; ++c) {
                    double s = 0;
                    for (int k = 0; k < 15; ++k) s += F[15 * r + k] * dP[j][15 * k + c];
                    T[15 * r + c] = s;
                }
            for (int r = 0; r < 15; ++r)
                for (int c = 0; c < 15; ++c) {
                    double s = 0;
                    for (int k = 0; k < 15; ++k) s += T[15 * r + k] * F[15 * c + k];
                    N[15 * r + c] = s + (r == c ? Kd[j][r] : 0.0);
                }
            std::copy(N, N + 225, dP[j].begin());
        }
        Dq = Dq1; Cint = Cint1; aint = aint1; cross_ = cross1; dv = dv1; time = next;
        if (next == t1) break;
    }
    if (!started) return false;
    std::vector<double> P(225, 0.0);
    const double s2[4] = {sgc * sgc, sac * sac, sgw * sgw, saw * saw};
    for (int j = 0; j < 4; ++j)
        for (int r = 0; r < 15; ++r)
            for (int c = 0; c < 15; ++c) P[15 * r + c] += (0.5 * dP[j][15 * r + c] + 0.5 * dP[j][15 * c + r]) * s2[j];
    std::vector<double> ev, V;
    jacobiEigen(15, P, ev, V);
    const double eps = std::numeric_limits<double>::epsilon();
    const double tol = std::max(eps, eps * 15 * *std::max_element(ev.begin(), ev.end()));
    // W = diag(sqrt(1/lambda)) * V^T, stored column-major
    for (int r = 0; r < 15; ++r) {
        const double s = std::sqrt(ev[r] > tol ? 1 / ev[r] : 1 / tol);
        for (int c = 0; c < 15; ++c) out.whitening[r + 15 * c] = s * V[(size_t)c * 15 + r];
    }
    out.duration = t1 - t0;
    out.gravity = g;
    out.sensor_position[0] = out.sensor_position[1] = out.sensor_position[2] = 0;
    out.sensor_quaternion[0] = out.sensor_quaternion[1] = out.sensor_quaternion[2] = 0;
    out.sensor_quaternion[3] = 1;
    out.delta_quaternion[0] = Dq.x; out.delta_quaternion[1] = Dq.y; out.delta_quaternion[2] = Dq.z; out.delta_quaternion[3] = Dq.w;
    for (int i = 0; i < 3; ++i) { out.delta_velocity[i] = aint[i]; out.delta_position[i] = adint[i]; }
    for (int i = 0; i < 6; ++i) out.reference_bias[i] = sbLin[3 + i];
    auto colmaj = [](const M3& M, double* dst) { for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) dst[r + 3 * c] = M[3 * r + c]; };
    colmaj(dalpha, out.rotation_gyro); colmaj(dv, out.velocity_gyro); colmaj(dp, out.position_gyro);
    colmaj(Cint, out.velocity_accel); colmaj(Cdint, out.position_accel);
    return true;
}

V3 gyroAt(const std::vector<ImuSample>& m, double t) {
    for (size_t i = 0; i + 1 < m.size(); ++i)
        if (m[i + 1].t >= t) {
            const double r = (t - m[i].t) / (m[i + 1].t - m[i].t);
            return add(scl(1 - r, m[i].gyro), scl(r, m[i + 1].gyro));
        }
    return m.back().gyro;
}

void setQuat(double* dst, const M3& R) { const Qt q = quatFromR(R); dst[0] = q.x; dst[1] = q.y; dst[2] = q.z; dst[3] = q.w; }

std::unique_ptr<Store> make(const Params& P, uint64_t seed) {
    std::mt19937_64 rng(seed * 0x9E3779B97F4A7C15ull + 12345);
    std::normal_distribution<double> N01(0.0, 1.0);
    std::uniform_real_distribution<double> U01(0.0, 1.0);
    auto st = std::make_unique<Store>();
    Store& s = *st;
    const int K = P.keyframes, C = P.cameras;
    const Camera cam;
    // Rig: camera c yawed c*360/C deg about body z, 5 cm from the IMU.
    const M3 R0 = {0, 0, 1, -1, 0, 0, 0, -1, 0};
    std::vector<M3> RBC(C);
    std::vector<V3> tBC(C);
    for (int c = 0; c < C; ++c) {
        const double yaw = 2 * M_PI * c / C;
        RBC[c] = mul(Rz(yaw), R0);
        tBC[c] = mv(Rz(yaw), V3{0.05, 0, 0});
    }
    const int E = P.per_camera_extrinsics ? C : 1;
    std::vector<M3> RBR(E), RBRtrue(E);
    std::vector<V3> tBR(E), tBRtrue(E);
    s.camR.resize(9 * C); s.camT.resize(3 * C); s.camExt.resize(C);
    for (int e = 0; e < E; ++e) {
        const int c = P.per_camera_extrinsics ? e : 0;
        RBR[e] = RBC[c]; tBR[e] = tBC[c];
        const V3 dr{P.extrinsic_jitter_rad * N01(rng), P.extrinsic_jitter_rad * N01(rng), P.extrinsic_jitter_rad * N01(rng)};
        const V3 dt{P.extrinsic_jitter_m * N01(rng), P.extrinsic_jitter_m * N01(rng), P.extrinsic_jitter_m * N01(rng)};
        RBRtrue[e] = mul(expSO3(dr), RBC[c]);
        tBRtrue[e] = add(tBC[c], dt);
    }
    for (int c = 0; c < C; ++c) {
        const int e = P.per_camera_extrinsics ? c : 0;
        s.camExt[c] = e;
        // T_RC = T_BR^-1 * T_BC (nominal)
        const M3 R = mul(tr(RBR[e]), RBC[c]);
        const V3 t = mv(tr(RBR[e]), sub(tBC[c], tBR[e]));
        for (int i = 0; i < 9; ++i) s.camR[9 * c + i] = R[i];
        for (int i = 0; i < 3; ++i) s.camT[3 * c + i] = t[i];
    }
    // True camera poses in body: T_BR_true * T_RC.
    std::vector<M3> RBCt(C);
    std::vector<V3> tBCt(C);
    for (int c = 0; c < C; ++c) {
        const int e = s.camExt[c];
        const M3 Rrc{s.camR[9 * c], s.camR[9 * c + 1], s.camR[9 * c + 2], s.camR[9 * c + 3], s.camR[9 * c + 4],
                     s.camR[9 * c + 5], s.camR[9 * c + 6], s.camR[9 * c + 7], s.camR[9 * c + 8]};
        RBCt[c] = mul(RBRtrue[e], Rrc);
        tBCt[c] = add(mv(RBRtrue[e], V3{s.camT[3 * c], s.camT[3 * c + 1], s.camT[3 * c + 2]}), tBRtrue[e]);
    }
    // Trajectory: ~1 m/s, keyframes 0.3 s apart (0.3 m, < 5 deg).
    Trajectory tj;
    tj.v0 = 1.0;
    for (int i = 0; i < 3; ++i) { tj.w[i] = 0.4 + 0.4 * U01(rng); tj.ph[i] = 2 * M_PI * U01(rng); }
    tj.a[0] = 0.05; tj.a[1] = 0.4 + 0.3 * U01(rng); tj.a[2] = 0.1;
    tj.yawAmp = 0.05; tj.yawW = 0.7 + 0.3 * U01(rng); tj.yawPh = 2 * M_PI * U01(rng);
    tj.pitchAmp = 0.03; tj.rollAmp = 0.03;
    for (int i = 0; i < 2; ++i) { tj.attW[i] = 0.8 + 0.5 * U01(rng); tj.attPh[i] = 2 * M_PI * U01(rng); }
    const double dtk = 0.3;
    std::vector<double> tk(K);
    for (int k = 0; k < K; ++k) tk[k] = 1.0 + dtk * k;
    std::vector<M3> Rwb(K);
    std::vector<V3> pwb(K);
    for (int k = 0; k < K; ++k) { Rwb[k] = tj.R(tk[k]); pwb[k] = tj.p(tk[k]); }
    // IMU truth: constant biases plus a random walk at 200 Hz.
    V3 bg{2e-3 * N01(rng), 2e-3 * N01(rng), 2e-3 * N01(rng)}, ba{2e-2 * N01(rng), 2e-2 * N01(rng), 2e-2 * N01(rng)};
    std::vector<ImuSample> imu;
    std::vector<V3> bgAt, baAt;
    const double rate = 200.0, h = 1.0 / rate;
    for (double t = tk[0] - 0.05; t <= tk[K - 1] + 0.05 + 1e-12; t += h) {
        const M3 R = tj.R(t);
        const V3 aW = add(tj.acc(t), V3{0, 0, 9.81});
        ImuSample smp;
        smp.t = t;
        smp.gyro = add(add(tj.omegaBody(t), bg), scl(1.7e-4 * std::sqrt(rate), V3{N01(rng), N01(rng), N01(rng)}));
        smp.acc = add(add(mv(tr(R), aW), ba), scl(2e-3 * std::sqrt(rate), V3{N01(rng), N01(rng), N01(rng)}));
        imu.push_back(smp);
        bgAt.push_back(bg); baAt.push_back(ba);
        bg = add(bg, scl(2e-5 * std::sqrt(h), V3{N01(rng), N01(rng), N01(rng)}));
        ba = add(ba, scl(3e-3 * std::sqrt(h), V3{N01(rng), N01(rng), N01(rng)}));
    }
    auto biasAt = [&](double t, V3& g, V3& a) {
        size_t i = (size_t)std::max(0.0, std::min((double)imu.size() - 1, std::round((t - imu[0].t) / h)));
        g = bgAt[i]; a = baAt[i];
    };
    // True states.
    s.truePoses.resize(7 * K); s.trueSb.resize(9 * K);
    for (int k = 0; k < K; ++k) {
        for (int i = 0; i < 3; ++i) s.truePoses[7 * k + i] = pwb[k][i];
        setQuat(&s.truePoses[7 * k + 3], Rwb[k]);
        const V3 v = tj.v(tk[k]);
        V3 g, a;
        biasAt(tk[k], g, a);
        for (int i = 0; i < 3; ++i) { s.trueSb[9 * k + i] = v[i]; s.trueSb[9 * k + 3 + i] = g[i]; s.trueSb[9 * k + 6 + i] = a[i]; }
    }
    s.trueExt.resize(7 * E);
    for (int e = 0; e < E; ++e) {
        for (int i = 0; i < 3; ++i) s.trueExt[7 * e + i] = tBRtrue[e][i];
        setQuat(&s.trueExt[7 * e + 3], RBRtrue[e]);
    }
    // Landmarks and tracks.  Camera poses at keyframe times (and +-1 ms for
    // bearing velocities) are computed once.
    std::vector<M3> Rwc((size_t)K * C), Rwp((size_t)K * C), Rwm((size_t)K * C);
    std::vector<V3> twc((size_t)K * C), twp((size_t)K * C), twm((size_t)K * C);
    const double ve = 1e-3;
    for (int k = 0; k < K; ++k) {
        const M3 Rp = tj.R(tk[k] + ve), Rm = tj.R(tk[k] - ve);
        const V3 pp = tj.p(tk[k] + ve), pm = tj.p(tk[k] - ve);
        for (int c = 0; c < C; ++c) {
            const size_t i = (size_t)k * C + c;
            Rwc[i] = mul(Rwb[k], RBCt[c]); twc[i] = add(mv(Rwb[k], tBCt[c]), pwb[k]);
            Rwp[i] = mul(Rp, RBCt[c]); twp[i] = add(mv(Rp, tBCt[c]), pp);
            Rwm[i] = mul(Rm, RBCt[c]); twm[i] = add(mv(Rm, tBCt[c]), pm);
        }
    }
    auto camPose = [&](int k, int c, M3& R, V3& t) { R = Rwc[(size_t)k * C + c]; t = twc[(size_t)k * C + c]; };
    auto project = [&](const V3& pW, int k, int c, double& u, double& v, V3& pc) {
        const size_t i = (size_t)k * C + c;
        pc = mv(tr(Rwc[i]), sub(pW, twc[i]));
        if (pc[2] < 0.1) return false;
        u = cam.fx * pc[0] / pc[2] + cam.cx;
        v = cam.fy * pc[1] / pc[2] + cam.cy;
        return u >= 0 && v >= 0 && u < cam.width && v < cam.height;
    };
    auto bearingVelocity = [&](const V3& pW, int k, int c) {
        // d/dt of the unit bearing at keyframe time, from the true motion.
        const size_t i = (size_t)k * C + c;
        const V3 a = mv(tr(Rwp[i]), sub(pW, twp[i])), b = mv(tr(Rwm[i]), sub(pW, twm[i]));
        return scl(1 / (2 * ve), sub(scl(1 / nrm(a), a), scl(1 / nrm(b), b)));
    };
    const double sigma = P.pixel_sigma;
    s.lmBegin.push_back(0);
    int made = 0, attempts = 0;
    while (made < P.landmarks && attempts < 50 * P.landmarks + 1000) {
        ++attempts;
        const int a = std::min(K - 1, (int)(U01(rng) * K)), ca = std::min(C - 1, (int)(U01(rng) * C));
        const double u0 = U01(rng) * cam.width, v0 = U01(rng) * cam.height;
        const double dist = 2 + 13 * U01(rng);
        const V3 ray{(u0 - cam.cx) / cam.fx, (v0 - cam.cy) / cam.fy, 1.0};
        const V3 bc = scl(1 / nrm(ray), ray);
        M3 Ra; V3 ta;
        camPose(a, ca, Ra, ta);
        const V3 pW = add(mv(Ra, scl(dist, bc)), ta);
        struct Cand { int k, c; double u, v; double order; };
        std::vector<Cand> cands;
        for (int k = 0; k < K; ++k)
            for (int c = 0; c < C; ++c) {
                if (k == a && c == ca) continue;
                double u, v; V3 pc;
                if (!project(pW, k, c, u, v, pc)) continue;
                cands.push_back({k, c, u, v, std::abs(k - a) + 0.5 * U01(rng)});
            }
        if (cands.empty()) continue;
        const int track = P.track_min + (int)(U01(rng) * (P.track_max - P.track_min + 1));
        std::sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) { return x.order < y.order; });
        const int nobs = std::min((int)cands.size(), std::max(1, track - 1));
        cands.resize(nobs);
        std::sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) { return x.k != y.k ? x.k < y.k : x.c < y.c; });
        // anchor measurement (inlier noise only)
        V3 ab; double Pa[6];
        if (!whiten(cam, std::min(cam.width - 1e-3, std::max(0.0, u0 + sigma * N01(rng))),
                    std::min(cam.height - 1e-3, std::max(0.0, v0 + sigma * N01(rng))), sigma, ab, Pa)) continue;
        s.lmKf.push_back(a); s.lmCam.push_back(ca);
        for (int i = 0; i < 3; ++i) s.lmBearing.push_back(ab[i]);
        // bearing velocities are tangent to the measured bearing (the factor's
        // time model moves the measured ray along a great circle)
        auto tangent = [](const V3& v, const V3& b) { return sub(v, scl(dot(v, b), b)); };
        const V3 av = P.with_velocity ? tangent(bearingVelocity(pW, a, ca), ab) : V3{0, 0, 0};
        for (int i = 0; i < 3; ++i) s.lmVel.push_back(av[i]);
        s.trueRho.push_back(1.0 / dist);
        s.rho.push_back((1.0 / dist) * std::max(0.2, 1 + 0.05 * N01(rng)));
        for (const auto& cd : cands) {
            double u = cd.u, v = cd.v;
            const bool outlier = U01(rng) < P.outlier_fraction;
            if (outlier) { u = U01(rng) * cam.width; v = U01(rng) * cam.height; }
            else {
                u = std::min(cam.width - 1e-3, std::max(0.0, u + sigma * N01(rng)));
                v = std::min(cam.height - 1e-3, std::max(0.0, v + sigma * N01(rng)));
            }
            V3 b; double Pm[6];
            whiten(cam, u, v, sigma, b, Pm);
            s.obsKf.push_back(cd.k); s.obsCam.push_back(cd.c);
            for (int i = 0; i < 3; ++i) s.obsBearing.push_back(b[i]);
            for (int i = 0; i < 6; ++i) s.obsP.push_back(Pm[i]);
            const V3 bv = P.with_velocity ? tangent(bearingVelocity(pW, cd.k, cd.c), b) : V3{0, 0, 0};
            for (int i = 0; i < 3; ++i) s.obsVel.push_back(bv[i]);
            s.obsOutlier.push_back(outlier);
        }
        s.lmBegin.push_back((int)s.obsKf.size());
        ++made;
    }
    const int L = made;
    // Initial estimate: perturbed poses, nominal extrinsics, zero biases.
    s.poses.resize(7 * K); s.sb.resize(9 * K);
    for (int k = 0; k < K; ++k) {
        const V3 dp{P.init_position_sigma * N01(rng), P.init_position_sigma * N01(rng), P.init_position_sigma * N01(rng)};
        const V3 dr{P.init_rotation_sigma * N01(rng), P.init_rotation_sigma * N01(rng), P.init_rotation_sigma * N01(rng)};
        for (int i = 0; i < 3; ++i) s.poses[7 * k + i] = pwb[k][i] + dp[i];
        setQuat(&s.poses[7 * k + 3], mul(expSO3(dr), Rwb[k]));
        for (int i = 0; i < 3; ++i) s.sb[9 * k + i] = s.trueSb[9 * k + i] + 0.05 * N01(rng);
        for (int i = 3; i < 9; ++i) s.sb[9 * k + i] = 0.0;
    }
    s.ext.resize(7 * E);
    for (int e = 0; e < E; ++e) {
        for (int i = 0; i < 3; ++i) s.ext[7 * e + i] = tBR[e][i];
        setQuat(&s.ext[7 * e + 3], RBR[e]);
    }
    s.trueTd = 0.0;
    s.td.assign(1, P.estimate_td ? 0.002 : 0.0);
    // IMU factors, preintegrated at the initial bias estimate.
    if (P.with_imu)
        for (int k = 0; k + 1 < K; ++k) {
            std::vector<ImuSample> seg;
            for (size_t i = 0; i < imu.size(); ++i)
                if (imu[i].t >= tk[k] - 2 * h && imu[i].t <= tk[k + 1] + 2 * h) seg.push_back(imu[i]);
            cgmli_frozen_imu f{};
            if (!preintegrate(seg, tk[k], tk[k + 1], &s.sb[9 * k], f)) continue;
            const V3 g0 = gyroAt(imu, tk[k]), g1 = gyroAt(imu, tk[k + 1]);
            for (int i = 0; i < 3; ++i) { f.gyros[i] = g0[i]; f.gyros[3 + i] = g1[i]; }
            s.imu.push_back(f);
            s.imuKf.push_back(k);
        }
    // Seeded square-root prior over the oldest keyframe's pose and speed/bias,
    // the second keyframe's pose, and the calibration blocks: the separator
    // that an OLD marginalization leaves behind.
    if (P.with_prior && K >= 2) {
        std::vector<int> kind{CGMLI_PRIOR_POSE, CGMLI_PRIOR_SPEED_BIAS, CGMLI_PRIOR_POSE}, index{0, 0, 1};
        std::vector<double> sig{0.01, 0.01, 0.01, 0.004, 0.004, 0.004, 0.05, 0.05, 0.05, 0.003, 0.003, 0.003, 0.03, 0.03, 0.03,
                                0.02, 0.02, 0.02, 0.006, 0.006, 0.006};
        if (P.estimate_extrinsics)
            for (int e = 0; e < E; ++e) {
                kind.push_back(CGMLI_PRIOR_EXTRINSIC); index.push_back(e);
                for (int i = 0; i < 3; ++i) sig.push_back(0.005);
                for (int i = 0; i < 3; ++i) sig.push_back(0.003);
            }
        if (P.estimate_td) { kind.push_back(CGMLI_PRIOR_TIME_OFFSET); index.push_back(0); sig.push_back(0.002); }
        const int n = (int)sig.size();
        // A = diag(1/sigma) * (I + 0.3 * G / sqrt(n)), G Gaussian (5 mixing rounds).
        std::vector<double> A((size_t)n * n, 0.0);
        for (int i = 0; i < n; ++i) A[(size_t)i * n + i] = 1.0;
        for (int round = 0; round < 5; ++round) {
            std::vector<double> G((size_t)n * n);
            for (auto& x : G) x = 0.3 * N01(rng) / std::sqrt((double)n);
            std::vector<double> B((size_t)n * n, 0.0);
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) {
                    double v = A[(size_t)i * n + j];
                    for (int k2 = 0; k2 < n; ++k2) v += G[(size_t)i * n + k2] * A[(size_t)k2 * n + j] * 0.2;
                    B[(size_t)i * n + j] = v;
                }
            A.swap(B);
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) A[(size_t)i * n + j] /= sig[j];
        // reference = current estimate; r0 = -A (x_true [-] x_ref) + N(0,1)
        std::vector<double> delta;
        for (size_t b = 0; b < kind.size(); ++b) {
            const double* x; const double* xt; int amb;
            if (kind[b] == CGMLI_PRIOR_POSE) { x = &s.poses[7 * index[b]]; xt = &s.truePoses[7 * index[b]]; amb = 7; }
            else if (kind[b] == CGMLI_PRIOR_SPEED_BIAS) { x = &s.sb[9 * index[b]]; xt = &s.trueSb[9 * index[b]]; amb = 9; }
            else if (kind[b] == CGMLI_PRIOR_EXTRINSIC) { x = &s.ext[7 * index[b]]; xt = &s.trueExt[7 * index[b]]; amb = 7; }
            else { x = &s.td[0]; xt = &s.trueTd; amb = 1; }
            s.priorRef.insert(s.priorRef.end(), x, x + amb);
            if (amb == 7) {  // small-angle chart of x_true relative to x_ref
                const Qt qt{xt[3], xt[4], xt[5], xt[6]}, qr{x[3], x[4], x[5], x[6]};
                const Qt dq = qmul(qt, Qt{-qr.x, -qr.y, -qr.z, qr.w});
                const V3 th = logSO3(qrot(dq));
                const V3 dpos = sub(V3{xt[0], xt[1], xt[2]}, mv(qrot(dq), V3{x[0], x[1], x[2]}));
                for (int i = 0; i < 3; ++i) delta.push_back(dpos[i]);
                for (int i = 0; i < 3; ++i) delta.push_back(th[i]);
            } else {
                for (int i = 0; i < amb; ++i) delta.push_back(xt[i] - x[i]);
            }
        }
        s.priorA = A;
        s.priorR0.assign(n, 0.0);
        for (int i = 0; i < n; ++i) {
            double v = N01(rng);
            for (int j = 0; j < n; ++j) v -= A[(size_t)i * n + j] * delta[j];
            s.priorR0[i] = v;
        }
        s.priorKind = kind; s.priorIndex = index;
    }
    // Assemble the window view.
    cgmli_window& w = s.w;
    w.num_keyframes = K; w.num_cameras = C; w.num_extrinsics = E;
    w.estimate_extrinsics = P.estimate_extrinsics; w.estimate_td = P.estimate_td;
    w.num_landmarks = L; w.num_observations = (int)s.obsKf.size(); w.num_imu = (int)s.imu.size();
    w.prior_rank = (int)s.priorR0.size(); w.prior_num_blocks = (int)s.priorKind.size();
    w.huber_scale = P.huber; w.min_inverse_distance = 1e-8;
    w.poses = s.poses.data(); w.speed_bias = s.sb.data(); w.extrinsics = s.ext.data(); w.td = s.td.data(); w.rho = s.rho.data();
    w.cam_R = s.camR.data(); w.cam_t = s.camT.data(); w.cam_ext = s.camExt.data();
    w.lm_anchor_kf = s.lmKf.data(); w.lm_anchor_cam = s.lmCam.data(); w.lm_obs_begin = s.lmBegin.data();
    w.lm_anchor_bearing = s.lmBearing.data();
    w.lm_anchor_velocity = P.with_velocity ? s.lmVel.data() : nullptr;
    w.lm_anchor_time = nullptr;
    w.obs_kf = s.obsKf.data(); w.obs_cam = s.obsCam.data(); w.obs_bearing = s.obsBearing.data(); w.obs_P = s.obsP.data();
    w.obs_velocity = P.with_velocity ? s.obsVel.data() : nullptr;
    w.obs_time = nullptr;
    w.imu = s.imu.empty() ? nullptr : s.imu.data(); w.imu_kf = s.imuKf.empty() ? nullptr : s.imuKf.data();
    w.prior_block_kind = s.priorKind.empty() ? nullptr : s.priorKind.data();
    w.prior_block_index = s.priorIndex.empty() ? nullptr : s.priorIndex.data();
    w.prior_ref = s.priorRef.empty() ? nullptr : s.priorRef.data();
    w.prior_A = s.priorA.empty() ? nullptr : s.priorA.data();
    w.prior_r0 = s.priorR0.empty() ? nullptr : s.priorR0.data();
    return st;
}
}  // namespace

extern "C" {
typedef struct cgmli_synth_params {
    int keyframes, landmarks, cameras, track_min, track_max;
    double outlier_fraction, pixel_sigma, huber;
    int with_imu, with_prior, estimate_extrinsics, per_camera_extrinsics, estimate_td, with_velocity;
    double extrinsic_jitter_m, extrinsic_jitter_rad, init_position_sigma, init_rotation_sigma;
} cgmli_synth_params;

void* cgmli_synth_make(const cgmli_synth_params* p, unsigned long long seed) {
    Params P;
    std::memcpy(&P, p, sizeof(Params));
    static_assert(sizeof(Params) == sizeof(cgmli_synth_params), "layout");
    return make(P, seed).release();
}
void cgmli_synth_free(void* h) { delete static_cast<Store*>(h); }
cgmli_window* cgmli_synth_window(void* h) { return &static_cast<Store*>(h)->w; }
// Ground truth: poses (K*7), speed/bias (K*9), extrinsics (E*7), rho (L), td (1).
void cgmli_synth_truth(void* h, double* poses, double* sb, double* ext, double* rho, double* td) {
    const Store& s = *static_cast<Store*>(h);
    if (poses) std::copy(s.truePoses.begin(), s.truePoses.end(), poses);
    if (sb) std::copy(s.trueSb.begin(), s.trueSb.end(), sb);
    if (ext) std::copy(s.trueExt.begin(), s.trueExt.end(), ext);
    if (rho) std::copy(s.trueRho.begin(), s.trueRho.end(), rho);
    if (td) *td = s.trueTd;
}
// Per observation: 1 if the synthetic measurement is an outlier.
void cgmli_synth_outliers(void* h, int* flags) {
    const Store& s = *static_cast<Store*>(h);
    std::copy(s.obsOutlier.begin(), s.obsOutlier.end(), flags);
}
}
