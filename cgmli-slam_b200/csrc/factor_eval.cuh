// Device evaluators shared by the LM kernels and the marginalization kernels:
// gathering of a bearing factor's inputs, the frozen IMU factor and the
// parameter-block accessor used by the prior.
#pragma once
#include "../../include/cgmli_backend.h"
#include "backend_internal.h"
#include "device_math.cuh"

namespace cgmli {

// Gathers the inputs of observation f of landmark l from state buffer `buf`.
__device__ __forceinline__ void gatherFactor(const DevBatch& B, const WinDesc& wd, int wdx, int l, int f, int buf, FactorIn& in,
                                             int& kfa, int& kfb, int& ea, int& eb) {
    kfa = B.lmKf[l];
    kfb = B.obKf[f];
    const int cama = B.lmCam[l], camb = B.obCam[f];
    ea = B.camExt[cama];
    eb = B.camExt[camb];
    in.xa = B.pose[buf] + 7ll * kfa;
    in.xb = B.pose[buf] + 7ll * kfb;
    in.xea = B.ext[buf] + 7ll * ea;
    in.xeb = B.ext[buf] + 7ll * eb;
    in.Ra = B.rotKf[buf] + 9ll * kfa;
    in.Rb = B.rotKf[buf] + 9ll * kfb;
    in.Rea = B.rotExt[buf] + 9ll * ea;
    in.Reb = B.rotExt[buf] + 9ll * eb;
    in.Rca = B.camR + 9ll * cama; in.tca = B.camT + 3ll * cama;
    in.Rcb = B.camR + 9ll * camb; in.tcb = B.camT + 3ll * camb;
    in.anchor = ld3(B.lmBearing + 3ll * l);
    in.anchorVel = ld3(B.lmVel + 3ll * l);
    in.measured = ld3(B.obBearing + 3ll * f);
    in.measuredVel = ld3(B.obVel + 3ll * f);
    in.meas = B.obP + 6ll * f;
    in.rho = B.rho[buf][l];
    in.anchorTime = B.lmTime[l];
    in.measuredTime = B.obTime[f];
    in.td = wd.hasTd ? B.td[buf][wdx] : in.anchorTime;
    in.sameKf = kfa == kfb;
    in.splitExt = ea != eb;
    in.wantExt = wd.estExt != 0;
    in.wantTd = wd.estTd != 0;
}

// Frozen IMU factor, evaluateImu of GpuRetainedFactorMath.hpp:53-140.
// evalImuRaw gives the unwhitened error e (15) and its Jacobian U (15 x 30
// row-major over [pose_i 6 | sb_i 9 | pose_j 6 | sb_j 9]); the factor's
// residual and Jacobian are r = W e and J = W U with W the 15 x 15 whitening
// (column-major in cgmli_frozen_imu).  evalImu applies W in the calling thread.
struct Sensor { d3 p, v, arm, lever; qd q; };
__device__ inline Sensor sensorState(const cgmli_frozen_imu& imu, const double* pose, const double* sb, int end) {
    const qd q = qnormalized(ldq(pose + 3));
    Sensor s;
    s.q = qnormalized(qmul(q, ldq(imu.sensor_quaternion)));
    s.arm = qapply(q, ld3(imu.sensor_position));
    s.lever = cross(qapply(s.q, ld3(imu.gyros + 3 * end) - ld3(sb + 3)), s.arm);
    s.p = ld3(pose) + s.arm;
    s.v = ld3(sb) + s.lever;
    return s;
}
// prepared: U is already zero (the caller cleared it in parallel) and the caller
// checks U's finiteness itself (through every product it forms from U).
__device__ inline bool evalImuRaw(const cgmli_frozen_imu& imu, const double* p0, const double* sb0, const double* p1,
                                  const double* sb1, double* e, double* U, bool prepared = false) {
    const Sensor s0 = sensorState(imu, p0, sb0, 0), s1 = sensorState(imu, p1, sb1, 1);
    const m3 A = colmajor(imu.rotation_gyro), V = colmajor(imu.velocity_gyro), P = colmajor(imu.position_gyro),
             Va = colmajor(imu.velocity_accel), Pa = colmajor(imu.position_accel);
    const m3 R = qrot(qconj(s0.q));
    const double dt = imu.duration;
    const d3 gravity = {0, 0, imu.gravity};
    const d3 bg = ld3(sb0 + 3) - ld3(imu.reference_bias), ba = ld3(sb0 + 6) - ld3(imu.reference_bias + 3);
    const d3 dp = (s0.p - s1.p) + dt * s0.v - (0.5 * dt * dt) * gravity;
    const d3 dv = (s0.v - s1.v) - dt * gravity;
    const d3 phi = -1.0 * mv(A, bg);
    const qd correction = rotationExp(phi), dq = qmul(correction, ldq(imu.delta_quaternion));
    const qd tail = qmul(qmul(ldq(imu.delta_quaternion), qconj(s1.q)), s0.q);
    const d3 e0 = mv(R, dp) + ld3(imu.delta_position) + mv(P, bg) - mv(Pa, ba);
    const d3 e1 = 2.0 * qvec(qmul(dq, qmul(qconj(s1.q), s0.q)));
    const d3 e2 = mv(R, dv) + ld3(imu.delta_velocity) + mv(V, bg) - mv(Va, ba);
    e[0] = e0.x; e[1] = e0.y; e[2] = e0.z; e[3] = e1.x; e[4] = e1.y; e[5] = e1.z; e[6] = e2.x; e[7] = e2.y; e[8] = e2.z;
    for (int i = 0; i < 6; ++i) e[9 + i] = sb0[3 + i] - sb1[3 + i];
    for (int i = 0; i < 15; ++i)
        if (!isfinite(e[i])) return false;
    if (!U) return true;
    const m3 gyroAngle = mscl(-1, mul(rotationJacobian(-1.0 * phi), A));
    m3 Jrot, Jbias;
    for (int j = 0; j < 3; ++j) {
        const qd ax = {j == 0 ? 1.0 : 0.0, j == 1 ? 1.0 : 0.0, j == 2 ? 1.0 : 0.0, 0.0};
        const qd db = {gyroAngle.a[j], gyroAngle.a[3 + j], gyroAngle.a[6 + j], 0.0};
        const d3 c1 = qvec(qmul(qmul(qmul(dq, qconj(s1.q)), ax), s0.q));
        const d3 c2 = qvec(qmul(qmul(correction, db), tail));
        Jrot.a[j] = c1.x; Jrot.a[3 + j] = c1.y; Jrot.a[6 + j] = c1.z;
        Jbias.a[j] = c2.x; Jbias.a[3 + j] = c2.y; Jbias.a[6 + j] = c2.z;
    }
    if (!prepared)
        for (int i = 0; i < 450; ++i) U[i] = 0;
    const int col0[4] = {0, 6, 15, 21};
    for (int k = 0; k < 4; ++k) {
        const bool first = k < 2;
        const double sign = first ? 1 : -1;
        const Sensor& s = first ? s0 : s1;
        auto put = [&](int r0, int c0, const m3& m, bool accumulate) {
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double& t = U[30 * (r0 + i) + col0[k] + c0 + j];
                    t = accumulate ? t + m.a[3 * i + j] : m.a[3 * i + j];
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
            const m3 leverBias = mul(skew(s.arm), qrot(s.q));
            put(6, 0, mscl(sign, R), false);
            put(6, 3, mscl(sign, mul(R, leverBias)), false);
            put(9, 3, mscl(sign, eye3()), false);
            put(12, 6, mscl(sign, eye3()), false);
            if (first) {
                put(0, 0, mscl(dt, R), false);
                put(0, 3, madd(mscl(dt, mul(R, leverBias)), P), false);
                put(0, 6, mscl(-1, Pa), false);
                put(3, 3, Jbias, false);
                put(6, 3, V, true);
                put(6, 6, mscl(-1, Va), false);
            }
        }
    }
    if (!prepared)
        for (int i = 0; i < 450; ++i)
            if (!isfinite(U[i])) return false;
    return true;
}
__device__ inline bool evalImu(const cgmli_frozen_imu& imu, const double* p0, const double* sb0, const double* p1, const double* sb1,
                               double* r, double* J) {
    double e[15];
    if (!evalImuRaw(imu, p0, sb0, p1, sb1, e, J)) return false;
    for (int i = 0; i < 15; ++i) {
        double v = 0;
        for (int k = 0; k < 15; ++k) v += imu.whitening[i + 15 * k] * e[k];
        r[i] = v;
        if (!isfinite(v)) return false;
    }
    if (!J) return true;
    for (int c = 0; c < 30; ++c) {
        double u[15];
        for (int m = 0; m < 15; ++m) u[m] = J[30 * m + c];
        for (int i = 0; i < 15; ++i) {
            double v = 0;
            for (int m = 0; m < 15; ++m) v += imu.whitening[i + 15 * m] * u[m];
            if (!isfinite(v)) return false;
            J[30 * i + c] = v;
        }
    }
    return true;
}

__device__ __forceinline__ const double* blockValue(const DevBatch& B, int buf, int kind, int index, int wdx) {
    switch (kind) {
        case CGMLI_PRIOR_POSE: return B.pose[buf] + 7ll * index;
        case CGMLI_PRIOR_SPEED_BIAS: return B.sb[buf] + 9ll * index;
        case CGMLI_PRIOR_EXTRINSIC: return B.ext[buf] + 7ll * index;
        default: return B.td[buf] + wdx;
    }
}

}  // namespace cgmli
