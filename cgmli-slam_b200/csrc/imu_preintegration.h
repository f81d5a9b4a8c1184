// Launch interface of the batched IMU preintegration kernel (host runtime <->
// imu_preintegration.cu).
#pragma once
#include <cuda_runtime.h>

#include "../../include/cgmli_backend.h"

namespace cgmli {

struct ImuLaunch {
    cgmli_imu_parameters prm;
    const long long* times;    // sample times, indexed by range - sampleOffset
    const double* readings;    // 6 per sample
    int sampleOffset;
    const int* ranges;         // 2 per interval
    const long long* t0s;
    const long long* t1s;
    cgmli_frozen_imu* out;     // the factors written (refresh: replaced in place)
    int* status;               // per interval: CGMLI_OK / _E_INVALID / _E_NONFINITE
    // Batched construction: the linearization bias of interval i is biases[6i..6i+5].
    const double* biases;
    // Refresh (biases == nullptr): interval i belongs to keyframe kf[i]; its bias
    // is the current [b_g, b_a] of sb + 9 kf[i]; it is re-integrated only when
    // that bias moved from out[i].reference_bias by more than the thresholds, into
    // scratch[i], which replaces out[i] when the result is finite; refreshed[i]
    // tells which intervals were replaced.
    const double* sb;
    const int* kf;
    double gyroThreshold, accelThreshold;
    cgmli_frozen_imu* scratch;
    int* refreshed;
    // With force, every interval is integrated at the keyframe's current bias and
    // written straight to out[i] (no drift check, no scratch): the merged IMU
    // factor of a SECOND_NEW marginalization.
    int force;
};

cudaError_t launchImuPreintegration(const ImuLaunch& L, int count, cudaStream_t s);

}  // namespace cgmli
