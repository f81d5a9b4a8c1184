// Register-tiled symmetric rank updates over rows held in shared memory.
//
// The upper triangle of an np x np accumulation (np a multiple of 32) is cut
// into 32 x 32 tiles; one warp works on one tile, each lane holding a 4 x 8
// block in registers: rows {2g, 2g+1, 16+2g, 16+2g+1} and columns
// {2c + 8q, 2c + 8q + 1 : q < 4} of the tile, g = lane / 4, c = lane % 4.
// With that split every shared load of a warp is one 128-byte wavefront (the
// row pairs of the 8 lane groups are contiguous, the column pairs of the 4
// lane columns too), and a k-step costs 6 double2 loads for 32 FMAs per lane.
#pragma once

namespace cgmli {

// Tile t of the packed upper enumeration of an nb x nb block triangle.
__device__ __forceinline__ void tileOf(int t, int nb, int& bi, int& bj) {
    bi = 0;
    while (t >= nb - bi) { t -= nb - bi; ++bi; }
    bj = bi + t;
}
// Row and column (within the np x np accumulation) of the lane's entry (r, c).
__device__ __forceinline__ int tileRow(int bi, int lane, int r) { return bi * 32 + (r < 2 ? 2 * (lane >> 2) + r : 16 + 2 * (lane >> 2) + r - 2); }
__device__ __forceinline__ int tileCol(int bj, int lane, int c) { return bj * 32 + 8 * (c >> 1) + 2 * (lane & 3) + (c & 1); }

__device__ __forceinline__ void zeroTile(double (&acc)[4][8]) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;
}

// acc += (or -=) sum over rows k = k0, k0 + step, ... < k1 of V[k][rows] V[k][cols]^T,
// V row-major with row length np; Va = V + 32 bi + 2 (lane / 4), Vb = V + 32 bj + 2 (lane % 4).
template <bool kSubtract>
__device__ __forceinline__ void rankUpdate(double (&acc)[4][8], const double* Va, const double* Vb, int k0, int k1, int step, int np) {
#pragma unroll 2
    for (int k = k0; k < k1; k += step) {
        const double2 a01 = *reinterpret_cast<const double2*>(Va + (long long)k * np);
        const double2 a23 = *reinterpret_cast<const double2*>(Va + (long long)k * np + 16);
        double a[4] = {a01.x, a01.y, a23.x, a23.y};
        if (kSubtract)
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = -a[r];
        double b[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double2 v = *reinterpret_cast<const double2*>(Vb + (long long)k * np + 8 * q);
            b[2 * q] = v.x;
            b[2 * q + 1] = v.y;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
}

}  // namespace cgmli
