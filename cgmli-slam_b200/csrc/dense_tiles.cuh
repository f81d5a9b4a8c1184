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

// The same tile Gram on the FP64 tensor path: mma.sync m8n8k4 (f64), each 32 x 32
// tile as 4 x 4 blocks of 8 x 8.  A k-step takes 4 rows of V (lane % 4 selects
// the row, lane / 4 the column within an 8-wide block) and issues 16 MMAs for the
// tile, 4096 FMAs, against 128 FMA instructions per lane on the scalar path.  The
// accumulator layout differs from rankUpdate's: acc[I][2 J + e] is entry
// (8 I + lane / 4, 8 J + 2 (lane % 4) + e) of the tile, so flushes use tileRowMma
// (columns are tileCol's).  Rows k = k0 + step (4 t + lane % 4) < k1.
__device__ __forceinline__ int tileRowMma(int bi, int lane, int r) { return bi * 32 + 8 * r + (lane >> 2); }
__device__ __forceinline__ void mmaF64Tile(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}
template <bool kSubtract>
__device__ __forceinline__ void rankUpdateMma(double (&acc)[4][8], const double* V, int rowBase, int colBase, int k0, int k1, int step,
                                              int np) {
    const int lane = threadIdx.x & 31, g = lane >> 2, kr = lane & 3;
    for (int k = k0 + kr * step; k - kr * step < k1; k += 4 * step) {
        const bool valid = k < k1;
        const double* row = V + (long long)k * np;
        double a[4], b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            a[q] = valid ? row[rowBase + 8 * q + g] : 0.0;
            b[q] = valid ? row[colBase + 8 * q + g] : 0.0;
            if (kSubtract) a[q] = -a[q];
        }
#pragma unroll
        for (int I = 0; I < 4; ++I)
#pragma unroll
            for (int J = 0; J < 4; ++J) mmaF64Tile(acc[I][2 * J], acc[I][2 * J + 1], a[I], b[J]);
    }
}

}  // namespace cgmli
