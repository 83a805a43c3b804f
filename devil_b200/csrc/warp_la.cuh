// Warp-cooperative FP64 dense linear algebra for the per-gene finalize
// kernels: p x p matrices (p <= 32) in shared memory, row i at A + i * ld
// with ld odd, so that the 32 lanes' rows fall in distinct banks.  Lane i
// owns row i during the factorisation and column i during solves.
#pragma once
#include "common.cuh"

namespace devil {

// leading dimension of a warp matrix: odd and >= P
__host__ __device__ constexpr int wla_ld(int P) { return P | 1; }

// LU with partial pivoting (the factorisation Eigen's inverse() uses),
// without moving rows: perm[k] is the row chosen as pivot k (largest
// |a_ik| among rows not chosen yet, the lowest index on ties; a NaN entry
// wins so that it propagates).  A row keeps its multipliers left of its
// pivot column.  Returns false in every lane when a pivot is zero or not
// finite.
DEV bool warp_lu(double* A, int ld, int P, int* perm) {
    const int lane = threadIdx.x & 31;
    bool chosen = lane >= P;
    bool ok = true;
    for (int k = 0; k < P; ++k) {
        double v = -1.0;
        if (!chosen) {
            const double a = A[lane * ld + k];
            v = a != a ? INFINITY : fabs(a);
        }
        int bl = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, v, o);
            const int ol = __shfl_xor_sync(0xffffffffu, bl, o);
            if (ov > v || (ov == v && ol < bl)) {
                v = ov;
                bl = ol;
            }
        }
        const int pv = bl;
        if (lane == pv) chosen = true;
        if (lane == 0) perm[k] = pv;
        const double d = A[pv * ld + k];
        if (!(d != 0.0) || !isfinite(d)) ok = false;
        if (!chosen) {
            const double l = A[lane * ld + k] / d;
            A[lane * ld + k] = l;
            for (int j = k + 1; j < P; ++j) A[lane * ld + j] -= l * A[pv * ld + j];
        }
        __syncwarp();
    }
    return ok;
}

// X = A^-1 from the factors of warp_lu; lane c solves for column c
// (forward substitution in pivot order, back substitution in column order)
DEV void warp_lu_inverse(const double* A, int ld, int P, const int* perm, double* X, int ldx) {
    const int c = threadIdx.x & 31;
    if (c < P) {
        for (int k = 0; k < P; ++k) {
            const double* r = A + perm[k] * ld;
            double y = perm[k] == c ? 1.0 : 0.0;
            for (int j = 0; j < k; ++j) y -= r[j] * X[j * ldx + c];
            X[k * ldx + c] = y;
        }
        for (int k = P - 1; k >= 0; --k) {
            const double* r = A + perm[k] * ld;
            double x = X[k * ldx + c];
            for (int j = k + 1; j < P; ++j) x -= r[j] * X[j * ldx + c];
            X[k * ldx + c] = x / r[k];
        }
    }
    __syncwarp();
}

// x = A^-1 b for one right-hand side (one thread; x may alias nothing)
DEV void lu_solve_perm(const double* A, int ld, int P, const int* perm, const double* b,
                       double* x) {
    for (int k = 0; k < P; ++k) {
        const double* r = A + perm[k] * ld;
        double y = b[perm[k]];
        for (int j = 0; j < k; ++j) y -= r[j] * x[j];
        x[k] = y;
    }
    for (int k = P - 1; k >= 0; --k) {
        const double* r = A + perm[k] * ld;
        double v = x[k];
        for (int j = k + 1; j < P; ++j) v -= r[j] * x[j];
        x[k] = v / r[k];
    }
}

// M (row-major, ld) = the symmetric matrix of packed upper-triangular
// storage (tri_index) times `scale`, plus `ridge` on the diagonal
DEV void warp_unpack_sym(int P, const double* packed, double scale, double ridge, double* M, int ld) {
    const int lane = threadIdx.x & 31;
    for (int q = lane; q < P * P; q += 32) {
        const int i = q / P, j = q - i * P;
        const double v = packed[i <= j ? tri_index(i, j) : tri_index(j, i)] * scale;
        M[i * ld + j] = i == j ? v + ridge : v;
    }
    __syncwarp();
}

// C = A B (all P x P, row-major); lane j computes column j
DEV void warp_matmul(int P, const double* A, const double* B, double* C, int ld) {
    const int j = threadIdx.x & 31;
    if (j < P)
        for (int i = 0; i < P; ++i) {
            double s = 0.0;
            for (int k = 0; k < P; ++k) s += A[i * ld + k] * B[k * ld + j];
            C[i * ld + j] = s;
        }
    __syncwarp();
}

// sum_{i,k} A_ik B_ki (every lane gets the value)
DEV double warp_trace_prod(int P, const double* A, const double* B, int ld) {
    const int i = threadIdx.x & 31;
    double s = 0.0;
    if (i < P)
        for (int k = 0; k < P; ++k) s += A[i * ld + k] * B[k * ld + i];
    return warp_sum(s);
}

}  // namespace devil
