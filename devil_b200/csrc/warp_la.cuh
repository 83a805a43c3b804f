// Warp-cooperative FP64 dense linear algebra for the per-gene finalize
// kernels: p x p matrices (p <= 32) in shared memory, row i at A + i * ld
// with ld odd, so that the 32 lanes' rows fall in distinct banks.  Lane i
// owns row i during the factorisation and column i during solves.
#pragma once
#include "common.cuh"

namespace devil {

// leading dimension of a warp matrix: odd and >= P
__host__ __device__ constexpr int wla_ld(int P) { return P | 1; }

// 1/x: the MUFU estimate refined by two Newton-Raphson steps (within an
// ulp of the quotient; ~2x lower latency than the division sequence)
DEV double wla_rcp(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

// LU with partial pivoting (the factorisation Eigen's inverse() uses),
// without moving rows: perm[k] is the row chosen as pivot k (largest
// |a_ik| among rows not chosen yet, the lowest index on ties; a NaN entry
// wins so that it propagates); step (optional) receives, per row, the step
// at which it was chosen.  A row keeps its multipliers left of its pivot
// column.  Returns false in every lane when a pivot is zero or not finite.
// The multipliers use the pivot's reciprocal (one rounding more than a
// quotient) and the row updates run four columns at a time.
DEV bool warp_lu(double* A, int ld, int P, int* perm, int* step = nullptr) {
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
        if (lane == pv) {
            chosen = true;
            if (step) step[lane] = k;
        }
        if (lane == 0) perm[k] = pv;
        const double d = A[pv * ld + k];
        if (!(d != 0.0) || !isfinite(d)) ok = false;
        if (!chosen) {
            const double l = A[lane * ld + k] * wla_rcp(d);
            A[lane * ld + k] = l;
            const double* pr = A + pv * ld;
            double* r = A + lane * ld;
            int j = k + 1;
            for (; j + 3 < P; j += 4) {
                const double p0 = pr[j], p1 = pr[j + 1], p2 = pr[j + 2], p3 = pr[j + 3];
                const double r0 = r[j], r1 = r[j + 1], r2 = r[j + 2], r3 = r[j + 3];
                r[j] = fma(-l, p0, r0);
                r[j + 1] = fma(-l, p1, r1);
                r[j + 2] = fma(-l, p2, r2);
                r[j + 3] = fma(-l, p3, r3);
            }
            for (; j < P; ++j) r[j] = fma(-l, pr[j], r[j]);
        }
        __syncwarp();
    }
    return ok;
}

// x = A^-1 b for one right-hand side with the whole warp, from the factors
// of warp_lu (perm and step filled).  b is indexed by row; lane k returns
// x_k (lanes >= P return 0).  Column-oriented substitutions: after x_k (or
// y_k) is known it is broadcast and every remaining lane folds it into its
// own entry, so each step is one shuffle and one FMA per lane.
DEV double warp_lu_solve(const double* A, int ld, int P, const int* perm, const int* step,
                         double b_own) {
    const int lane = threadIdx.x & 31;
    // forward: rows in pivot order, unit lower factor; lane r holds the
    // running value of row r, y_k is row perm[k]'s value at step k
    const int my_step = lane < P ? step[lane] : -1;  // lanes without a row take no part
    double c = lane < P ? b_own : 0.0;
    double y_mine = 0.0;  // y_{lane}: lane k keeps y_k
    for (int k = 0; k < P; ++k) {
        const double yk = __shfl_sync(0xffffffffu, c, perm[k]);
        if (lane == k) y_mine = yk;
        if (my_step > k) c = fma(-A[lane * ld + k], yk, c);
    }
    // back: x_k = (y_k - sum_{j>k} U_kj x_j) / U_kk with U_kj = A[perm[k]][j]
    double d = y_mine;
    double x_mine = 0.0;
    for (int k = P - 1; k >= 0; --k) {
        double xk = 0.0;
        if (lane == k) xk = d / A[perm[k] * ld + k];
        xk = __shfl_sync(0xffffffffu, xk, k);
        if (lane == k) x_mine = xk;
        if (lane < k) d = fma(-A[perm[lane] * ld + k], xk, d);
    }
    return x_mine;
}

// X = A^-1 from the factors of warp_lu; lane c solves for column c
// (forward substitution in pivot order, back substitution in column order)
// (the inner products run with two partial sums so that consecutive FMAs
// do not wait on each other)
DEV void warp_lu_inverse(const double* A, int ld, int P, const int* perm, double* X, int ldx) {
    const int c = threadIdx.x & 31;
    if (c < P) {
        for (int k = 0; k < P; ++k) {
            const double* r = A + perm[k] * ld;
            double y0 = perm[k] == c ? 1.0 : 0.0, y1 = 0.0;
            int j = 0;
            for (; j + 1 < k; j += 2) {
                y0 = fma(-r[j], X[j * ldx + c], y0);
                y1 = fma(-r[j + 1], X[(j + 1) * ldx + c], y1);
            }
            if (j < k) y0 = fma(-r[j], X[j * ldx + c], y0);
            X[k * ldx + c] = y0 + y1;
        }
        for (int k = P - 1; k >= 0; --k) {
            const double* r = A + perm[k] * ld;
            double x0 = X[k * ldx + c], x1 = 0.0;
            int j = k + 1;
            for (; j + 1 < P; j += 2) {
                x0 = fma(-r[j], X[j * ldx + c], x0);
                x1 = fma(-r[j + 1], X[(j + 1) * ldx + c], x1);
            }
            if (j < P) x0 = fma(-r[j], X[j * ldx + c], x0);
            X[k * ldx + c] = (x0 + x1) / r[k];
        }
    }
    __syncwarp();
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
            double s0 = 0.0, s1 = 0.0;
            int k = 0;
            for (; k + 1 < P; k += 2) {
                s0 = fma(A[i * ld + k], B[k * ld + j], s0);
                s1 = fma(A[i * ld + k + 1], B[(k + 1) * ld + j], s1);
            }
            if (k < P) s0 = fma(A[i * ld + k], B[k * ld + j], s0);
            C[i * ld + j] = s0 + s1;
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
