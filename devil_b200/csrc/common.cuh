// Device helpers shared by every kernel of the devil B200 path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DEV __device__ __forceinline__

namespace devil {

constexpr float kLog2e = 1.4426950408889634f;

// MUFU.EX2 / MUFU.RCP through PTX (approximate, ~1-2 ulp; FTZ).
DEV float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
DEV float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
DEV float fast_exp(float x) { return ex2_approx(x * kLog2e); }

template <class T>
DEV T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <class T>
DEV T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// value loaders for the two CSR value types
DEV float load_val(const uint16_t* v, int64_t e) { return (float)__ldg(v + e); }
DEV float load_val(const float* v, int64_t e) { return __ldg(v + e); }

// ---------------------------------------------------------------------
// small dense FP64 linear algebra on column-major p x p matrices held by
// one thread (local memory / registers).  LU with partial pivoting, the
// factorisation Eigen's MatrixXd::inverse() uses for dynamic sizes.
// Returns false when a pivot is exactly zero or not finite.
// ---------------------------------------------------------------------
DEV bool lu_factor(int p, double* A, int* piv) {
    bool ok = true;
    for (int k = 0; k < p; ++k) {
        int mx = k;
        double mv = fabs(A[k * p + k]);
        for (int i = k + 1; i < p; ++i) {
            double v = fabs(A[k * p + i]);
            if (v > mv) { mv = v; mx = i; }
        }
        piv[k] = mx;
        if (mx != k)
            for (int j = 0; j < p; ++j) {
                double t = A[j * p + k];
                A[j * p + k] = A[j * p + mx];
                A[j * p + mx] = t;
            }
        double d = A[k * p + k];
        if (!(d != 0.0) || !isfinite(d)) ok = false;
        double rd = 1.0 / d;
        for (int i = k + 1; i < p; ++i) {
            double l = A[k * p + i] * rd;
            A[k * p + i] = l;
            for (int j = k + 1; j < p; ++j) A[j * p + i] -= l * A[j * p + k];
        }
    }
    return ok;
}

DEV void lu_solve(int p, const double* LU, const int* piv, double* x) {
    for (int k = 0; k < p; ++k)
        if (piv[k] != k) { double t = x[k]; x[k] = x[piv[k]]; x[piv[k]] = t; }
    for (int i = 0; i < p; ++i) {
        double s = x[i];
        for (int j = 0; j < i; ++j) s -= LU[j * p + i] * x[j];
        x[i] = s;
    }
    for (int i = p - 1; i >= 0; --i) {
        double s = x[i];
        for (int j = i + 1; j < p; ++j) s -= LU[j * p + i] * x[j];
        x[i] = s / LU[i * p + i];
    }
}

// inverse of an LU-factored matrix into Ainv (column-major)
DEV void lu_inverse(int p, const double* LU, const int* piv, double* Ainv) {
    for (int c = 0; c < p; ++c) {
        double* x = Ainv + c * p;
        for (int i = 0; i < p; ++i) x[i] = (i == c) ? 1.0 : 0.0;
        lu_solve(p, LU, piv, x);
    }
}

// index of (i, j), i <= j, in packed upper-triangular storage by rows of j:
// pairs are enumerated (0,0),(0,1),(1,1),(0,2),(1,2),(2,2),...
DEV constexpr int tri_index(int i, int j) { return j * (j + 1) / 2 + i; }

}  // namespace devil
