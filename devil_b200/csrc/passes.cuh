// Per-gene reductions over cells ("passes") for devil's NB GLM path.
//
// Every step of the path -- an IRLS iteration, the MOM moments, one Newton
// evaluation of the dispersion score, the bread and the clustered meat --
// is a reduction over all n cells of per-cell terms that depend on
// mu_c = exp(x_c . beta_g + off_c) and on the count y_gc.  Counts are
// sparse, so each pass is split into
//   dense : the y = 0 value of the per-cell terms, evaluated for every cell
//           (needs only X, the offsets and the gene's parameters), and
//   sparse: the correction term(y) - term(0), evaluated for the nonzero
//           entries of the gene's CSR row.
// A pass "trait" states its terms; two engines evaluate any trait:
//   reg_pass_kernel : p <= 8, GT genes per CTA held in registers, each cell
//                     row of X loaded once and reused by all GT genes.
//   gen_pass_kernel : any p <= 32, shared-memory tiles of cells; outputs
//                     are owned one per thread.
// Terms are of three kinds: outer(w) adds w * x x^T (packed upper
// triangle), vec(w) adds w * x, scal(v) adds v.  Per-segment partial sums
// go to global memory and a finalize kernel per pass reduces them in FP64.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace devil {

// ---------------------------------------------------------------------
// geometry shared by both engines
// ---------------------------------------------------------------------
struct PassGeom {
    const float* X;        // [n][xs] row-major float
    int xs;                // row stride of X (>= p)
    const float* off;      // [n]
    const double* Xd;      // [n][xs] row-major double (FP64 passes)
    const double* offd;    // [n] (FP64 passes)
    const int32_t* col;    // CSR cell index
    const void* val;       // CSR values (uint16 or float)
    const int64_t* segptr; // [G][nbound] first CSR entry with col >= bound[b]
    const int32_t* bound;  // [nbound] cell boundaries
    int nbound;            // fine segments + 1
    int nseg;              // work items along the cells: item s covers fine
                           // segments [s*(nbound-1)/nseg, (s+1)*(nbound-1)/nseg)
    int32_t* err;          // set to 1 when a bounded wait gives up
    const int32_t* act;    // active gene list
    const int32_t* n_act;  // its length (device)
    int32_t* reset_next;   // counter zeroed by block (0,0) (may be null)
    void* partW;           // [seg][slot_stride][NA] of Pass::AW
    double* partS;         // [seg][slot_stride][NS]
    int slot_stride;
};

// ---------------------------------------------------------------------
// accumulators
// ---------------------------------------------------------------------
// zz holds the cell's products x_i x_j (packed upper triangle), computed
// once per cell and shared by the gene tile.
// (a0, a1) += (b, b) * (c0, c1) as one packed FP32x2 FMA (sm_100): two
// correctly rounded FMAs, the same results as two fmaf, in one instruction
DEV void fma_x2(float& a0, float& a1, float b, float c0, float c1) {
    uint64_t acc, bb, cc;
    asm("mov.b64 %0, {%1, %2};" : "=l"(acc) : "f"(a0), "f"(a1));
    asm("mov.b64 %0, {%1, %1};" : "=l"(bb) : "f"(b));
    asm("mov.b64 %0, {%1, %2};" : "=l"(cc) : "f"(c0), "f"(c1));
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(bb), "l"(cc));
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a0), "=f"(a1) : "l"(acc));
}

template <int P, int NA, int NS, class AW, class AS, class R>
struct RegAcc {
    AW* a;
    AS* s;
    const R* x;
    const R* zz;
    static constexpr bool X2 = std::is_same<AW, float>::value && std::is_same<R, float>::value;
    template <int W>
    DEV void outer(R w) {
        constexpr int NE = P * (P + 1) / 2;
        constexpr int base = W * NE;
        if constexpr (X2) {
#pragma unroll
            for (int q = 0; q + 1 < NE; q += 2) fma_x2(a[base + q], a[base + q + 1], w, zz[q], zz[q + 1]);
            if constexpr (NE & 1) a[base + NE - 1] = fmaf(w, zz[NE - 1], a[base + NE - 1]);
        } else {
#pragma unroll
            for (int q = 0; q < NE; ++q) a[base + q] += (AW)(w * zz[q]);
        }
    }
    template <int V, int NW>
    DEV void vec(R w) {
        constexpr int base = NW * (P * (P + 1) / 2) + V * P;
        if constexpr (X2) {
#pragma unroll
            for (int i = 0; i + 1 < P; i += 2) fma_x2(a[base + i], a[base + i + 1], w, x[i], x[i + 1]);
            if constexpr (P & 1) a[base + P - 1] = fmaf(w, x[P - 1], a[base + P - 1]);
        } else {
#pragma unroll
            for (int i = 0; i < P; ++i) a[base + i] += (AW)(w * x[i]);
        }
    }
    template <int K>
    DEV void scal(AS v) { s[K] += v; }
    // scalar accumulated with the FP32 weight sums (after outer and vec terms)
    template <int K, int NW, int NV>
    DEV void fscal(R v) { a[NW * (P * (P + 1) / 2) + NV * P + K] += (AW)v; }
};

// recorder used by the shared-memory engine: captures the weights only
template <int NWV, int NS, class AS, class R>
struct RecAcc {
    R w[NWV > 0 ? NWV : 1];
    AS s[NS > 0 ? NS : 1];
    DEV void zero() {
#pragma unroll
        for (int i = 0; i < NWV; ++i) w[i] = 0;
#pragma unroll
        for (int i = 0; i < NS; ++i) s[i] = 0;
    }
    template <int W>
    DEV void outer(R v) { w[W] += v; }
    template <int V, int NW>
    DEV void vec(R v) { w[NW + V] += v; }
    template <int K>
    DEV void scal(AS v) { s[K] += v; }
    template <int K, int NW, int NV>
    DEV void fscal(R v) { w[NW + NV + K] += v; }
};

// 1/x in FP64 for x > 0: the MUFU estimate (rcp.approx.ftz.f64, about 20
// correct bits) refined by Newton-Raphson steps r <- r + r (1 - x r), each
// of which doubles the number of correct bits: two steps give the quotient
// to within an ulp, one step to ~1e-12 relative (plenty for terms that are
// summed over cells).  rcp_nr gives 0 for x = +inf, as the quotient does.
DEV double rcp_nr(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    return isinf(x) ? 0.0 : r;
}
// (one step, and no special case for x = +inf: there the pass's dense term
// mu / (mu + k) is already NaN, whatever the reciprocal returns)
DEV double rcp_nr1(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

// reciprocal in the arithmetic of the pass: MUFU estimate in FP32, the
// estimate refined by one Newton step in FP64 (the per-cell terms are summed
// over cells; ~1e-11 relative per term is far below what the sums carry)
DEV float rcp_r(float x) { return rcp_approx(x); }
DEV double rcp_r(double x) { return rcp_nr1(x); }

// ---------------------------------------------------------------------
// pass traits
// ---------------------------------------------------------------------

// One IRLS iteration of beta_fit (src/beta.cpp:35-42):
//   w_q = exp(-eta - off), mu_g = (k + y) / (1 + k w_q)
//   H = k X' diag(mu_g w_q) X,  score = k X' (mu_g w_q - 1)
// With mu = 1/w_q and r = 1/(mu + k):  k mu_g w_q = k (k + y) r  and
//   k (mu_g w_q - 1) = k (y - mu) r.  The pass accumulates
//   outer0 = sum r x x' + sum_{y>0} (y/k) r x x'      (H = k^2 outer0)
//   vec0   = sum mu r x - sum_{y>0} y r x            (score = -k vec0)
// so a zero cell costs one reciprocal, one product and the FMAs; the
// constant factors are applied in FP64 by the finalize.
struct PassIRLS {
    static constexpr int NF = 0;
    static constexpr int NW = 1, NV = 1, NS = 0;
    static constexpr bool F64 = false;
    static constexpr bool TABLES = false;
    using AW = float;
    using AS = float;
    struct Params { const float* beta; const double* beta_d; const float* k; };
    struct Gene { float k, rk; };
    static DEV Gene load(const Params& p, int g) {
        float k = p.k[g];
        return Gene{k, 1.f / k};
    }
    template <class R, class A>
    static DEV void dense(const Gene& G, R mu, A& acc) {
        R r = rcp_r(mu + (R)G.k);
        acc.template outer<0>(r);
        acc.template vec<0, NW>(mu * r);
    }
    // (y: the count, float or -- from integer counts -- converted straight to R)
    template <class R, class A, class Y>
    static DEV void sparse(const Gene& G, R mu, Y y, A& acc) {
        R r = rcp_r(mu + (R)G.k);
        R yr = (R)y * r;
        acc.template outer<0>(yr * (R)G.rk);  // rk scales H only, not the score
        acc.template vec<0, NW>(-yr);
    }
};

// estimate_mom_dispersion_cpp (src/mom_overdispersion.cpp:34-45):
//   num = sum (y - mu)^2 - mu,  den = sum mu^2
// One pass, evaluated in FP64 per cell (num cancels for near-Poisson genes).
struct PassMOM {
    static constexpr int NF = 0;
    static constexpr int NW = 0, NV = 0, NS = 2;
    static constexpr bool F64 = true;
    static constexpr bool TABLES = false;
    using AW = float;
    using AS = double;
    struct Params { const float* beta; const double* beta_d; };
    struct Gene { int dummy; };
    static DEV Gene load(const Params&, int) { return Gene{0}; }
    template <class R, class A>
    static DEV void dense(const Gene&, R mu, A& acc) {
        double m = mu;
        acc.template scal<0>(m * m - m);
        acc.template scal<1>(m * m);
    }
    template <class R, class A>
    static DEV void sparse(const Gene&, R mu, float y, A& acc) {
        double m = mu, yy = y;
        acc.template scal<0>(yy * yy - 2.0 * yy * m);
    }
};

// g(x) = log(1 + x) - x / (1 + x), x = mu * theta >= 0, to full relative
// precision.  With u = x / (1 + x):  log(1 + x) = -log(1 - u), so
// g = sum_{m>=2} u^m / m, a series of positive terms (no cancellation);
// for x >= 1/4 (u >= 1/5) the direct difference loses < 4 bits.
DEV float nb_g(float x, float r) {
    // r = 1/(1 + x) from the caller; u = x r.  Series error < 2e-8 relative
    // for u <= 0.2.
    float u = x * r;
    if (x < 0.25f) {
        float t = 1.f / 12.f;
        t = fmaf(t, u, 1.f / 11.f);
        t = fmaf(t, u, 1.f / 10.f);
        t = fmaf(t, u, 1.f / 9.f);
        t = fmaf(t, u, 1.f / 8.f);
        t = fmaf(t, u, 1.f / 7.f);
        t = fmaf(t, u, 1.f / 6.f);
        t = fmaf(t, u, 1.f / 5.f);
        t = fmaf(t, u, 1.f / 4.f);
        t = fmaf(t, u, 1.f / 3.f);
        t = fmaf(t, u, 0.5f);
        return u * u * t;
    }
    return log1pf(x) - u;
}

DEV double nb_g(double x, double r) {
    double u = x * r;
    if (x < 0.25) {
        double t = 0.0;
        for (int m = 24; m >= 3; --m) t = fma(t, u, 1.0 / m);
        t = fma(t, u, 0.5);
        return u * u * t;
    }
    return log1p(x) - u;
}

// The per-cell part of conventional_score_function_fast's ll_part
// (src/overdispersion.cpp:159-173) for y = 0: the reference's branches on
// mu*theta < 1e-10 and < 1e-4 with the clamp to its Taylor bounds.
template <class R>
DEV R nb_ll_term(R x, R r) {
    if (x < (R)1e-10) return x * x * (r - (R)0.5);
    R gx = nb_g(x, r);
    if (x < (R)1e-4) {
        R ub = x * x * r, lb = x * x * (r - (R)0.5);
        gx = fmax(fmin(gx, ub), lb);
    }
    return gx;
}

// psi(y + a) - psi(a) and psi1(y + a) - psi1(a) for a count y > 0
DEV double digamma_d(double x) {
    double r = 0.0;
    while (x < 10.0) { r -= 1.0 / x; x += 1.0; }
    double f = 1.0 / (x * x);
    double t = f * (-1.0 / 12 + f * (1.0 / 120 + f * (-1.0 / 252 + f * (1.0 / 240 +
               f * (-1.0 / 132 + f * (691.0 / 32760 + f * (-1.0 / 12)))))));
    return r + log(x) - 0.5 / x + t;
}
DEV double trigamma_d(double x) {
    double r = 0.0;
    while (x < 10.0) { r += 1.0 / (x * x); x += 1.0; }
    double f = 1.0 / (x * x);
    double t = 1.0 / x + f / 2.0 + (f / x) * (1.0 / 6 + f * (-1.0 / 30 + f * (1.0 / 42 +
               f * (-1.0 / 30 + f * (5.0 / 66 + f * (-691.0 / 2730 + f * (7.0 / 6)))))));
    return r + t;
}

// Per-gene tables of psi(v + a) - psi(a) and psi1(v + a) - psi1(a) for
// v = 0..kPsiTab-1, from psi(x + 1) = psi(x) + 1/x (prefix sums of 1/(a+j)
// and -1/(a+j)^2).  Counts are integers, so most nonzeros read a table
// entry; larger counts evaluate the asymptotic series.  This plays the role
// of the reference's count table (make_table_if_small,
// src/overdispersion.cpp:32-46): the digamma work no longer scales with
// the nonzeros.
constexpr int kPsiTab = 64;
struct PsiTable {
    const double* d1;  // [kPsiTab]
    const double* d2;  // [kPsiTab]
    double pa, ta;     // psi(a), psi1(a) for counts beyond the table
};
// build tables for GTn genes with parameter a[j] using all threads of the
// block (one thread per (gene, v)); tab layout [gene][2][kPsiTab]
DEV void build_psi_tables(int GTn, const double* a, double* tab, double* scratch) {
    // scratch: [GTn][kPsiTab] terms; inclusive scan by one warp per gene
    for (int i = threadIdx.x; i < GTn * kPsiTab; i += blockDim.x) {
        int j = i / kPsiTab, v = i - j * kPsiTab;
        double t = (v == 0) ? 0.0 : 1.0 / (a[j] + (v - 1));
        scratch[i] = t;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int j = warp; j < GTn; j += nw) {
        double c1 = 0.0, c2 = 0.0;
        for (int base = 0; base < kPsiTab; base += 32) {
            double t = scratch[j * kPsiTab + base + lane];
            double s1 = t, s2 = -t * t;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                double u1 = __shfl_up_sync(0xffffffffu, s1, o);
                double u2 = __shfl_up_sync(0xffffffffu, s2, o);
                if (lane >= o) { s1 += u1; s2 += u2; }
            }
            tab[(j * 2 + 0) * kPsiTab + base + lane] = c1 + s1;
            tab[(j * 2 + 1) * kPsiTab + base + lane] = c2 + s2;
            c1 += __shfl_sync(0xffffffffu, s1, 31);
            c2 += __shfl_sync(0xffffffffu, s2, 31);
        }
    }
    __syncthreads();
}
DEV void psi_diffs_tab(double y, double a, const PsiTable& T, double& d1, double& d2) {
    if (y < (double)kPsiTab && y == floor(y)) {
        int v = (int)y;
        d1 = T.d1[v];
        d2 = T.d2[v];
    } else {
        d1 = digamma_d(y + a) - T.pa;
        d2 = trigamma_d(y + a) - T.ta;
    }
}

// One evaluation of the dispersion score and its derivative in log theta
// (src/overdispersion.cpp:95-242) at theta, with x = mu theta, a = 1/theta,
// w = mu/(1 + x):
//   fscal0 = sum ll_term(x)        fscal1 = sum mu x/(1+x)^2    (FP32 sums)
//   scal0  = sum y theta/(1+x)     scal1  = sum y/(1+x)^2       (FP64)
//   scal2  = sum psi(y+a) - psi(a) scal3  = sum psi1(y+a) - psi1(a)
//   outer0 = X' diag(w) X, outer1 = X' diag(-w^2) X, outer2 = X' diag(2 w^3) X
// (the Cox-Reid b, db, d2b).  The nonzero terms stay FP64: their sum nearly
// cancels the digamma sum in the score.
struct PassMLE {
    static constexpr int NF = 2;
    static constexpr int NW = 3, NV = 0, NS = 4;
    static constexpr bool F64 = false;
    static constexpr bool TABLES = true;
    using AW = float;
    using AS = double;
    struct Params { const float* beta; const double* beta_d; const double* log_theta; };
    struct Gene { double theta, a; float thf; PsiTable tab; };
    static DEV Gene load(const Params& p, int g) {
        double th = exp(p.log_theta[g]);
        return Gene{th, 1.0 / th, (float)th, PsiTable{nullptr, nullptr, 0.0, 0.0}};
    }
    template <class R, class A>
    static DEV void dense(const Gene& G, R mu, A& acc) {
        R x = mu * (sizeof(R) == 4 ? (R)G.thf : (R)G.theta);
        R r = rcp_r((R)1 + x);
        R w = mu * r;
        acc.template outer<0>(w);
        acc.template outer<1>(-w * w);
        acc.template outer<2>((R)2 * w * w * w);
        acc.template fscal<0, NW, NV>(nb_ll_term<R>(x, r));
        acc.template fscal<1, NW, NV>(w * x * r);
    }
    template <class R, class A, class Y>
    static DEV void sparse(const Gene& G, R mu, Y y, A& acc) {
        double m = mu, yy = y;
        double den = 1.0 + m * G.theta;
        // reciprocal: MUFU estimate refined by one FP64 Newton step
        double r = (double)rcp_approx((float)den);
        r = r + r * (1.0 - den * r);
        acc.template scal<0>(yy * G.theta * r);
        acc.template scal<1>(yy * r * r);
        double d1, d2;
        psi_diffs_tab(yy, G.a, G.tab, d1, d2);
        acc.template scal<2>(d1);
        acc.template scal<3>(d2);
    }
};

// init_beta's right-hand side on a grouped design (R/beta.R:12-24): the sum
// over the gene's nonzeros of log1p(y / exp(offset)) (zero counts give
// log1p(0) = 0).  Run by the slice-major pass with beta = 0, where mu is
// exp(offset) itself.
struct PassInitZ {
    static constexpr int NF = 0;
    static constexpr int NW = 0, NV = 0, NS = 1;
    static constexpr bool F64 = true;
    static constexpr bool TABLES = false;
    using AW = double;
    using AS = double;
    struct Params { const float* beta; const double* beta_d; };
    struct Gene { int dummy; };
    static DEV Gene load(const Params&, int) { return Gene{0}; }
    template <class R, class A>
    static DEV void dense(const Gene&, R, A&) {}
    template <class R, class A>
    static DEV void sparse(const Gene&, R mu, float y, A& acc) {
        acc.template scal<0>(log1p((double)y / (double)mu));
    }
};

// compute_hessian (src/variance.cpp:22-47) and the per-cluster score sums of
// compute_clustered_meat_fast (src/variance.cpp:207-217) in one pass:
//   outer0 = X' diag((y theta + 1) mu / (1 + theta mu)^2) X
//   vec0   = X' (y - mu)/(1 + mu theta)       (per segment; segments never
//                                              cross a cluster boundary)
// One pass, evaluated in FP64 per cell with FP64 sums: the bread is an
// inverse, so cond(H) multiplies every relative error of H.
struct PassSandwich {
    static constexpr int NF = 0;
    static constexpr int NW = 1, NV = 1, NS = 0;
    static constexpr bool F64 = true;
    static constexpr bool TABLES = false;
    using AW = double;
    using AS = float;
    struct Params { const float* beta; const double* beta_d; const double* theta; };
    struct Gene { double th; };
    static DEV Gene load(const Params& p, int g) { return Gene{p.theta[g]}; }
    template <class R, class A>
    static DEV void dense(const Gene& G, R mu, A& acc) {
        R r = (R)1 / ((R)1 + (R)G.th * mu);
        acc.template outer<0>(mu * r * r);
        acc.template vec<0, NW>(-mu * r);
    }
    template <class R, class A>
    static DEV void sparse(const Gene& G, R mu, float y, A& acc) {
        R r = (R)1 / ((R)1 + (R)G.th * mu);
        acc.template outer<0>((R)y * (R)G.th * mu * r * r);
        acc.template vec<0, NW>((R)y * r);
    }
};

// ---------------------------------------------------------------------
// engine 1: registers, p <= 8
// ---------------------------------------------------------------------
template <int P, int PP>
DEV void load_row(const float* __restrict__ X, int64_t c, float* x) {
    const float* r = X + c * PP;
    if constexpr (PP == 8) {
        float4 a = __ldg(reinterpret_cast<const float4*>(r));
        float4 b = __ldg(reinterpret_cast<const float4*>(r) + 1);
        float t[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < P; ++i) x[i] = t[i];
    } else if constexpr (PP == 4) {
        float4 a = __ldg(reinterpret_cast<const float4*>(r));
        float t[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int i = 0; i < P; ++i) x[i] = t[i];
    } else if constexpr (PP == 2) {
        float2 a = __ldg(reinterpret_cast<const float2*>(r));
        float t[2] = {a.x, a.y};
#pragma unroll
        for (int i = 0; i < P; ++i) x[i] = t[i];
    } else {
#pragma unroll
        for (int i = 0; i < P; ++i) x[i] = __ldg(r + i);
    }
}

template <int P, int PP, int GT, int NT, class Pass, class VT>
DEV void reg_pass_body(PassGeom geo, typename Pass::Params prm) {
    constexpr int NE = P * (P + 1) / 2;
    constexpr int NA = Pass::NW * NE + Pass::NV * P + Pass::NF;
    constexpr int NS = Pass::NS;
    constexpr int NAc = NA > 0 ? NA : 1;
    constexpr int NSc = NS > 0 ? NS : 1;
    using AW = typename Pass::AW;
    using AS = typename Pass::AS;

    if (geo.reset_next && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *geo.reset_next = 0;
    const int nact = *geo.n_act;
    const int tile = blockIdx.y;
    if (tile * GT >= nact) return;
    const int seg = blockIdx.x;
    const VT* __restrict__ val = static_cast<const VT*>(geo.val);

    constexpr bool F64 = Pass::F64;
    int gid[GT];
    float beta[GT][P];                 // FP32 passes: log2(e)-scaled
    double betad[GT][F64 ? P : 1];     // FP64 passes
    typename Pass::Gene gp[GT];
#pragma unroll
    for (int j = 0; j < GT; ++j) {
        int slot = tile * GT + j;
        if (slot >= nact) slot = tile * GT;  // duplicate a valid gene; not written
        int g = __ldg(geo.act + slot);
        gid[j] = g;
        if constexpr (F64) {
#pragma unroll
            for (int i = 0; i < P; ++i) betad[j][i] = __ldg(prm.beta_d + (int64_t)g * P + i);
        } else {
#pragma unroll
            for (int i = 0; i < P; ++i) beta[j][i] = __ldg(prm.beta + (int64_t)g * P + i) * kLog2e;
        }
        gp[j] = Pass::load(prm, g);
    }
    if constexpr (Pass::TABLES) {
        __shared__ double psitab[GT * 2 * kPsiTab];
        __shared__ double psiscr[GT * kPsiTab];
        __shared__ double psia[GT];
        if (threadIdx.x < GT) {
#pragma unroll
            for (int j = 0; j < GT; ++j)
                if (j == (int)threadIdx.x) psia[j] = gp[j].a;
        }
        __syncthreads();
        build_psi_tables(GT, psia, psitab, psiscr);
#pragma unroll
        for (int j = 0; j < GT; ++j) {
            gp[j].tab.d1 = psitab + (j * 2 + 0) * kPsiTab;
            gp[j].tab.d2 = psitab + (j * 2 + 1) * kPsiTab;
            gp[j].tab.pa = digamma_d(gp[j].a);
            gp[j].tab.ta = trigamma_d(gp[j].a);
        }
    }

    AW aw[GT][NAc];
    AS as[GT][NSc];
#pragma unroll
    for (int j = 0; j < GT; ++j) {
#pragma unroll
        for (int a = 0; a < NAc; ++a) aw[j][a] = 0;
#pragma unroll
        for (int s = 0; s < NSc; ++s) as[j][s] = 0;
    }

    const int nfs = geo.nbound - 1;
    const int b0 = (int)(((int64_t)seg * nfs) / geo.nseg);
    const int b1 = (int)(((int64_t)(seg + 1) * nfs) / geo.nseg);
    const int c0 = __ldg(geo.bound + b0), c1 = __ldg(geo.bound + b1);

    if constexpr (F64) {
        for (int c = c0 + threadIdx.x; c < c1; c += NT) {
            double x[P];
#pragma unroll
            for (int i = 0; i < P; ++i) x[i] = __ldg(geo.Xd + (int64_t)c * PP + i);
            const double o = __ldg(geo.offd + c);
            double zz[P * (P + 1) / 2];
#pragma unroll
            for (int jj = 0; jj < P; ++jj)
#pragma unroll
                for (int ii = 0; ii <= jj; ++ii) zz[tri_index(ii, jj)] = x[ii] * x[jj];
#pragma unroll
            for (int j = 0; j < GT; ++j) {
                double e = o;
#pragma unroll
                for (int i = 0; i < P; ++i) e = fma(x[i], betad[j][i], e);
                double mu = exp(e);
                RegAcc<P, NAc, NSc, AW, AS, double> acc{aw[j], as[j], x, zz};
                Pass::template dense<double>(gp[j], mu, acc);
            }
        }
    } else {
        // software pipeline: the next cell's row is in flight while the gene
        // tile works on the current one
        int c = c0 + threadIdx.x;
        float xn[P];
        float on = 0.f;
        if (c < c1) {
            load_row<P, PP>(geo.X, c, xn);
            on = __ldg(geo.off + c);
        }
        for (; c < c1; c += NT) {
            float x[P];
#pragma unroll
            for (int i = 0; i < P; ++i) x[i] = xn[i];
            const float o = on * kLog2e;
            const int cn = c + NT;
            if (cn < c1) {
                load_row<P, PP>(geo.X, cn, xn);
                on = __ldg(geo.off + cn);
            }
            float zz[P * (P + 1) / 2];
#pragma unroll
            for (int jj = 0; jj < P; ++jj)
#pragma unroll
                for (int ii = 0; ii <= jj; ++ii) zz[tri_index(ii, jj)] = x[ii] * x[jj];
            // eta of the gene tile, two genes per packed FMA
            float e[GT];
#pragma unroll
            for (int j = 0; j < GT; ++j) e[j] = o;
#pragma unroll
            for (int j = 0; j + 1 < GT; j += 2)
#pragma unroll
                for (int i = 0; i < P; ++i) fma_x2(e[j], e[j + 1], x[i], beta[j][i], beta[j + 1][i]);
            if constexpr (GT & 1) {
#pragma unroll
                for (int i = 0; i < P; ++i) e[GT - 1] = fmaf(x[i], beta[GT - 1][i], e[GT - 1]);
            }
#pragma unroll
            for (int j = 0; j < GT; ++j) {
                float mu = ex2_approx(e[j]);
                RegAcc<P, NAc, NSc, AW, AS, float> acc{aw[j], as[j], x, zz};
                Pass::template dense<float>(gp[j], mu, acc);
            }
        }
    }
    // sparse corrections: UNR independent nonzeros per thread per step, so
    // their dependent (index -> design row) loads overlap
    constexpr int UNR = (F64 || Pass::NS > 0) ? (P <= 4 ? 2 : 1) : 4;
#pragma unroll
    for (int j = 0; j < GT; ++j) {
        const int64_t* sp = geo.segptr + (int64_t)gid[j] * geo.nbound;
        const int64_t e0 = __ldg(sp + b0), e1 = __ldg(sp + b1);
        for (int64_t eb = e0 + threadIdx.x; eb < e1; eb += (int64_t)UNR * NT) {
            int cc[UNR];
            float yy[UNR];
            bool ok[UNR];
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                const int64_t e = eb + (int64_t)u * NT;
                ok[u] = e < e1;
                cc[u] = ok[u] ? __ldg(geo.col + e) : c0;
                yy[u] = ok[u] ? load_val(val, e) : 0.f;
            }
            if constexpr (F64) {
                double xr[UNR][P];
                double ol[UNR];
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
#pragma unroll
                    for (int i = 0; i < P; ++i) xr[u][i] = __ldg(geo.Xd + (int64_t)cc[u] * PP + i);
                    ol[u] = __ldg(geo.offd + cc[u]);
                }
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
                    if (!ok[u]) continue;
                    double el = ol[u];
#pragma unroll
                    for (int i = 0; i < P; ++i) el = fma(xr[u][i], betad[j][i], el);
                    double mu = exp(el);
                    double zz[P * (P + 1) / 2];
#pragma unroll
                    for (int jj = 0; jj < P; ++jj)
#pragma unroll
                        for (int ii = 0; ii <= jj; ++ii) zz[tri_index(ii, jj)] = xr[u][ii] * xr[u][jj];
                    RegAcc<P, NAc, NSc, AW, AS, double> acc{aw[j], as[j], xr[u], zz};
                    Pass::template sparse<double>(gp[j], mu, yy[u], acc);
                }
            } else {
                float xr[UNR][P];
                float ol[UNR];
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
                    load_row<P, PP>(geo.X, cc[u], xr[u]);
                    ol[u] = __ldg(geo.off + cc[u]);
                }
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
                    if (!ok[u]) continue;
                    float el = ol[u] * kLog2e;
#pragma unroll
                    for (int i = 0; i < P; ++i) el = fmaf(xr[u][i], beta[j][i], el);
                    float mu = ex2_approx(el);
                    float zz[P * (P + 1) / 2];
#pragma unroll
                    for (int jj = 0; jj < P; ++jj)
#pragma unroll
                        for (int ii = 0; ii <= jj; ++ii) zz[tri_index(ii, jj)] = xr[u][ii] * xr[u][jj];
                    RegAcc<P, NAc, NSc, AW, AS, float> acc{aw[j], as[j], xr[u], zz};
                    Pass::template sparse<float>(gp[j], mu, yy[u], acc);
                }
            }
        }
    }

    // block reduction: warp shuffles, then across warps through shared memory
    constexpr int NWARP = NT / 32;
    __shared__ AW redW[NWARP][GT * NAc];
    __shared__ AS redS[NWARP][GT * NSc];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < GT; ++j) {
        if constexpr (NA > 0) {
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                AW v = warp_sum(aw[j][a]);
                if (lane == 0) redW[warp][j * NAc + a] = v;
            }
        }
        if constexpr (NS > 0) {
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                AS v = warp_sum(as[j][s]);
                if (lane == 0) redS[warp][j * NSc + s] = v;
            }
        }
    }
    __syncthreads();
    if constexpr (NA > 0) {
        for (int t = threadIdx.x; t < GT * NA; t += NT) {
            int j = t / NA, a = t - j * NA;
            int slot = tile * GT + j;
            if (slot >= nact) continue;
            AW s = 0;
#pragma unroll
            for (int w = 0; w < NWARP; ++w) s += redW[w][j * NAc + a];
            static_cast<AW*>(geo.partW)[((int64_t)seg * geo.slot_stride + slot) * NA + a] = s;
        }
    }
    if constexpr (NS > 0) {
        for (int t = threadIdx.x; t < GT * NS; t += NT) {
            int j = t / NS, s = t - j * NS;
            int slot = tile * GT + j;
            if (slot >= nact) continue;
            double v = 0.0;
#pragma unroll
            for (int w = 0; w < NWARP; ++w) v += (double)redS[w][j * NSc + s];
            geo.partS[((int64_t)seg * geo.slot_stride + slot) * NS + s] = v;
        }
    }
}

// Two entry points with the same body.  The IRLS pass runs best with the
// compiler's default register budget for 256 threads (120 registers at
// p = 4, four genes per thread); the MOM, MLE and bread passes measured
// faster when told one block per SM is enough (more registers, no spills).
template <int P, int PP, int GT, int NT, class Pass, class VT>
__global__ void __launch_bounds__(NT) reg_pass_kernel(PassGeom geo, typename Pass::Params prm) {
    reg_pass_body<P, PP, GT, NT, Pass, VT>(geo, prm);
}
template <int P, int PP, int GT, int NT, class Pass, class VT>
__global__ void __launch_bounds__(NT, 1) reg_pass_kernel_b1(PassGeom geo, typename Pass::Params prm) {
    reg_pass_body<P, PP, GT, NT, Pass, VT>(geo, prm);
}

// ---------------------------------------------------------------------
// engine 2: shared-memory tiles, any p <= 32 (runtime p)
// ---------------------------------------------------------------------
// Threads 0..NT-1 are split into GT gene groups of TC = NT/GT threads.  Per
// chunk of TC cells: X rows are staged in shared memory, the genes' nonzero
// counts are scattered into a dense shared tile, each thread evaluates the
// per-cell weights of one (gene, cell) pair, and then every thread adds the
// cell terms of the outputs it owns.
constexpr int kGenNT = 256;
constexpr int kGenKMAX = 16;

// byte offset of the design/weight tiles in the generic engine's shared
// memory: after the FP64 scalar tile and the per-gene bookkeeping, 16-byte
// aligned
__host__ __device__ __forceinline__ size_t gen_wt_offset(int NS, int GT) {
    size_t b = (size_t)NS * kGenNT * 8 + (size_t)GT * (8 + 8 + 4 + 4);
    return (b + 15) & ~(size_t)15;
}

// F32W: the plain comparison form -- per-(gene, cell) weights computed in
// FP32 from the FP32 design, offsets and beta (exp2 / reciprocal on the
// special function units), staged and contracted in FP32 with FP32 sums per
// chunk of cells.  Only for passes whose per-cell arithmetic is FP32
// (Pass::F64 false); the FP64 passes (MOM, bread/meat) are FP64 in every form.
template <class Pass, class VT, bool F32W = false>
__global__ void __launch_bounds__(kGenNT) gen_pass_kernel(PassGeom geo, typename Pass::Params prm,
                                                          int P, int GT) {
    static_assert(!(F32W && Pass::F64), "FP32 staging only for FP32 passes");
    constexpr int NWV = Pass::NW + Pass::NV + Pass::NF;
    constexpr int NS = Pass::NS;
    using AS = typename Pass::AS;
    const int NE = P * (P + 1) / 2;
    const int NA = Pass::NW * NE + Pass::NV * P + Pass::NF;
    const int TC = kGenNT / GT;
    const int XS = (P + 1) | 1;  // odd row stride: conflict-free column reads

    if (geo.reset_next && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *geo.reset_next = 0;
    const int nact = *geo.n_act;
    const int tile = blockIdx.y;
    if (tile * GT >= nact) return;
    const int seg = blockIdx.x;
    const VT* __restrict__ val = static_cast<const VT*>(geo.val);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* wsc = reinterpret_cast<double*>(smem_raw);              // [NS][GT][TC]
    int64_t* cursor = reinterpret_cast<int64_t*>(wsc + NS * kGenNT); // [GT]
    int64_t* cend = cursor + GT;                                    // [GT]
    int* cnt = reinterpret_cast<int*>(cend + GT);                   // [GT]
    int* gids = cnt + GT;                                           // [GT]
    // design rows and per-cell weights are staged in double in the chosen
    // form: FP32 staging left errors of ~1.5e-5 in beta for slowly converging
    // genes at p = 12, and FP64 FMAs run at half the FP32 rate on this part
    // while the engine is bound by shared-memory traffic anyway
    using WT = typename std::conditional<F32W, float, double>::type;
    WT* xsm = reinterpret_cast<WT*>(smem_raw + gen_wt_offset(NS, GT));  // [TC][XS]
    WT* wts = xsm + TC * XS;                                        // [NWV][GT][TC]
    float* ys = reinterpret_cast<float*>(wts + NWV * kGenNT);       // [GT][TC]
    float* betas = ys + kGenNT;                                     // [GT][P]
    const int t = threadIdx.x;
    const int nfs = geo.nbound - 1;
    const int b0 = (int)(((int64_t)seg * nfs) / geo.nseg);
    const int b1 = (int)(((int64_t)(seg + 1) * nfs) / geo.nseg);
    const int c0 = __ldg(geo.bound + b0), c1 = __ldg(geo.bound + b1);
    if (t < GT) {
        int slot = tile * GT + t;
        if (slot >= nact) slot = tile * GT;
        int g = __ldg(geo.act + slot);
        gids[t] = g;
        const int64_t* sp = geo.segptr + (int64_t)g * geo.nbound;
        cursor[t] = __ldg(sp + b0);
        cend[t] = __ldg(sp + b1);
    }
    __syncthreads();
    for (int i = t; i < GT * P; i += kGenNT) {
        int j = i / P, k = i - j * P;
        betas[i] = __ldg(prm.beta + (int64_t)gids[j] * P + k) * (F32W ? kLog2e : 1.f);
    }
    const int gA = t / TC, cA = t - gA * TC;
    typename Pass::Gene gpar = Pass::load(prm, gids[gA]);
    if constexpr (Pass::TABLES) {
        __shared__ double psitab[8 * 2 * kPsiTab];
        __shared__ double psiscr[8 * kPsiTab];
        __shared__ double psia[8];
        if (cA == 0) psia[gA] = gpar.a;
        __syncthreads();
        build_psi_tables(GT, psia, psitab, psiscr);
        gpar.tab.d1 = psitab + (gA * 2 + 0) * kPsiTab;
        gpar.tab.d2 = psitab + (gA * 2 + 1) * kPsiTab;
        gpar.tab.pa = digamma_d(gpar.a);
        gpar.tab.ta = trigamma_d(gpar.a);
    }

    // owned outputs (W-type): o = t + k*NT over [0, GT*NA); per-chunk sums
    // are folded into FP64 accumulators
    double acc[kGenKMAX];
    short oi[kGenKMAX], oj[kGenKMAX], og[kGenKMAX], ow[kGenKMAX];
    int nown = 0;
#pragma unroll
    for (int k = 0; k < kGenKMAX; ++k) {
        acc[k] = 0;
        int o = t + k * kGenNT;
        og[k] = 0; ow[k] = 0; oi[k] = 0; oj[k] = 0;
        if (o < GT * NA) {
            nown = k + 1;
            int g = o / NA, a = o - g * NA;
            og[k] = (short)g;
            if (a < Pass::NW * NE) {
                int w = a / NE, q = a - w * NE;
                int j = 0;
                while ((j + 1) * (j + 2) / 2 <= q) ++j;
                int i = q - j * (j + 1) / 2;
                ow[k] = (short)w; oi[k] = (short)i; oj[k] = (short)j;
            } else if (a < Pass::NW * NE + Pass::NV * P) {
                int r = a - Pass::NW * NE;
                int v = r / P, i = r - v * P;
                ow[k] = (short)(Pass::NW + v); oi[k] = (short)i; oj[k] = (short)P;  // x_P == 1
            } else {
                int f = a - Pass::NW * NE - Pass::NV * P;  // FP32 scalar: w * 1 * 1
                ow[k] = (short)(Pass::NW + Pass::NV + f); oi[k] = (short)P; oj[k] = (short)P;
            }
        }
    }
    // owned scalar outputs: thread t < GT*NS owns (gene t/NS, scalar t%NS)
    AS sacc = 0;
    __syncthreads();

    const double* bd = prm.beta_d + (int64_t)gids[gA] * P;

    for (int cb = c0; cb < c1; cb += TC) {
        const int nc = min(TC, c1 - cb);
        // stage X rows (+ the constant 1 column) and offsets; clear the tile
        for (int i = t; i < nc * P; i += kGenNT) {
            int c = i / P, k = i - c * P;
            if constexpr (Pass::F64 || !F32W)
                xsm[c * XS + k] = (WT)__ldg(geo.Xd + (int64_t)(cb + c) * geo.xs + k);
            else
                xsm[c * XS + k] = __ldg(geo.X + (int64_t)(cb + c) * geo.xs + k);
        }
        for (int c = t; c < TC; c += kGenNT) xsm[c * XS + P] = (WT)1;
        ys[t] = 0.f;
        if (t < GT) cnt[t] = 0;
        __syncthreads();
        // scatter this chunk's nonzeros of gene gA (at most TC entries)
        {
            int64_t e = cursor[gA] + cA;
            if (e < cend[gA]) {
                int c = __ldg(geo.col + e);
                if (c >= cb && c < cb + nc) {
                    ys[gA * TC + (c - cb)] = load_val(val, e);
                    atomicAdd(&cnt[gA], 1);
                }
            }
        }
        __syncthreads();
        if (cA == 0) cursor[gA] += cnt[gA];
        // per-(gene, cell) weights
        {
            // per-(gene, cell) weights: FP64 in the chosen form (this engine's
            // cost is the outer-product phase, and FP64 here keeps the
            // per-step error of slowly converging genes small), FP32 in the
            // plain form
            RecAcc<NWV, NS, AS, WT> rec;
            rec.zero();
            if (cA < nc) {
                const int64_t c = cb + cA;
                const float y = ys[gA * TC + cA];
                if constexpr (F32W) {
                    // eta in log2 units: x . (log2(e) beta) + log2(e) off
                    const float* bf = betas + gA * P;
                    float e = __ldg(geo.off + c) * kLog2e;
                    for (int i = 0; i < P; ++i) e = fmaf(xsm[cA * XS + i], bf[i], e);
                    const float mu = ex2_approx(e);
                    Pass::template dense<float>(gpar, mu, rec);
                    if (y != 0.f) Pass::template sparse<float>(gpar, mu, y, rec);
                } else {
                    double e = __ldg(geo.offd + c);
                    for (int i = 0; i < P; ++i) e = fma(__ldg(geo.Xd + c * geo.xs + i), __ldg(bd + i), e);
                    double mu = exp(e);
                    Pass::template dense<double>(gpar, mu, rec);
                    if (y != 0.f) Pass::template sparse<double>(gpar, mu, y, rec);
                }
            }
#pragma unroll
            for (int w = 0; w < NWV; ++w) wts[(w * GT + gA) * TC + cA] = (WT)rec.w[w];
#pragma unroll
            for (int s = 0; s < NS; ++s) wsc[(s * GT + gA) * TC + cA] = rec.s[s];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kGenKMAX; ++k) {
            if (k >= nown) break;
            const WT* wp = wts + (ow[k] * GT + og[k]) * TC;
            const WT* xi = xsm + oi[k];
            const WT* xj = xsm + oj[k];
            WT s = 0;
            for (int c = 0; c < nc; ++c) s = fma(wp[c] * xi[c * XS], xj[c * XS], s);
            acc[k] += (double)s;
        }
        if (NS > 0 && t < GT * NS) {
            constexpr int NSd = NS > 0 ? NS : 1;
            int g = t / NSd, s = t - g * NSd;
            const double* sp = wsc + (s * GT + g) * TC;
            AS v = sacc;
            for (int c = 0; c < nc; ++c) v += sp[c];
            sacc = v;
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < kGenKMAX; ++k) {
        if (k >= nown) break;
        int o = t + k * kGenNT;
        int g = o / NA, a = o - g * NA;
        int slot = tile * GT + g;
        if (slot < nact)  // FP64 partial sums for every pass of this engine
            static_cast<double*>(geo.partW)[((int64_t)seg * geo.slot_stride + slot) * NA + a] = acc[k];
    }
    if (NS > 0 && t < GT * NS) {
        constexpr int NSd = NS > 0 ? NS : 1;
        int g = t / NSd, s = t - g * NSd;
        int slot = tile * GT + g;
        if (slot < nact) geo.partS[((int64_t)seg * geo.slot_stride + slot) * NS + s] = (double)sacc;
    }
}

}  // namespace devil
