// test_de on the device (R/test.R:85-134): contrast LFCs, t-test p-values
// in FP64, stats::p.adjust, LFC clipping; and the per-cell NB
// log-likelihood adjoint.
#include <cub/cub.cuh>

#include "internal.h"

namespace devil {

static inline unsigned nblk(int64_t m, int t) { return (unsigned)((m + t - 1) / t); }

// Continued fraction of the regularised incomplete beta I_x(a, b) by the
// modified Lentz method; converges for x < (a + 1)/(a + b + 2).
DEV double betacf_d(double a, double b, double x) {
    const double tiny = 1e-300, eps = 1e-16;
    double qab = a + b, qap = a + 1.0, qam = a - 1.0;
    double c = 1.0, d = 1.0 - qab * x / qap;
    if (fabs(d) < tiny) d = tiny;
    d = 1.0 / d;
    double h = d;
    for (int m = 1; m <= 20000; ++m) {
        int m2 = 2 * m;
        double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
        d = 1.0 + aa * d; if (fabs(d) < tiny) d = tiny;
        c = 1.0 + aa / c; if (fabs(c) < tiny) c = tiny;
        d = 1.0 / d; h *= d * c;
        aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
        d = 1.0 + aa * d; if (fabs(d) < tiny) d = tiny;
        c = 1.0 + aa / c; if (fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (fabs(del - 1.0) < eps) break;
    }
    return h;
}

// lgamma(a + b) - lgamma(a) for a >= 100 from the Stirling series of
// ln G(z) = (z - 1/2) ln z - z + ln(2 pi)/2 + 1/(12 z) - 1/(360 z^3) + ...,
// the leading terms differenced analytically (df up to 1e6 keeps full
// relative precision).
DEV double lgamma_diff_large(double a, double b) {
    double z = a + b;
    double d = (a - 0.5) * log1p(b / a) + b * log(z) - b;
    d += (1.0 / 12.0) * (1.0 / z - 1.0 / a);
    d -= (1.0 / 360.0) * (1.0 / (z * z * z) - 1.0 / (a * a * a));
    d += (1.0 / 1260.0) * (1.0 / (z * z * z * z * z) - 1.0 / (a * a * a * a * a));
    return d;
}
DEV double log_beta_d(double a, double b) {
    if (a >= 100.0 && b < a) return lgamma(b) - lgamma_diff_large(a, b);
    if (b >= 100.0 && a < b) return lgamma(a) - lgamma_diff_large(b, a);
    return lgamma(a) + lgamma(b) - lgamma(a + b);
}

// I_x(a, b) with both x and 1 - x supplied (no cancellation in either)
DEV double ibeta_d(double a, double b, double x, double omx) {
    if (x <= 0.0) return 0.0;
    if (omx <= 0.0) return 1.0;
    double lbeta = log_beta_d(a, b);
    double lfront = (x > 0.5) ? a * log1p(-omx) + b * log(omx) : a * log(x) + b * log1p(-x);
    lfront -= lbeta;
    if (x < (a + 1.0) / (a + b + 2.0)) return exp(lfront) * betacf_d(a, b, x) / a;
    return 1.0 - exp(lfront) * betacf_d(b, a, omx) / b;
}

// 2 * pt(|t|, df, lower.tail = FALSE) = I_{df/(df+t^2)}(df/2, 1/2)
DEV double t_two_sided(double t, double df) {
    if (isnan(t) || isnan(df) || df <= 0.0) return NAN;
    t = fabs(t);
    if (isinf(t)) return 0.0;
    double t2 = t * t;
    return ibeta_d(0.5 * df, 0.5, df / (df + t2), t2 / (df + t2));
}

__global__ void test_pvalues_kernel(int64_t G, int P, const double* beta, const double* bread,
                                    const double* sandwich, double df, const double* c,
                                    double max_lfc, double* pval, double* lfc) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G;
         g += (int64_t)gridDim.x * blockDim.x) {
        double l = 0.0;
        for (int j = 0; j < P; ++j) l += beta[g * P + j] * c[j];
        const double* Hn = bread + g * P * P;
        double vn = 0.0;
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i) vn += c[i] * Hn[j * P + i] * c[j];
        double pn = t_two_sided(fabs(l) / sqrt(vn), df);
        double p = pn;
        if (sandwich) {
            const double* Hc = sandwich + g * P * P;
            double vc = 0.0;
            for (int j = 0; j < P; ++j)
                for (int i = 0; i < P; ++i) vc += c[i] * Hc[j * P + i] * c[j];
            double pc = t_two_sided(fabs(l) / sqrt(vc), df);
            p = (isnan(pc) || isnan(pn)) ? NAN : fmax(pc, pn);
        }
        pval[g] = p;
        double lf = l / log(2.0);
        if (lf >= max_lfc) lf = max_lfc;
        if (lf <= -max_lfc) lf = -max_lfc;
        lfc[g] = lf;
    }
}

cudaError_t launch_test_pvalues(int64_t G, int P, const double* beta, const double* bread,
                                const double* sandwich, double df, const double* contrast_dev,
                                double max_lfc, double* pval, double* lfc, cudaStream_t st) {
    if (G == 0) return cudaSuccess;
    test_pvalues_kernel<<<(unsigned)std::min<int64_t>(nblk(G, 128), 4096), 128, 0, st>>>(
        G, P, beta, bread, sandwich, df, contrast_dev, max_lfc, pval, lfc);
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// stats::p.adjust.  NaN p-values are excluded from n and stay NaN.
// ------------------------------------------------------------------
__global__ void padj_prepare_kernel(const double* p, int64_t m, double* keys, int32_t* idx,
                                    int32_t* nvalid) {
    int cnt = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        double v = p[i];
        bool ok = !isnan(v);
        keys[i] = ok ? v : INFINITY;
        idx[i] = (int32_t)i;
        cnt += ok;
    }
    cnt = warp_sum(cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(nvalid, cnt);
}

DEV double dm_times(int64_t m, double v) { return (double)m * v; }

// s + e += v as a double-double (error-free TwoSum of the high parts)
DEV void dd_add(double& s, double& e, double v) {
    const double t = s + v;
    const double bp = t - s;
    e += (s - (t - bp)) + (v - bp);
    s = t;
}

// one block: scan over the sorted valid p-values (ascending ranks 1..n)
__global__ void padj_scan_kernel(const double* sk, const int32_t* sidx, const int32_t* nvalid_p,
                                 int64_t m, const double* p, int method, double* out) {
    const int64_t n = *nvalid_p;
    const int T = blockDim.x, t = threadIdx.x;
    // pass-through: NaN stay NaN, method none or n <= 1 returns p
    for (int64_t i = t; i < m; i += T) out[i] = p[i];
    __syncthreads();
    if (method == 0 || n <= 1) return;
    // hommel with two p-values is hochberg (as stats::p.adjust switches);
    // n >= 3 runs in the hommel kernels
    if (method == 6) {
        if (n >= 3) return;
        method = 4;
    }
    const double dn = (double)n;
    double q = 1.0;
    if (method == 5) {
        // q = sum(1/(1:n)) of the double-rounded terms, summed in
        // double-double and rounded once: the correctly rounded sum (R sums
        // in extended precision)
        double hs = 0.0, he = 0.0;
        for (int64_t k = 1 + t; k <= n; k += T) dd_add(hs, he, 1.0 / (double)k);
        __shared__ double qh[1024], ql[1024];
        qh[t] = hs;
        ql[t] = he;
        __syncthreads();
        if (t == 0) {
            double a = 0.0, ae = 0.0;
            for (int w = 0; w < T; ++w) {
                dd_add(a, ae, qh[w]);
                ae += ql[w];
            }
            qh[0] = a + ae;
        }
        __syncthreads();
        q = qh[0];
    }
    auto val = [&](int64_t k) -> double {  // k = 0-based ascending rank
        double pk = sk[k];
        double i = (double)(k + 1);
        switch (method) {
            case 1: return dn / i * pk;            // BH
            case 5: return q * dn / i * pk;        // BY
            case 4: return (dn + 1.0 - i) * pk;    // hochberg
            case 3: return (dn + 1.0 - i) * pk;    // holm
            case 2: return dn * pk;                // bonferroni
        }
        return pk;
    };
    if (method == 2) {
        for (int64_t k = t; k < n; k += T) out[sidx[k]] = fmin(1.0, val(k));
        return;
    }
    const bool suffix_min = (method == 1 || method == 5 || method == 4);
    const int64_t chunk = (n + T - 1) / T;
    const int64_t k0 = (int64_t)t * chunk, k1 = min(n, k0 + chunk);
    double agg = suffix_min ? INFINITY : -INFINITY;
    for (int64_t k = k0; k < k1; ++k) {
        double v = val(k);
        agg = suffix_min ? fmin(agg, v) : fmax(agg, v);
    }
    __shared__ double aggs[1024];
    aggs[t] = agg;
    __syncthreads();
    if (t == 0) {
        if (suffix_min) {
            double run = INFINITY;
            for (int w = T - 1; w >= 0; --w) { double a = aggs[w]; aggs[w] = run; run = fmin(run, a); }
        } else {
            double run = -INFINITY;
            for (int w = 0; w < T; ++w) { double a = aggs[w]; aggs[w] = run; run = fmax(run, a); }
        }
    }
    __syncthreads();
    double run = aggs[t];  // exclusive aggregate from the other side
    if (suffix_min) {
        for (int64_t k = k1 - 1; k >= k0; --k) {
            run = fmin(run, val(k));
            out[sidx[k]] = fmin(1.0, run);
        }
    } else {
        for (int64_t k = k0; k < k1; ++k) {
            run = fmax(run, val(k));
            out[sidx[k]] = fmin(1.0, run);
        }
    }
}

// Hommel (stats::p.adjust, "hommel") on the ascending p-values s[0..n):
//   pa = min_i n s_i / i;  for m = n-1 .. 2:
//     q1 = min_{j=2..m} m s_{n-m+j} / j                  (1-based ranks)
//     q_i = min(m s_i, q1) for i <= n-m+1, q_{n-m+1} beyond
//     pa = max(pa, q)
//   result = max(pa, s).
// Every m is independent given the sorted p-values, and pa is a max over
// m, so the O(n^2) loop of the reference runs as two parallel kernels:
// q1 for every m (a block per m), then, per rank i, the max over m.
__global__ void hommel_q1_kernel(const double* s, const int32_t* nvalid_p, double* q1) {
    const int64_t n = *nvalid_p;
    const int64_t m = blockIdx.x + 2;  // 2 .. n-1
    if (n < 3 || m > n - 1) return;
    const double dm = (double)m;
    double v = INFINITY;
    for (int64_t j = 2 + threadIdx.x; j <= m; j += blockDim.x)
        v = fmin(v, dm * s[n - m + j - 1] / (double)j);
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmin(r, red[w]);
        q1[m] = r;
    }
}

__global__ void hommel_pa_kernel(const double* s, const int32_t* sidx, const int32_t* nvalid_p,
                                 const double* q1, double* out) {
    const int64_t n = *nvalid_p;
    if (n < 3) return;
    const double dn = (double)n;
    // pa0 = min_i n s_i / i, the same in every thread (one warp-strided pass
    // per thread over all ranks would cost n^2: read it from the block)
    __shared__ double red[32];
    __shared__ double pa0s;
    double v = INFINITY;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) v = fmin(v, dn * s[i] / (double)(i + 1));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmin(r, red[w]);
        pa0s = r;
    }
    __syncthreads();
    const double pa0 = pa0s;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r1 = i + 1;  // 1-based rank
        double pa = pa0;
        for (int64_t m = 2; m <= n - 1; ++m) {
            const int64_t k = r1 <= n - m + 1 ? i : n - m;  // rank n-m+1, 0-based
            pa = fmax(pa, fmin(dm_times(m, s[k]), q1[m]));
        }
        out[sidx[i]] = fmax(pa, s[i]);  // <= 1: every q_m is at most s_n
    }
}

static size_t cub_sort_bytes(int64_t m) {
    size_t b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b, (const double*)nullptr, (double*)nullptr,
                                    (const int32_t*)nullptr, (int32_t*)nullptr, (int)m);
    return b;
}

static size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

size_t p_adjust_temp_bytes(int64_t m) {
    return align_up(cub_sort_bytes(m)) + 2 * align_up(8 * (size_t)m) + 2 * align_up(4 * (size_t)m) +
           256;
}

cudaError_t launch_p_adjust(int64_t m, const double* p, int method, double* out, void* temp,
                            size_t temp_bytes, cudaStream_t st) {
    if (m == 0) return cudaSuccess;
    if (temp_bytes < p_adjust_temp_bytes(m)) return cudaErrorInvalidValue;
    char* b = static_cast<char*>(temp);
    size_t sb = cub_sort_bytes(m);
    void* cub_tmp = b; b += align_up(sb);
    double* k_in = reinterpret_cast<double*>(b); b += align_up(8 * (size_t)m);
    double* k_out = reinterpret_cast<double*>(b); b += align_up(8 * (size_t)m);
    int32_t* i_in = reinterpret_cast<int32_t*>(b); b += align_up(4 * (size_t)m);
    int32_t* i_out = reinterpret_cast<int32_t*>(b); b += align_up(4 * (size_t)m);
    int32_t* nvalid = reinterpret_cast<int32_t*>(b);
    double* q1 = k_in;  // hommel's per-m minima: the unsorted keys are dead after the sort
    cudaError_t e = cudaMemsetAsync(nvalid, 0, sizeof(int32_t), st);
    if (e != cudaSuccess) return e;
    padj_prepare_kernel<<<(unsigned)std::min<int64_t>(nblk(m, 256), 1024), 256, 0, st>>>(p, m, k_in, i_in, nvalid);
    e = cub::DeviceRadixSort::SortPairs(cub_tmp, sb, k_in, k_out, i_in, i_out, (int)m, 0, 64, st);
    if (e != cudaSuccess) return e;
    padj_scan_kernel<<<1, 1024, 0, st>>>(k_out, i_out, nvalid, m, p, method, out);
    if (method == 6 && m >= 3) {
        // blocks for every m the valid count can reach; those beyond n - 1 exit
        hommel_q1_kernel<<<(unsigned)(m - 2), 256, 0, st>>>(k_out, nvalid, q1);
        hommel_pa_kernel<<<(unsigned)std::min<int64_t>(nblk(m, 256), 1184), 256, 0, st>>>(
            k_out, i_out, nvalid, q1, out);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------
// Per-cell NB log-likelihood and its adjoint.  With a = 1/theta and
// mu = exp(eta):
//   l   = lgamma(y+a) - lgamma(a) - lgamma(y+1) + y eta - (y+a) log(mu+a)
//         + a log a
//   dl/deta      = (y - mu) / (1 + mu theta)
//   dl/dlogtheta = -a [psi(y+a) - psi(a) - log1p(mu theta) + (mu - y)/(mu + a)]
// dl/deta times x_c is the per-cell score of src/variance.cpp:64-85; the
// sum over cells of dl/dlogtheta is the non-Cox-Reid part of the
// dispersion score of src/overdispersion.cpp:95-178.
// ------------------------------------------------------------------
__global__ void nb_adjoint_kernel(int64_t n, const double* y, const double* eta, double log_theta,
                                  double* ll, double* d_eta, double* d_lt) {
    const double theta = exp(log_theta), a = 1.0 / theta;
    const double pa = digamma_d(a);
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        double yy = y[c], e = eta[c];
        double mu = exp(e);
        if (ll)
            ll[c] = lgamma(yy + a) - lgamma(a) - lgamma(yy + 1.0) + yy * e -
                    (yy + a) * log(mu + a) + a * log(a);
        if (d_eta) d_eta[c] = (yy - mu) / (1.0 + mu * theta);
        if (d_lt) {
            double dpsi = (yy == 0.0) ? 0.0 : digamma_d(yy + a) - pa;
            d_lt[c] = -a * (dpsi - log1p(mu * theta) + (mu - yy) / (mu + a));
        }
    }
}
cudaError_t launch_nb_adjoint(int64_t n, const double* y, const double* eta, double log_theta,
                              double* ll, double* d_eta, double* d_lt, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    nb_adjoint_kernel<<<(unsigned)std::min<int64_t>(nblk(n, 256), 4096), 256, 0, st>>>(
        n, y, eta, log_theta, ll, d_eta, d_lt);
    return cudaGetLastError();
}

}  // namespace devil
