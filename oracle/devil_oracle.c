/*
 * devil_oracle.c -- FP64 CPU restatement of devil's per-gene negative-binomial
 * GLM path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and
 * the CPU-baseline leg of bench.py compare against it or time it.  The product
 * (libdevil_b200.so) never links or calls anything in this directory.
 *
 * Every function names the reference file:line it restates (paths are
 * relative to the devil source tree).  Third-party arithmetic the reference
 * reaches (Eigen inverse, R nmath digamma/trigamma/pt, LINPACK qr,
 * stats::p.adjust, stats::nlminb) is restated here from its published
 * mathematics:
 *   - digamma / trigamma: recurrence psi(x) = psi(x+1) - 1/x up to x >= 10,
 *     then the Stirling-type asymptotic series with Bernoulli coefficients.
 *   - t upper tail: 2*pt(t, df, upper) = I_x(df/2, 1/2), x = df/(df+t^2),
 *     the regularised incomplete beta evaluated by its continued fraction
 *     with the modified Lentz algorithm.
 *   - qr: Householder QR (no pivoting; full column rank is required, as
 *     R's solve(R, .) requires).
 *   - nlminb on log(theta): replaced by a bracketed Newton root search on the
 *     same score function, converged to |d log theta| < 1e-10 (the oracle's
 *     definition of the MLE; the reference's nlminb stops at rel.tol=1e-3).
 *
 * Parity status: the formulas pinned by the reference's own tests
 * (tests/testthat/test-size_factors.R, test-overdispersion.R, test-beta.R,
 * test-test.R) are checked in tests/test_oracle_known_answers.py.  For
 * beta_fit iterates, the MLE theta, bread/meat and p-values the reference
 * ships no golden vectors and cannot be built here (R, Rcpp, Eigen,
 * Armadillo absent): parity for those values is unpinned beyond this
 * restatement.
 *
 * Layouts (shared with the CUDA library):
 *   counts  CSR, gene-major: rowptr[G+1] (int64), col[nnz] (int32, sorted
 *           within a row), val[nnz] (double)
 *   X       n x p, column-major (R layout): X[j*n + c]
 *   matrices per gene p x p column-major, genes consecutive.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_ZERO_COLUMN 1
#define ORC_ERR_SINGULAR 2
#define ORC_ERR_ARG 3
#define ORC_ERR_UNSORTED 4
#define ORC_ERR_ALLOC 5

/* ------------------------------------------------------------------ */
/* special functions                                                   */
/* ------------------------------------------------------------------ */

double orc_digamma(double x)
{
    if (isnan(x)) return x;
    if (x <= 0.0 && floor(x) == x) return NAN;
    double r = 0.0;
    if (x < 0.0) { /* reflection: psi(1-x) - psi(x) = pi cot(pi x) */
        return orc_digamma(1.0 - x) - M_PI / tan(M_PI * x);
    }
    while (x < 10.0) { r -= 1.0 / x; x += 1.0; }
    double f = 1.0 / (x * x);
    /* B2k/(2k) coefficients: 1/12, 1/120, 1/252, 1/240, 1/132, 691/32760, 1/12 */
    double t = f * (-1.0 / 12 + f * (1.0 / 120 + f * (-1.0 / 252 + f * (1.0 / 240 +
               f * (-1.0 / 132 + f * (691.0 / 32760 + f * (-1.0 / 12)))))));
    return r + log(x) - 0.5 / x + t;
}

double orc_trigamma(double x)
{
    if (isnan(x)) return x;
    if (x <= 0.0 && floor(x) == x) return NAN;
    double r = 0.0;
    if (x < 0.0) { /* psi1(1-x) + psi1(x) = pi^2 / sin^2(pi x) */
        double s = sin(M_PI * x);
        return -orc_trigamma(1.0 - x) + M_PI * M_PI / (s * s);
    }
    while (x < 10.0) { r += 1.0 / (x * x); x += 1.0; }
    double f = 1.0 / (x * x);
    /* psi1(x) ~ 1/x + 1/(2x^2) + sum B2k / x^(2k+1) */
    double t = 1.0 / x + f / 2.0 + (f / x) * (1.0 / 6 + f * (-1.0 / 30 + f * (1.0 / 42 +
               f * (-1.0 / 30 + f * (5.0 / 66 + f * (-691.0 / 2730 + f * (7.0 / 6)))))));
    return r + t;
}

/* continued fraction for I_x(a,b) (modified Lentz); valid when
 * x < (a+1)/(a+b+2).  Returns the fraction value. */
static double betacf(double a, double b, double x)
{
    const double tiny = 1e-300, eps = 1e-16;
    double qab = a + b, qap = a + 1.0, qam = a - 1.0;
    double c = 1.0, d = 1.0 - qab * x / qap;
    if (fabs(d) < tiny) d = tiny;
    d = 1.0 / d;
    double h = d;
    for (int m = 1; m <= 100000; m++) {
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

/* lgamma(a + b) - lgamma(a) for a >= 100, from the Stirling series
 * ln G(z) = (z - 1/2) ln z - z + ln(2 pi)/2 + 1/(12 z) - 1/(360 z^3) + ...
 * with the leading terms differenced analytically (no cancellation). */
static double lgamma_diff_large(double a, double b)
{
    double z = a + b;
    double d = (a - 0.5) * log1p(b / a) + b * log(z) - b;
    d += (1.0 / 12.0) * (1.0 / z - 1.0 / a);
    d -= (1.0 / 360.0) * (1.0 / (z * z * z) - 1.0 / (a * a * a));
    d += (1.0 / 1260.0) * (1.0 / (z * z * z * z * z) - 1.0 / (a * a * a * a * a));
    return d;
}

static double log_beta(double a, double b)
{
    if (a >= 100.0 && b < a) return lgamma(b) - lgamma_diff_large(a, b);
    if (b >= 100.0 && a < b) return lgamma(a) - lgamma_diff_large(b, a);
    return lgamma(a) + lgamma(b) - lgamma(a + b);
}

/* regularised incomplete beta I_x(a,b) with x and (1-x) both supplied so
 * that neither is formed by cancellation. */
static double ibeta(double a, double b, double x, double omx)
{
    if (x <= 0.0) return 0.0;
    if (omx <= 0.0) return 1.0;
    double lbeta = log_beta(a, b);
    double lfront = a * log(x) + b * log1p(-x);
    if (x > 0.5) lfront = a * log1p(-omx) + b * log(omx);
    lfront -= lbeta;
    if (x < (a + 1.0) / (a + b + 2.0))
        return exp(lfront) * betacf(a, b, x) / a;
    return 1.0 - exp(lfront) * betacf(b, a, omx) / b;
}

/* 2 * pt(|t|, df, lower.tail = FALSE)  (R/test.R:108-116) */
double orc_two_sided_t_pvalue(double t, double df)
{
    if (isnan(t) || isnan(df)) return NAN;
    if (df <= 0) return NAN;
    t = fabs(t);
    if (isinf(t)) return 0.0;
    double t2 = t * t;
    double x = df / (df + t2);
    double omx = t2 / (df + t2);
    return ibeta(0.5 * df, 0.5, x, omx);
}

/* ------------------------------------------------------------------ */
/* small dense linear algebra (column-major p x p)                     */
/* ------------------------------------------------------------------ */

/* inverse by LU with partial pivoting, as Eigen's MatrixXd::inverse() does
 * for dynamic sizes.  Returns 0 on success, 1 when a pivot is exactly 0 (the
 * result then holds inf/nan like Eigen's would). */
static int lu_inverse(int p, const double *A, double *Ainv)
{
    double *LU = (double *)malloc(sizeof(double) * p * p);
    int *piv = (int *)malloc(sizeof(int) * p);
    memcpy(LU, A, sizeof(double) * p * p);
    int sing = 0;
    for (int k = 0; k < p; k++) {
        int mx = k; double mv = fabs(LU[k * p + k]);
        for (int i = k + 1; i < p; i++) {
            double v = fabs(LU[k * p + i]);
            if (v > mv) { mv = v; mx = i; }
        }
        piv[k] = mx;
        if (mx != k)
            for (int j = 0; j < p; j++) { double t = LU[j * p + k]; LU[j * p + k] = LU[j * p + mx]; LU[j * p + mx] = t; }
        double d = LU[k * p + k];
        if (d == 0.0) sing = 1;
        for (int i = k + 1; i < p; i++) {
            LU[k * p + i] /= d;
            double l = LU[k * p + i];
            for (int j = k + 1; j < p; j++) LU[j * p + i] -= l * LU[j * p + k];
        }
    }
    /* solve for each unit vector, applying the row swaps */
    for (int col = 0; col < p; col++) {
        double *x = Ainv + col * p;
        for (int i = 0; i < p; i++) x[i] = (i == col) ? 1.0 : 0.0;
        for (int k = 0; k < p; k++) if (piv[k] != k) { double t = x[k]; x[k] = x[piv[k]]; x[piv[k]] = t; }
        for (int i = 0; i < p; i++) { double s = x[i]; for (int j = 0; j < i; j++) s -= LU[j * p + i] * x[j]; x[i] = s; }
        for (int i = p - 1; i >= 0; i--) { double s = x[i]; for (int j = i + 1; j < p; j++) s -= LU[j * p + i] * x[j]; x[i] = s / LU[i * p + i]; }
    }
    free(LU); free(piv);
    return sing;
}

/* log|det| through LU: sum log(L diag)=0 plus U diag floored at 1e-50,
 * as src/overdispersion.cpp:62-68 does with arma::lu. */
static double lu_logdet_floored(int p, const double *A)
{
    double *LU = (double *)malloc(sizeof(double) * p * p);
    memcpy(LU, A, sizeof(double) * p * p);
    double ld = 0.0;
    for (int k = 0; k < p; k++) {
        int mx = k; double mv = fabs(LU[k * p + k]);
        for (int i = k + 1; i < p; i++) { double v = fabs(LU[k * p + i]); if (v > mv) { mv = v; mx = i; } }
        if (mx != k) for (int j = 0; j < p; j++) { double t = LU[j * p + k]; LU[j * p + k] = LU[j * p + mx]; LU[j * p + mx] = t; }
        double d = LU[k * p + k];
        if (d != 0.0)
            for (int i = k + 1; i < p; i++) {
                LU[k * p + i] /= d;
                double l = LU[k * p + i];
                for (int j = k + 1; j < p; j++) LU[j * p + i] -= l * LU[j * p + k];
            }
    }
    /* arma::lu returns U with the sign carried by the permutation; log of a
     * negative U diagonal is NaN there too.  Mirror: log(e) with floor. */
    for (int k = 0; k < p; k++) {
        double e = LU[k * p + k];
        ld += e < 1e-50 ? log(1e-50) : log(e);
    }
    free(LU);
    return ld;
}

/* ------------------------------------------------------------------ */
/* helpers                                                             */
/* ------------------------------------------------------------------ */

static void row_dense(const int64_t *rowptr, const int32_t *col, const double *val,
                      int64_t g, int64_t n, double *y)
{
    memset(y, 0, sizeof(double) * n);
    for (int64_t i = rowptr[g]; i < rowptr[g + 1]; i++) y[col[i]] = val[i];
}

static void linear_predictor(int64_t n, int p, const double *X, const double *beta, double *eta)
{
    for (int64_t c = 0; c < n; c++) {
        double s = 0.0;
        for (int j = 0; j < p; j++) s += X[(int64_t)j * n + c] * beta[j];
        eta[c] = s;
    }
}

/* Sums over the cells of one gene.  The cells are taken in blocks of
 * ORC_BLK whose design rows are copied into a row-major buffer; a callback
 * fills, per cell of the block, nw "outer" weights, nv "vector" weights and
 * ns scalars, and the helper adds
 *     out[k]          += sum_c w_k(c) x_c x_c^T     (k < nw, p x p)
 *     out[nw p^2 + k] += sum_c v_k(c) x_c           (k < nv, p)
 *     out[... + k]    += sum_c s_k(c)                (k < ns)
 * with the p x p sums over the upper triangle of contiguous rows (a loop
 * the compiler vectorises) and mirrored at the end.  When the caller is not
 * already inside a parallel region and n is large, the blocks are split
 * into one contiguous range per thread and the per-thread partial sums are
 * added in thread order, so the result does not depend on scheduling.  The
 * arithmetic of every term is the reference's; only the order of the
 * floating-point additions differs from a plain loop over the cells. */
#define ORC_BLK 128
typedef void (*orc_cellfn)(void *ctx, int64_t c0, int nc, int p, const double *xr, double *w);

static void orc_cell_sums(int64_t n, int p, const double *X, int nw, int nv, int ns,
                          orc_cellfn fn, void *ctx, double *out)
{
    const int nq = nw + nv + ns;
    const size_t per = (size_t)nw * p * p + (size_t)nv * p + (size_t)ns;
    int nt = 1;
#ifdef _OPENMP
    const int par = !omp_in_parallel() && n >= 32768;
    if (par) nt = omp_get_max_threads();
#else
    const int par = 0;
#endif
    double *part = (double *)calloc((size_t)nt * (per > 0 ? per : 1), sizeof(double));
    #pragma omp parallel num_threads(nt) if (par)
    {
        int t = 0, T = 1;
#ifdef _OPENMP
        t = omp_get_thread_num();
        T = omp_get_num_threads();
#endif
        double *xr = (double *)malloc(sizeof(double) * ORC_BLK * p);
        double *w = (double *)malloc(sizeof(double) * ORC_BLK * (nq > 0 ? nq : 1));
        double *acc = part + (size_t)t * per;
        const int64_t nb = (n + ORC_BLK - 1) / ORC_BLK;
        const int64_t b0 = nb * t / T, b1 = nb * (t + 1) / T;
        for (int64_t blk = b0; blk < b1; blk++) {
            const int64_t c0 = blk * ORC_BLK;
            const int nc = (int)(n - c0 < ORC_BLK ? n - c0 : ORC_BLK);
            for (int j = 0; j < p; j++) {
                const double *xc = X + (int64_t)j * n + c0;
                for (int c = 0; c < nc; c++) xr[c * p + j] = xc[c];
            }
            fn(ctx, c0, nc, p, xr, w);
            for (int k = 0; k < nw; k++) {
                double *H = acc + (size_t)k * p * p;
                const double *wk = w + k * ORC_BLK;
                for (int c = 0; c < nc; c++) {
                    const double *x = xr + c * p;
                    for (int a = 0; a < p; a++) {
                        const double sa = wk[c] * x[a];
                        double *Ha = H + a * p;
                        for (int b = a; b < p; b++) Ha[b] += sa * x[b];
                    }
                }
            }
            for (int k = 0; k < nv; k++) {
                double *v = acc + (size_t)nw * p * p + (size_t)k * p;
                const double *wk = w + (nw + k) * ORC_BLK;
                for (int c = 0; c < nc; c++)
                    for (int a = 0; a < p; a++) v[a] += wk[c] * xr[c * p + a];
            }
            for (int k = 0; k < ns; k++) {
                double *sv = acc + (size_t)nw * p * p + (size_t)nv * p + k;
                const double *wk = w + (nw + nv + k) * ORC_BLK;
                for (int c = 0; c < nc; c++) *sv += wk[c];
            }
        }
        free(xr); free(w);
    }
    if (per) memset(out, 0, sizeof(double) * per);
    for (int t = 0; t < nt; t++)
        for (size_t i = 0; i < per; i++) out[i] += part[(size_t)t * per + i];
    for (int k = 0; k < nw; k++) {  /* upper triangle (row a, col b >= a) -> symmetric */
        double *H = out + (size_t)k * p * p;
        for (int a = 0; a < p; a++)
            for (int b = a + 1; b < p; b++) H[b * p + a] = H[a * p + b];
    }
    free(part);
}

/* ------------------------------------------------------------------ */
/* size factors and offset  (R/size_factors.R)                         */
/* ------------------------------------------------------------------ */

/* method: 0 = normed_sum (R/size_factors.R:75-88), 1 = psinorm (:100-117).
 * calculate_sf returns unit factors when the matrix has <= 1 row (:38-42). */
int orc_calculate_sf(int64_t G, int64_t n, const int64_t *rowptr, const int32_t *col,
                     const double *val, int method, double *sf)
{
    if (G <= 1) { for (int64_t c = 0; c < n; c++) sf[c] = 1.0; return ORC_OK; }
    if (method == 0) {
        for (int64_t c = 0; c < n; c++) sf[c] = 0.0;
        for (int64_t g = 0; g < G; g++)
            for (int64_t i = rowptr[g]; i < rowptr[g + 1]; i++) sf[col[i]] += val[i];
        for (int64_t c = 0; c < n; c++) if (sf[c] == 0.0) return ORC_ERR_ZERO_COLUMN;
        double ml = 0.0;
        for (int64_t c = 0; c < n; c++) ml += log(sf[c]);
        double gm = exp(ml / (double)n);
        for (int64_t c = 0; c < n; c++) sf[c] /= gm;
        return ORC_OK;
    }
    if (method == 1) {
        double *mn = (double *)malloc(sizeof(double) * n);
        int64_t *cnt = (int64_t *)calloc(n, sizeof(int64_t));
        for (int64_t c = 0; c < n; c++) { sf[c] = 0.0; mn[c] = INFINITY; }
        for (int64_t g = 0; g < G; g++)
            for (int64_t i = rowptr[g]; i < rowptr[g + 1]; i++) {
                double l = log1p(val[i]);
                sf[col[i]] += l;
                if (l < mn[col[i]]) mn[col[i]] = l;
                cnt[col[i]]++;
            }
        for (int64_t c = 0; c < n; c++) {
            double m = (cnt[c] < G) ? 0.0 : mn[c];     /* zeros present -> log1p(0)=0 */
            if (cnt[c] < G && mn[c] < 0.0) m = mn[c];  /* negative entries (not counts) */
            sf[c] = sf[c] / (double)G - m;
        }
        /* mean(log(sf), na.rm=TRUE): NaN logs dropped, -Inf kept */
        double ml = 0.0; int64_t k = 0;
        for (int64_t c = 0; c < n; c++) { double l = log(sf[c]); if (!isnan(l)) { ml += l; k++; } }
        double gm = exp(ml / (double)k);
        for (int64_t c = 0; c < n; c++) sf[c] /= gm;
        free(mn); free(cnt);
        return ORC_OK;
    }
    return ORC_ERR_ARG;
}

/* compute_offset_vector (R/size_factors.R:172-184): off + log(sf) */
void orc_offset_vector(int64_t n, double off, const double *sf, double *out)
{
    for (int64_t c = 0; c < n; c++) out[c] = off + (sf ? log(sf[c]) : 0.0);
}

/* ------------------------------------------------------------------ */
/* theta_0  (R/overdispersion.R:129-135)                               */
/* ------------------------------------------------------------------ */
void orc_estimate_dispersion(int64_t G, int64_t n, const int64_t *rowptr, const int32_t *col,
                             const double *val, const double *offv, double *theta0)
{
    (void)col;
    double me = 0.0;
    for (int64_t c = 0; c < n; c++) me += exp(offv[c]);
    double moi = 1.0 / (me / (double)n);
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t g = 0; g < G; g++) {
        double s = 0.0;
        for (int64_t i = rowptr[g]; i < rowptr[g + 1]; i++) s += val[i];
        double mean = s / (double)n;
        /* two-pass sample variance; zeros contribute mean^2 each */
        double ss = 0.0;
        int64_t nz = rowptr[g + 1] - rowptr[g];
        for (int64_t i = rowptr[g]; i < rowptr[g + 1]; i++) { double d = val[i] - mean; ss += d * d; }
        ss += (double)(n - nz) * mean * mean;
        double var = ss / (double)(n - 1);
        double d = (var - moi * mean) / (mean * mean);
        theta0[g] = (isnan(d) || d < 0.0) ? 0.01 : d;
    }
}

/* ------------------------------------------------------------------ */
/* beta init  (R/beta.R:13-20; rough init R/main.R:404-406)            */
/* ------------------------------------------------------------------ */

/* Householder QR of X (n x p, column-major).  On exit QR holds the
 * reflectors below the diagonal and R on/above it; tau[p]. */
static int householder_qr(int64_t n, int p, double *QR, double *tau)
{
    for (int k = 0; k < p; k++) {
        double *a = QR + (int64_t)k * n;
        double nrm = 0.0;
        for (int64_t i = k; i < n; i++) nrm += a[i] * a[i];
        nrm = sqrt(nrm);
        if (nrm == 0.0) return ORC_ERR_SINGULAR;
        double alpha = a[k] > 0 ? -nrm : nrm;
        double v0 = a[k] - alpha;
        for (int64_t i = k + 1; i < n; i++) a[i] /= v0;
        tau[k] = -v0 / alpha;
        a[k] = alpha;
        for (int j = k + 1; j < p; j++) {
            double *b = QR + (int64_t)j * n;
            double s = b[k];
            for (int64_t i = k + 1; i < n; i++) s += a[i] * b[i];
            s *= tau[k];
            b[k] -= s;
            for (int64_t i = k + 1; i < n; i++) b[i] -= s * a[i];
        }
    }
    /* rank check as R's solve(R, .) would report an exactly singular R */
    double rmax = 0.0;
    for (int k = 0; k < p; k++) { double v = fabs(QR[(int64_t)k * n + k]); if (v > rmax) rmax = v; }
    for (int k = 0; k < p; k++) if (fabs(QR[(int64_t)k * n + k]) <= 1e-7 * rmax) return ORC_ERR_SINGULAR;
    return ORC_OK;
}

int orc_init_beta(int64_t G, int64_t n, int p, const int64_t *rowptr, const int32_t *col,
                  const double *val, const double *X, const double *offv, double *beta0)
{
    double *QR = (double *)malloc(sizeof(double) * n * p);
    double *tau = (double *)malloc(sizeof(double) * p);
    memcpy(QR, X, sizeof(double) * n * p);
    int st = householder_qr(n, p, QR, tau);
    if (st) { free(QR); free(tau); return st; }
    int err = 0;
    #pragma omp parallel
    {
        double *z = (double *)malloc(sizeof(double) * n);
        double *b = (double *)malloc(sizeof(double) * p);
        if (!z || !b) err = 1;
        #pragma omp for schedule(dynamic, 16)
        for (int64_t g = 0; g < G; g++) {
            if (!z || !b) continue;
            memset(z, 0, sizeof(double) * n);
            for (int64_t i = rowptr[g]; i < rowptr[g + 1]; i++)
                z[col[i]] = log1p(val[i] / exp(offv[col[i]]));
            /* Q^T z */
            for (int k = 0; k < p; k++) {
                const double *a = QR + (int64_t)k * n;
                double s = z[k];
                for (int64_t i = k + 1; i < n; i++) s += a[i] * z[i];
                s *= tau[k];
                z[k] -= s;
                for (int64_t i = k + 1; i < n; i++) z[i] -= s * a[i];
            }
            for (int k = p - 1; k >= 0; k--) {
                double s = z[k];
                for (int j = k + 1; j < p; j++) s -= QR[(int64_t)j * n + k] * b[j];
                b[k] = s / QR[(int64_t)k * n + k];
            }
            for (int j = 0; j < p; j++) beta0[g * p + j] = b[j];
        }
        free(z); free(b);
    }
    free(QR); free(tau);
    return err ? ORC_ERR_ALLOC : ORC_OK;
}

void orc_init_beta_rough(int64_t G, int64_t n, int p, const int64_t *rowptr, const double *val,
                         double *beta0)
{
    for (int64_t g = 0; g < G; g++) {
        double s = 0.0;
        for (int64_t i = rowptr[g]; i < rowptr[g + 1]; i++) s += val[i];
        beta0[g * p] = log1p(s / (double)n);
        for (int j = 1; j < p; j++) beta0[g * p + j] = 0.0;
    }
}

/* ------------------------------------------------------------------ */
/* IRLS beta fit  (src/beta.cpp:25-51)                                 */
/* ------------------------------------------------------------------ */

/* k_in is the float the reference receives (theta_0 rounded to float);
 * eps is the float tolerance.  beta holds beta_0 on entry, the fit on exit.
 * Returns the iteration count. */
/* per cell of one IRLS iteration: outer weight mu_g w_q, score weight
 * mu_g w_q - 1 */
typedef struct { const double *beta, *off, *y; double k; } irls_cells;
static void irls_cellfn(void *vc, int64_t c0, int nc, int p, const double *xr, double *w)
{
    const irls_cells *q = (const irls_cells *)vc;
    for (int c = 0; c < nc; c++) {
        double eta = 0.0;
        for (int j = 0; j < p; j++) eta += xr[c * p + j] * q->beta[j];
        const double w_q = exp(-eta - q->off[c0 + c]);
        const double mu_g = (q->k + q->y[c0 + c]) / (1.0 + q->k * w_q);
        const double mw = mu_g * w_q;
        w[c] = mw;
        w[ORC_BLK + c] = mw - 1.0;
    }
}

int orc_beta_fit(int64_t n, int p, const double *y, const double *X, double *beta,
                 const double *offv, float k_in, int max_iter, float eps)
{
    float k = (float)(1.0 / (double)k_in);       /* k = 1.0 / k; stored in a float */
    double kd = (double)k;
    double epsd = (double)eps;
    double *sums = (double *)calloc((size_t)p * p + p, sizeof(double));
    double *H = sums, *sc = sums + (size_t)p * p;
    double *Z = (double *)calloc((size_t)p * p, sizeof(double));
    double *delta = (double *)calloc(p, sizeof(double));
    irls_cells q = { beta, offv, y, kd };
    int converged = 0, iter = 0;
    while (!converged && iter < max_iter) {
        /* H = X' diag(mu_g w_q) X, sc = X' (mu_g w_q - 1) */
        orc_cell_sums(n, p, X, 1, 1, 0, irls_cellfn, &q, sums);
        for (int i = 0; i < p * p; i++) H[i] *= kd;
        lu_inverse(p, H, Z);
        for (int a = 0; a < p; a++) {
            double s = 0.0;
            for (int b = 0; b < p; b++) s += Z[b * p + a] * (kd * sc[b]);
            delta[a] = s;
        }
        double mx = 0.0;
        for (int a = 0; a < p; a++) { beta[a] += delta[a]; if (fabs(delta[a]) > mx) mx = fabs(delta[a]); }
        converged = mx < epsd;
        iter++;
        if (delta[0] != delta[0]) converged = 1;
    }
    free(sums); free(Z); free(delta);
    return iter;
}

/* ------------------------------------------------------------------ */
/* MOM theta  (src/mom_overdispersion.cpp:24-53)                       */
/* ------------------------------------------------------------------ */
typedef struct { const double *beta, *sf, *y; } mom_cells;
static void mom_cellfn(void *vc, int64_t c0, int nc, int p, const double *xr, double *w)
{
    const mom_cells *q = (const mom_cells *)vc;
    for (int c = 0; c < nc; c++) {
        double eta = 0.0;
        for (int j = 0; j < p; j++) eta += xr[c * p + j] * q->beta[j];
        const double mu = q->sf[c0 + c] * exp(eta);
        const double diff = q->y[c0 + c] - mu;
        w[c] = diff * diff - mu;
        w[ORC_BLK + c] = mu * mu;
    }
}

double orc_mom_dispersion(int64_t n, int p, const double *y, const double *X, const double *beta,
                          const double *sf)
{
    double corr = (double)n / (double)(n - p);
    mom_cells q = { beta, sf, y };
    double nd[2];
    orc_cell_sums(n, p, X, 0, 0, 2, mom_cellfn, &q, nd);
    const double num = nd[0], den = nd[1];
    double th = 0.0;
    if (den > 0.0) { th = corr * num / den; if (th < 0.0) th = 0.0; }
    return th;
}

/* ------------------------------------------------------------------ */
/* NB log-likelihood in log(theta) with Cox-Reid adjustment            */
/* (src/overdispersion.cpp:53-242)                                     */
/* ------------------------------------------------------------------ */
static const double CR_FACTOR = 0.99;   /* src/overdispersion.cpp:25 */

typedef struct {
    int64_t n; int p;
    const double *y, *mu, *X;
} nbdata;

/* b = X^T diag(w) X and friends for the Cox-Reid terms */
typedef struct { const double *mu; double theta; int nw; } cr_cells;
static void cr_cellfn(void *vc, int64_t c0, int nc, int p, const double *xr, double *w)
{
    const cr_cells *q = (const cr_cells *)vc;
    (void)p; (void)xr;
    for (int c = 0; c < nc; c++) {
        const double ww = 1.0 / (1.0 / q->mu[c0 + c] + q->theta);
        const double dw = -ww * ww;
        w[c] = ww;
        if (q->nw > 1) w[ORC_BLK + c] = dw;
        if (q->nw > 2) w[2 * ORC_BLK + c] = -2.0 * dw * ww;
    }
}

static void cr_mats(const nbdata *d, double theta, double *b, double *db, double *d2b)
{
    const int p = d->p;
    const int nw = d2b ? 3 : (db ? 2 : 1);
    const size_t pp = (size_t)p * p;
    double *m = (double *)malloc(sizeof(double) * nw * pp);
    cr_cells q = { d->mu, theta, nw };
    orc_cell_sums(d->n, p, d->X, nw, 0, 0, cr_cellfn, &q, m);
    memcpy(b, m, sizeof(double) * pp);
    if (db) memcpy(db, m + pp, sizeof(double) * pp);
    if (d2b) memcpy(d2b, m + 2 * pp, sizeof(double) * pp);
    free(m);
}

/* inv_sympd(b + 1e-6 I) -- symmetric positive definite inverse */
static int spd_inverse_ridge(int p, const double *b, double *binv)
{
    double *m = (double *)malloc(sizeof(double) * p * p);
    memcpy(m, b, sizeof(double) * p * p);
    for (int i = 0; i < p; i++) m[i * p + i] += 1e-6;
    int s = lu_inverse(p, m, binv);
    free(m);
    return s;
}

double orc_nb_loglik(const nbdata *d, double log_theta, int cr)
{
    int p = d->p; int64_t n = d->n;
    double theta = exp(log_theta);
    double cr_term = 0.0;
    if (cr) {
        double *b = (double *)malloc(sizeof(double) * p * p);
        cr_mats(d, theta, b, NULL, NULL);
        cr_term = -0.5 * lu_logdet_floored(p, b) * CR_FACTOR;
        free(b);
    }
    double a = 1.0 / theta;
    double lg = 0.0, ll = 0.0;
    for (int64_t c = 0; c < n; c++) {
        lg += lgamma(d->y[c] + a);
        ll += (-d->y[c] - a) * log(d->mu[c] + a);
    }
    lg -= (double)n * lgamma(a);
    ll -= (double)n * a * log(theta);
    return lg + ll + cr_term;
}

/* Sum over cells of psi(y+a) - psi(a) (exact for integer y by the
 * recurrence psi(x+1) = psi(x) + 1/x) and likewise for trigamma.  The
 * reference forms sum(psi(y+a)) - n psi(a); both are the same quantity. */
static void digamma_sums(const nbdata *d, double a, double *dig, double *trig)
{
    double sd = 0.0, st = 0.0;
    double pa = 0.0, ta = 0.0; int have = 0;
    for (int64_t c = 0; c < d->n; c++) {
        double y = d->y[c];
        if (y == 0.0) continue;
        if (y == floor(y) && y <= 64.0) {
            for (int j = 0; j < (int)y; j++) { double v = 1.0 / (a + j); sd += v; st -= v * v; }
        } else {
            if (!have) { pa = orc_digamma(a); ta = orc_trigamma(a); have = 1; }
            sd += orc_digamma(y + a) - pa;
            st += orc_trigamma(y + a) - ta;
        }
    }
    *dig = sd; if (trig) *trig = st;
}

/* per-cell terms of the score's ll_part (src/overdispersion.cpp:159-175),
 * including the reference's branches on mu*theta */
typedef struct { const double *mu, *y; double theta, a; } score_cells;
static void score_cellfn(void *vc, int64_t c0, int nc, int p, const double *xr, double *w)
{
    const score_cells *q = (const score_cells *)vc;
    (void)p; (void)xr;
    for (int c = 0; c < nc; c++) {
        const double mu = q->mu[c0 + c], y = q->y[c0 + c];
        const double mt = mu * q->theta;
        double ll;
        if (mt < 1e-10) {
            ll = mt * mt * (1.0 / (1.0 + mt) - 0.5);
        } else if (mt < 1e-4) {
            double inv = 1.0 / (1.0 + mt);
            double ub = mt * mt * inv, lb = mt * mt * (inv - 0.5);
            double sug = log1p(mt) - mu / (mu + q->a);
            ll = fmax(fmin(sug, ub), lb);
        } else {
            ll = log1p(mt) - mu / (mu + q->a);
        }
        w[c] = ll + y / (mu + q->a);
    }
}

/* conventional_score_function_fast (src/overdispersion.cpp:95-178) */
double orc_nb_score(const nbdata *d, double log_theta, int cr)
{
    int p = d->p; int64_t n = d->n;
    double theta = exp(log_theta);
    double a = 1.0 / theta;
    double cr_term = 0.0;
    if (cr) {
        double *b = (double *)malloc(sizeof(double) * p * p);
        double *db = (double *)malloc(sizeof(double) * p * p);
        double *bi = (double *)malloc(sizeof(double) * p * p);
        cr_mats(d, theta, b, db, NULL);
        spd_inverse_ridge(p, b, bi);
        double tr = 0.0;
        for (int i = 0; i < p; i++) for (int k = 0; k < p; k++) tr += bi[k * p + i] * db[i * p + k];
        cr_term = -0.5 * tr * CR_FACTOR;
        free(b); free(db); free(bi);
    }
    double max_y = 0.0, sum_y = 0.0, sum_prod_y = 0.0;
    for (int64_t c = 0; c < n; c++) {
        double y = d->y[c];
        sum_y += y; sum_prod_y += (y - 1.0) * y;
        if (y > max_y) max_y = y;
    }
    double corr = a > 1e5 ? sum_prod_y / (2.0 * a) : 0.0;
    double dig;
    if (max_y * 1e6 < a) {
        dig = sum_y - corr;
    } else {
        double sd; digamma_sums(d, a, &sd, NULL);
        dig = sd * a;
        if (dig > sum_y - corr) dig = sum_y - corr;
    }
    score_cells q = { d->mu, d->y, theta, a };
    double ll;
    orc_cell_sums(n, 0, NULL, 0, 0, 1, score_cellfn, &q, &ll);
    ll *= a;
    return ll - dig + cr_term * theta;
}

/* per-cell terms of the derivative (src/overdispersion.cpp:223-233) */
static void deriv_cellfn(void *vc, int64_t c0, int nc, int p, const double *xr, double *w)
{
    const score_cells *q = (const score_cells *)vc;
    (void)p; (void)xr;
    for (int c = 0; c < nc; c++) {
        const double mu = q->mu[c0 + c], y = q->y[c0 + c];
        const double den = 1.0 + mu * q->theta;
        w[c] = log1p(mu * q->theta) + (y - mu) / (mu + q->a);
        w[ORC_BLK + c] = (mu * mu * q->theta + y) / den / den;
    }
}

/* conventional_deriv_score_function_fast (src/overdispersion.cpp:186-242) */
double orc_nb_deriv_score(const nbdata *d, double log_theta, int cr)
{
    int p = d->p; int64_t n = d->n;
    double theta = exp(log_theta);
    double cr_term = 0.0, cr_term2 = 0.0;
    if (cr) {
        size_t sz = sizeof(double) * p * p;
        double *b = malloc(sz), *db = malloc(sz), *d2b = malloc(sz), *bi = malloc(sz), *m = malloc(sz);
        cr_mats(d, theta, b, db, d2b);
        spd_inverse_ridge(p, b, bi);
        /* m = bi * db */
        for (int i = 0; i < p; i++) for (int j = 0; j < p; j++) {
            double s = 0.0; for (int k = 0; k < p; k++) s += bi[k * p + i] * db[j * p + k];
            m[j * p + i] = s;
        }
        double ddetb = 0.0, trmm = 0.0, trbd2 = 0.0;
        for (int i = 0; i < p; i++) ddetb += m[i * p + i];
        for (int i = 0; i < p; i++) for (int k = 0; k < p; k++) trmm += m[k * p + i] * m[i * p + k];
        for (int i = 0; i < p; i++) for (int k = 0; k < p; k++) trbd2 += bi[k * p + i] * d2b[i * p + k];
        double d2detb = ddetb * ddetb - trmm + trbd2;
        cr_term = (0.5 * ddetb * ddetb - 0.5 * d2detb) * CR_FACTOR;
        cr_term2 = -0.5 * ddetb * CR_FACTOR;
        free(b); free(db); free(d2b); free(bi); free(m);
    }
    double a = 1.0 / theta, a2 = a * a;
    double sd, st;
    digamma_sums(d, a, &sd, &st);
    double dig = sd;
    double trig = a2 * st;
    score_cells q = { d->mu, d->y, theta, a };
    double l12[2];
    orc_cell_sums(n, 0, NULL, 0, 0, 2, deriv_cellfn, &q, l12);
    const double l1 = l12[0], l2 = l12[1];
    double ll = -2.0 * a * (l1 - dig) + (l2 + trig);
    return ll + cr_term * theta * theta + (l1 - dig) * a + cr_term2 * theta;
}

/* mu = exp(X beta + off), 0 -> 1e-6 (R/overdispersion.R:41-42); written per
 * cell, no sums */
typedef struct { const double *beta, *off; double *mu; } mu_cells;
static void mu_cellfn(void *vc, int64_t c0, int nc, int p, const double *xr, double *w)
{
    const mu_cells *q = (const mu_cells *)vc;
    (void)w;
    for (int c = 0; c < nc; c++) {
        double eta = 0.0;
        for (int j = 0; j < p; j++) eta += xr[c * p + j] * q->beta[j];
        double m = exp(eta + q->off[c0 + c]);
        q->mu[c0 + c] = m == 0.0 ? 1e-6 : m;
    }
}

/* fit_dispersion (R/overdispersion.R:25-115), re-expressed as a bracketed
 * Newton search for the root of the score in log(theta).
 * Returns theta; *iters gets the Newton iteration count. */
double orc_fit_dispersion(int64_t n, int p, const double *y, const double *X, const double *beta,
                          const double *offv, int max_iter, int cr, int *iters)
{
    *iters = 0;
    int allzero = 1;
    for (int64_t c = 0; c < n; c++) if (y[c] != 0.0) { allzero = 0; break; }
    if (allzero) return 0.0;
    double *mu = (double *)malloc(sizeof(double) * n);
    mu_cells mq = { beta, offv, mu };
    orc_cell_sums(n, p, X, 0, 0, 0, mu_cellfn, &mq, NULL);
    nbdata d = { n, p, y, mu, X };
    double m = 0.0;
    for (int64_t c = 0; c < n; c++) m += y[c];
    m /= (double)n;
    double v = 0.0;
    for (int64_t c = 0; c < n; c++) v += (y[c] - m) * (y[c] - m);
    v /= (double)(n - 1);
    double start = (v - m) / (m * m);
    if (isnan(start) || start <= 0.0) start = 0.5;

    double lo = log(1e-8);
    if (orc_nb_score(&d, lo, cr) < 0.0) { free(mu); return 0.0; }
    double hi = log(1e16);
    double x = log(start);
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    double dx = hi - lo, dxold = hi - lo;
    int it = 0;
    for (; it < max_iter; it++) {
        double s = orc_nb_score(&d, x, cr);
        if (s == 0.0) break;
        if (s > 0.0) lo = x; else hi = x;
        double dd = orc_nb_deriv_score(&d, x, cr);
        double xn = (dd < 0.0) ? x - s / dd : NAN;
        /* Newton inside the bracket; bisect when the step leaves it or fails
         * to halve the step before last (safeguarded Newton, "rtsafe") */
        if (!(xn > lo && xn < hi) || fabs(xn - x) > 0.5 * fabs(dxold)) {
            dxold = dx;
            dx = 0.5 * (hi - lo);
            xn = lo + dx;
        } else {
            dxold = dx;
            dx = fabs(xn - x);
        }
        x = xn;
        if (dx < 1e-10 || hi - lo < 1e-10) { it++; break; }
    }
    *iters = it;
    free(mu);
    return exp(x);
}

/* ------------------------------------------------------------------ */
/* bread and meat  (src/variance.cpp:22-47, :64-85, :104-137, :157-178, */
/* :186-228)                                                            */
/* ------------------------------------------------------------------ */
typedef struct { const double *beta, *sf, *y; double th; } hess_cells;
static void hess_cellfn(void *vc, int64_t c0, int nc, int p, const double *xr, double *w)
{
    const hess_cells *q = (const hess_cells *)vc;
    for (int c = 0; c < nc; c++) {
        double eta = 0.0;
        for (int j = 0; j < p; j++) eta += xr[c * p + j] * q->beta[j];
        const double mu = q->sf[c0 + c] * exp(eta);
        const double den = 1.0 + q->th * mu;
        w[c] = (q->y[c0 + c] * q->th + 1.0) * mu / (den * den);
    }
}

int orc_compute_hessian(int64_t n, int p, const double *beta, double overdispersion,
                        const double *y, const double *X, const double *sf, double *bread)
{
    double *H = (double *)calloc((size_t)p * p, sizeof(double));
    hess_cells q = { beta, sf, y, overdispersion };
    orc_cell_sums(n, p, X, 1, 0, 0, hess_cellfn, &q, H);
    int st = lu_inverse(p, H, bread);
    free(H);
    return st;
}

/* per-cell score vectors (the NB log-likelihood adjoint with respect to
 * eta, times x): (y - mu) / (1 + mu theta) * x_c  (src/variance.cpp:64-85) */
void orc_compute_scores(int64_t n, int p, const double *X, const double *y, const double *beta,
                        double overdispersion, const double *sf, double *scores /* n x p colmajor */)
{
    for (int64_t c = 0; c < n; c++) {
        double eta = 0.0;
        for (int j = 0; j < p; j++) eta += X[(int64_t)j * n + c] * beta[j];
        double mu = sf[c] * exp(eta);
        double alpha = 1.0 / overdispersion;
        double wr = (y[c] - mu) / mu * (mu / (1.0 + mu / alpha));
        for (int j = 0; j < p; j++) scores[(int64_t)j * n + c] = X[(int64_t)j * n + c] * wr;
    }
}

/* compute_clustered_meat_fast: contiguous blocks with 1-based exclusive
 * ends (cumsum(rle(clusters)$lengths), R/main.R:193). */
void orc_clustered_meat_fast(int64_t n, int p, const double *X, const double *y, const double *beta,
                             double overdispersion, const double *sf, const int32_t *ends, int ng,
                             double *meat)
{
    double *S = (double *)calloc((size_t)ng * p, sizeof(double));
    int64_t start = 0;
    for (int g = 0; g < ng; g++) {
        int64_t end = ends[g];
        for (int64_t c = start; c < end; c++) {
            double eta = 0.0;
            for (int j = 0; j < p; j++) eta += X[(int64_t)j * n + c] * beta[j];
            double mu = sf[c] * exp(eta);
            double wr = (y[c] - mu) / (1.0 + mu * overdispersion);
            for (int j = 0; j < p; j++) S[g * p + j] += X[(int64_t)j * n + c] * wr;
        }
        start = end;
    }
    double adj = ng > 1 ? (double)ng / (ng - 1.0) : 1.0;
    for (int a = 0; a < p; a++)
        for (int b = 0; b < p; b++) {
            double s = 0.0;
            for (int g = 0; g < ng; g++) s += S[g * p + a] * S[g * p + b];
            meat[b * p + a] = adj / (double)n * s;
        }
    free(S);
}

/* compute_clustered_meat with arbitrary 1-based cluster labels
 * (src/variance.cpp:104-137) and compute_meat (:157-178). */
void orc_clustered_meat(int64_t n, int p, const double *X, const double *y, const double *beta,
                        double overdispersion, const double *sf, const int32_t *clusters,
                        double *meat)
{
    int ng = 0;
    for (int64_t c = 0; c < n; c++) if (clusters[c] > ng) ng = clusters[c];
    double *S = (double *)calloc((size_t)(ng > 0 ? ng : 1) * p, sizeof(double));
    double *sc = (double *)malloc(sizeof(double) * n * p);
    orc_compute_scores(n, p, X, y, beta, overdispersion, sf, sc);
    for (int64_t c = 0; c < n; c++) {
        int g = clusters[c] - 1;
        if (g >= 0 && g < ng) for (int j = 0; j < p; j++) S[g * p + j] += sc[(int64_t)j * n + c];
    }
    double adj = ng > 1 ? (double)ng / (ng - 1.0) : 1.0;
    for (int a = 0; a < p; a++)
        for (int b = 0; b < p; b++) {
            double s = 0.0;
            for (int g = 0; g < ng; g++) s += S[g * p + a] * S[g * p + b];
            meat[b * p + a] = adj / (double)n * s;
        }
    free(S); free(sc);
}

void orc_meat(int64_t n, int p, const double *X, const double *y, const double *beta,
              double overdispersion, const double *sf, double *meat)
{
    double *sc = (double *)malloc(sizeof(double) * n * p);
    orc_compute_scores(n, p, X, y, beta, overdispersion, sf, sc);
    for (int a = 0; a < p; a++)
        for (int b = 0; b < p; b++) {
            double s = 0.0;
            for (int64_t c = 0; c < n; c++) s += sc[(int64_t)a * n + c] * sc[(int64_t)b * n + c];
            meat[b * p + a] = s / (double)n;
        }
    free(sc);
}

/* ------------------------------------------------------------------ */
/* cluster handling  (R/main.R:190-196, R/group_data.R:38-69)           */
/* ------------------------------------------------------------------ */

/* factor(clusters, levels = unique(clusters)) -> 1-based levels by first
 * appearance.  Returns the number of levels. */
int orc_factor_first_appearance(int64_t n, const int64_t *clusters, int32_t *levels)
{
    int64_t cap = 16, nu = 0;
    int64_t *uniq = (int64_t *)malloc(sizeof(int64_t) * cap);
    for (int64_t c = 0; c < n; c++) {
        int64_t k;
        for (k = 0; k < nu; k++) if (uniq[k] == clusters[c]) break;
        if (k == nu) {
            if (nu == cap) { cap *= 2; uniq = (int64_t *)realloc(uniq, sizeof(int64_t) * cap); }
            uniq[nu++] = clusters[c];
        }
        levels[c] = (int32_t)(k + 1);
    }
    free(uniq);
    return (int)nu;
}

/* cluster_blocks_indexes = cumsum(rle(levels)$lengths); error when the
 * levels are unsorted.  ends must hold n entries; returns count or -1. */
int orc_cluster_blocks(int64_t n, const int32_t *levels, int32_t *ends)
{
    for (int64_t c = 1; c < n; c++) if (levels[c] < levels[c - 1]) return -1;
    int nb = 0;
    for (int64_t c = 0; c < n; c++)
        if (c == n - 1 || levels[c + 1] != levels[c]) ends[nb++] = (int32_t)(c + 1);
    return nb;
}

/* order(levels): stable ascending permutation (0-based) */
void orc_group_order(int64_t n, const int32_t *levels, int nlev, int64_t *ord)
{
    int64_t *cnt = (int64_t *)calloc((size_t)nlev + 2, sizeof(int64_t));
    for (int64_t c = 0; c < n; c++) cnt[levels[c] + 1]++;
    for (int i = 1; i <= nlev + 1; i++) cnt[i] += cnt[i - 1];
    for (int64_t c = 0; c < n; c++) ord[cnt[levels[c]]++] = c;
    free(cnt);
}

/* ------------------------------------------------------------------ */
/* multiple testing  (R/test.R:127 -> stats::p.adjust)                 */
/* ------------------------------------------------------------------ */
typedef struct { double p; int64_t i; } pi_pair;
static int cmp_desc(const void *a, const void *b)
{
    const pi_pair *x = a, *y = b;
    if (x->p > y->p) return -1;
    if (x->p < y->p) return 1;
    return (x->i < y->i) ? -1 : (x->i > y->i);
}
static int cmp_asc(const void *a, const void *b)
{
    const pi_pair *x = a, *y = b;
    if (x->p < y->p) return -1;
    if (x->p > y->p) return 1;
    return (x->i < y->i) ? -1 : (x->i > y->i);
}

/* sum(1/(1:n)) of the double-rounded terms, rounded once (double-double
 * accumulation); R's sum() accumulates in extended precision */
static double harmonic_rounded(int64_t n)
{
    double s = 0.0, e = 0.0;
    for (int64_t k = 1; k <= n; k++) {
        double v = 1.0 / (double)k;
        double t = s + v, bp = t - s;
        e += (s - (t - bp)) + (v - bp);
        s = t;
    }
    return s + e;
}

/* Hommel's method as stats::p.adjust states it, on the ascending valid
 * p-values s[0..n) (n >= 3); writes the adjusted value of rank k to r[k]. */
static void hommel_sorted(int64_t n, const double *s, double *r)
{
    double *q = (double *)malloc(sizeof(double) * n);
    double *pa = (double *)malloc(sizeof(double) * n);
    double mn = INFINITY;
    for (int64_t i = 1; i <= n; i++) { double t = (double)n * s[i - 1] / (double)i; if (t < mn) mn = t; }
    for (int64_t i = 0; i < n; i++) q[i] = pa[i] = mn;
    for (int64_t m = n - 1; m >= 2; m--) {
        /* i1 = 1..n-m+1, i2 = n-m+2..n */
        double q1 = INFINITY;
        for (int64_t j = 2; j <= m; j++) {
            double t = (double)m * s[n - m + j - 1] / (double)j;
            if (t < q1) q1 = t;
        }
        for (int64_t i = 1; i <= n - m + 1; i++) q[i - 1] = fmin((double)m * s[i - 1], q1);
        for (int64_t i = n - m + 2; i <= n; i++) q[i - 1] = q[n - m];
        for (int64_t i = 0; i < n; i++) pa[i] = fmax(pa[i], q[i]);
    }
    for (int64_t i = 0; i < n; i++) r[i] = fmax(pa[i], s[i]);
    free(q); free(pa);
}

/* method: 0 none, 1 BH, 2 bonferroni, 3 holm, 4 hochberg, 5 BY, 6 hommel
 * (stats::p.adjust, called at R/test.R:127).  NaN entries are left NaN and
 * do not count toward n (p.adjust's default n = length(p) is evaluated
 * after the NAs are dropped).  With n = 2, hommel is hochberg, as
 * p.adjust switches. */
int orc_p_adjust(int64_t m, const double *p, int method, double *out)
{
    pi_pair *v = (pi_pair *)malloc(sizeof(pi_pair) * (m > 0 ? m : 1));
    int64_t n = 0;
    for (int64_t i = 0; i < m; i++) { out[i] = p[i]; if (!isnan(p[i])) { v[n].p = p[i]; v[n].i = i; n++; } }
    if (n <= 1 || method == 0) { free(v); return ORC_OK; }
    if (method == 6 && n == 2) method = 4;
    double dn = (double)n;
    if (method == 6) {
        qsort(v, n, sizeof(pi_pair), cmp_asc);
        double *s = (double *)malloc(sizeof(double) * n), *r = (double *)malloc(sizeof(double) * n);
        for (int64_t k = 0; k < n; k++) s[k] = v[k].p;
        hommel_sorted(n, s, r);
        for (int64_t k = 0; k < n; k++) out[v[k].i] = r[k];
        free(s); free(r); free(v);
        return ORC_OK;
    }
    if (method == 2) {
        for (int64_t k = 0; k < n; k++) out[v[k].i] = fmin(1.0, dn * v[k].p);
    } else if (method == 1 || method == 5 || method == 4) {
        qsort(v, n, sizeof(pi_pair), cmp_desc);
        double q = 1.0;
        if (method == 5) q = harmonic_rounded(n);
        double cm = INFINITY;
        for (int64_t k = 0; k < n; k++) {
            double i = (double)(n - k);               /* i = lp:1 */
            double val = (method == 4) ? (dn + 1.0 - i) * v[k].p : q * dn / i * v[k].p;
            if (val < cm) cm = val;
            out[v[k].i] = fmin(1.0, cm);
        }
    } else if (method == 3) {
        qsort(v, n, sizeof(pi_pair), cmp_asc);
        double cm = -INFINITY;
        for (int64_t k = 0; k < n; k++) {
            double val = (dn - (double)k) * v[k].p;  /* (n+1-i) with i = k+1 */
            if (val > cm) cm = val;
            out[v[k].i] = fmin(1.0, cm);
        }
    } else { free(v); return ORC_ERR_ARG; }
    free(v);
    return ORC_OK;
}

/* test_de (R/test.R:85-134).  sandwich may be NULL (no clusters).
 * lfc output is log2 and clipped to +-max_lfc. */
int orc_test_de(int64_t G, int p, const double *beta, const double *bread, const double *sandwich,
                int64_t nsamples, const double *contrast, int method, double max_lfc,
                double *pval, double *padj, double *lfc)
{
    double df = (double)(nsamples - 2);
    for (int64_t g = 0; g < G; g++) {
        double l = 0.0;
        for (int j = 0; j < p; j++) l += beta[g * p + j] * contrast[j];
        const double *Hn = bread + g * p * p;
        double vn = 0.0;
        for (int a = 0; a < p; a++) for (int b = 0; b < p; b++) vn += contrast[a] * Hn[b * p + a] * contrast[b];
        double pn = orc_two_sided_t_pvalue(fabs(l) / sqrt(vn), df);
        if (sandwich) {
            const double *Hc = sandwich + g * p * p;
            double vc = 0.0;
            for (int a = 0; a < p; a++) for (int b = 0; b < p; b++) vc += contrast[a] * Hc[b * p + a] * contrast[b];
            double pc = orc_two_sided_t_pvalue(fabs(l) / sqrt(vc), df);
            pval[g] = (isnan(pc) || isnan(pn)) ? NAN : fmax(pc, pn);
        } else {
            pval[g] = pn;
        }
        double lf = l / log(2.0);
        if (lf >= max_lfc) lf = max_lfc;
        if (lf <= -max_lfc) lf = -max_lfc;
        lfc[g] = lf;
    }
    return orc_p_adjust(G, pval, method, padj);
}

/* ------------------------------------------------------------------ */
/* cpu_fit pipeline  (R/main.R:375-523)                                */
/* ------------------------------------------------------------------ */
double orc_fit_overdispersion_new(int64_t n, int p, const double *y, const double *X,
                                  const double *beta, const double *off, int max_iter,
                                  double eps_theta, int newton_max, int *iters, int *converged,
                                  int *err);

/* overdispersion: 0 = FALSE (Poisson), 1 = MOM, 2 = MLE ("old"/"MLE").
 * theta0: per-gene initial dispersion (estimate_dispersion or user value).
 * beta0 : G x p initial coefficients (row-major per gene).
 * ends  : cluster block ends (NULL when no clusters).
 * outputs: beta (G x p), theta (G), iters (G), theta_iters (G; -1 = NA),
 *          bread (G p^2), sandwich (G p^2, only when ends != NULL),
 *          theta_mom (G, optional: MOM estimate at the fitted beta). */
int orc_cpu_fit(int64_t G, int64_t n, int p, const int64_t *rowptr, const int32_t *col,
                const double *val, const double *X, const double *offv, const double *theta0,
                const double *beta0, int overdispersion, int max_iter, double tolerance,
                const int32_t *ends, int nclust, int64_t g_begin, int64_t g_end,
                double *beta, double *theta, int32_t *iters, int32_t *theta_iters,
                double *bread, double *sandwich, double *theta_mom)
{
    double *sf = (double *)malloc(sizeof(double) * n);
    for (int64_t c = 0; c < n; c++) sf[c] = exp(offv[c]);
    if (g_end > G) g_end = G;
    /* many genes: one thread per gene; few genes: one gene at a time with
     * its cell sums split over the threads (orc_cell_sums) */
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    #pragma omp parallel if (g_end - g_begin >= 4 * (int64_t)nth)
    {
        double *y = (double *)malloc(sizeof(double) * n);
        double *meat = (double *)malloc(sizeof(double) * p * p);
        double *tmp = (double *)malloc(sizeof(double) * p * p);
        #pragma omp for schedule(dynamic, 1)
        for (int64_t g = g_begin; g < g_end; g++) {
            row_dense(rowptr, col, val, g, n, y);
            double *b = beta + g * p;
            for (int j = 0; j < p; j++) b[j] = beta0[g * p + j];
            iters[g] = orc_beta_fit(n, p, y, X, b, offv, (float)theta0[g], max_iter, (float)tolerance);
            double th = theta0[g];
            int32_t ti = -1;
            if (theta_mom) theta_mom[g] = orc_mom_dispersion(n, p, y, X, b, sf);
            if (overdispersion == 2) {
                int it;
                th = orc_fit_dispersion(n, p, y, X, b, offv, max_iter, 1, &it);
                ti = -1;  /* theta_iters is NA for "old"/"MLE" (R/main.R:424-435) */
            } else if (overdispersion == 1) {
                th = theta_mom ? theta_mom[g] : orc_mom_dispersion(n, p, y, X, b, sf);
                ti = 0;
            } else if (overdispersion == 3) {
                int it, cv, er;
                th = orc_fit_overdispersion_new(n, p, y, X, b, offv, max_iter, tolerance, 16, &it,
                                                &cv, &er);
                ti = it;
            } else {
                th = 0.0; ti = 0;
            }
            theta[g] = th;
            theta_iters[g] = ti;
            double *br = bread + g * p * p;
            orc_compute_hessian(n, p, b, th, y, X, sf, br);
            if (ends && sandwich) {
                orc_clustered_meat_fast(n, p, X, y, b, th, sf, ends, nclust, meat);
                /* s_clust = bread %*% meat %*% bread * n */
                for (int i = 0; i < p; i++) for (int j = 0; j < p; j++) {
                    double s = 0.0; for (int k = 0; k < p; k++) s += br[k * p + i] * meat[j * p + k];
                    tmp[j * p + i] = s;
                }
                double *sw = sandwich + g * p * p;
                for (int i = 0; i < p; i++) for (int j = 0; j < p; j++) {
                    double s = 0.0; for (int k = 0; k < p; k++) s += tmp[k * p + i] * br[j * p + k];
                    sw[j * p + i] = s * (double)n;
                }
            }
        }
        free(y); free(meat); free(tmp);
    }
    free(sf);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* overdispersion = "new" / "I": fit_overdispersion_cppp                 */
/* (src/new_overdispersion.cpp:195-481)                                 */
/* ------------------------------------------------------------------ */

/* Gauss-Hermite rule (weight exp(-x^2)) of order m: nodes are the
 * eigenvalues of the Jacobi matrix (zero diagonal, off-diagonal sqrt(k/2)),
 * found by bisection on Sturm counts; weights sqrt(pi) / sum_k q_k(x)^2
 * with q_k the orthonormal Hermite polynomials (Christoffel numbers).  The
 * reference builds the same rule with an Eigen eigensolver
 * (src/new_overdispersion.cpp:22-47). */
void orc_gauss_hermite(int m, double *x, double *w)
{
    const double hi0 = sqrt(2.0 * m) + 1.0;
    for (int j = 0; j < m; j++) {
        double lo = -hi0, hi = hi0;
        for (int it = 0; it < 200; it++) {
            double mid = 0.5 * (lo + hi);
            if (mid <= lo || mid >= hi) break;
            int c = 0;
            double d = 1.0;
            for (int i = 0; i < m; i++) {
                double b2 = i ? 0.5 * i : 0.0;
                d = -mid - (i ? b2 / d : 0.0);
                if (d == 0.0) d = -1e-300;
                c += d < 0.0;
            }
            if (c > j) hi = mid; else lo = mid;
        }
        double xj = 0.5 * (lo + hi);
        double qm = 0.0, q = 1.0, sum = 1.0;
        for (int k = 0; k + 1 < m; k++) {
            double qn = (xj * q - (k ? sqrt(0.5 * k) : 0.0) * qm) / sqrt(0.5 * (k + 1));
            qm = q; q = qn;
            sum += q * q;
        }
        x[j] = xj;
        w[j] = sqrt(M_PI) / sum;
    }
}

typedef struct { double mu0, sigma0, h_mu0; } orc_laplace;

/* h(x) = p log x + s (x log x - lgamma x) - t x and its derivatives
 * (src/new_overdispersion.cpp:55-68) */
static double nod_g(double s, double t, double x) { return s * (x * log(x) - lgamma(x)) - t * x; }
static double nod_g1(double s, double t, double x) { return s * (log(x) + 1.0 - orc_digamma(x)) - t; }
static double nod_g2(double s, double x) { return s * (1.0 / x - orc_trigamma(x)); }

/* find_mode (src/new_overdispersion.cpp:71-97); returns -1 on failure */
static int nod_mode(double p, double s, double t, int max_newton, double tol, double x0,
                    orc_laplace *lp)
{
    double x = x0 > 1e-9 ? x0 : 1e-9;
    for (int i = 0; i < max_newton; i++) {
        double g1v = p / x + nod_g1(s, t, x);
        if (fabs(g1v) < tol) break;
        double g2v = -p / (x * x) + nod_g2(s, x);
        double xn = x - g1v / g2v;
        if (!(xn > 0.0) || !isfinite(xn)) xn = 0.5 * x;
        if (fabs(xn - x) < tol * (1.0 + fabs(x))) { x = xn; break; }
        x = xn;
    }
    double curv = -(-p / (x * x) + nod_g2(s, x));
    if (!(curv > 0.0) || !isfinite(curv)) return -1;
    lp->mu0 = x > 1e-12 ? x : 1e-12;
    lp->sigma0 = sqrt(1.0 / curv);
    lp->h_mu0 = p * log(lp->mu0) + nod_g(s, t, lp->mu0);
    return 0;
}

/* log_integral_at (src/new_overdispersion.cpp:99-126); -1 on underflow */
static int nod_log_integral(double p, double s, double t, int m, const double *gx,
                            const double *gw, const orc_laplace *lp, double *out)
{
    const double scale = lp->sigma0 * sqrt(2.0);
    double max_lt = -INFINITY;
    for (int i = 0; i < m; i++) {
        double xx = lp->mu0 + scale * gx[i];
        if (xx <= 0.0 || !isfinite(xx)) continue;
        double r = (p * log(xx) + nod_g(s, t, xx)) - lp->h_mu0 + gx[i] * gx[i];
        double lt = log(gw[i]) + r;
        if (lt > max_lt) max_lt = lt;
    }
    long double acc = 0.0L;
    for (int i = 0; i < m; i++) {
        double xx = lp->mu0 + scale * gx[i];
        if (xx <= 0.0 || !isfinite(xx)) continue;
        double r = (p * log(xx) + nod_g(s, t, xx)) - lp->h_mu0 + gx[i] * gx[i];
        acc += expl((long double)(log(gw[i]) + r - max_lt));
    }
    if (!(acc > 0.0L)) return -1;
    *out = lp->h_mu0 + log(scale) + max_lt + log((double)acc);
    return 0;
}

/* H_log_gh_cpp (src/new_overdispersion.cpp:129-141): log of the integral
 * of x^p exp(s (x log x - lgamma x) - t x) over x > 0 by Laplace-centred
 * Gauss-Hermite quadrature; NAN when t <= s or the mode search fails */
double orc_h_log_gh(double p, double s, double t, int m, int max_newton, double tol)
{
    if (!(t > s)) return NAN;
    if (m < 4) m = 4;
    if (m > 64) m = 64;
    double gx[64], gw[64], out;
    orc_gauss_hermite(m, gx, gw);
    double x0 = (p + s) / (t - s);
    if (x0 < 1e-3) x0 = 1e-3;
    orc_laplace lp;
    if (nod_mode(p, s, t, max_newton, tol, x0, &lp)) return NAN;
    if (nod_log_integral(p, s, t, m, gx, gw, &lp, &out)) return NAN;
    return out;
}

/* per-gene state of fit_overdispersion_cppp */
typedef struct {
    int64_t n;
    int p;
    const double *y, *wq;
    double xbeta_sum;
    int gh_m, max_newton;
    double tol;
    const double *gx, *gw;
    int err;   /* 1: C1 <= n, 2: mode search failed, 3: quadrature underflow */
} nod_ctx;

/* F_k (src/new_overdispersion.cpp:288-311): the fixed-point map */
static double nod_F(nod_ctx *c, double kk)
{
    if (c->err) return NAN;
    double sd = 0.0, sl = 0.0, sm = 0.0;
    for (int64_t i = 0; i < c->n; i++) {
        double wi = c->wq[i], yi = c->y[i];
        double kw = kk * wi;
        sd += orc_digamma(kk + yi);
        sl += log1p(kw);
        sm += (kk + yi) * wi / (1.0 + kw);
    }
    double C1 = c->xbeta_sum - (sd - sl) + sm;
    if (!(C1 > (double)c->n)) { c->err = 1; return NAN; }
    double sN = (double)c->n;
    orc_laplace l1, l2;
    double x01 = (0.5 + sN) / (C1 - sN);
    if (x01 < 1e-3) x01 = 1e-3;
    if (nod_mode(0.5, sN, C1, c->max_newton, c->tol, x01, &l1)) { c->err = 2; return NAN; }
    if (nod_mode(-0.5, sN, C1, c->max_newton, c->tol, l1.mu0, &l2)) { c->err = 2; return NAN; }
    double lp, lm;
    if (nod_log_integral(0.5, sN, C1, c->gh_m, c->gx, c->gw, &l1, &lp)) { c->err = 3; return NAN; }
    if (nod_log_integral(-0.5, sN, C1, c->gh_m, c->gx, c->gw, &l2, &lm)) { c->err = 3; return NAN; }
    return exp(lp - lm);
}
static double nod_f(nod_ctx *c, double kk) { return log(nod_F(c, kk)) - log(kk); }

static double nod_clamp(double k) { return k < 1e-4 ? 1e-4 : (k > 1e4 ? 1e4 : k); }

/* the reference's Brent root finder (src/new_overdispersion.cpp:343-373) */
static double nod_brent(nod_ctx *c, double a, double b, double fa, double fb)
{
    double cc = a, fc = fa, d = b - a, e = d;
    const double tol = c->tol, epsm = DBL_EPSILON;
    for (int it = 0; it < 60; it++) {
        if (fabs(fc) < fabs(fb)) { a = b; b = cc; cc = a; fa = fb; fb = fc; fc = fa; }
        double tol1 = 2.0 * epsm * fabs(b) + 0.5 * tol;
        double xm = 0.5 * (cc - b);
        if (fabs(xm) <= tol1 || fb == 0.0) return b;
        double sv, pv, qv;
        if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
            sv = fb / fa;
            if (a == cc) { pv = 2.0 * xm * sv; qv = 1.0 - sv; }
            else {
                double r = fb / fc, t = fa / fc;
                pv = sv * (2.0 * xm * t * (t - r) - (b - a) * (r - 1.0));
                qv = (t - 1.0) * (r - 1.0) * (sv - 1.0);
            }
            if (pv > 0) qv = -qv;
            pv = fabs(pv);
            double m1 = 3.0 * xm * qv - fabs(tol1 * qv), m2 = fabs(e * qv);
            if (2.0 * pv < (m1 < m2 ? m1 : m2)) { e = d; d = pv / qv; }
            else { d = xm; e = d; }
        } else { d = xm; e = d; }
        a = b; fa = fb;
        b += (fabs(d) > tol1 ? d : (xm > 0 ? tol1 : -tol1));
        fb = nod_f(c, b);
        if ((fb > 0 && fc > 0) || (fb < 0 && fc < 0)) { cc = a; fc = fa; e = d = b - a; }
    }
    return b;
}

/* fit_overdispersion_cppp for one gene (dense y): returns kappa (= theta);
 * *iters = kappa_iters, *converged, *err as in nod_ctx (4: residual not
 * finite at the start).  The kappa argument of the reference is unused
 * there (it restarts from the moment estimate of y) and is not taken. */
double orc_fit_overdispersion_new(int64_t n, int p, const double *y, const double *X,
                                  const double *beta, const double *off, int max_iter,
                                  double eps_theta, int newton_max, int *iters, int *converged,
                                  int *err)
{
    double *wq = (double *)malloc(sizeof(double) * n);
    double xbs = 0.0;
    for (int64_t i = 0; i < n; i++) {
        double xb = 0.0;
        for (int j = 0; j < p; j++) xb += X[(int64_t)j * n + i] * beta[j];
        xbs += xb;
        wq[i] = exp(-(xb + off[i]));
    }
    double gx[64], gw[64];
    int m = newton_max < 4 ? 4 : (newton_max > 64 ? 64 : newton_max);
    orc_gauss_hermite(m, gx, gw);
    nod_ctx c = {n, p, y, wq, xbs, m, newton_max, eps_theta, gx, gw, 0};
    /* moment start (src/new_overdispersion.cpp:225-254) */
    double ym = 0.0;
    for (int64_t i = 0; i < n; i++) ym += y[i];
    ym /= (double)n;
    double yv = 0.0;
    if (n > 1) {
        for (int64_t i = 0; i < n; i++) yv += (y[i] - ym) * (y[i] - ym);
        yv /= (double)(n - 1);
    }
    double kap = (yv - ym) / (ym * ym);
    if (!isfinite(kap) || kap <= 0.0) kap = 0.01;
    double k = 1.0 / kap;
    if (!isfinite(k)) k = 1e-4;
    k = nod_clamp(k);
    const double kmin = 1e-4, jump = 10.0;
    int conv = 0, it_k = 0, bad = 0;
    *err = 0;

    double k0 = nod_clamp(k), f0 = nod_f(&c, k0);
    if (!isfinite(f0)) { *err = c.err ? c.err : 4; free(wq); *iters = 0; *converged = 0; return NAN; }
    double h = 1e-6 * k0 > 1e-8 ? 1e-6 * k0 : 1e-8;
    double fp0 = (nod_f(&c, k0 + h) - f0) / h;
    if (isfinite(fp0) && fabs(fp0) > 1e-10) {
        double kn = nod_clamp(k0 - f0 / fp0), fn = nod_f(&c, kn);
        if (isfinite(fn) && fabs(fn) < fabs(f0)) { k0 = kn; f0 = fn; }
    }
    double k1 = nod_F(&c, k0);
    double cap = jump * (k0 > 1.0 ? k0 : 1.0);
    if (k1 > cap) k1 = cap;
    k1 = nod_clamp(k1);
    double f1 = nod_f(&c, k1);
    if (f0 * f1 < 0) {
        k = nod_brent(&c, k0 < k1 ? k0 : k1, k0 < k1 ? k1 : k0, f0, f1);
        conv = 1;
    } else {
        for (it_k = 0; it_k < max_iter; it_k++) {
            double aj = jump / (1.0 + 0.1 * it_k);
            double k2 = nod_F(&c, k1);
            double c2 = aj * (k1 > 1.0 ? k1 : 1.0);
            if (k2 > c2) k2 = c2;
            k2 = nod_clamp(k2);
            double f2 = nod_f(&c, k2);
            double d1 = k1 - k0, d2 = k2 - k1, den = d2 - d1;
            double ka = fabs(den) > 1e-14 ? k0 - d1 * d1 / den : k2;
            if (!(ka > 0) || !isfinite(ka)) ka = k2;
            double c3 = aj * (k2 > 1.0 ? k2 : 1.0);
            if (ka > c3) ka = c3;
            ka = nod_clamp(ka);
            double kp = ka, fp = nod_f(&c, kp);
            int bt = 0;
            while ((fabs(fp) >= fabs(f1) || !isfinite(fp)) && bt < 8) {
                kp = 0.5 * (kp + k1);
                fp = nod_f(&c, kp);
                bt++;
            }
            if (!(fabs(fp) < fabs(f1))) {
                bad++;
                if (bad == 1 && fabs(f1 - f0) > 1e-14) {
                    double ks = nod_clamp(k1 - f1 * (k1 - k0) / (f1 - f0)), fs = nod_f(&c, ks);
                    if (isfinite(fs) && fabs(fs) < fabs(f1)) { kp = ks; fp = fs; bad = 0; }
                }
                if (bad >= 1) {
                    double a = k1 < k2 ? k1 : k2, b = k1 < k2 ? k2 : k1;
                    if (f1 * f2 < 0) { k = nod_brent(&c, a, b, f1, f2); conv = 1; break; }
                }
                if (bad >= 1) {
                    /* find_bracket (src/new_overdispersion.cpp:324-339) */
                    double lo = -1.0, hi = -1.0, fc = nod_f(&c, k1);
                    for (int ex = 1; ex <= 10; ex++) {
                        double fac = pow(2.0, ex);
                        double l = k1 / fac > kmin ? k1 / fac : kmin;
                        double u = k1 * fac < 1e4 ? k1 * fac : 1e4;
                        double fl = nod_f(&c, l);
                        if (fl * fc < 0) { lo = l; hi = k1; break; }
                        double fu = nod_f(&c, u);
                        if (fc * fu < 0) { lo = k1; hi = u; break; }
                        if (fl * fu < 0) { lo = l; hi = u; break; }
                    }
                    if (lo > 0) {
                        double flo = nod_f(&c, lo), fhi = nod_f(&c, hi);
                        k = nod_brent(&c, lo, hi, flo, fhi);
                        conv = 1;
                        break;
                    }
                }
                kp = k2; fp = f2;
            } else {
                bad = 0;
            }
            if (fabs(kp - k1) < eps_theta * (1.0 + k1)) { k = kp; conv = 1; break; }
            k0 = k1; f0 = f1; k1 = kp; f1 = fp;
        }
        if (!conv) k = k1 > kmin ? k1 : kmin;
    }
    free(wq);
    *iters = it_k + 1;
    *converged = conv;
    if (c.err) { *err = c.err; return NAN; }
    return 1.0 / k;
}

/* single-gene wrappers used by the tests (dense y) */
double orc_score_dense(int64_t n, int p, const double *y, const double *mu, const double *X,
                       double log_theta, int cr)
{
    nbdata d = { n, p, y, mu, X };
    return orc_nb_score(&d, log_theta, cr);
}
double orc_deriv_score_dense(int64_t n, int p, const double *y, const double *mu, const double *X,
                             double log_theta, int cr)
{
    nbdata d = { n, p, y, mu, X };
    return orc_nb_deriv_score(&d, log_theta, cr);
}
double orc_loglik_dense(int64_t n, int p, const double *y, const double *mu, const double *X,
                        double log_theta, int cr)
{
    nbdata d = { n, p, y, mu, X };
    return orc_nb_loglik(&d, log_theta, cr);
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
