/*
 * devil_b200.h -- C ABI of the B200 (sm_100a) implementation of devil's
 * per-gene negative-binomial GLM path.
 *
 * Every entry point returns an int status (DEVIL_OK = 0) and never exits the
 * process; devil_last_error() gives the message of the last failure on a
 * context.  Arrays are plain pointers with explicit sizes.  Unless a
 * function says "_device", pointers are HOST pointers and the call is
 * synchronous (it copies in, computes on the GPU, copies out).  "_device"
 * variants take device pointers and run asynchronously on the context's
 * stream (devil_ctx_stream()).
 *
 * Layout conventions (the same as R's, so an Rcpp shim passes R memory
 * straight through):
 *   design X        n x p doubles, column-major:  X[j*n + c]
 *   per-gene p x p  column-major, genes consecutive: M[g*p*p + j*p + i]
 *   beta            G x p, row-major by gene:       beta[g*p + j]
 *   counts          see devil_counts below.
 *
 * One context per host thread; a context owns its device buffers and one
 * CUDA stream.  Calls on one context are not re-entrant.
 */
#ifndef DEVIL_B200_H
#define DEVIL_B200_H

#include <stdint.h>
#include <stddef.h>

#if defined(__GNUC__)
#define DEVIL_API __attribute__((visibility("default")))
#else
#define DEVIL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define DEVIL_OK               0
#define DEVIL_ERR_ARG          1   /* invalid argument / shape            */
#define DEVIL_ERR_CUDA         2   /* CUDA runtime error                  */
#define DEVIL_ERR_ZERO_COLUMN  3   /* normed_sum: a cell has no counts    */
#define DEVIL_ERR_SINGULAR     4   /* design matrix rank deficient        */
#define DEVIL_ERR_UNSORTED     5   /* clusters not in contiguous blocks   */
#define DEVIL_ERR_NOMEM        6   /* device allocation failed            */
#define DEVIL_ERR_UNSUPPORTED  7   /* option outside this implementation  */
#define DEVIL_ERR_NUMERIC      8   /* a numerical stop() of the reference  */

/* ---- per-gene fit status (devil_fit_result.status) ------------------- */
#define DEVIL_GENE_CONVERGED   0   /* max|delta| < tolerance               */
#define DEVIL_GENE_MAX_ITER    1   /* stopped at max_iter                  */
#define DEVIL_GENE_NAN         2   /* delta[0] was NaN (reference stops)   */

/* ---- count matrix ---------------------------------------------------- */
#define DEVIL_COUNTS_DENSE_F64   0  /* values: G x n doubles              */
#define DEVIL_COUNTS_DENSE_F32   1  /* values: G x n floats               */
#define DEVIL_COUNTS_CSR_U16     2  /* gene-major CSR, uint16 values      */
#define DEVIL_COUNTS_CSR_F32     3  /* gene-major CSR, float values       */
#define DEVIL_COUNTS_CSC_F64     4  /* cell-major (R dgCMatrix), doubles  */

#define DEVIL_DENSE_GENE_MAJOR   0  /* Y[g*n + c]                          */
#define DEVIL_DENSE_CELL_MAJOR   1  /* Y[c*G + g]  (R's column-major G x n) */

typedef struct devil_counts {
    int format;            /* DEVIL_COUNTS_*                               */
    int dense_layout;      /* DEVIL_DENSE_* (dense formats only)           */
    int64_t n_genes;       /* G                                            */
    int64_t n_cells;       /* n                                            */
    int64_t nnz;           /* sparse formats                               */
    const void *values;    /* dense matrix or nnz values                   */
    const int64_t *ptr;    /* CSR: rowptr[G+1]; CSC: colptr[n+1]           */
    const int32_t *idx;    /* CSR: cell index; CSC: gene index (sorted)    */
} devil_counts;

/* ---- options --------------------------------------------------------- */
#define DEVIL_SF_NONE        0   /* size_factors = NULL -> all ones        */
#define DEVIL_SF_NORMED_SUM  1
#define DEVIL_SF_PSINORM     2
#define DEVIL_SF_GIVEN       3   /* use devil_fit_opts.size_factors        */

#define DEVIL_OD_NONE        0   /* overdispersion = FALSE (Poisson)       */
#define DEVIL_OD_MOM         1
#define DEVIL_OD_MLE         2   /* "old" / "MLE"                          */
#define DEVIL_OD_NEW         3   /* "new" / "I": fit_overdispersion_cppp   */

#define DEVIL_FORM_CHOSEN    0   /* tiled, compacted, grouped kernels       */
#define DEVIL_FORM_PLAIN     1   /* comparison form: every pass per cell on */
                                 /* the shared-memory SIMT engine, FP32     */
                                 /* per-cell arithmetic and chunk sums for  */
                                 /* IRLS and MLE (MOM, bread/meat FP64 as   */
                                 /* in every form), no design grouping      */

/* arithmetic of the per-cell Hessian contractions (IRLS and MLE passes) */
#define DEVIL_PREC_FP32      0   /* FP32 FMAs on the CUDA cores (default)   */
#define DEVIL_PREC_TC_TF32   1   /* tcgen05 MMAs on split TF32 (hi + lo)    */
                                 /* operands, FP32 accumulation: IRLS and   */
                                 /* MLE passes at every p (designs without  */
                                 /* few distinct rows; from p = 9 on this   */
                                 /* is also what DEVIL_PREC_FP32 runs);     */
                                 /* other passes as DEVIL_PREC_FP32         */
#define DEVIL_PREC_TC_BF16X3 2   /* not provided (DEVIL_ERR_UNSUPPORTED):   */
                                 /* the split-TF32 path already reaches     */
                                 /* FP32 accuracy                           */

typedef struct devil_fit_opts {
    int max_iter;                 /* default 200                           */
    double tolerance;             /* default 1e-3 (rounded to float, as    */
                                  /* the reference's beta_fit receives it)  */
    int overdispersion;           /* DEVIL_OD_*                            */
    int init_beta_rough;          /* 0: QR least squares, 1: log1p(mean)   */
    int size_factors;             /* DEVIL_SF_*                            */
    const double *size_factor_values;   /* n, when DEVIL_SF_GIVEN          */
    double offset;                /* scalar offset (default 0)             */
    int has_init_overdispersion;  /* 1: theta_0 = init_overdispersion      */
    double init_overdispersion;
    int compute_theta_mom;        /* also return the MOM theta at beta     */
    int form;                     /* DEVIL_FORM_*                          */
    int precision;                /* DEVIL_PREC_* (default FP32)           */
} devil_fit_opts;

DEVIL_API void devil_fit_opts_default(devil_fit_opts *opts);

typedef struct devil_fit_result {
    double  *beta;          /* G x p                       (required)       */
    double  *theta;         /* G                           (required)       */
    int32_t *beta_iters;    /* G                           (required)       */
    int32_t *theta_iters;   /* G; INT32_MIN = NA (MLE)     (optional)       */
    double  *bread;         /* G x p x p  = beta_sandwiches_null (optional) */
    double  *sandwich;      /* G x p x p, clusters only    (optional)       */
    double  *theta_mom;     /* G (opts.compute_theta_mom)  (optional)       */
    int32_t *status;        /* G  DEVIL_GENE_*             (optional)       */
    double  *size_factors;  /* n                           (optional)       */
    double  *offset_vector; /* n                           (optional)       */
    double  *meat;          /* G x p x p, clusters only    (optional)       */
} devil_fit_result;

typedef struct devil_ctx devil_ctx;

/* ---- context --------------------------------------------------------- */
/* replaces the per-call device setup of cuda/src/batch.cpp:184-311 */
DEVIL_API int  devil_ctx_create(int device, devil_ctx **out);
DEVIL_API int  devil_ctx_destroy(devil_ctx *ctx);
DEVIL_API const char *devil_last_error(const devil_ctx *ctx);
DEVIL_API void *devil_ctx_stream(devil_ctx *ctx);         /* cudaStream_t            */
DEVIL_API int  devil_ctx_synchronize(devil_ctx *ctx);
/* kernel launches issued by this context since creation (for accounting) */
DEVIL_API int64_t devil_ctx_launch_count(const devil_ctx *ctx);

/* Profiling (no counterpart in the reference, whose only timing is wall
 * clock prints in src/beta.cpp:89-124): when enabled, every per-gene cell
 * pass launch is bracketed by CUDA events on the context stream and its
 * algorithmic bytes are accounted from the per-gene pass counts.
 * pass_kind: 0 IRLS, 1 MOM, 2 MLE, 3 bread/meat.  Enabling resets. */
DEVIL_API int devil_ctx_set_profiling(devil_ctx *ctx, int enable);
DEVIL_API int devil_ctx_profile(devil_ctx *ctx, int pass_kind, int64_t *launches, double *ms,
                                double *alg_bytes);
/* Tensor-core FLOPs the profiled launches of a pass kind issued (MMA
 * shapes, padding included; no counterpart in the reference).  Counted for
 * the tensor-core IRLS engine of p = 5..32 (engine 4); 0 otherwise. */
DEVIL_API int devil_ctx_profile_tc(devil_ctx *ctx, int pass_kind, double *tc_flops);
/* Genes of the last fit on this context that the tensor-core engine of
 * p = 5..32 handed back to the CUDA-core engine, which fitted them again
 * from beta_0: a coefficient beyond +-8 (DEVIL_TCW_RESCUE_BETA) or more
 * IRLS steps than DEVIL_TCW_RESCUE (default: none) (no counterpart in the
 * reference); 0 when that engine did not run. */
DEVIL_API int64_t devil_ctx_irls_rescued(const devil_ctx *ctx);
/* Engine of the last launch of a pass kind on this context (no counterpart
 * in the reference): 0 register tiles (p <= 8), 1 shared-memory tiles,
 * 2 design groups (few distinct design rows), 3 tensor cores (IRLS and MLE
 * passes, p <= 4), 4 tensor cores (IRLS and MLE passes, p = 5..32: the
 * p x p contractions as split-TF32 MMAs over a dense count image), -1 none
 * yet. */
DEVIL_API int devil_ctx_engine(const devil_ctx *ctx, int pass_kind);

/* ---- full pipeline --------------------------------------------------- */
/* fit_devil(x, design_matrix, clusters, overdispersion, init_overdispersion,
 *           init_beta_rough, offset, size_factors, max_iter, tolerance)
 * with the cpu_fit order theta_0 -> beta | theta_0 -> theta | beta ->
 * bread, meat (R/main.R:164-273, :375-523).  cluster_ends are the 1-based
 * exclusive block ends cumsum(rle(clusters)$lengths) (R/main.R:190-196);
 * n_clusters = 0 for no clusters. */
DEVIL_API int devil_fit(devil_ctx *ctx, const devil_counts *counts, const double *X, int p,
              const int32_t *cluster_ends, int n_clusters, const devil_fit_opts *opts,
              devil_fit_result *res);

/* Many independent problems (each its own genes, cells, design and
 * clusters; the configuration of many uneven DE problems): the fit of
 * every problem as devil_fit, spread over `workers` concurrent streams of
 * the context's device (1..8; each worker holds its own context) so that
 * the kernels of small problems overlap.  results[i] receives problem i.
 * On failure the status of the first failing problem is returned and the
 * context's message names the problem.  The reference fits one problem
 * per fit_devil call (R/main.R:164-273). */
typedef struct devil_problem {
    devil_counts counts;           /* host counts                           */
    const double *X;               /* n x p column-major                    */
    int p;
    const int32_t *cluster_ends;   /* NULL or n_clusters ends               */
    int n_clusters;
} devil_problem;
DEVIL_API int devil_fit_batch(devil_ctx *ctx, int n_problems, const devil_problem *problems,
                              const devil_fit_opts *opts, devil_fit_result *results, int workers);

/* same, with the count matrix (CSR formats only) and every input/output
 * already in device memory.  X_dev is n x p column-major doubles.
 * Asynchronous on the context stream. */
DEVIL_API int devil_fit_device(devil_ctx *ctx, const devil_counts *counts_dev, const double *X_dev, int p,
                     const int32_t *cluster_ends_host, int n_clusters,
                     const devil_fit_opts *opts, devil_fit_result *res_dev);

/* devil_fit_device ordered on the caller's CUDA stream (cudaStream_t;
 * NULL = the context's own stream) instead of the context's: the work
 * starts after everything the caller queued on `stream` before the call,
 * and the results are complete once the work queued on `stream` by the
 * call has finished.  The host thread still waits inside the call for the
 * active-gene counts of the IRLS and theta loops (read through mapped
 * memory).  The context's own stream is restored before returning. */
DEVIL_API int devil_fit_async(devil_ctx *ctx, void *stream, const devil_counts *counts_dev,
                              const double *X_dev, int p, const int32_t *cluster_ends_host,
                              int n_clusters, const devil_fit_opts *opts,
                              devil_fit_result *res_dev);

/* ---- DE test --------------------------------------------------------- */
#define DEVIL_ADJ_NONE        0
#define DEVIL_ADJ_BH          1   /* "BH" / "fdr"                          */
#define DEVIL_ADJ_BONFERRONI  2
#define DEVIL_ADJ_HOLM        3
#define DEVIL_ADJ_HOCHBERG    4
#define DEVIL_ADJ_BY          5
#define DEVIL_ADJ_HOMMEL      6   /* O(n^2) as in stats::p.adjust; n = 2 is */
                                  /* hochberg                              */

/* test_de (R/test.R:85-134): lfc = beta . contrast; p from the t
 * distribution with df = n_samples - 2 using contrast' H contrast; when
 * sandwich != NULL p = max(p_clust, p_null); p.adjust(method); lfc / log 2
 * clipped to +-max_lfc.  bread / sandwich are G x p x p (column-major). */
DEVIL_API int devil_test_de(devil_ctx *ctx, int64_t n_genes, int p, const double *beta,
                  const double *bread, const double *sandwich, int64_t n_samples,
                  const double *contrast, int adjust_method, double max_lfc,
                  double *pval, double *adj_pval, double *lfc);
DEVIL_API int devil_test_de_device(devil_ctx *ctx, int64_t n_genes, int p, const double *beta_dev,
                         const double *bread_dev, const double *sandwich_dev, int64_t n_samples,
                         const double *contrast_host, int adjust_method, double max_lfc,
                         double *pval_dev, double *adj_pval_dev, double *lfc_dev);

/* stats::p.adjust (called at R/test.R:127) on the device (NaN = NA,
 * excluded from n) */
DEVIL_API int devil_p_adjust(devil_ctx *ctx, int64_t m, const double *p, int method, double *out);
DEVIL_API int devil_p_adjust_device(devil_ctx *ctx, int64_t m, const double *p_dev, int method,
                                    double *out_dev);

/* The same adjustment for callers that cannot allocate device memory (no
 * counterpart in the reference): no context, no cudaMalloc / cudaFree; the
 * scratch is a 4 MiB file-scope device array held by every GPU that loads
 * the library, so m <= 65536 (larger m: DEVIL_ERR_ARG with a message in
 * errbuf).  Runs on `stream` (cudaStream_t, NULL = legacy default) of the
 * current device.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) and should come before any stream capture.  The
 * array is shared by every call on a device: calls must not overlap in
 * time (serialise them, e.g. on one stream).  errbuf (may be NULL)
 * receives a message on failure. */
DEVIL_API int devil_p_adjust_device_static(int64_t m, const double *p_dev, int method,
                                           double *out_dev, void *stream, char *errbuf,
                                           size_t errlen);

/* ---- single steps (each mirrors one reference function) -------------- */
/* calculate_sf / normed_sum_sf / psinorm_sf (R/size_factors.R:37-117) */
DEVIL_API int devil_calculate_sf(devil_ctx *ctx, const devil_counts *counts, int method, double *sf);

/* estimate_dispersion (R/overdispersion.R:129-135) */
DEVIL_API int devil_estimate_dispersion(devil_ctx *ctx, const devil_counts *counts,
                              const double *offset_vector, double *theta0);

/* init_beta (R/beta.R:13-20) or the rough init (R/main.R:404-406) */
DEVIL_API int devil_init_beta(devil_ctx *ctx, const devil_counts *counts, const double *X, int p,
                    const double *offset_vector, int rough, double *beta0);

/* beta_fit (src/beta.cpp:25-51) for every gene: k = theta0 per gene */
DEVIL_API int devil_beta_fit(devil_ctx *ctx, const devil_counts *counts, const double *X, int p,
                   const double *beta0, const double *offset_vector, const double *theta0,
                   int max_iter, double eps, int form, double *beta, int32_t *iters);

/* estimate_mom_dispersion_cpp (src/mom_overdispersion.cpp:6-56) */
DEVIL_API int devil_estimate_mom_dispersion(devil_ctx *ctx, const devil_counts *counts, const double *X,
                                  int p, const double *beta, const double *size_factors,
                                  double *theta);

/* fit_dispersion (R/overdispersion.R:25-115), MLE of log theta with the
 * Cox-Reid adjustment; Newton root search of the same score. */
DEVIL_API int devil_fit_dispersion(devil_ctx *ctx, const devil_counts *counts, const double *X, int p,
                         const double *beta, const double *offset_vector, int max_iter,
                         int cox_reid, double *theta, int32_t *newton_iters);

/* fit_overdispersion_cppp (src/new_overdispersion.cpp:195-481), the
 * overdispersion = "new" / "I" method: fixed-point search for k = 1/kappa
 * with Laplace-centred Gauss-Hermite integrals (order newton_max = 16) and
 * Aitken / secant / Brent safeguards, tolerance eps_theta.  kappa_iters is
 * the reference's kappa_iters.  DEVIL_ERR_NUMERIC (with the reference's
 * message) when a gene reaches one of the reference's stop() conditions. */
DEVIL_API int devil_fit_overdispersion_new(devil_ctx *ctx, const devil_counts *counts,
                                           const double *X, int p, const double *beta,
                                           const double *offset_vector, int max_iter,
                                           double eps_theta, double *theta, int32_t *kappa_iters);

/* compute_hessian (src/variance.cpp:22-47): bread = (X' W X)^-1 per gene */
DEVIL_API int devil_compute_hessian(devil_ctx *ctx, const devil_counts *counts, const double *X, int p,
                          const double *beta, const double *overdispersion,
                          const double *size_factors, double *bread);

/* compute_clustered_meat_fast (src/variance.cpp:186-228) per gene */
DEVIL_API int devil_compute_clustered_meat(devil_ctx *ctx, const devil_counts *counts, const double *X,
                                 int p, const double *beta, const double *overdispersion,
                                 const double *size_factors, const int32_t *cluster_ends,
                                 int n_clusters, double *meat);

/* Per-cell NB log-likelihood adjoint for one gene: for every cell c,
 * dl_c/d eta_c = (y - mu)/(1 + mu theta)  (times x_c it is the score
 * vector of src/variance.cpp:64-85) and dl_c/d log theta.  Also returns
 * the per-cell log-likelihood l_c (used for finite-difference checks).
 * y, eta (linear predictor incl. offset) are n-vectors. */
DEVIL_API int devil_nb_adjoint(devil_ctx *ctx, int64_t n, const double *y, const double *eta,
                     double log_theta, double *loglik, double *d_eta, double *d_log_theta);

/* ---- cluster handling (host-side, R/main.R:190-196, R/group_data.R) -- */
/* levels = factor(clusters, levels = unique(clusters)) (1-based); returns
 * DEVIL_ERR_UNSORTED when the levels are not in contiguous blocks.
 * ends must have room for n entries; *n_blocks receives the count. */
DEVIL_API int devil_cluster_blocks(int64_t n, const int64_t *clusters, int32_t *levels, int32_t *ends,
                         int *n_blocks);
/* order(factor(clusters, levels = unique(clusters))): stable permutation */
DEVIL_API int devil_group_order(int64_t n, const int64_t *clusters, int64_t *order);

/* version string */
DEVIL_API const char *devil_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DEVIL_B200_H */
