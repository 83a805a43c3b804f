// Rcpp bindings of libdevil_b200.so for the devil R package.
//
// Source only: R, Rcpp and RcppEigen are not available where this library
// is built and tested, so this file is not compiled here.  It shows the
// binding a devil maintainer adds to src/ (with -ldevil_b200 in
// src/Makevars) so that fit_devil(..., CUDA = TRUE) and test_de run on the
// B200 path.  Every function returns R objects with the names the reference
// already uses (R/main.R:261-272, :297-371; R/test.R:124-133).
//
//   devil_b200_fit(...)      -> list(beta, theta, iter, theta_iters, status,
//                               hessian_inv, sandwich, size_factors,
//                               offset_vector)
//   beta_fit_gpu(...)        -> the reference's beta_fit_gpu signature
//                               (src/beta.cpp:83-161) on the new backend
//   devil_b200_test_de(...)  -> list(pval, adj_pval, lfc)
#include <Rcpp.h>

#include <cstring>
#include <string>

#include "devil_b200.h"

using namespace Rcpp;

namespace {

devil_ctx* context() {
    static devil_ctx* ctx = nullptr;
    if (!ctx) {
        if (devil_ctx_create(0, &ctx) != DEVIL_OK) stop("devil_b200: no usable CUDA device");
    }
    return ctx;
}

void check(int rc) {
    if (rc != DEVIL_OK) stop(std::string("devil_b200: ") + devil_last_error(context()));
}

// a dense R matrix is genes x cells, column-major: cell-major storage
devil_counts dense_counts(const NumericMatrix& y) {
    devil_counts c;
    std::memset(&c, 0, sizeof c);
    c.format = DEVIL_COUNTS_DENSE_F64;
    c.dense_layout = DEVIL_DENSE_CELL_MAJOR;
    c.n_genes = y.nrow();
    c.n_cells = y.ncol();
    c.values = REAL(y);
    return c;
}

// a dgCMatrix (genes x cells) is compressed by cell: the CSC format
devil_counts sparse_counts(S4 m, std::vector<int64_t>& ptr64) {
    IntegerVector dim = m.slot("Dim"), p = m.slot("p"), i = m.slot("i");
    NumericVector x = m.slot("x");
    ptr64.assign(p.begin(), p.end());
    devil_counts c;
    std::memset(&c, 0, sizeof c);
    c.format = DEVIL_COUNTS_CSC_F64;
    c.n_genes = dim[0];
    c.n_cells = dim[1];
    c.nnz = x.size();
    c.values = REAL(x);
    c.ptr = ptr64.data();
    c.idx = INTEGER(i);  // 0-based row (gene) indices
    return c;
}

}  // namespace

// [[Rcpp::export]]
List devil_b200_fit(SEXP input_matrix, NumericMatrix design_matrix, SEXP size_factors,
                    SEXP overdispersion, Nullable<NumericVector> init_overdispersion,
                    bool init_beta_rough, double offset, int max_iter, double tolerance,
                    Nullable<IntegerVector> cluster_ends) {
    std::vector<int64_t> ptr64;
    devil_counts counts = Rf_isS4(input_matrix) ? sparse_counts(S4(input_matrix), ptr64)
                                                : dense_counts(NumericMatrix(input_matrix));
    const int64_t G = counts.n_genes, n = counts.n_cells;
    const int p = design_matrix.ncol();
    devil_fit_opts o;
    devil_fit_opts_default(&o);
    o.max_iter = max_iter;
    o.tolerance = tolerance;
    o.init_beta_rough = init_beta_rough;
    o.offset = offset;
    // overdispersion: "MOM", "old"/"MLE", "new"/"I" or FALSE (R/main.R:415-459)
    if (TYPEOF(overdispersion) == LGLSXP && !as<bool>(overdispersion)) {
        o.overdispersion = DEVIL_OD_NONE;
    } else {
        std::string od = as<std::string>(overdispersion);
        if (od == "MOM") o.overdispersion = DEVIL_OD_MOM;
        else if (od == "old" || od == "MLE") o.overdispersion = DEVIL_OD_MLE;
        else if (od == "new" || od == "I") o.overdispersion = DEVIL_OD_NEW;
        else stop("Unknown overdispersion mode: " + od);
    }
    NumericVector sf_given;
    if (Rf_isNull(size_factors)) {
        o.size_factors = DEVIL_SF_NONE;
    } else if (TYPEOF(size_factors) == STRSXP) {
        std::string m = as<std::string>(size_factors);
        o.size_factors = m == "psinorm" ? DEVIL_SF_PSINORM : DEVIL_SF_NORMED_SUM;
    } else {
        sf_given = NumericVector(size_factors);
        o.size_factors = DEVIL_SF_GIVEN;
        o.size_factor_values = REAL(sf_given);
    }
    if (init_overdispersion.isNotNull()) {
        o.has_init_overdispersion = 1;
        o.init_overdispersion = NumericVector(init_overdispersion)[0];
    }
    IntegerVector ends;
    if (cluster_ends.isNotNull()) ends = IntegerVector(cluster_ends);

    NumericMatrix beta(p, G);  // filled gene-major, transposed below
    NumericVector theta(G), sf(n), offv(n);
    IntegerVector iter(G), titers(G), status(G);
    NumericVector bread(p * p * G), sandwich(ends.size() ? p * p * G : 0);
    devil_fit_result r;
    std::memset(&r, 0, sizeof r);
    r.beta = REAL(beta);
    r.theta = REAL(theta);
    r.beta_iters = INTEGER(iter);
    r.theta_iters = INTEGER(titers);  // INT32_MIN is R's NA_integer_
    r.bread = REAL(bread);
    r.sandwich = ends.size() ? REAL(sandwich) : nullptr;
    r.status = INTEGER(status);
    r.size_factors = REAL(sf);
    r.offset_vector = REAL(offv);
    check(devil_fit(context(), &counts, REAL(design_matrix), p,
                    ends.size() ? INTEGER(ends) : nullptr, ends.size(), &o, &r));
    return List::create(Named("beta") = transpose(beta), Named("theta") = theta,
                        Named("iter") = iter, Named("theta_iters") = titers,
                        Named("status") = status, Named("hessian_inv") = bread,
                        Named("sandwich") = sandwich, Named("size_factors") = sf,
                        Named("offset_vector") = offv);
}

// The reference's GPU entry point, same arguments (src/beta.cpp:83-161):
// counts G x n, design n x p, offsets, cluster ends.  Returns the list
// gpu_fit() consumes (mu_beta, theta, hessian_inv, meat, iter).
// [[Rcpp::export]]
List beta_fit_gpu(NumericMatrix y, NumericMatrix X, NumericVector off, int max_iter, float eps,
                  int batch_size, bool TEST = false,
                  IntegerVector cluster_ends = IntegerVector(), int n_clusters = 0) {
    (void)batch_size;
    (void)TEST;
    devil_counts counts = dense_counts(y);
    const int64_t G = counts.n_genes;
    const int p = X.ncol();
    devil_fit_opts o;
    devil_fit_opts_default(&o);
    o.max_iter = max_iter;
    o.tolerance = eps;
    o.overdispersion = DEVIL_OD_MOM;  // the reference GPU path returns MOM theta
    o.init_beta_rough = 1;            // and starts from the rough init
    o.size_factors = DEVIL_SF_GIVEN;
    NumericVector sf = exp(off);
    o.size_factor_values = REAL(sf);
    NumericMatrix beta(p, G);
    NumericVector theta(G), bread(p * p * G), meat(n_clusters > 0 ? p * p * G : 0);
    NumericVector sandwich(n_clusters > 0 ? p * p * G : 0);
    IntegerVector iter(G);
    devil_fit_result r;
    std::memset(&r, 0, sizeof r);
    r.beta = REAL(beta);
    r.theta = REAL(theta);
    r.beta_iters = INTEGER(iter);
    r.bread = REAL(bread);
    r.sandwich = n_clusters > 0 ? REAL(sandwich) : nullptr;
    r.meat = n_clusters > 0 ? REAL(meat) : nullptr;
    check(devil_fit(context(), &counts, REAL(X), p,
                    n_clusters > 0 ? INTEGER(cluster_ends) : nullptr, n_clusters, &o, &r));
    // gpu_fit (R/main.R:312-328) forms (H %*% M %*% H) * n from these two
    List out = List::create(Named("mu_beta") = transpose(beta), Named("theta") = theta,
                            Named("hessian_inv") = NumericMatrix(p * p, G, bread.begin()),
                            Named("iter") = iter);
    if (n_clusters > 0) out["meat"] = NumericMatrix(p * p, G, meat.begin());
    return out;
}

// [[Rcpp::export]]
List devil_b200_test_de(NumericMatrix beta, NumericVector bread, Nullable<NumericVector> sandwich,
                        int n_samples, NumericVector contrast, std::string method, double max_lfc) {
    const int64_t G = beta.nrow();
    const int p = beta.ncol();
    int adj = DEVIL_ADJ_BH;
    if (method == "bonferroni") adj = DEVIL_ADJ_BONFERRONI;
    else if (method == "holm") adj = DEVIL_ADJ_HOLM;
    else if (method == "hochberg") adj = DEVIL_ADJ_HOCHBERG;
    else if (method == "BY") adj = DEVIL_ADJ_BY;
    else if (method == "none") adj = DEVIL_ADJ_NONE;
    else if (method != "BH" && method != "fdr") stop("p-value adjustment not supported: " + method);
    NumericMatrix bt = transpose(beta);  // gene-major rows
    NumericVector sw;
    if (sandwich.isNotNull()) sw = NumericVector(sandwich);
    NumericVector pv(G), pa(G), lf(G);
    check(devil_test_de(context(), G, p, REAL(bt), REAL(bread), sw.size() ? REAL(sw) : nullptr,
                        n_samples, REAL(contrast), adj, max_lfc, REAL(pv), REAL(pa), REAL(lf)));
    return List::create(Named("pval") = pv, Named("adj_pval") = pa, Named("lfc") = lf);
}
