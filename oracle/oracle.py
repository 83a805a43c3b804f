"""ctypes front end of the FP64 oracle (libdevil_oracle.so).

TEST INFRASTRUCTURE ONLY.  The parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` compare against this module or time it;
the product package ``devil_b200`` never imports it.

Each wrapper restates one function of devil's R/C++ path; the C source
(devil_oracle.c) cites the reference file:line of each.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

SF_NORMED_SUM = 0
SF_PSINORM = 1
OD_NONE, OD_MOM, OD_MLE, OD_NEW = 0, 1, 2, 3
ADJ = {"none": 0, "BH": 1, "fdr": 1, "bonferroni": 2, "holm": 3, "hochberg": 4, "BY": 5,
       "hommel": 6}

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "libdevil_oracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libdevil_oracle.so")
        src = os.path.join(_HERE, "devil_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = C.CDLL(path)
        L.orc_digamma.restype = C.c_double
        L.orc_digamma.argtypes = [C.c_double]
        L.orc_trigamma.restype = C.c_double
        L.orc_trigamma.argtypes = [C.c_double]
        L.orc_two_sided_t_pvalue.restype = C.c_double
        L.orc_two_sided_t_pvalue.argtypes = [C.c_double, C.c_double]
        L.orc_calculate_sf.argtypes = [C.c_int64, C.c_int64, _i64, _i32, _d, C.c_int, _d]
        L.orc_offset_vector.argtypes = [C.c_int64, C.c_double, _d, _d]
        L.orc_offset_vector.restype = None
        L.orc_estimate_dispersion.argtypes = [C.c_int64, C.c_int64, _i64, _i32, _d, _d, _d]
        L.orc_estimate_dispersion.restype = None
        L.orc_init_beta.argtypes = [C.c_int64, C.c_int64, C.c_int, _i64, _i32, _d, _d, _d, _d]
        L.orc_init_beta_rough.argtypes = [C.c_int64, C.c_int64, C.c_int, _i64, _d, _d]
        L.orc_init_beta_rough.restype = None
        L.orc_beta_fit.argtypes = [C.c_int64, C.c_int, _d, _d, _d, _d, C.c_float, C.c_int, C.c_float]
        L.orc_mom_dispersion.restype = C.c_double
        L.orc_mom_dispersion.argtypes = [C.c_int64, C.c_int, _d, _d, _d, _d]
        L.orc_fit_dispersion.restype = C.c_double
        L.orc_fit_dispersion.argtypes = [C.c_int64, C.c_int, _d, _d, _d, _d, C.c_int, C.c_int,
                                         C.POINTER(C.c_int)]
        for nm in ("orc_score_dense", "orc_deriv_score_dense", "orc_loglik_dense"):
            f = getattr(L, nm)
            f.restype = C.c_double
            f.argtypes = [C.c_int64, C.c_int, _d, _d, _d, C.c_double, C.c_int]
        L.orc_compute_hessian.argtypes = [C.c_int64, C.c_int, _d, C.c_double, _d, _d, _d, _d]
        L.orc_gauss_hermite.argtypes = [C.c_int, _d, _d]
        L.orc_gauss_hermite.restype = None
        L.orc_h_log_gh.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double]
        L.orc_h_log_gh.restype = C.c_double
        _ip = C.POINTER(C.c_int)
        L.orc_fit_overdispersion_new.argtypes = [C.c_int64, C.c_int, _d, _d, _d, _d, C.c_int,
                                                 C.c_double, C.c_int, _ip, _ip, _ip]
        L.orc_fit_overdispersion_new.restype = C.c_double
        L.orc_compute_scores.argtypes = [C.c_int64, C.c_int, _d, _d, _d, C.c_double, _d, _d]
        L.orc_compute_scores.restype = None
        L.orc_clustered_meat_fast.argtypes = [C.c_int64, C.c_int, _d, _d, _d, C.c_double, _d, _i32,
                                              C.c_int, _d]
        L.orc_clustered_meat_fast.restype = None
        L.orc_clustered_meat.argtypes = [C.c_int64, C.c_int, _d, _d, _d, C.c_double, _d, _i32, _d]
        L.orc_clustered_meat.restype = None
        L.orc_meat.argtypes = [C.c_int64, C.c_int, _d, _d, _d, C.c_double, _d, _d]
        L.orc_meat.restype = None
        L.orc_factor_first_appearance.argtypes = [C.c_int64, _i64, _i32]
        L.orc_cluster_blocks.argtypes = [C.c_int64, _i32, _i32]
        L.orc_group_order.argtypes = [C.c_int64, _i32, C.c_int, _i64]
        L.orc_group_order.restype = None
        L.orc_p_adjust.argtypes = [C.c_int64, _d, C.c_int, _d]
        L.orc_test_de.argtypes = [C.c_int64, C.c_int, _d, _d, _d, C.c_int64, _d, C.c_int,
                                  C.c_double, _d, _d, _d]
        L.orc_cpu_fit.argtypes = [C.c_int64, C.c_int64, C.c_int, _i64, _i32, _d, _d, _d, _d, _d,
                                  C.c_int, C.c_int, C.c_double, _i32, C.c_int, C.c_int64,
                                  C.c_int64, _d, _d, _i32, _i32, _d, _d, _d]
        L.orc_num_threads.restype = C.c_int
        _LIB = L
    return _LIB


def _p(a, t=_d):
    return None if a is None else a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _csr(y):
    """Accept a dense (G x n) array or a (rowptr, col, val, n) tuple."""
    if isinstance(y, tuple):
        rowptr, col, val, n = y
        return (np.ascontiguousarray(rowptr, np.int64), np.ascontiguousarray(col, np.int32),
                _f64(val), int(n))
    y = np.asarray(y, dtype=np.float64)
    G, n = y.shape
    nz = y != 0
    rowptr = np.zeros(G + 1, np.int64)
    rowptr[1:] = np.cumsum(nz.sum(1))
    rows, cols = np.nonzero(nz)
    return rowptr, cols.astype(np.int32), _f64(y[rows, cols]), n


def _colmajor(X):
    X = np.asarray(X, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    return np.asfortranarray(X), X.shape[0], X.shape[1]


def digamma(x):
    return lib().orc_digamma(float(x))


def trigamma(x):
    return lib().orc_trigamma(float(x))


def two_sided_t_pvalue(t, df):
    return lib().orc_two_sided_t_pvalue(float(t), float(df))


def calculate_sf(Y, method="normed_sum"):
    rowptr, col, val, n = _csr(Y)
    G = len(rowptr) - 1
    sf = np.empty(n)
    m = {"normed_sum": SF_NORMED_SUM, "psinorm": SF_PSINORM}[method]
    st = lib().orc_calculate_sf(G, n, _p(rowptr, _i64), _p(col, _i32), _p(val), m, _p(sf))
    if st == 1:
        raise ValueError("At least one column (sample) contains all zeros, unable to compute size factor.")
    return sf


def offset_vector(off, n, sf=None):
    out = np.empty(n)
    sfa = None if sf is None else _f64(sf)
    lib().orc_offset_vector(n, float(off), _p(sfa), _p(out))
    return out


def estimate_dispersion(Y, offv):
    rowptr, col, val, n = _csr(Y)
    G = len(rowptr) - 1
    out = np.empty(G)
    offv = _f64(offv)
    lib().orc_estimate_dispersion(G, n, _p(rowptr, _i64), _p(col, _i32), _p(val), _p(offv), _p(out))
    return out


def init_beta(Y, X, offv, rough=False):
    rowptr, col, val, n = _csr(Y)
    G = len(rowptr) - 1
    Xc, n2, p = _colmajor(X)
    assert n2 == n
    out = np.empty((G, p))
    if rough:
        lib().orc_init_beta_rough(G, n, p, _p(rowptr, _i64), _p(val), _p(out))
        return out
    offv = _f64(offv)
    st = lib().orc_init_beta(G, n, p, _p(rowptr, _i64), _p(col, _i32), _p(val), _p(Xc), _p(offv),
                             _p(out))
    if st:
        raise np.linalg.LinAlgError("design matrix is rank deficient")
    return out


def beta_fit(y, X, beta0, offv, k, max_iter=200, eps=1e-3):
    Xc, n, p = _colmajor(X)
    b = _f64(beta0).copy()
    y = _f64(y)
    offv = _f64(offv)
    it = lib().orc_beta_fit(n, p, _p(y), _p(Xc), _p(b), _p(offv), float(k), int(max_iter), float(eps))
    return b, it


def mom_dispersion(y, X, beta, sf):
    Xc, n, p = _colmajor(X)
    return lib().orc_mom_dispersion(n, p, _p(_f64(y)), _p(Xc), _p(_f64(beta)), _p(_f64(sf)))


def fit_dispersion(beta, X, y, offv, max_iter=200, cr=True):
    Xc, n, p = _colmajor(X)
    it = C.c_int(0)
    th = lib().orc_fit_dispersion(n, p, _p(_f64(y)), _p(Xc), _p(_f64(beta)), _p(_f64(offv)),
                                  int(max_iter), int(bool(cr)), C.byref(it))
    return th, it.value


def gauss_hermite(m):
    """Gauss-Hermite nodes and weights (weight exp(-x^2)) of order m."""
    x = np.zeros(m)
    w = np.zeros(m)
    lib().orc_gauss_hermite(int(m), _p(x), _p(w))
    return x, w


def h_log_gh(p, s, t, m=32, max_newton=8, tol=1e-12):
    """H_log_gh_cpp (src/new_overdispersion.cpp:129-141)."""
    return lib().orc_h_log_gh(float(p), float(s), float(t), int(m), int(max_newton), float(tol))


def fit_overdispersion_new(y, X, beta, offv, max_iter=200, eps=1e-3, newton_max=16):
    """fit_overdispersion_cppp (src/new_overdispersion.cpp:195-481) for one
    gene; returns (kappa, kappa_iters, converged, err)."""
    Xc, n, p = _colmajor(X)
    it, cv, er = C.c_int(0), C.c_int(0), C.c_int(0)
    k = lib().orc_fit_overdispersion_new(n, p, _p(_f64(y)), _p(Xc), _p(_f64(beta)), _p(_f64(offv)),
                                         int(max_iter), float(eps), int(newton_max), C.byref(it),
                                         C.byref(cv), C.byref(er))
    return k, it.value, cv.value, er.value


def nb_score(y, mu, X, log_theta, cr=True):
    Xc, n, p = _colmajor(X)
    return lib().orc_score_dense(n, p, _p(_f64(y)), _p(_f64(mu)), _p(Xc), float(log_theta), int(cr))


def nb_deriv_score(y, mu, X, log_theta, cr=True):
    Xc, n, p = _colmajor(X)
    return lib().orc_deriv_score_dense(n, p, _p(_f64(y)), _p(_f64(mu)), _p(Xc), float(log_theta),
                                       int(cr))


def nb_loglik(y, mu, X, log_theta, cr=True):
    Xc, n, p = _colmajor(X)
    return lib().orc_loglik_dense(n, p, _p(_f64(y)), _p(_f64(mu)), _p(Xc), float(log_theta), int(cr))


def compute_hessian(beta, overdispersion, y, X, sf):
    Xc, n, p = _colmajor(X)
    out = np.empty((p, p), order="F")
    lib().orc_compute_hessian(n, p, _p(_f64(beta)), float(overdispersion), _p(_f64(y)), _p(Xc),
                              _p(_f64(sf)), _p(out))
    return np.array(out)


def compute_scores(X, y, beta, overdispersion, sf):
    Xc, n, p = _colmajor(X)
    out = np.empty((n, p), order="F")
    lib().orc_compute_scores(n, p, _p(Xc), _p(_f64(y)), _p(_f64(beta)), float(overdispersion),
                             _p(_f64(sf)), _p(out))
    return np.array(out)


def clustered_meat_fast(X, y, beta, overdispersion, sf, ends):
    Xc, n, p = _colmajor(X)
    ends = np.ascontiguousarray(ends, np.int32)
    out = np.empty((p, p), order="F")
    lib().orc_clustered_meat_fast(n, p, _p(Xc), _p(_f64(y)), _p(_f64(beta)), float(overdispersion),
                                  _p(_f64(sf)), _p(ends, _i32), len(ends), _p(out))
    return np.array(out)


def clustered_meat(X, y, beta, overdispersion, sf, clusters):
    Xc, n, p = _colmajor(X)
    cl = np.ascontiguousarray(clusters, np.int32)
    out = np.empty((p, p), order="F")
    lib().orc_clustered_meat(n, p, _p(Xc), _p(_f64(y)), _p(_f64(beta)), float(overdispersion),
                             _p(_f64(sf)), _p(cl, _i32), _p(out))
    return np.array(out)


def meat(X, y, beta, overdispersion, sf):
    Xc, n, p = _colmajor(X)
    out = np.empty((p, p), order="F")
    lib().orc_meat(n, p, _p(Xc), _p(_f64(y)), _p(_f64(beta)), float(overdispersion), _p(_f64(sf)),
                   _p(out))
    return np.array(out)


def factor_first_appearance(clusters):
    cl = np.ascontiguousarray(clusters, np.int64)
    lev = np.empty(len(cl), np.int32)
    nl = lib().orc_factor_first_appearance(len(cl), _p(cl, _i64), _p(lev, _i32))
    return lev, nl


def cluster_blocks(levels):
    lev = np.ascontiguousarray(levels, np.int32)
    ends = np.empty(max(len(lev), 1), np.int32)
    nb = lib().orc_cluster_blocks(len(lev), _p(lev, _i32), _p(ends, _i32))
    if nb < 0:
        raise ValueError("Input data should be grouped in blocks of patients.")
    return ends[:nb].copy()


def group_order(levels, nlev):
    lev = np.ascontiguousarray(levels, np.int32)
    out = np.empty(len(lev), np.int64)
    lib().orc_group_order(len(lev), _p(lev, _i32), int(nlev), _p(out, _i64))
    return out


def p_adjust(p, method="BH"):
    p = _f64(p)
    out = np.empty_like(p)
    lib().orc_p_adjust(len(p), _p(p), ADJ[method], _p(out))
    return out


def test_de(beta, bread, sandwich, nsamples, contrast, method="BH", max_lfc=10.0):
    beta = _f64(beta)
    G, p = beta.shape
    br = _f64(bread).reshape(G, p, p)
    br = np.ascontiguousarray(np.transpose(br, (0, 2, 1)))  # to column-major per gene
    sw = None
    if sandwich is not None:
        sw = np.ascontiguousarray(np.transpose(_f64(sandwich).reshape(G, p, p), (0, 2, 1)))
    c = _f64(contrast)
    pv, pa, lf = np.empty(G), np.empty(G), np.empty(G)
    lib().orc_test_de(G, p, _p(beta), _p(br), _p(sw), int(nsamples), _p(c), ADJ[method],
                      float(max_lfc), _p(pv), _p(pa), _p(lf))
    return pv, pa, lf


def cpu_fit(Y, X, offv, theta0, beta0, overdispersion=OD_MOM, max_iter=200, tolerance=1e-3,
            ends=None, genes=None, theta_mom=False):
    """Restates cpu_fit (R/main.R:375-523).  Matrices per gene come back as
    (G, p, p) arrays in the usual row/column sense.  ``genes`` = (begin, end)
    restricts the work to a gene range (other rows are left NaN)."""
    rowptr, col, val, n = _csr(Y)
    G = len(rowptr) - 1
    Xc, n2, p = _colmajor(X)
    assert n2 == n
    g0, g1 = (0, G) if genes is None else genes
    beta = np.full((G, p), np.nan)
    theta = np.full(G, np.nan)
    iters = np.zeros(G, np.int32)
    titers = np.zeros(G, np.int32)
    bread = np.full((G, p, p), np.nan)
    sw = np.full((G, p, p), np.nan) if ends is not None else None
    tm = np.full(G, np.nan) if theta_mom else None
    e = None if ends is None else np.ascontiguousarray(ends, np.int32)
    lib().orc_cpu_fit(G, n, p, _p(rowptr, _i64), _p(col, _i32), _p(val), _p(Xc), _p(_f64(offv)),
                      _p(_f64(theta0)), _p(_f64(beta0)), int(overdispersion), int(max_iter),
                      float(tolerance), _p(e, _i32), 0 if e is None else len(e), int(g0), int(g1),
                      _p(beta), _p(theta), _p(iters, _i32), _p(titers, _i32), _p(bread),
                      _p(sw), _p(tm))
    # per-gene matrices were written column-major; transpose to row-major view
    bread = np.transpose(bread, (0, 2, 1)).copy()
    if sw is not None:
        sw = np.transpose(sw, (0, 2, 1)).copy()
    return dict(beta=beta, theta=theta, iters=iters, theta_iters=titers, bread=bread,
                sandwich=sw, theta_mom=tm)


def num_threads():
    return lib().orc_num_threads()
