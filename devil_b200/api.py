"""Python mirror of devil's R surface for the NB GLM path.

``fit_devil`` / ``test_de`` / ``group_data`` and the single-step helpers take
the same arguments, with the same meaning and error messages, as the R
functions they mirror (R/main.R:164-273, R/test.R:85-134,
R/group_data.R:38-69, R/size_factors.R, R/overdispersion.R, R/beta.R,
src/*.cpp).  Every computation runs through libdevil_b200.so on a GPU;
there is no CPU path.

Matrices follow R's orientation: the count matrix is genes x cells, the
design matrix cells x features.  Per-gene p x p matrices come back as a
(G, p, p) array.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

_ADJ = {"BH": L.ADJ_BH, "fdr": L.ADJ_BH, "bonferroni": L.ADJ_BONFERRONI, "holm": L.ADJ_HOLM,
        "hochberg": L.ADJ_HOCHBERG, "BY": L.ADJ_BY, "hommel": L.ADJ_HOMMEL, "none": L.ADJ_NONE}


def _adjust_code(method):
    """stats::p.adjust's method argument (match.arg over p.adjust.methods)."""
    if method not in _ADJ:
        raise ValueError("'arg' should be one of \u201cholm\u201d, \u201chochberg\u201d, "
                         "\u201chommel\u201d, \u201cbonferroni\u201d, \u201cBH\u201d, "
                         "\u201cBY\u201d, \u201cfdr\u201d, \u201cnone\u201d")
    return _ADJ[method]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ----------------------------------------------------------------------
# count matrix marshalling
# ----------------------------------------------------------------------
class _CountsHold:
    """Keeps the host arrays of a devil_counts alive."""

    def __init__(self, x):
        self.keep = []
        self.s = L.Counts()
        s = self.s
        try:
            import scipy.sparse as sp
        except Exception:  # pragma: no cover
            sp = None
        if sp is not None and sp.issparse(x):
            if x.format == "csc":
                x = x.copy()
                x.sort_indices()
                G, n = x.shape
                ptr = np.ascontiguousarray(x.indptr, np.int64)
                idx = np.ascontiguousarray(x.indices, np.int32)
                val = np.ascontiguousarray(x.data, np.float64)
                s.format = L.COUNTS_CSC_F64
            else:
                x = x.tocsr()
                x.sort_indices()
                G, n = x.shape
                ptr = np.ascontiguousarray(x.indptr, np.int64)
                idx = np.ascontiguousarray(x.indices, np.int32)
                data = x.data
                if (np.issubdtype(data.dtype, np.integer) and data.size
                        and data.min() >= 0 and data.max() <= 65535):
                    val = np.ascontiguousarray(data, np.uint16)
                    s.format = L.COUNTS_CSR_U16
                else:
                    val = np.ascontiguousarray(data, np.float32)
                    s.format = L.COUNTS_CSR_F32
            s.n_genes, s.n_cells, s.nnz = G, n, int(ptr[-1])
            self.keep += [ptr, idx, val]
            s.values, s.ptr, s.idx = _ptr(val), _ptr(ptr), _ptr(idx)
            self.shape = (G, n)
            return
        if isinstance(x, tuple):  # (rowptr, col, val, n_cells): gene-major CSR
            rowptr, col, val, n = x
            ptr = np.ascontiguousarray(rowptr, np.int64)
            idx = np.ascontiguousarray(col, np.int32)
            if np.asarray(val).dtype == np.uint16:
                v = np.ascontiguousarray(val, np.uint16)
                s.format = L.COUNTS_CSR_U16
            else:
                v = np.ascontiguousarray(val, np.float32)
                s.format = L.COUNTS_CSR_F32
            s.n_genes, s.n_cells, s.nnz = len(ptr) - 1, int(n), int(ptr[-1])
            self.keep += [ptr, idx, v]
            s.values, s.ptr, s.idx = _ptr(v), _ptr(ptr), _ptr(idx)
            self.shape = (len(ptr) - 1, int(n))
            return
        a = np.asarray(x)
        if a.ndim != 2:
            raise ValueError("'x' must be a matrix (genes x cells)")
        G, n = a.shape
        if a.flags.f_contiguous and not a.flags.c_contiguous:
            a = np.asfortranarray(a, dtype=np.float64)
            s.dense_layout = L.DENSE_CELL_MAJOR
        else:
            a = np.ascontiguousarray(a, dtype=np.float64)
            s.dense_layout = L.DENSE_GENE_MAJOR
        s.format = L.COUNTS_DENSE_F64
        s.n_genes, s.n_cells, s.nnz = G, n, 0
        self.keep.append(a)
        s.values = _ptr(a)
        self.shape = (G, n)

    @property
    def ref(self):
        return C.byref(self.s)


def _design(X, n=None):
    X = np.asarray(X, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    if n is not None and X.shape[0] != n:
        raise ValueError("nrow(design_matrix) must equal ncol(x)")
    return np.asfortranarray(X), X.shape[1]


def _gene_names(x):
    return getattr(x, "gene_names", None)


# ----------------------------------------------------------------------
# clusters (R/main.R:190-196, R/group_data.R)
# ----------------------------------------------------------------------
def _cluster_codes(clusters):
    cl = np.asarray(clusters)
    if cl.dtype.kind in "iu":
        return np.ascontiguousarray(cl, np.int64)
    _, inv = np.unique(cl, return_inverse=True)  # any labels -> integer codes
    return np.ascontiguousarray(inv, np.int64)


def cluster_blocks(clusters):
    """levels = factor(clusters, levels = unique(clusters)); error when the
    cells of a cluster are not contiguous; returns (levels, ends) with ends =
    cumsum(rle(levels)$lengths) (1-based exclusive)."""
    codes = _cluster_codes(clusters)
    n = len(codes)
    levels = np.empty(n, np.int32)
    ends = np.empty(max(n, 1), np.int32)
    nb = C.c_int(0)
    rc = L.load().devil_cluster_blocks(n, _ptr(codes), _ptr(levels), _ptr(ends), C.byref(nb))
    if rc == L.ERR_UNSORTED:
        raise ValueError("Input data should be grouped in blocks of patients. "
                         "Use the `group_data` function to group them.")
    if rc != L.OK:
        raise L.DevilError(rc, "devil_cluster_blocks failed")
    return levels, ends[:nb.value].copy()


def group_data(input_matrix, design_matrix, clusters):
    """Reorder cells so that each cluster is contiguous (R/group_data.R:38-69)."""
    X = np.asarray(design_matrix)
    shape = input_matrix.shape
    if shape[1] != X.shape[0]:
        raise ValueError("Dimension mismatch: ncol(input_matrix) must equal nrow(design_matrix)")
    if len(clusters) != shape[1]:
        raise ValueError("Dimension mismatch: length(clusters) must match the number of cells")
    codes = _cluster_codes(clusters)
    order = np.empty(len(codes), np.int64)
    rc = L.load().devil_group_order(len(codes), _ptr(codes), _ptr(order))
    if rc != L.OK:
        raise L.DevilError(rc, "devil_group_order failed")
    levels, _ = _levels_only(codes)
    return dict(input_matrix=input_matrix[:, order], design_matrix=X[order],
                clusters=levels[order].astype(np.float64))


def _levels_only(codes):
    n = len(codes)
    levels = np.empty(n, np.int32)
    ends = np.empty(max(n, 1), np.int32)
    nb = C.c_int(0)
    L.load().devil_cluster_blocks(n, _ptr(codes), _ptr(levels), _ptr(ends), C.byref(nb))
    return levels, nb.value


# ----------------------------------------------------------------------
# fit_devil (R/main.R:164-273)
# ----------------------------------------------------------------------
def _od_mode(overdispersion):
    if overdispersion is False:
        return L.OD_NONE
    if isinstance(overdispersion, str):
        if overdispersion in ("old", "MLE"):
            return L.OD_MLE
        if overdispersion == "MOM":
            return L.OD_MOM
        if overdispersion in ("new", "I"):
            return L.OD_NEW
    raise ValueError(f"Unknown overdispersion mode: {overdispersion}")


def _sf_mode(size_factors, n):
    if size_factors is None:
        return L.SF_NONE, None
    if isinstance(size_factors, str):
        if size_factors == "normed_sum":
            return L.SF_NORMED_SUM, None
        if size_factors == "psinorm":
            return L.SF_PSINORM, None
        if size_factors == "edgeR":
            raise RuntimeError('To use the "edgeR" method for size factor calculation, you need to '
                               "install the 'edgeR' package from Bioconductor.")
        raise ValueError("'arg' should be one of \"normed_sum\", \"psinorm\", \"edgeR\"")
    sf = np.ascontiguousarray(size_factors, np.float64)
    if sf.shape != (n,):
        raise ValueError("size_factors must have one value per cell")
    return L.SF_GIVEN, sf


_PRECISION = {"fp32": 0, "tc_tf32": 1, "tc_bf16x3": 2}


def _fit_opts(overdispersion, init_overdispersion, init_beta_rough, offset, sfm, sfv, max_iter,
              tolerance, compute_theta_mom, form, precision="fp32"):
    opts = L.FitOpts()
    L.load().devil_fit_opts_default(C.byref(opts))
    opts.max_iter = int(max_iter)
    opts.tolerance = float(tolerance)
    opts.overdispersion = _od_mode(overdispersion)
    opts.init_beta_rough = int(bool(init_beta_rough))
    opts.size_factors = sfm
    opts.size_factor_values = _ptr(sfv)
    opts.offset = float(offset)
    if init_overdispersion is not None:
        opts.has_init_overdispersion = 1
        opts.init_overdispersion = float(init_overdispersion)
    opts.compute_theta_mom = int(bool(compute_theta_mom))
    opts.form = L.FORM_PLAIN if form == "plain" else L.FORM_CHOSEN
    if precision not in _PRECISION:
        raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
    opts.precision = _PRECISION[precision]
    return opts


class _FitSlots:
    """Host inputs and output arrays of one fit (kept alive for the call)."""

    def __init__(self, x, design_matrix, clusters, compute_theta_mom):
        self.x = x
        self.design_matrix = design_matrix
        self.counts = _CountsHold(x)
        G, n = self.counts.shape
        self.G, self.n = G, n
        self.Xf, self.p = _design(design_matrix, n)
        p = self.p
        self.ends = None
        if clusters is not None:
            if len(clusters) != n:
                raise ValueError("clusters must have one entry per cell")
            _, self.ends = cluster_blocks(clusters)
        self.beta = np.empty((G, p))
        self.theta = np.empty(G)
        self.iters = np.empty(G, np.int32)
        self.titers = np.empty(G, np.int32)
        self.bread = np.empty((G, p, p))
        self.sw = np.empty((G, p, p)) if self.ends is not None else None
        self.tm = np.empty(G) if compute_theta_mom else None
        self.status = np.empty(G, np.int32)
        self.sfo = np.empty(n)
        self.offo = np.empty(n)
        self.meat = np.empty((G, p, p)) if self.ends is not None else None
        self.res = L.FitResult(_ptr(self.beta), _ptr(self.theta), _ptr(self.iters),
                               _ptr(self.titers), _ptr(self.bread), _ptr(self.sw), _ptr(self.tm),
                               _ptr(self.status), _ptr(self.sfo), _ptr(self.offo),
                               _ptr(self.meat))

    def result(self, size_factors, max_iter, tolerance):
        # per-gene matrices are column-major p x p; present them as [g, i, j]
        bread = np.ascontiguousarray(np.transpose(self.bread, (0, 2, 1)))
        sw = meat = None
        if self.sw is not None:
            sw = np.ascontiguousarray(np.transpose(self.sw, (0, 2, 1)))
            meat = np.ascontiguousarray(np.transpose(self.meat, (0, 2, 1)))
        th_it = self.titers.astype(np.float64)
        th_it[self.titers == L.NA_INT] = np.nan
        return dict(
            beta=self.beta,
            beta_sandwiches_null=bread,
            beta_sandwiches=sw,
            overdispersion=self.theta,
            iterations=dict(beta_iters=self.iters, theta_iters=th_it),
            size_factors=self.sfo if size_factors is not None else np.ones(self.n),
            offset_vector=self.offo,
            design_matrix=np.asarray(self.design_matrix),
            input_matrix=self.x,
            input_parameters=dict(max_iter=max_iter, tolerance=tolerance),
            status=self.status,
            theta_mom=self.tm,
            meat=meat,
        )


def fit_devil(x, design_matrix, clusters=None, overdispersion="MOM", init_overdispersion=None,
              init_beta_rough=False, offset=0.0, size_factors=None, verbose=False, max_iter=200,
              tolerance=1e-3, CUDA=True, batch_size=1024, form="chosen", compute_theta_mom=False,
              device=0, precision="fp32"):
    """Fit the per-gene NB GLM (fit_devil, R/main.R:164-273) on the GPU.

    ``CUDA`` and ``batch_size`` are accepted for signature compatibility;
    the B200 path always runs on the GPU and schedules genes itself.
    ``form`` = "chosen" (default) or "plain" (the per-cell, one gene per
    block comparison form).  ``precision`` = "fp32" (default: FP32 FMAs on
    the CUDA cores) or "tc_tf32" (the IRLS and MLE Hessian contractions as
    tcgen05 MMAs on split-TF32 operands, p <= 4); "tc_bf16x3" is rejected."""
    del verbose, CUDA, batch_size
    f = _FitSlots(x, design_matrix, clusters, compute_theta_mom)
    sfm, sfv = _sf_mode(size_factors, f.n)
    opts = _fit_opts(overdispersion, init_overdispersion, init_beta_rough, offset, sfm, sfv,
                     max_iter, tolerance, compute_theta_mom, form, precision)
    ctx = L.context(device)
    rc = L.load().devil_fit(ctx.h, f.counts.ref, _ptr(f.Xf), f.p, _ptr(f.ends),
                            0 if f.ends is None else len(f.ends), C.byref(opts), C.byref(f.res))
    if rc == L.ERR_ZERO_COLUMN:
        raise ValueError(L.load().devil_last_error(ctx.h).decode())
    ctx.check(rc)
    return f.result(size_factors, max_iter, tolerance)


def fit_devil_batch(problems, overdispersion="MOM", init_overdispersion=None,
                    init_beta_rough=False, offset=0.0, size_factors=None, max_iter=200,
                    tolerance=1e-3, form="chosen", compute_theta_mom=False, workers=4, device=0,
                    precision="fp32"):
    """fit_devil for many independent problems in one call (devil_fit_batch).

    ``problems`` is a sequence of (x, design_matrix) or (x, design_matrix,
    clusters); the options apply to every problem (size_factors: None or a
    method name).  The problems run on ``workers`` concurrent GPU streams.
    Returns one fit dict per problem, as fit_devil."""
    if size_factors is not None and not isinstance(size_factors, str):
        raise ValueError("fit_devil_batch takes size_factors as None or a method name")
    slots = []
    for pr in problems:
        x, X = pr[0], pr[1]
        cl = pr[2] if len(pr) > 2 else None
        slots.append(_FitSlots(x, X, cl, compute_theta_mom))
    sfm, _ = _sf_mode(size_factors, 1)
    opts = _fit_opts(overdispersion, init_overdispersion, init_beta_rough, offset, sfm, None,
                     max_iter, tolerance, compute_theta_mom, form, precision)
    n = len(slots)
    arr = (L.Problem * max(n, 1))()
    res = (L.FitResult * max(n, 1))()
    for i, f in enumerate(slots):
        arr[i].counts = f.counts.s
        arr[i].X = _ptr(f.Xf)
        arr[i].p = f.p
        arr[i].cluster_ends = _ptr(f.ends)
        arr[i].n_clusters = 0 if f.ends is None else len(f.ends)
        res[i] = f.res
    ctx = L.context(device)
    ctx.check(L.load().devil_fit_batch(ctx.h, n, arr, C.byref(opts), res, int(workers)))
    return [f.result(size_factors, max_iter, tolerance) for f in slots]


# ----------------------------------------------------------------------
# test_de (R/test.R:85-134)
# ----------------------------------------------------------------------
def test_de(devil_fit, contrast, clusters=None, pval_adjust_method="BH", max_lfc=10.0, device=0):
    """Wald/t test of a contrast per gene with multiple-testing adjustment.

    Returns a dict of arrays name / pval / adj_pval / lfc (log2, clipped)."""
    del clusters  # accepted but unused, as in the reference (R/test.R:85-134)
    if "beta_sandwiches_null" not in devil_fit:
        raise ValueError("The fit object was created with an older version of devil and is no "
                         "longer supported. Please re-fit your model with the current version of "
                         "fit_devil().")
    adj = _adjust_code(pval_adjust_method)
    beta = np.ascontiguousarray(devil_fit["beta"], np.float64)
    G, p = beta.shape
    c = np.ascontiguousarray(np.asarray(contrast, np.float64).reshape(-1))
    if c.shape[0] != p:
        raise ValueError("contrast length must equal the number of coefficients")
    bread = _stack_mats(devil_fit["beta_sandwiches_null"], G, p)
    sw = devil_fit.get("beta_sandwiches")
    sw = None if sw is None else _stack_mats(sw, G, p)
    nsamples = np.asarray(devil_fit["design_matrix"]).shape[0]
    pv, pa, lf = np.empty(G), np.empty(G), np.empty(G)
    ctx = L.context(device)
    ctx.check(L.load().devil_test_de(ctx.h, G, p, _ptr(beta), _ptr(bread), _ptr(sw), nsamples,
                                     _ptr(c), adj, float(max_lfc), _ptr(pv),
                                     _ptr(pa), _ptr(lf)))
    names = devil_fit.get("gene_names")
    if names is None:
        names = np.array([f"gene{i + 1}" for i in range(G)])
    return dict(name=names, pval=pv, adj_pval=pa, lfc=lf)


def _stack_mats(mats, G, p):
    """(G, p, p) array or list of p x p (None allowed only when all None)
    -> column-major per gene, contiguous."""
    if isinstance(mats, (list, tuple)):
        if all(m is None for m in mats):
            return None
        mats = np.stack([np.asarray(m, np.float64) for m in mats])
    a = np.asarray(mats, np.float64).reshape(G, p, p)
    return np.ascontiguousarray(np.transpose(a, (0, 2, 1)))


def p_adjust(p, method="BH", device=0):
    """stats::p.adjust on the GPU (NaN = NA)."""
    p = np.ascontiguousarray(p, np.float64)
    out = np.empty_like(p)
    ctx = L.context(device)
    ctx.check(L.load().devil_p_adjust(ctx.h, len(p), _ptr(p), _adjust_code(method), _ptr(out)))
    return out


# ----------------------------------------------------------------------
# single steps
# ----------------------------------------------------------------------
def calculate_sf(Y, method="normed_sum", verbose=False, device=0):
    """calculate_sf (R/size_factors.R:37-63)."""
    del verbose
    if method not in ("normed_sum", "psinorm", "edgeR"):
        raise ValueError("'arg' should be one of \"normed_sum\", \"psinorm\", \"edgeR\"")
    if method == "edgeR":
        raise RuntimeError('To use the "edgeR" method for size factor calculation, you need to '
                           "install the 'edgeR' package from Bioconductor.")
    counts = _CountsHold(Y)
    G, n = counts.shape
    sf = np.empty(n)
    ctx = L.context(device)
    rc = L.load().devil_calculate_sf(ctx.h, counts.ref,
                                     L.SF_NORMED_SUM if method == "normed_sum" else L.SF_PSINORM,
                                     _ptr(sf))
    if rc == L.ERR_ZERO_COLUMN:
        raise ValueError("At least one column (sample) contains all zeros, unable to compute size "
                         "factor. Please filter out empty samples from input matrix.")
    ctx.check(rc)
    return sf


def normed_sum_sf(Y, device=0):
    return calculate_sf(Y, "normed_sum", device=device)


def psinorm_sf(Y, device=0):
    return calculate_sf(Y, "psinorm", device=device)


def compute_offset_vector(off, Y, size_factors=None):
    """compute_offset_vector (R/size_factors.R:172-184): off + log(sf).
    Host arithmetic on an n-vector; the device path computes the same inside
    fit_devil."""
    n = Y.shape[1]
    v = np.full(n, float(off))
    if size_factors is not None:
        v = v + np.log(np.asarray(size_factors, np.float64))
    return v


def estimate_dispersion(count_matrix, offset_vector, device=0):
    """estimate_dispersion (R/overdispersion.R:129-135)."""
    counts = _CountsHold(count_matrix)
    G, n = counts.shape
    off = np.ascontiguousarray(offset_vector, np.float64)
    out = np.empty(G)
    ctx = L.context(device)
    ctx.check(L.load().devil_estimate_dispersion(ctx.h, counts.ref, _ptr(off), _ptr(out)))
    return out


def init_beta(y, design_matrix, offset_vector, rough=False, device=0):
    """init_beta (R/beta.R:13-20); rough=True gives (log1p(rowMeans), 0...)."""
    counts = _CountsHold(y)
    G, n = counts.shape
    Xf, p = _design(design_matrix, n)
    off = np.ascontiguousarray(offset_vector, np.float64)
    out = np.empty((G, p))
    ctx = L.context(device)
    rc = L.load().devil_init_beta(ctx.h, counts.ref, _ptr(Xf), p, _ptr(off), int(rough), _ptr(out))
    if rc == L.ERR_SINGULAR:
        raise np.linalg.LinAlgError("design matrix is rank deficient")
    ctx.check(rc)
    return out


def beta_fit(Y, design_matrix, beta0, offset_vector, theta0, max_iter=200, eps=1e-3,
             form="chosen", device=0):
    """beta_fit (src/beta.cpp:25-51) for all genes; k = theta0 per gene."""
    counts = _CountsHold(Y)
    G, n = counts.shape
    Xf, p = _design(design_matrix, n)
    b0 = np.ascontiguousarray(beta0, np.float64).reshape(G, p)
    off = np.ascontiguousarray(offset_vector, np.float64)
    th = np.ascontiguousarray(theta0, np.float64)
    out = np.empty((G, p))
    it = np.empty(G, np.int32)
    ctx = L.context(device)
    ctx.check(L.load().devil_beta_fit(ctx.h, counts.ref, _ptr(Xf), p, _ptr(b0), _ptr(off), _ptr(th),
                                      int(max_iter), float(eps),
                                      L.FORM_PLAIN if form == "plain" else L.FORM_CHOSEN,
                                      _ptr(out), _ptr(it)))
    return out, it


def estimate_mom_dispersion(count_matrix, design_matrix, beta_matrix, sf, device=0):
    """estimate_mom_dispersion_cpp (src/mom_overdispersion.cpp:6-56)."""
    counts = _CountsHold(count_matrix)
    G, n = counts.shape
    Xf, p = _design(design_matrix, n)
    b = np.ascontiguousarray(beta_matrix, np.float64).reshape(G, p)
    s = np.ascontiguousarray(sf, np.float64)
    out = np.empty(G)
    ctx = L.context(device)
    ctx.check(L.load().devil_estimate_mom_dispersion(ctx.h, counts.ref, _ptr(Xf), p, _ptr(b),
                                                     _ptr(s), _ptr(out)))
    return out


def fit_overdispersion_new(y, X, mu_beta, off, max_iter=200, eps_theta=1e-3, device=0):
    """fit_overdispersion_cppp (src/new_overdispersion.cpp:195-481), the
    overdispersion = "new" / "I" method, for every gene (rows of y).
    Returns (kappa, kappa_iters).  Raises DevilError (status ERR_NUMERIC,
    with the reference's message) where the reference would stop()."""
    counts = _CountsHold(y)
    G, n = counts.shape
    Xf, p = _design(X, n)
    b = np.ascontiguousarray(mu_beta, np.float64).reshape(G, p)
    o = np.ascontiguousarray(off, np.float64)
    out = np.empty(G)
    it = np.empty(G, np.int32)
    ctx = L.context(device)
    ctx.check(L.load().devil_fit_overdispersion_new(ctx.h, counts.ref, _ptr(Xf), p, _ptr(b), _ptr(o),
                                                    int(max_iter), float(eps_theta), _ptr(out),
                                                    _ptr(it)))
    return out, it


def fit_dispersion(beta, model_matrix, y, offset_vector, tolerance=1e-3, max_iter=200,
                   do_cox_reid_adjustment=True, device=0):
    """fit_dispersion (R/overdispersion.R:25-115) for every gene (rows of y)."""
    del tolerance
    counts = _CountsHold(y)
    G, n = counts.shape
    Xf, p = _design(model_matrix, n)
    b = np.ascontiguousarray(beta, np.float64).reshape(G, p)
    off = np.ascontiguousarray(offset_vector, np.float64)
    out = np.empty(G)
    it = np.empty(G, np.int32)
    ctx = L.context(device)
    ctx.check(L.load().devil_fit_dispersion(ctx.h, counts.ref, _ptr(Xf), p, _ptr(b), _ptr(off),
                                            int(max_iter), int(bool(do_cox_reid_adjustment)),
                                            _ptr(out), _ptr(it)))
    return out, it


def compute_hessian(beta, overdispersion, y, design_matrix, size_factors, device=0):
    """compute_hessian (src/variance.cpp:22-47): the bread per gene."""
    counts = _CountsHold(y)
    G, n = counts.shape
    Xf, p = _design(design_matrix, n)
    b = np.ascontiguousarray(beta, np.float64).reshape(G, p)
    th = np.ascontiguousarray(np.broadcast_to(overdispersion, (G,)), np.float64)
    sf = np.ascontiguousarray(size_factors, np.float64)
    out = np.empty((G, p, p))
    ctx = L.context(device)
    ctx.check(L.load().devil_compute_hessian(ctx.h, counts.ref, _ptr(Xf), p, _ptr(b), _ptr(th),
                                             _ptr(sf), _ptr(out)))
    return np.ascontiguousarray(np.transpose(out, (0, 2, 1)))


def compute_clustered_meat(design_matrix, y, beta, overdispersion, size_factors,
                           cluster_blocks_indexes, device=0):
    """compute_clustered_meat_fast (src/variance.cpp:186-228) per gene."""
    counts = _CountsHold(y)
    G, n = counts.shape
    Xf, p = _design(design_matrix, n)
    b = np.ascontiguousarray(beta, np.float64).reshape(G, p)
    th = np.ascontiguousarray(np.broadcast_to(overdispersion, (G,)), np.float64)
    sf = np.ascontiguousarray(size_factors, np.float64)
    ends = np.ascontiguousarray(cluster_blocks_indexes, np.int32)
    out = np.empty((G, p, p))
    ctx = L.context(device)
    ctx.check(L.load().devil_compute_clustered_meat(ctx.h, counts.ref, _ptr(Xf), p, _ptr(b),
                                                    _ptr(th), _ptr(sf), _ptr(ends), len(ends),
                                                    _ptr(out)))
    return np.ascontiguousarray(np.transpose(out, (0, 2, 1)))


def compute_sandwich(design_matrix, y, beta, overdispersion, size_factors, clusters=None,
                     device=0):
    """compute_sandwich (R/variance.R:16-26), including its use of
    1/overdispersion for the bread.  Unclustered meat uses one block per cell."""
    Y = np.atleast_2d(np.asarray(y, np.float64))
    n = Y.shape[1]
    b = np.atleast_2d(np.asarray(beta, np.float64))
    th = np.atleast_1d(np.asarray(overdispersion, np.float64))
    bread = compute_hessian(b, 1.0 / th, Y, design_matrix, size_factors, device=device)
    if clusters is not None:
        levels, _ = _levels_only(_cluster_codes(clusters))
        order = np.argsort(levels, kind="stable")
        lv = levels[order]
        ends = (np.flatnonzero(np.r_[lv[1:] != lv[:-1], True]) + 1).astype(np.int32)
        meat = compute_clustered_meat(np.asarray(design_matrix)[order], Y[:, order], b, th,
                                      np.asarray(size_factors)[order], ends, device=device)
    else:
        # compute_meat (src/variance.cpp:157-178): sum_i s_i s_i' / n; every
        # cell is its own block with adj = n/(n-1) removed again
        ends = np.arange(1, n + 1, dtype=np.int32)
        meat = compute_clustered_meat(design_matrix, Y, b, th, size_factors, ends, device=device)
        meat = meat * (n - 1.0) / n
    return np.einsum("gij,gjk,gkl->gil", bread, meat, bread) * n


def nb_adjoint(y, eta, log_theta, device=0):
    """Per-cell NB log-likelihood l_c and its adjoint (dl/deta, dl/dlog theta)."""
    y = np.ascontiguousarray(y, np.float64)
    e = np.ascontiguousarray(eta, np.float64)
    n = len(y)
    ll, de, dt = np.empty(n), np.empty(n), np.empty(n)
    ctx = L.context(device)
    ctx.check(L.load().devil_nb_adjoint(ctx.h, n, _ptr(y), _ptr(e), float(log_theta), _ptr(ll),
                                        _ptr(de), _ptr(dt)))
    return ll, de, dt
