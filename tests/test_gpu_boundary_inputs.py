"""The inputs an R caller hands the library, through the C ABI:

* a dgCMatrix (cell-compressed, DEVIL_COUNTS_CSC_F64) -- the format
  fit_devil receives for sparse single-cell data -- must fit exactly as the
  same counts in gene-major CSR;
* the call sequence of the Rcpp shim's beta_fit_gpu (devil_b200/rcpp,
  replacing src/beta.cpp:83-161): dense counts in R's column-major genes x
  cells layout, offsets turned into size factors sf = exp(off), the rough
  beta initialisation (log1p of the gene mean, cuda/src/batch.cpp:352-356),
  MOM theta, cluster ends for the meat; its outputs laid out as gpu_fit
  (R/main.R:312-328) reads them: hessian_inv p^2 x G column-major per gene,
  sandwich = H M H n.  Checked against the oracle run with the same options.
"""
import ctypes as C

import numpy as np
import pytest

from devil_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_dgcmatrix_fits_like_csr(dv):
    sp = pytest.importorskip("scipy.sparse")
    P = synthetic.make("plain_sparse", seed=31, G=120, n=3000)
    csr = sp.csr_matrix((P.val.astype(np.float64), P.col, P.rowptr), shape=(P.G, P.n))
    a = dv.fit_devil((P.rowptr, P.col, P.val, P.n), P.X, overdispersion="MLE",
                     size_factors="normed_sum")
    b = dv.fit_devil(csr.tocsc(), P.X, overdispersion="MLE", size_factors="normed_sum")
    np.testing.assert_array_equal(a["size_factors"], b["size_factors"])
    np.testing.assert_array_equal(a["iterations"]["beta_iters"], b["iterations"]["beta_iters"])
    np.testing.assert_array_equal(a["beta"], b["beta"])
    np.testing.assert_array_equal(a["overdispersion"], b["overdispersion"])
    np.testing.assert_array_equal(a["beta_sandwiches_null"], b["beta_sandwiches_null"])
    # the same through the single-step entry points
    np.testing.assert_array_equal(dv.calculate_sf(csr.tocsc()),
                                  dv.calculate_sf((P.rowptr, P.col, P.val, P.n)))


def _shim_beta_fit_gpu(dv, y_gxn, X, off, max_iter, eps, cluster_ends):
    """The C-ABI calls of devil_b200_rcpp.cpp: beta_fit_gpu, in Python."""
    from devil_b200 import _lib as L

    lib = L.load()
    ctx = L.context(0)
    G, n = y_gxn.shape
    p = X.shape[1]
    yc = np.asfortranarray(y_gxn, np.float64)       # R NumericMatrix: column-major G x n
    Xc = np.asfortranarray(X, np.float64)
    counts = L.Counts()
    counts.format = L.COUNTS_DENSE_F64
    counts.dense_layout = 1                          # DEVIL_DENSE_CELL_MAJOR
    counts.n_genes, counts.n_cells = G, n
    counts.values = yc.ctypes.data
    o = L.FitOpts()
    lib.devil_fit_opts_default(C.byref(o))
    o.max_iter = max_iter
    o.tolerance = float(np.float32(eps))
    o.overdispersion = L.OD_MOM
    o.init_beta_rough = 1
    o.size_factors = L.SF_GIVEN
    sf = np.exp(off)
    o.size_factor_values = sf.ctypes.data
    ncl = 0 if cluster_ends is None else len(cluster_ends)
    beta = np.empty((p, G), order="F")               # NumericMatrix beta(p, G)
    theta, bread = np.empty(G), np.empty(p * p * G)
    meat = np.empty(p * p * G) if ncl else None
    sandwich = np.empty(p * p * G) if ncl else None
    it = np.empty(G, np.int32)
    r = L.FitResult(beta.ctypes.data, theta.ctypes.data, it.ctypes.data, None, bread.ctypes.data,
                    None if sandwich is None else sandwich.ctypes.data, None, None, None, None,
                    None if meat is None else meat.ctypes.data)
    ends = None if cluster_ends is None else np.ascontiguousarray(cluster_ends, np.int32)
    ctx.check(lib.devil_fit(ctx.h, C.byref(counts), Xc.ctypes.data, p,
                            None if ends is None else ends.ctypes.data, ncl, C.byref(o), C.byref(r)))
    out = {"mu_beta": beta.T.copy(), "theta": theta, "iter": it,
           "hessian_inv": bread.reshape(G, p * p).T}  # p^2 x G, column-major per gene
    if ncl:
        out["meat"] = meat.reshape(G, p * p).T
        out["sandwich"] = sandwich
    return out


def test_beta_fit_gpu_shim_mapping(dv, orc):
    P = synthetic.make("clustered", seed=37, G=60, n=2500)
    _, ends = dv.cluster_blocks(P.clusters)
    Y = P.dense()
    off = np.log(P.sf_true)
    res = _shim_beta_fit_gpu(dv, Y, P.X, off, 200, 1e-3, ends)
    # the oracle with the same options: rough init, theta_0 from
    # estimate_dispersion, MOM theta, offsets as given
    Yc = P.csr_f64()
    th0 = orc.estimate_dispersion(Yc, off)
    b0 = orc.init_beta(Yc, P.X, off, rough=True)
    ref = orc.cpu_fit(Yc, P.X, off, th0, b0, orc.OD_MOM, 200, 1e-3, ends=ends)
    same = res["iter"] == ref["iters"]
    assert same.mean() >= 0.97
    conv = same & (ref["iters"] < 200)
    assert np.abs(res["mu_beta"] - ref["beta"])[conv].max() <= 1e-5
    ok = conv & (ref["theta"] > 1e-3)
    r = np.abs(res["theta"] - ref["theta"])[ok] / ref["theta"][ok]
    assert r.max() <= 1e-4
    p = P.p
    # gpu_fit's assembly: matrix(hessian_inv[, g], p, p) and (H M H) * n
    for g in np.flatnonzero(conv)[:10]:
        H = res["hessian_inv"][:, g].reshape(p, p, order="F")
        M = res["meat"][:, g].reshape(p, p, order="F")
        np.testing.assert_allclose(H, ref["bread"][g], rtol=1e-4,
                                   atol=1e-4 * np.abs(np.diag(ref["bread"][g])).max())
        S = res["sandwich"].reshape(P.G, p, p)[g].T    # column-major per gene
        np.testing.assert_allclose((H @ M @ H) * P.n, S, rtol=1e-9, atol=1e-12 * np.abs(S).max())
