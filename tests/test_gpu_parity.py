"""GPU parity: fit_devil / test_de through libdevil_b200.so against the FP64
oracle (cpu_fit, R/main.R:375-523) on the same seeded inputs.

Bars (from the path's acceptance criteria):
  * beta: |d beta| <= 1e-5 (absolute) on genes that converge in both with
    the same IRLS iteration count;
    iteration counts agree on >= 97% of genes (a gene whose max|delta|
    lands within FP32 rounding of the tolerance may take one step more or
    less; those genes differ by at most one step < tolerance);
  * theta: relative <= 1e-4 (MOM, MLE) on genes that converge in both and
    whose theta is resolvable (see _theta_mask);
  * bread: relative <= 1e-4 of the diagonal scale; clustered sandwich
    1e-3 (its meat sums residuals, see test_fit_clustered_p12);
  * p-values: relative |d log10 p| <= 1e-3.
"""
import numpy as np
import pytest

from devil_b200 import synthetic

pytestmark = pytest.mark.gpu

BETA_TOL = 1e-5
ITER_AGREE = 0.97


def oracle_fit(orc, P, od, clusters_ends=None, sf="normed_sum", max_iter=200, tol=1e-3,
               init_rough=False):
    Y = P.csr_f64()
    if sf is None:
        sfv = np.ones(P.n)
        off = orc.offset_vector(0.0, P.n, None)
    elif isinstance(sf, str):
        sfv = orc.calculate_sf(Y, sf)
        off = orc.offset_vector(0.0, P.n, sfv)
    else:
        sfv = np.asarray(sf, float)
        off = orc.offset_vector(0.0, P.n, sfv)
    th0 = orc.estimate_dispersion(Y, off)
    b0 = orc.init_beta(Y, P.X, off, rough=init_rough)
    r = orc.cpu_fit(Y, P.X, off, th0, b0, od, max_iter, tol, ends=clusters_ends, theta_mom=True)
    r.update(sf=sfv, off=off, theta0=th0, beta0=b0)
    return r


def gpu_fit(dv, P, od, clusters=None, sf="normed_sum", max_iter=200, tol=1e-3, form="chosen",
            init_rough=False, precision="fp32"):
    return dv.fit_devil((P.rowptr, P.col, P.val, P.n), P.X, clusters=clusters, overdispersion=od,
                        size_factors=sf, max_iter=max_iter, tolerance=tol, form=form,
                        compute_theta_mom=True, init_beta_rough=init_rough, precision=precision)


def check_beta(fit, ref, tol=BETA_TOL, agree=ITER_AGREE, max_iter=200):
    """|d beta| <= tol (absolute, the acceptance bar) on genes that converge
    in both with the same iteration count.  Genes stopped by max_iter have
    not converged (the bar does not apply: e.g. an intercept drifting
    towards -inf for a cell group without counts moves by ~1 per step);
    they are checked at 1e-4 relative.  Genes one step apart differ by that
    step, which is below the tolerance (1e-3)."""
    it_g = fit["iterations"]["beta_iters"]
    it_o = ref["iters"]
    same = it_g == it_o
    assert same.mean() >= agree, f"iteration counts agree on only {same.mean():.3f}"
    d = np.abs(fit["beta"] - ref["beta"])
    conv = same & (it_o < max_iter)
    if conv.any():
        g = np.flatnonzero(conv)[np.argmax(np.nanmax(d[conv], axis=1))]
        assert np.nanmax(d[conv]) <= tol, (
            f"max |dbeta| = {np.nanmax(d[conv]):.3e} at gene {g}: iters {it_o[g]}, "
            f"beta {ref['beta'][g]}, gpu {fit['beta'][g]}")
    capped = same & (it_o >= max_iter)
    if capped.any():
        rel = d[capped] / np.maximum(1.0, np.abs(ref["beta"][capped]))
        assert np.nanmax(rel) <= 10 * tol, f"max-iter genes: rel |dbeta| {np.nanmax(rel):.3e}"
    # genes off by one iteration: the extra step is below the tolerance
    if (~same).any():
        assert np.all(np.abs(it_g[~same] - it_o[~same]) <= 1)
        assert np.nanmax(d[~same] / np.maximum(1.0, np.abs(ref["beta"][~same]))) <= 10 * 1e-3
    return conv


def _theta_mask(th_ref, same):
    return same & (th_ref > 1e-3) & (th_ref < 1e3)


def check_rel(a, b, mask, tol, what):
    a, b = np.asarray(a)[mask], np.asarray(b)[mask]
    r = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    assert r.size == 0 or r.max() <= tol, f"{what}: max rel err {r.max():.3e}"


def check_mats(A, B, mask, tol, what):
    A, B = np.asarray(A)[mask], np.asarray(B)[mask]
    diag = np.sqrt(np.abs(np.einsum("gii->gi", B)))
    scale = diag[:, :, None] * diag[:, None, :]
    r = np.abs(A - B) / np.maximum(scale, 1e-300)
    assert r.size == 0 or r.max() <= tol, f"{what}: max rel err {r.max():.3e}"


def check_pvals(p_g, p_o, mask, tol=1e-3):
    ok = mask & np.isfinite(p_o) & (p_o > 1e-300) & np.isfinite(p_g) & (p_g > 0)
    lg, lo = np.log10(p_g[ok]), np.log10(p_o[ok])
    r = np.abs(lg - lo) / np.maximum(1.0, np.abs(lo))
    assert r.size == 0 or r.max() <= tol, f"log10 p rel err {r.max():.3e}"


def small_problem(cfg, seed, G, n):
    """A config at test size; the wide design with gene means LogNormal(-1, 2)
    so that a few dozen genes at a few thousand cells carry counts."""
    return synthetic.make(cfg, seed=seed, G=G, n=n, mean_loc=-1.0 if cfg == "wide" else None)


@pytest.fixture(scope="module")
def sparse_problem():
    return synthetic.make("plain_sparse", seed=11, G=300, n=6000)


@pytest.mark.parametrize("od", ["MOM", "MLE", False])
def test_fit_sparse_p4(dv, orc, sparse_problem, od):
    P = sparse_problem
    code = {"MOM": orc.OD_MOM, "MLE": orc.OD_MLE, False: orc.OD_NONE}[od]
    ref = oracle_fit(orc, P, code)
    fit = gpu_fit(dv, P, od)
    np.testing.assert_allclose(fit["size_factors"], ref["sf"], rtol=1e-12)
    np.testing.assert_allclose(fit["offset_vector"], ref["off"], rtol=0, atol=1e-12)
    same = check_beta(fit, ref)
    check_rel(fit["theta_mom"], ref["theta_mom"], _theta_mask(ref["theta_mom"], same), 1e-4,
              "theta MOM")
    if od == "MLE":
        check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4,
                  "theta MLE")
        assert np.isnan(fit["iterations"]["theta_iters"]).all()
    elif od is False:
        assert (fit["overdispersion"] == 0).all()
    check_mats(fit["beta_sandwiches_null"], ref["bread"], same & (ref["theta"] < 1e3), 1e-4, "bread")
    c = np.array([0.0, 1.0, 0.0, 0.0])
    res = dv.test_de(fit, c)
    pv, pa, lf = orc.test_de(ref["beta"], ref["bread"], None, P.n, c)
    check_pvals(res["pval"], pv, same)


def test_fit_dense_p2(dv, orc):
    P = synthetic.make("plain_small", seed=5, G=200, n=1500)
    Y = P.dense()
    ref = oracle_fit(orc, P, orc.OD_MLE)
    fit = dv.fit_devil(Y, P.X, overdispersion="MLE", size_factors="normed_sum",
                       compute_theta_mom=True)
    same = check_beta(fit, ref)
    check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta")
    res = dv.test_de(fit, [0, 1])
    pv, _, _ = orc.test_de(ref["beta"], ref["bread"], None, P.n, [0, 1])
    check_pvals(res["pval"], pv, same)


def test_fit_clustered_p12(dv, orc):
    P = synthetic.make("clustered", seed=7, G=200, n=4000)
    # 40 patients are drawn for the full config; sizes here scale with n
    levels, ends = dv.cluster_blocks(P.clusters)
    ref = oracle_fit(orc, P, orc.OD_MOM, clusters_ends=ends)
    fit = gpu_fit(dv, P, "MOM", clusters=P.clusters)
    same = check_beta(fit, ref)
    check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta")
    check_mats(fit["beta_sandwiches_null"], ref["bread"], same, 1e-4, "bread")
    # the meat is built from per-cluster sums of residuals y - mu: a relative
    # change of mu (beta agrees to ~1e-6 in eta) moves it by ~sqrt(sum mu)
    # times more; the p-value bar below is the acceptance criterion
    check_mats(fit["beta_sandwiches"], ref["sandwich"], same, 1e-3, "sandwich")
    c = np.zeros(P.p)
    c[1] = 1.0
    res = dv.test_de(fit, c)
    pv, _, _ = orc.test_de(ref["beta"], ref["bread"], ref["sandwich"], P.n, c)
    check_pvals(res["pval"], pv, same)


def test_fit_wide_p32(dv, orc):
    # gene means LogNormal(-1, 2): at n = 4000 the headline location (-3.8)
    # leaves most of 24 genes with a handful of counts
    P = synthetic.make("wide", seed=2, G=24, n=4000, mean_loc=-1.0)
    ref = oracle_fit(orc, P, orc.OD_MOM, sf=None)
    fit = gpu_fit(dv, P, "MOM", sf=None)
    same = check_beta(fit, ref)
    check_mats(fit["beta_sandwiches_null"], ref["bread"], same, 1e-4, "bread")


def test_groups_match_per_cell_form(dv):
    """The design-group engine (22 distinct design rows x 40 patients; the
    zero-count terms of each group from a Gauss rule of its offsets, the
    nonzeros from the group-ordered CSR) against the per-cell FP64 form on
    the same data: the two differ only in summation order and the rule's
    ~1e-15 quadrature error."""
    P = synthetic.make("clustered", seed=21, G=48, n=40000)
    ctx = dv.context()
    # 48 genes leave empty cells: size factors are given (the truth)
    a = gpu_fit(dv, P, "MLE", clusters=P.clusters, sf=P.sf_true)
    assert [ctx.engine(k) for k in range(4)] == ["groups"] * 4
    b = gpu_fit(dv, P, "MLE", clusters=P.clusters, sf=P.sf_true, form="plain")
    assert ctx.engine(0) == "shared"
    ia, ib = a["iterations"]["beta_iters"], b["iterations"]["beta_iters"]
    same = ia == ib
    assert same.mean() >= 0.97
    conv = same & (ib < 200)
    d = np.abs(a["beta"] - b["beta"]) / np.maximum(1.0, np.abs(b["beta"]))
    assert d[conv].max() <= 1e-7, d[conv].max()
    check_rel(a["overdispersion"], b["overdispersion"], _theta_mask(b["overdispersion"], conv),
              1e-6, "theta")
    check_mats(a["beta_sandwiches_null"], b["beta_sandwiches_null"], conv, 1e-7, "bread")
    check_mats(a["beta_sandwiches"], b["beta_sandwiches"], conv, 1e-5, "sandwich")


def test_groups_single_cell_groups(dv, orc):
    """Groups of at most ten cells per offset bin use the cells themselves
    as nodes: a two-group design at n = 300 must match the oracle."""
    P = synthetic.make("plain_small", seed=13, G=40, n=300)
    Y = (P.rowptr, P.col, P.val.astype(np.float64), P.n)
    ref = oracle_fit(orc, P, orc.OD_MLE)
    fit = dv.fit_devil(Y, P.X, overdispersion="MLE", size_factors="normed_sum",
                       compute_theta_mom=True)
    assert dv.context().engine(0) == "groups"
    same = check_beta(fit, ref)
    check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta")
    check_mats(fit["beta_sandwiches_null"], ref["bread"], same, 1e-4, "bread")


def test_plain_form_matches_oracle(dv, orc, sparse_problem):
    P = sparse_problem.subset_genes(np.arange(80))
    ref = oracle_fit(orc, P, orc.OD_MOM, sf=P.sf_true)
    fit = gpu_fit(dv, P, "MOM", form="plain", sf=P.sf_true)
    check_beta(fit, ref)


def test_rough_init_and_given_sf(dv, orc, sparse_problem):
    P = sparse_problem.subset_genes(np.arange(64))
    Y = P.csr_f64()
    sf = P.sf_true
    off = orc.offset_vector(0.0, P.n, sf)
    th0 = orc.estimate_dispersion(Y, off)
    b0 = orc.init_beta(Y, P.X, off, rough=True)
    ref = orc.cpu_fit(Y, P.X, off, th0, b0, orc.OD_MOM, 200, 1e-3)
    fit = dv.fit_devil((P.rowptr, P.col, P.val, P.n), P.X, size_factors=sf,
                       init_beta_rough=True)
    check_beta(fit, ref)


def test_single_steps(dv, orc, sparse_problem):
    Pf = sparse_problem
    for m in ("normed_sum", "psinorm"):
        np.testing.assert_allclose(dv.calculate_sf((Pf.rowptr, Pf.col, Pf.val, Pf.n), m),
                                   orc.calculate_sf(Pf.csr_f64(), m), rtol=1e-12)
    P = sparse_problem.subset_genes(np.arange(50))
    Y = P.csr_f64()
    csr = (P.rowptr, P.col, P.val, P.n)
    sf = P.sf_true
    off = orc.offset_vector(0.0, P.n, sf)
    np.testing.assert_allclose(dv.estimate_dispersion(csr, off), orc.estimate_dispersion(Y, off),
                               rtol=1e-12)
    np.testing.assert_allclose(dv.init_beta(csr, P.X, off), orc.init_beta(Y, P.X, off),
                               rtol=0, atol=1e-10)
    b = P.beta_true
    th = P.theta_true
    np.testing.assert_allclose(dv.estimate_mom_dispersion(csr, P.X, b, sf),
                               [orc.mom_dispersion(y, P.X, bb, sf) for y, bb in zip(P.dense(), b)],
                               rtol=1e-5, atol=1e-9)
    bread = dv.compute_hessian(b, th, csr, P.X, sf)
    ref = np.stack([orc.compute_hessian(bb, t, y, P.X, sf) for bb, t, y in zip(b, th, P.dense())])
    check_mats(bread, ref, np.ones(P.G, bool), 1e-5, "compute_hessian")


def test_beta_fit_entry(dv, orc, sparse_problem):
    P = sparse_problem.subset_genes(np.arange(40))
    Y = P.dense()
    csr = (P.rowptr, P.col, P.val, P.n)
    off = np.log(P.sf_true)
    b0 = orc.init_beta(P.csr_f64(), P.X, off)
    th0 = P.theta_true
    b, it = dv.beta_fit(csr, P.X, b0, off, th0, 200, 1e-3)
    ref = [orc.beta_fit(y, P.X, bb, off, t, 200, 1e-3) for y, bb, t in zip(Y, b0, th0)]
    rb = np.stack([r[0] for r in ref])
    ri = np.array([r[1] for r in ref])
    same = it == ri
    assert same.mean() >= ITER_AGREE
    assert np.abs(b - rb)[same].max() <= BETA_TOL


def test_fit_dispersion_entry(dv, orc, sparse_problem):
    P = sparse_problem.subset_genes(np.arange(60))
    Y = P.dense()
    csr = (P.rowptr, P.col, P.val, P.n)
    off = np.log(P.sf_true)
    b = P.beta_true
    for cr in (True, False):
        th, _ = dv.fit_dispersion(b, P.X, csr, off, do_cox_reid_adjustment=cr)
        ref = np.array([orc.fit_dispersion(bb, P.X, y, off, 200, cr)[0] for bb, y in zip(b, Y)])
        mask = (ref > 1e-3) & (ref < 1e3)
        check_rel(th, ref, mask, 1e-4, f"fit_dispersion cr={cr}")
        assert np.all((ref == 0) == (th == 0))


def test_clustered_meat_entry(dv, orc):
    P = synthetic.make("clustered", seed=9, G=20, n=3000)
    levels, ends = dv.cluster_blocks(P.clusters)
    b, th, sf = P.beta_true, P.theta_true, P.sf_true
    meat = dv.compute_clustered_meat(P.X, (P.rowptr, P.col, P.val, P.n), b, th, sf, ends)
    ref = np.stack([orc.clustered_meat_fast(P.X, y, bb, t, sf, ends)
                    for y, bb, t in zip(P.dense(), b, th)])
    check_mats(meat, ref, np.ones(P.G, bool), 1e-4, "meat")


NEW_OD_EPS = 1e-3  # eps_theta of the fit (its tolerance)


def _k_close(theta_a, theta_b, width):
    """|k_a - k_b| <= width * eps * (1 + k_b) with k = 1 / theta: the "new"
    method only determines k to its tolerance eps (1 + k)."""
    ka, kb = 1.0 / np.asarray(theta_a), 1.0 / np.asarray(theta_b)
    return np.abs(ka - kb) <= width * NEW_OD_EPS * (1.0 + kb)


def _new_od_stable(orc, P, beta, off, theta, pert):
    """Genes whose oracle k = 1/kappa stays within the method's tolerance
    when beta is scaled by 1 +- pert and when the offsets move by 1e-13.  fit_overdispersion_cppp stops its
    search at |dk| < eps (1 + k) and takes discrete branches (Aitken,
    backtracking, secant, bracketing, Brent) on the sign and size of
    f(k) = log F(k) - log k, which is nearly flat for near-Poisson genes:
    there the reference's own result moves by orders of magnitude under
    rounding-level changes of its inputs, so no second implementation can
    match it.  Parity is asserted on the genes where it is well defined."""
    D = P.dense()
    rng = np.random.default_rng(0)
    off2 = off + 1e-13 * rng.choice([-1.0, 1.0], size=len(off))
    ok = np.ones(P.G, bool)
    for g in range(P.G):
        for b, o in ((beta[g] * (1.0 + pert), off), (beta[g] * (1.0 - pert), off), (beta[g], off2)):
            k = orc.fit_overdispersion_new(D[g], P.X, b, o)[0]
            if not _k_close(k, theta[g], 1.0):
                ok[g] = False
                break
    return ok


def test_new_overdispersion_fit_matches_oracle(dv, orc):
    """fit_devil(overdispersion = "new") against the oracle's
    fit_overdispersion_cppp at the fitted beta (normed_sum size factors:
    no gene reaches the reference's stop conditions)."""
    P = synthetic.make("plain_sparse", seed=11, G=200, n=2000)
    ref = oracle_fit(orc, P, orc.OD_NEW)
    fit = gpu_fit(dv, P, "new")
    check_beta(fit, ref)
    # kappa given beta: the oracle's search at the GPU's beta (the FP32
    # per-cell beta differs from the FP64 one at ~1e-7, which moves the
    # search's discrete branches on some genes)
    D = P.dense()
    offg = fit["offset_vector"]
    kg = np.array([orc.fit_overdispersion_new(D[g], P.X, fit["beta"][g], offg)[0]
                   for g in range(P.G)])
    stable = _new_od_stable(orc, P, fit["beta"], offg, kg, 1e-12)
    assert stable.mean() >= 0.4
    close = _k_close(fit["overdispersion"], kg, 2.0)
    # a gene left on the flat part of f(k) can still branch differently on
    # the GPU's own rounding (summation order over cells, digamma ulps)
    assert close[stable].mean() >= 0.95, np.flatnonzero(stable & ~close)
    # and against the FP64 fit where both searches are stable
    both = stable & _new_od_stable(orc, P, ref["beta"], ref["off"], ref["theta"], 1e-6)
    assert _k_close(fit["overdispersion"], ref["theta"], 2.0)[both].mean() >= 0.95


def test_new_overdispersion_single_step(dv, orc):
    """devil_fit_overdispersion_new at the oracle's beta (FP64 on both
    sides), checked on the genes where the reference's search is stable."""
    P = synthetic.make("clustered", seed=4, G=60, n=2000)
    Y = P.csr_f64()
    off = np.zeros(P.n)  # logs summing to zero, as normed_sum size factors give
    th0 = orc.estimate_dispersion(Y, off)
    b0 = orc.init_beta(Y, P.X, off)
    r = orc.cpu_fit(Y, P.X, off, th0, b0, orc.OD_MOM, 200, 1e-3)
    k, it = dv.fit_overdispersion_new((P.rowptr, P.col, P.val, P.n), P.X, r["beta"], off)
    D = P.dense()
    ref = [orc.fit_overdispersion_new(D[g], P.X, r["beta"][g], off) for g in range(P.G)]
    ko = np.array([x[0] for x in ref])
    io = np.array([x[1] for x in ref])
    stable = _new_od_stable(orc, P, r["beta"], off, ko, 1e-12)
    assert stable.mean() >= 0.4
    close = _k_close(k, ko, 2.0)
    assert close[stable].mean() >= 0.95, np.flatnonzero(stable & ~close)
    assert (it[stable] == io[stable]).mean() >= 0.9


def test_new_overdispersion_stop_is_an_error(dv, orc):
    """Where the reference stops (C1 <= n for some gene) the call fails
    with DEVIL_ERR_NUMERIC and the reference's message."""
    from devil_b200 import DevilError
    from devil_b200 import _lib as L
    P = synthetic.make("plain_sparse", seed=5, G=20, n=3000)
    off = np.log(P.sf_true)
    Y = P.csr_f64()
    r = orc.cpu_fit(Y, P.X, off, orc.estimate_dispersion(Y, off), orc.init_beta(Y, P.X, off),
                    orc.OD_MOM, 200, 1e-3)
    with pytest.raises(DevilError) as e:
        dv.fit_overdispersion_new((P.rowptr, P.col, P.val, P.n), P.X, r["beta"], off)
    assert e.value.code == L.ERR_NUMERIC
    assert "C1 > n" in str(e.value)


def test_fit_batch_uneven_problems(dv):
    """devil_fit_batch over uneven problems (different genes, cells, design
    width and clusters) on concurrent streams gives, problem by problem,
    exactly what devil_fit gives."""
    cases = [("plain_small", 1, 40, 400, False), ("plain_sparse", 2, 120, 3000, False),
             ("clustered", 3, 80, 2500, True), ("wide", 4, 24, 4000, False),
             ("plain_sparse", 5, 60, 800, False)]
    probs = []
    for cfg, seed, G, n, cl in cases:
        P = small_problem(cfg, seed, G, n)
        x = (P.rowptr, P.col, P.val.astype(np.float64) if P.val.dtype != np.uint16 else P.val, P.n)
        probs.append((x, P.X, P.clusters) if cl else (x, P.X))
    kw = dict(overdispersion="MOM", size_factors=None)
    fits = dv.fit_devil_batch(probs, workers=3, **kw)
    assert len(fits) == len(probs)
    for pr, f in zip(probs, fits):
        one = dv.fit_devil(pr[0], pr[1], clusters=pr[2] if len(pr) > 2 else None, **kw)
        np.testing.assert_array_equal(f["beta"], one["beta"])
        np.testing.assert_array_equal(f["overdispersion"], one["overdispersion"])
        np.testing.assert_array_equal(f["iterations"]["beta_iters"], one["iterations"]["beta_iters"])
        np.testing.assert_array_equal(f["beta_sandwiches_null"], one["beta_sandwiches_null"])
        if len(pr) > 2:
            np.testing.assert_array_equal(f["beta_sandwiches"], one["beta_sandwiches"])


def test_fit_batch_names_the_failing_problem(dv):
    from devil_b200 import DevilError
    P = synthetic.make("plain_sparse", seed=2, G=30, n=500)
    x = (P.rowptr, P.col, P.val, P.n)
    bad_X = np.zeros_like(P.X)  # rank deficient design
    with pytest.raises(DevilError, match="problem 1"):
        dv.fit_devil_batch([(x, P.X), (x, bad_X)], workers=2)


@pytest.mark.parametrize("p", [4, 3, 2, 1])
def test_tensor_core_irls_matches_oracle(dv, orc, sparse_problem, monkeypatch, p):
    """The opt-in tcgen05 IRLS engine (DEVIL_TC=1, p <= 4): the Hessian's
    dense part as split-TF32 MMAs, the score and the nonzero corrections in
    FP32.  Same bars as the register engine against the oracle, and the two
    engines agree to FP32 rounding on genes with the same iteration count."""
    import dataclasses

    # continuous covariates in every design (a design of few distinct rows
    # goes to the design-group engine instead)
    cols = {4: [0, 1, 2, 3], 3: [0, 1, 2], 2: [0, 2], 1: [2]}[p]
    P = dataclasses.replace(sparse_problem, X=np.ascontiguousarray(sparse_problem.X[:, cols]), p=p)
    ref = oracle_fit(orc, P, orc.OD_MLE)
    reg = gpu_fit(dv, P, "MLE")
    assert dv.context().engine(0) == "register"
    monkeypatch.setenv("DEVIL_TC", "1")
    tc = gpu_fit(dv, P, "MLE")
    assert dv.context().engine(0) == "tensor"
    same = check_beta(tc, ref)
    check_rel(tc["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta MLE")
    it_tc, it_reg = tc["iterations"]["beta_iters"], reg["iterations"]["beta_iters"]
    assert (it_tc == it_reg).mean() >= 0.97
    both = (it_tc == it_reg) & (it_reg < 200)
    d = np.abs(tc["beta"] - reg["beta"]) / np.maximum(1.0, np.abs(reg["beta"]))
    assert d[both].max() <= 2e-6, d[both].max()


@pytest.mark.parametrize("p", [4, 3])
def test_tensor_core_mle_matches_oracle(dv, orc, sparse_problem, monkeypatch, p):
    """The opt-in tcgen05 MLE pass (DEVIL_TC_MLE=1, p <= 4): the Cox-Reid
    matrices b, db, d2b as split-TF32 MMAs over 32-gene tiles, the scalar
    and nonzero terms on the CUDA cores.  theta against the oracle with the
    register engine's bar."""
    import dataclasses

    cols = {4: [0, 1, 2, 3], 3: [0, 1, 2]}[p]
    P = dataclasses.replace(sparse_problem, X=np.ascontiguousarray(sparse_problem.X[:, cols]), p=p)
    ref = oracle_fit(orc, P, orc.OD_MLE)
    monkeypatch.setenv("DEVIL_TC_MLE", "1")
    tc = gpu_fit(dv, P, "MLE")
    assert dv.context().engine(2) == "tensor"
    same = check_beta(tc, ref)
    check_rel(tc["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta MLE")


def test_precision_tc_tf32_option(dv, orc, sparse_problem):
    """precision="tc_tf32" (DEVIL_PREC_TC_TF32 in the C ABI) puts the IRLS and
    MLE passes on the tensor-core engines; results keep the oracle bars.
    "tc_bf16x3" is refused with DEVIL_ERR_UNSUPPORTED."""
    P = sparse_problem
    ref = oracle_fit(orc, P, orc.OD_MLE)
    fit = gpu_fit(dv, P, "MLE", precision="tc_tf32")
    ctx = dv.context()
    assert [ctx.engine(k) for k in range(4)] == ["tensor", "register", "tensor", "register"]
    same = check_beta(fit, ref)
    check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta MLE")
    check_mats(fit["beta_sandwiches_null"], ref["bread"], same & (ref["theta"] < 1e3), 1e-4, "bread")
    with pytest.raises(RuntimeError, match="tc_bf16x3"):
        gpu_fit(dv, P, "MLE", precision="tc_bf16x3")


def test_fit_batch_concurrent_shapes(dv):
    """Workers that fit problems of different shapes at the same time need
    different dynamic shared memory for the same kernels (design-group pass,
    finalizes); the per-kernel cap is process-wide, so a worker must never
    lower it under another worker's launch.  Grouped designs of different
    widths and group counts, many workers, several rounds."""
    cases = [("clustered", 31, 64, 3000, True), ("wide", 32, 16, 4000, False),
             ("clustered", 33, 48, 1500, False), ("wide", 34, 24, 2500, False),
             ("plain_small", 35, 40, 600, False), ("plain_sparse", 36, 64, 2000, False)]
    probs = []
    for cfg, seed, G, n, cl in cases:
        P = small_problem(cfg, seed, G, n)
        x = (P.rowptr, P.col, P.val.astype(np.float64) if P.val.dtype != np.uint16 else P.val, P.n)
        probs.append((x, P.X, P.clusters) if cl else (x, P.X))
    kw = dict(overdispersion="MLE", size_factors=None)
    ref = [dv.fit_devil(pr[0], pr[1], clusters=pr[2] if len(pr) > 2 else None, **kw) for pr in probs]
    for _ in range(3):
        fits = dv.fit_devil_batch(probs * 2, workers=8, **kw)
        for f, one in zip(fits, ref * 2):
            np.testing.assert_array_equal(f["beta"], one["beta"])
            np.testing.assert_array_equal(f["overdispersion"], one["overdispersion"])
