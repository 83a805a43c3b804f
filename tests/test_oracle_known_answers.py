"""Pins the FP64 oracle to the known answers of devil's own test suite
(tests/testthat/*.R).  R's set.seed/rpois streams cannot be reproduced
here, so each check restates the test's property or formula on seeded
numpy data; matrices with explicit values are copied as given."""
import numpy as np
import pytest
from scipy import special, stats

from conftest import rel_err


# -- test-size_factors.R --------------------------------------------------
def test_calculate_sf_single_row_is_unit(orc):
    # test-size_factors.R:1-7
    Y = np.arange(1, 6, dtype=float).reshape(1, 5)
    np.testing.assert_array_equal(orc.calculate_sf(Y, "normed_sum"), np.ones(5))


def test_normed_sum_matches_manual_geomean(orc):
    # test-size_factors.R:57-70 (explicit 3 x 2 matrix)
    Y = np.array([[1, 2], [3, 4], [5, 6]], dtype=float)
    cs = Y.sum(0)
    expected = cs / np.exp(np.mean(np.log(cs)))
    np.testing.assert_allclose(orc.calculate_sf(Y, "normed_sum"), expected, rtol=1e-15)


def test_normed_sum_errors_on_zero_column(orc):
    # test-size_factors.R:72-83
    Y = np.array([[0, 1], [0, 2], [0, 4]], dtype=float)
    with pytest.raises(ValueError, match="all zeros"):
        orc.calculate_sf(Y, "normed_sum")


@pytest.mark.parametrize("method", ["normed_sum", "psinorm"])
def test_sf_positive_geomean_one(orc, method):
    # test-size_factors.R:21-35, :85-98
    rng = np.random.default_rng(1)
    Y = rng.poisson(10, (10, 10)).astype(float)
    sf = orc.calculate_sf(Y, method)
    assert np.all(np.isfinite(sf)) and np.all(sf > 0)
    assert abs(np.exp(np.mean(np.log(sf))) - 1) < 1e-8


def test_psinorm_matches_formula_and_is_monotone(orc):
    # R/size_factors.R:100-117 and test-size_factors.R:100-114
    rng = np.random.default_rng(123)
    base = rng.poisson(10, (20, 10)).astype(float)
    Y = np.stack([base[:, 0], 2 * base[:, 0], 4 * base[:, 0]], 1)
    sf = orc.calculate_sf(Y, "psinorm")
    L = np.log1p(Y)
    raw = L.mean(0) - L.min(0)
    np.testing.assert_allclose(sf, raw / np.exp(np.mean(np.log(raw))), rtol=1e-14)
    assert sf[1] > sf[0] and sf[2] > sf[1]


def test_offset_vector(orc):
    # test-size_factors.R:144-163
    np.testing.assert_array_equal(orc.offset_vector(1.2, 4, None), np.full(4, 1.2))
    np.testing.assert_allclose(orc.offset_vector(0.5, 3, np.array([1.0, 2.0, 4.0])),
                               0.5 + np.log([1.0, 2.0, 4.0]), rtol=1e-15)


# -- test-overdispersion.R ------------------------------------------------
def test_estimate_dispersion_formula(orc):
    # test-overdispersion.R:1-15: (var - mean) / mean^2, truncated to 0.01
    rng = np.random.default_rng(1)
    Y = rng.poisson(10, (5, 10)).astype(float)
    d = orc.estimate_dispersion(Y, np.zeros(10))
    v, m = Y.var(1, ddof=1), Y.mean(1)
    mom = (v - m) / m ** 2
    mom[(mom < 0) | np.isnan(mom)] = 0.01
    np.testing.assert_allclose(d, mom, rtol=1e-14)


def test_estimate_dispersion_depends_on_offset(orc):
    # test-overdispersion.R:17-28
    rng = np.random.default_rng(2)
    Y = rng.poisson(20, (10, 10)).astype(float)
    d0 = orc.estimate_dispersion(Y, np.zeros(10))
    d1 = orc.estimate_dispersion(Y, np.full(10, np.log(2)))
    assert not np.allclose(d0, d1)
    v, m = Y.var(1, ddof=1), Y.mean(1)
    exp1 = (v - m / 2.0) / m ** 2
    exp1[(exp1 < 0) | np.isnan(exp1)] = 0.01
    np.testing.assert_allclose(d1, exp1, rtol=1e-14)


def test_estimate_dispersion_truncation(orc):
    # test-overdispersion.R:30-45 (Poisson rows truncated; all-zero row 0.01)
    rng = np.random.default_rng(3)
    Y = rng.poisson(5, (5, 10)).astype(float)
    d = orc.estimate_dispersion(Y, np.zeros(10))
    assert np.all(d >= 0.01)
    Y2 = np.vstack([np.zeros(10), Y])
    assert orc.estimate_dispersion(Y2, np.zeros(10))[0] == 0.01


def test_fit_dispersion_all_zero_is_exactly_zero(orc):
    # test-overdispersion.R:47-65
    th, _ = orc.fit_dispersion(np.zeros(1), np.ones((20, 1)), np.zeros(20), np.zeros(20))
    assert th == 0.0


def test_fit_dispersion_poisson_small(orc):
    # test-overdispersion.R:67-91
    rng = np.random.default_rng(10)
    y = rng.poisson(10, 200).astype(float)
    th, _ = orc.fit_dispersion(np.array([np.log(10.0)]), np.ones((200, 1)), y, np.zeros(200))
    assert np.isfinite(th) and 0 <= th < 0.2


def test_fit_dispersion_nb_near_truth(orc):
    # test-overdispersion.R:93-125
    rng = np.random.default_rng(11)
    y_p = rng.poisson(10, 400).astype(float)
    lam = rng.gamma(2.0, 0.5 * 10, 400)
    y_nb = rng.poisson(lam).astype(float)
    X = np.ones((400, 1))
    b = np.array([np.log(10.0)])
    t_p, _ = orc.fit_dispersion(b, X, y_p, np.zeros(400))
    t_nb, _ = orc.fit_dispersion(b, X, y_nb, np.zeros(400))
    assert t_nb > t_p and np.isfinite(t_nb)
    assert abs(t_nb - 0.5) <= 0.3 * 0.5 + 1e-9 or abs(t_nb - 0.5) / 0.5 <= 0.3


def test_fit_dispersion_depends_on_cox_reid(orc):
    # test-overdispersion.R:127-152
    rng = np.random.default_rng(12)
    lam = rng.gamma(1 / 0.8, 0.8 * 5, 200)
    y = rng.poisson(lam).astype(float)
    X = np.ones((200, 1))
    b = np.array([np.log(5.0)])
    a, _ = orc.fit_dispersion(b, X, y, np.zeros(200), cr=True)
    c, _ = orc.fit_dispersion(b, X, y, np.zeros(200), cr=False)
    assert np.isfinite(a) and np.isfinite(c) and a != c


# -- test-beta.R ----------------------------------------------------------
def test_init_beta_intercept_only_is_mean_log1p(orc):
    # test-beta.R:19-39
    rng = np.random.default_rng(2)
    Y = rng.poisson(5, (4, 6)).astype(float)
    b = orc.init_beta(Y, np.ones((6, 1)), np.zeros(6))
    np.testing.assert_allclose(b[:, 0], np.log1p(Y).mean(1), rtol=0, atol=1e-10)


def test_init_beta_matches_least_squares(orc):
    # test-beta.R:41-77 (tolerance 1e-10; offsets vary by cell here)
    rng = np.random.default_rng(3)
    Y = rng.poisson(10, (3, 10)).astype(float)
    X = np.column_stack([np.ones(10), rng.normal(size=10), rng.normal(size=10)])
    off = rng.uniform(-0.5, 0.5, 10)
    b = orc.init_beta(Y, X, off)
    Z = np.log1p(Y / np.exp(off)[None, :])
    manual = np.linalg.solve(X.T @ X, X.T @ Z.T).T
    np.testing.assert_allclose(b, manual, rtol=0, atol=1e-10)


def test_init_beta_scaling(orc):
    # test-beta.R:79-100
    rng = np.random.default_rng(4)
    Y = rng.poisson(7, (3, 12)).astype(float)
    X = np.column_stack([np.ones(12), rng.normal(size=12)])
    b1 = orc.init_beta(Y, X, np.zeros(12))
    Xs = X.copy()
    Xs[:, 1] *= 5
    b2 = orc.init_beta(Y, Xs, np.zeros(12))
    np.testing.assert_allclose(b1[:, 0], b2[:, 0], atol=1e-8)
    np.testing.assert_allclose(b1[:, 1], b2[:, 1] * 5, atol=1e-8)


# -- test-test.R ----------------------------------------------------------
def test_test_de_lfc_clipping(orc):
    # test-test.R:32-62 (explicit betas)
    beta = np.array([[0, 0.5], [0, -1], [0, 4], [0, -5]], dtype=float)
    bread = np.stack([np.eye(2) / 6] * 4)
    _, _, lfc = orc.test_de(beta, bread, None, 6, [0, 1], "BH", 2.0)
    raw = beta @ np.array([0, 1.0]) / np.log(2)
    np.testing.assert_array_equal(lfc, np.clip(raw, -2, 2))


def test_test_de_bh_le_bonferroni(orc):
    # test-test.R:64-73
    rng = np.random.default_rng(2)
    beta = rng.normal(size=(10, 2))
    bread = np.stack([np.eye(2) / 8] * 10)
    p1, a1, _ = orc.test_de(beta, bread, None, 8, [0, 1], "BH")
    p2, a2, _ = orc.test_de(beta, bread, None, 8, [0, 1], "bonferroni")
    np.testing.assert_array_equal(p1, p2)
    assert np.all(a2 >= a1)


def test_test_de_clustered_is_more_conservative(orc):
    # test-test.R:88-118
    rng = np.random.default_rng(4)
    beta = rng.normal(size=(6, 2))
    b1 = np.stack([np.eye(2) / 12] * 6)
    b5 = np.stack([5 * np.eye(2) / 12] * 6)
    p_nc, _, _ = orc.test_de(beta, b1, None, 12, [0, 1])
    p_c, _, _ = orc.test_de(beta, b1, b5, 12, [0, 1])
    assert np.all(p_c >= p_nc)


def test_test_de_pvalue_formula(orc):
    # R/test.R:108-116: 2 * pt(|lfc| / sqrt(c'Hc), df = n - 2, upper)
    rng = np.random.default_rng(5)
    beta = rng.normal(size=(50, 3))
    A = rng.normal(size=(50, 3, 3))
    H = np.einsum("gij,gkj->gik", A, A) / 30 + np.eye(3) * 0.01
    c = np.array([0.0, 1.0, -1.0])
    p, _, _ = orc.test_de(beta, H, None, 40, c)
    t = np.abs(beta @ c) / np.sqrt(np.einsum("i,gij,j->g", c, H, c))
    np.testing.assert_allclose(p, 2 * stats.t.sf(t, 38), rtol=1e-12)


# -- test-variance.R ------------------------------------------------------
def test_sandwich_properties(orc):
    # test-variance.R:1-82 via the clustered meat and bread of the oracle
    rng = np.random.default_rng(2)
    n, p = 12, 2
    X = rng.normal(size=(n, p))
    y = rng.poisson(10, n).astype(float)
    b = rng.normal(size=p) * 0.1
    sf = np.ones(n)
    bread = orc.compute_hessian(b, 1.0, y, X, sf)
    clusters = np.repeat([1, 2, 3], 4).astype(np.int32)
    m_cl = orc.clustered_meat(X, y, b, 1.0, sf, clusters)
    m_fast = orc.clustered_meat_fast(X, y, b, 1.0, sf, np.array([4, 8, 12], np.int32))
    np.testing.assert_allclose(m_cl, m_fast, rtol=1e-12)
    S = bread @ m_cl @ bread * n
    np.testing.assert_allclose(S, S.T, rtol=1e-12)


# -- special functions behind the reference's nmath calls ------------------
@pytest.mark.parametrize("x", [1e-3, 0.1, 0.5, 1.0, 3.7, 9.99, 10.0, 55.5, 1e4, 1e8])
def test_digamma_trigamma_vs_scipy(orc, x):
    assert rel_err(orc.digamma(x), special.digamma(x)) < 1e-13
    assert rel_err(orc.trigamma(x), special.polygamma(1, x)) < 1e-13


@pytest.mark.parametrize("df", [1, 3, 10, 98, 5000, 99998, 999998])
def test_t_pvalue_vs_scipy(orc, df):
    for t in [0.0, 0.01, 0.5, 1.0, 2.5, 5.0, 10.0, 30.0]:
        ref = 2 * stats.t.sf(t, df)
        got = orc.two_sided_t_pvalue(t, df)
        if ref > 1e-300:
            assert rel_err(got, ref) < 1e-10, (t, df, got, ref)


# ----------------------------------------------------------------------
# overdispersion = "new" (src/new_overdispersion.cpp)
# ----------------------------------------------------------------------
@pytest.mark.parametrize("m", [4, 16, 32])
def test_gauss_hermite_matches_numpy(orc, m):
    """The Golub-Welsch Hermite rule of get_gh (src/new_overdispersion.cpp:22-47)."""
    x, w = orc.gauss_hermite(m)
    xr, wr = np.polynomial.hermite.hermgauss(m)
    assert np.abs(x - xr).max() < 1e-12
    assert np.abs(w / wr - 1.0).max() < 1e-10


@pytest.mark.parametrize("p,s,t", [(0.5, 100.0, 130.0), (-0.5, 100.0, 130.0),
                                   (0.5, 20.0, 60.0), (0.5, 5000.0, 5100.5)])
def test_h_log_gh_matches_quadrature(orc, p, s, t):
    """H_log_gh_cpp (src/new_overdispersion.cpp:129-141): the log of
    int x^p exp(s (x log x - lgamma x) - t x) dx by Laplace-centred
    Gauss-Hermite, against adaptive quadrature around the mode."""
    from scipy import integrate, special

    def h(x):
        return p * np.log(x) + s * (x * np.log(x) - special.gammaln(x)) - t * x

    xs = np.linspace(1e-3, 200, 400001)
    hv = h(xs)
    i = int(np.argmax(hv))
    hm, xm = hv[i], xs[i]
    width = 40 * xm / np.sqrt(s) + 1.0
    val = integrate.quad(lambda x: np.exp(h(x) - hm), max(1e-9, xm - width), xm + width,
                         points=[xm], limit=500, epsabs=0, epsrel=1e-12)[0]
    assert abs(orc.h_log_gh(p, s, t, 32, 8, 1e-12) - (hm + np.log(val))) < 1e-3


def test_new_overdispersion_near_truth_and_mle(orc):
    """fit_overdispersion_cppp on large simulated NB genes lands near the
    generating theta and the Cox-Reid MLE."""
    rng = np.random.default_rng(3)
    n = 20000
    X = np.ones((n, 1))
    off = np.zeros(n)
    for th, mu in [(0.5, 2.0), (2.0, 5.0)]:
        y = rng.poisson(rng.gamma(1 / th, th * mu, n)).astype(float)
        beta = np.array([np.log(y.mean())])
        k, it, conv, err = orc.fit_overdispersion_new(y, X, beta, off)
        mle, _ = orc.fit_dispersion(beta, X, y, off)
        assert err == 0 and conv == 1 and it >= 1
        assert abs(k - th) / th < 0.1
        assert abs(k - mle) / mle < 0.01


def test_new_overdispersion_stop_condition(orc):
    """The reference stops when C1 <= n (src/new_overdispersion.cpp:303-304):
    with size factors whose logs do not sum to zero a near-Poisson gene
    reaches it at the large-k end of the search."""
    from devil_b200 import synthetic
    P = synthetic.make("plain_sparse", seed=5, G=20, n=3000)
    off = np.log(P.sf_true)
    Y = P.csr_f64()
    b0 = orc.init_beta(Y, P.X, off)
    th0 = orc.estimate_dispersion(Y, off)
    r = orc.cpu_fit(Y, P.X, off, th0, b0, orc.OD_MOM, 200, 1e-3)
    D = P.dense()
    errs = [orc.fit_overdispersion_new(D[g], P.X, r["beta"][g], off)[3] for g in range(P.G)]
    assert 1 in errs and 0 in errs


def _hommel_as_in_p_adjust(p):
    """stats::p.adjust(p, "hommel") line by line in numpy (no NAs)."""
    p = np.asarray(p, float)
    n = len(p)
    i = np.arange(1, n + 1)
    o = np.argsort(p, kind="stable")
    ps = p[o]
    ro = np.argsort(o, kind="stable")
    q = pa = np.full(n, np.min(n * ps / i))
    for m in range(n - 1, 1, -1):
        i1 = np.arange(1, n - m + 2)
        i2 = np.arange(n - m + 2, n + 1)
        q1 = np.min(m * ps[i2 - 1] / np.arange(2, m + 1))
        q = q.copy()
        q[i1 - 1] = np.minimum(m * ps[i1 - 1], q1)
        q[i2 - 1] = q[n - m]
        pa = np.maximum(pa, q)
    return np.maximum(pa, ps)[ro]


def test_p_adjust_hommel(orc):
    # the restatement of p.adjust's hommel branch; n = 2 switches to hochberg
    rng = np.random.default_rng(8)
    for n in (3, 4, 11, 60):
        p = rng.uniform(size=n) ** 2
        np.testing.assert_array_equal(orc.p_adjust(p, "hommel"), _hommel_as_in_p_adjust(p))
    np.testing.assert_allclose(orc.p_adjust([0.01, 0.02, 0.03, 0.04, 0.05], "hommel"),
                               [0.05] * 5, rtol=1e-15)
    p2 = np.array([0.04, 0.01])
    np.testing.assert_array_equal(orc.p_adjust(p2, "hommel"), orc.p_adjust(p2, "hochberg"))
    # Hommel is never less powerful than Hochberg
    p = rng.uniform(size=40) ** 3
    assert np.all(orc.p_adjust(p, "hommel") <= orc.p_adjust(p, "hochberg") + 1e-15)


def test_p_adjust_by_constant_is_correctly_rounded(orc):
    from fractions import Fraction
    n = 1000
    exact = float(sum(Fraction(1.0 / k) for k in range(1, n + 1)))  # sum of the double terms
    p = np.full(n, 1e-6)
    got = orc.p_adjust(p, "BY")
    # BY on equal p-values: min over ranks of q n / i p = q p at i = n
    assert got[0] == min(1.0, exact * n / n * 1e-6)
