"""test_de on the device against the oracle (R/test.R:94-133).

* stats::p.adjust for every method (R/test.R:127) on p-value vectors large
  enough for CUB's multi-pass radix sort (60,000 values), with NA (NaN)
  entries and exact ties: bit for bit, since each method is rank
  arithmetic in the same floating-point expression order as p.adjust;
  Hommel is O(n^2), as in p.adjust, and runs on 20,000 values;
* on real fits (plain and clustered, where the p-value is the max of the
  clustered and plain ones), the device test_de against the oracle's
  test_de given the same beta / bread / sandwich: lfc (log2, clipped at
  max_lfc) bit for bit, p-values to 1e-12 relative (the t tail is the
  incomplete beta's continued fraction in both), adjusted p-values equal
  to the oracle's adjustment of the device p-values bit for bit.
"""
import numpy as np
import pytest

from devil_b200 import synthetic

pytestmark = pytest.mark.gpu

METHODS = ["none", "BH", "fdr", "BY", "holm", "hochberg", "bonferroni", "hommel"]


def pvals_with_nas_and_ties(m, seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(size=m) ** 3
    p[rng.choice(m, m // 50, replace=False)] = np.nan
    src, dst = rng.choice(m, m // 10), rng.choice(m, m // 10)
    p[dst] = p[src]                      # exact ties
    p[rng.choice(m, 20)] = 0.0
    p[rng.choice(m, 20)] = 1.0
    p[rng.choice(m, 200)] = 1e-300       # a run of equal tiny values
    return p


@pytest.mark.parametrize("method", METHODS)
def test_p_adjust_bit_equal(dv, orc, method):
    m = 20000 if method == "hommel" else 60000
    p = pvals_with_nas_and_ties(m, 7)
    got = dv.p_adjust(p, method)
    exp = orc.p_adjust(p, method)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(p))
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("method", METHODS)
def test_p_adjust_small_n(dv, orc, method):
    rng = np.random.default_rng(3)
    for n in (0, 1, 2, 3, 4, 17):
        p = rng.uniform(size=n)
        np.testing.assert_array_equal(dv.p_adjust(p, method), orc.p_adjust(p, method))
        q = p.copy()
        if n:
            q[0] = np.nan  # one NA: n counts the others only
        np.testing.assert_array_equal(dv.p_adjust(q, method), orc.p_adjust(q, method))


def test_p_adjust_hommel_two_is_hochberg(dv):
    p = np.array([0.03, 0.02])
    np.testing.assert_array_equal(dv.p_adjust(p, "hommel"), dv.p_adjust(p, "hochberg"))


def test_unknown_method_message(dv):
    fit = {"beta": np.zeros((2, 2)), "beta_sandwiches_null": np.ones((2, 2, 2)),
           "design_matrix": np.ones((10, 2))}
    with pytest.raises(ValueError, match="should be one of"):
        dv.test_de(fit, [0, 1], pval_adjust_method="sidak")


def _compare_test_de(dv, orc, fit, n, c, sandwich):
    for method in ("BH", "BY", "holm", "hommel", "none"):
        for max_lfc in (10.0, 0.5):
            res = dv.test_de(fit, c, pval_adjust_method=method, max_lfc=max_lfc)
            pv, pa, lf = orc.test_de(fit["beta"], fit["beta_sandwiches_null"],
                                     fit["beta_sandwiches"] if sandwich else None, n, c,
                                     method, max_lfc)
            np.testing.assert_array_equal(res["lfc"], lf)
            np.testing.assert_array_equal(np.isnan(res["pval"]), np.isnan(pv))
            ok = np.isfinite(pv) & (pv > 0)
            r = np.abs(res["pval"][ok] - pv[ok]) / pv[ok]
            assert r.max() <= 1e-12, r.max()
            np.testing.assert_array_equal(res["adj_pval"], orc.p_adjust(res["pval"], method))
            okp = np.isfinite(pa) & (pa > 0)
            ra = np.abs(res["adj_pval"][okp] - pa[okp]) / pa[okp]
            assert ra.max() <= 1e-12, ra.max()
        assert np.abs(res["lfc"]).max() <= 0.5


def test_test_de_plain_fit(dv, orc):
    P = synthetic.make("plain_sparse", seed=41, G=400, n=3000)
    fit = dv.fit_devil((P.rowptr, P.col, P.val, P.n), P.X, overdispersion="MOM",
                       size_factors="normed_sum")
    _compare_test_de(dv, orc, fit, P.n, np.array([0.0, 1.0, 0.0, 0.0]), sandwich=False)
    # a contrast of two coefficients
    _compare_test_de(dv, orc, fit, P.n, np.array([0.0, 1.0, -0.5, 0.25]), sandwich=False)


def test_test_de_clustered_fit_max_rule(dv, orc):
    P = synthetic.make("clustered", seed=42, G=300, n=4000)
    fit = dv.fit_devil((P.rowptr, P.col, P.val, P.n), P.X, clusters=P.clusters,
                       overdispersion="MOM", size_factors=P.sf_true)
    assert fit["beta_sandwiches"] is not None
    c = np.zeros(P.p)
    c[1] = 1.0
    _compare_test_de(dv, orc, fit, P.n, c, sandwich=True)
