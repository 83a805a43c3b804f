"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py).

CPU: the oracle reproduces every stored vector (regression pin of the
oracle).  GPU: fit_devil / test_de through libdevil_b200.so match the
stored vectors to the path's tolerances."""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT

FIXTURES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
SF_NAME = {"normed_sum": "normed_sum", "psinorm": "psinorm"}


def load(path):
    z = np.load(path, allow_pickle=False)
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p))
def test_oracle_reproduces_golden(orc, path):
    g = load(path)
    Y = (g["rowptr"], g["col"], g["val"], int(g["n"]))
    sf = orc.calculate_sf(Y, str(g["sf_method"]))
    np.testing.assert_array_equal(sf, g["sf"])
    off = orc.offset_vector(0.0, int(g["n"]), sf)
    th0 = orc.estimate_dispersion(Y, off)
    np.testing.assert_array_equal(th0, g["theta0"])
    b0 = orc.init_beta(Y, g["X"], off)
    np.testing.assert_allclose(b0, g["beta0"], rtol=0, atol=1e-13)
    ends = g["ends"] if g["ends"].size else None
    r = orc.cpu_fit(Y, g["X"], off, th0, g["beta0"], int(g["od"]), 200, 1e-3, ends=ends,
                    theta_mom=True)
    np.testing.assert_array_equal(r["iters"], g["iters"])
    np.testing.assert_allclose(r["beta"], g["beta"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(r["theta"], g["theta"], rtol=1e-10, atol=0)
    np.testing.assert_allclose(r["bread"], g["bread"], rtol=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p))
def test_gpu_matches_golden(dv, path):
    g = load(path)
    n = int(g["n"])
    csr = (g["rowptr"], g["col"], g["val"].astype(np.float32), n)
    od = {0: False, 1: "MOM", 2: "MLE"}[int(g["od"])]
    clusters = g["clusters"] if g["clusters"].size else None
    fit = dv.fit_devil(csr, g["X"], clusters=clusters, overdispersion=od,
                       size_factors=str(g["sf_method"]), compute_theta_mom=True)
    assert np.all(np.isfinite(g["sf"]))
    np.testing.assert_allclose(fit["size_factors"], g["sf"], rtol=1e-12)
    same = fit["iterations"]["beta_iters"] == g["iters"]
    assert same.mean() >= 0.95
    conv = same & (g["iters"] < 200)
    # the acceptance bar: |d beta| <= 1e-5 absolute on genes converging in both
    da = np.abs(fit["beta"] - g["beta"])
    assert da[conv].max() <= 1e-5
    capped = same & (g["iters"] >= 200)
    if capped.any():
        rel = np.abs(fit["beta"] - g["beta"])[capped] / np.maximum(1, np.abs(g["beta"][capped]))
        assert rel.max() <= 1e-4  # not converged: looser check
    mask = same & (g["theta"] > 1e-3)
    rel = np.abs(fit["overdispersion"] - g["theta"])[mask] / g["theta"][mask]
    assert rel.size == 0 or rel.max() <= 1e-4
    res = dv.test_de(fit, g["contrast"])
    # a bread whose condition number exceeds 1/eps of FP64 (an intercept
    # drifting to -75 for a gene without counts in a cell group) gives a
    # sandwich made of rounding in both implementations, the sign of the
    # contrast variance included: such genes carry no p-value to compare
    well = np.array([bool(np.all(np.isfinite(b))) and np.linalg.cond(b) < 1e15 for b in g["bread"]])
    ok = same & well & (g["pval"] > 1e-300)
    lr = np.abs(np.log10(res["pval"][ok]) - np.log10(g["pval"][ok])) / np.maximum(
        1, np.abs(np.log10(g["pval"][ok])))
    assert lr.max() <= 1e-3
