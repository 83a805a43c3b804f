"""fit_devil's surface as the reference's own tests check it
(tests/testthat/test-main.R): result names and shapes, size factors from a
method name, Poisson mode, rough initialisation, MOM and "old" (MLE) theta
with their theta_iters conventions.  The matrices are larger than the
reference's (a few cells are enough for R's dense solver; the GPU path
wants more cells than design columns per segment) but the assertions are
the reference's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _poisson(seed, G, n, lam):
    rng = np.random.default_rng(seed)
    Y = rng.poisson(lam, (G, n)).astype(np.float64)
    X = np.column_stack([np.ones(n), rng.normal(size=n)])
    return Y, X


def test_fit_devil_returns_well_formed_result(dv):
    # test-main.R:1-57
    Y, X = _poisson(123, 5, 200, 10)
    res = dv.fit_devil(Y, X, overdispersion=False, size_factors=None, CUDA=False, verbose=False)
    for name in ("beta", "overdispersion", "iterations", "size_factors", "offset_vector",
                 "design_matrix", "input_matrix", "input_parameters"):
        assert name in res
    assert res["beta"].shape == (5, 2)
    assert len(res["overdispersion"]) == 5
    assert len(res["iterations"]["beta_iters"]) == 5
    assert len(res["iterations"]["theta_iters"]) == 5
    np.testing.assert_array_equal(res["size_factors"], np.ones(200))
    assert len(res["offset_vector"]) == 200
    assert (res["overdispersion"] == 0).all()
    np.testing.assert_array_equal(res["design_matrix"], X)
    assert res["input_matrix"] is Y
    assert {"max_iter", "tolerance"} <= set(res["input_parameters"])


def test_fit_devil_size_factors_from_method_name(dv, orc):
    # test-main.R:59-86
    Y, X = _poisson(13, 5, 200, 10)
    res = dv.fit_devil(Y, X, overdispersion=False, size_factors="normed_sum")
    rows = [np.flatnonzero(Y[g]) for g in range(Y.shape[0])]  # the oracle takes CSR
    rowptr = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    col = np.concatenate(rows).astype(np.int32)
    val = np.concatenate([Y[g, r] for g, r in enumerate(rows)])
    expected = orc.calculate_sf((rowptr, col, val, Y.shape[1]), "normed_sum")
    np.testing.assert_allclose(res["size_factors"], expected, rtol=1e-12)


def test_poisson_mode_theta_is_zero(dv):
    # test-main.R:88-118
    Y, X = _poisson(10, 4, 200, 5)
    res = dv.fit_devil(Y, X, overdispersion=False, max_iter=50, tolerance=1e-3)
    assert res["beta"].shape == (4, 2)
    np.testing.assert_array_equal(res["overdispersion"], np.zeros(4))
    assert (res["iterations"]["theta_iters"] == 0).all()


def test_rough_initialisation(dv):
    # test-main.R:120-149
    Y, X = _poisson(11, 3, 200, 10)
    res = dv.fit_devil(Y, X, overdispersion=False, init_beta_rough=True, max_iter=5)
    assert np.isfinite(res["beta"][:, 0]).all()
    assert len(res["iterations"]["beta_iters"]) == 3


def test_mom_theta_non_negative(dv):
    # test-main.R:151-181
    Y, X = _poisson(12, 4, 200, 8)
    res = dv.fit_devil(Y, X, overdispersion="MOM", max_iter=50)
    assert len(res["overdispersion"]) == 4
    assert (res["overdispersion"] >= 0).all()
    assert (res["iterations"]["theta_iters"] == 0).all()


def test_old_mode_theta_finite_and_iterations_na(dv):
    # test-main.R:183-214 ("old" is the MLE of fit_dispersion)
    Y, X = _poisson(13, 4, 200, 8)
    res = dv.fit_devil(Y, X, overdispersion="old", max_iter=50)
    assert len(res["overdispersion"]) == 4
    assert np.isfinite(res["overdispersion"]).all()
    assert np.isnan(res["iterations"]["theta_iters"]).all()
