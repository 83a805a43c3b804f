"""The hand-written adjoint of the per-cell NB log-likelihood
(devil_nb_adjoint) on the device:

* against central finite differences of its own log-likelihood, in eta
  (per cell) and in log theta;
* d l/d eta times the design row against the oracle's per-cell score
  vectors (compute_scores, src/variance.cpp:64-85);
* the sum over cells of d l/d log theta against the oracle's dispersion
  score without the Cox-Reid term (src/overdispersion.cpp:95-178);
* the patient-clustered meat built from the adjoint's per-cell scores
  against the device's compute_clustered_meat and the oracle's
  compute_clustered_meat_fast (src/variance.cpp:186-228).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _nb_cells(seed, n=4000, p=4):
    rng = np.random.default_rng(seed)
    X = np.column_stack([np.ones(n), (np.arange(n) % 2).astype(float), rng.normal(size=n),
                         rng.integers(0, 3, n).astype(float)])[:, :p]
    beta = np.array([0.4, -0.6, 0.2, 0.1])[:p]
    sf = rng.lognormal(0.0, 0.3, n)
    eta = X @ beta + np.log(sf)
    mu = np.exp(eta)
    th = 0.8
    a = 1.0 / th
    y = rng.negative_binomial(a, a / (a + mu)).astype(float)
    y[:5] = [0.0, 1.0, 150.0, 3.0, 0.0]
    return X, beta, sf, eta, y, th


@pytest.mark.parametrize("theta", [0.05, 0.8, 20.0])
def test_adjoint_matches_finite_differences(dv, theta):
    X, beta, sf, eta, y, _ = _nb_cells(1)
    lt = np.log(theta)
    ll, de, dt = dv.nb_adjoint(y, eta, lt)
    assert np.all(np.isfinite(ll)) and np.all(np.isfinite(de)) and np.all(np.isfinite(dt))
    h = 1e-5
    lp, _, _ = dv.nb_adjoint(y, eta + h, lt)
    lm, _, _ = dv.nb_adjoint(y, eta - h, lt)
    fd = (lp - lm) / (2 * h)
    np.testing.assert_allclose(de, fd, rtol=1e-6, atol=1e-8 * np.abs(de).max())
    lp, _, _ = dv.nb_adjoint(y, eta, lt + h)
    lm, _, _ = dv.nb_adjoint(y, eta, lt - h)
    fd = (lp - lm) / (2 * h)
    np.testing.assert_allclose(dt, fd, rtol=1e-5, atol=1e-7 * np.abs(dt).max())
    fd_sum = (lp.sum() - lm.sum()) / (2 * h)
    assert abs(dt.sum() - fd_sum) <= 1e-6 * max(1.0, abs(fd_sum))


def test_adjoint_scores_match_oracle(dv, orc):
    X, beta, sf, eta, y, th = _nb_cells(2)
    _, de, dt = dv.nb_adjoint(y, eta, np.log(th))
    sc = orc.compute_scores(X, y, beta, th, sf)
    np.testing.assert_allclose(de[:, None] * X, sc, rtol=1e-12, atol=1e-14)
    # the non-Cox-Reid dispersion score is the sum of the log-theta adjoints
    s = orc.nb_score(y, np.exp(eta), X, np.log(th), cr=False)
    assert abs(dt.sum() - s) <= 1e-10 * max(1.0, abs(s))


def test_clustered_meat_from_adjoint_scores(dv, orc):
    X, beta, sf, eta, y, th = _nb_cells(3, n=6000)
    sizes = np.random.default_rng(4).multinomial(6000 - 40 * 5, np.ones(40) / 40) + 5
    ends = np.cumsum(sizes).astype(np.int32)
    _, de, _ = dv.nb_adjoint(y, eta, np.log(th))
    S = np.add.reduceat(de[:, None] * X, np.r_[0, ends[:-1]], axis=0)  # per-patient scores
    C = len(ends)
    meat_adj = C / (C - 1) / len(y) * S.T @ S
    meat_orc = orc.clustered_meat_fast(X, y, beta, th, sf, ends)
    np.testing.assert_allclose(meat_adj, meat_orc, rtol=1e-10, atol=1e-14 * np.abs(meat_orc).max())
    nz = np.flatnonzero(y)
    csr = (np.array([0, len(nz)], np.int64), nz.astype(np.int32), y[nz].astype(np.float32), len(y))
    meat_dev = dv.compute_clustered_meat(X, csr, beta[None, :], th, sf, ends)[0]
    np.testing.assert_allclose(meat_dev, meat_adj, rtol=1e-9, atol=1e-13 * np.abs(meat_adj).max())
