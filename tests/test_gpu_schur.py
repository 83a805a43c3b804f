"""The design-group engine's structured Newton steps: when some design
columns are exclusive (no design row with two of them nonzero, e.g. one-hot
cell types), the IRLS step and the Cox-Reid traces of the MLE step go
through the Schur complement on the remaining dense columns.  Designs with
1, 3 and 5 dense columns (intercept; + condition + batch; + two more
binary covariates) against the FP64 oracle with the path's bars
(src/beta.cpp:35-46, src/overdispersion.cpp:95-242)."""
import numpy as np
import pytest

from devil_b200 import synthetic
from test_gpu_parity import _theta_mask, check_beta, check_mats, check_rel, gpu_fit, oracle_fit

pytestmark = pytest.mark.gpu


def _problem(seed, G, n, n_types, n_bin):
    """Counts from the NB model of the synthetic workloads on a design of an
    intercept, n_bin binary covariates and n_types - 1 one-hot cell types."""
    rng = np.random.default_rng(seed)
    cols = [np.ones(n)]
    for _ in range(n_bin):
        cols.append((rng.random(n) < 0.5).astype(np.float64))
    t = rng.integers(0, n_types, n)
    for k in range(1, n_types):
        cols.append((t == k).astype(np.float64))
    X = np.stack(cols, 1)
    p = X.shape[1]
    sf = rng.lognormal(0.0, 0.3, n)
    theta = rng.lognormal(0.0, 1.0, G)
    beta = np.zeros((G, p))
    beta[:, 0] = rng.normal(-1.0, 1.0, G)
    beta[:, 1:] = rng.normal(0.0, 0.4, (G, p - 1))
    mu = sf[None, :] * np.exp(beta @ X.T)
    y = rng.poisson(rng.gamma(1.0 / theta[:, None], theta[:, None] * mu))
    y = np.minimum(y, 65535)
    nz = y != 0
    r, c = np.nonzero(nz)
    rowptr = np.zeros(G + 1, np.int64)
    rowptr[1:] = np.cumsum(nz.sum(1))
    return synthetic.Problem(G, n, p, rowptr, c.astype(np.int32), y[r, c].astype(np.uint16), X, sf,
                             beta, theta, None, {})


@pytest.mark.parametrize("n_types,n_bin", [(9, 0), (9, 2), (7, 4)])
def test_structured_steps_match_oracle(dv, orc, n_types, n_bin):
    P = _problem(100 + n_types + n_bin, G=160, n=6000, n_types=n_types, n_bin=n_bin)
    ref = oracle_fit(orc, P, orc.OD_MLE)
    fit = gpu_fit(dv, P, "MLE")
    assert [dv.context().engine(k) for k in (0, 2)] == ["groups", "groups"]
    same = check_beta(fit, ref)
    check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta MLE")
    check_mats(fit["beta_sandwiches_null"], ref["bread"], same & (ref["theta"] < 1e3), 1e-4, "bread")
