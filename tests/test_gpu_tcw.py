"""The tensor-core IRLS engine for designs of p = 5..32 columns without few
distinct rows (continuous covariates): the per-gene Hessian as split-TF32
tcgen05 MMAs over a dense count image, the score on the CUDA cores in FP32
(devil_b200/csrc/kernels_tcw.cu).  It replaces the per-cell contraction of
beta_fit (src/beta.cpp:35-42); the bars are the path's: |d beta| <= 1e-5
absolute on genes that converge in both with equal iteration counts, MOM /
MLE theta 1e-4 relative, bread 1e-4 of the diagonal scale."""
import numpy as np
import pytest

from devil_b200 import synthetic
from test_gpu_parity import _theta_mask, check_beta, check_mats, check_rel, gpu_fit, oracle_fit

pytestmark = pytest.mark.gpu


def _agree(a, b, tol=1e-5):
    """Two GPU fits of one problem: equal iteration counts on >= 97 % of the
    genes, |d beta| <= tol on the genes converged in both with equal counts."""
    ia, ib = a["iterations"]["beta_iters"], b["iterations"]["beta_iters"]
    same = ia == ib
    assert same.mean() >= 0.97, same.mean()
    both = same & (ia < 200)
    d = np.abs(a["beta"] - b["beta"])[both]
    assert d.size == 0 or d.max() <= tol, d.max()


@pytest.mark.parametrize("p,n", [(8, 4000), (16, 4001), (32, 3001)])
def test_tcw_irls_matches_oracle(dv, orc, monkeypatch, p, n):
    """p = 8, 16, 32 with continuous covariates; n not a multiple of the
    32-cell chunk (zero padding), 300 genes (a partial last tile), several
    cell segments and, at p = 32, three product blocks."""
    P = synthetic.make("continuous", seed=40 + p, G=300, n=n, p=p)
    ref = oracle_fit(orc, P, orc.OD_MOM)
    ctx = dv.context()
    ctx.set_profiling(True)
    fit = gpu_fit(dv, P, "MOM", precision="tc_tf32")
    assert ctx.engine(0) == "tensor_wide"
    assert ctx.profile_tc_flops(0) > 0
    ctx.set_profiling(False)
    same = check_beta(fit, ref)
    check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta MOM")
    check_mats(fit["beta_sandwiches_null"], ref["bread"], same & (ref["theta"] < 1e3), 1e-4, "bread")
    # the CUDA-core engine on the same problem (FP32 register tiles at
    # p <= 8, FP64 shared-memory tiles above)
    monkeypatch.setenv("DEVIL_TCW", "0")
    base = gpu_fit(dv, P, "MOM")
    monkeypatch.delenv("DEVIL_TCW")
    assert ctx.engine(0) in ("register", "shared")
    _agree(fit, base)
    # the default precision: the tensor-core engines from p = 9 on
    gpu_fit(dv, P, "MLE")
    want = "register" if p <= 8 else "tensor_wide"
    assert [ctx.engine(k) for k in (0, 2)] == [want, want]


def test_tcw_float_counts_and_mle(dv, orc):
    """Float counts (the dense image holds FP32 values) and the MLE theta
    that follows the IRLS."""
    P = synthetic.make("continuous", seed=77, G=200, n=2500, p=12)
    ref = oracle_fit(orc, P, orc.OD_MLE)
    fit = dv.fit_devil((P.rowptr, P.col, P.val.astype(np.float64), P.n), P.X, overdispersion="MLE",
                       size_factors="normed_sum", compute_theta_mom=True, precision="tc_tf32")
    assert [dv.context().engine(k) for k in (0, 2)] == ["tensor_wide", "tensor_wide"]
    same = check_beta(fit, ref)
    check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta MLE")


@pytest.mark.parametrize("p,n", [(9, 3000), (20, 2501), (32, 2000)])
def test_tcw_mle_matches_oracle(dv, orc, monkeypatch, p, n):
    """The dispersion pass on the tensor cores (precision "tc_tf32"): the
    Cox-Reid matrices b, db, d2b as split-TF32 MMAs (32 genes x 3 weights
    per tile), the scalar sums on the CUDA cores (FP64 at the nonzeros).
    MLE theta 1e-4 relative against the oracle and against the CUDA-core
    pass (FP64 per cell above p = 8; the two differ by FP32-level terms,
    measured 2.6e-5 at most)."""
    P = synthetic.make("continuous", seed=60 + p, G=160, n=n, p=p)
    ref = oracle_fit(orc, P, orc.OD_MLE)
    fit = gpu_fit(dv, P, "MLE", precision="tc_tf32")
    assert dv.context().engine(2) == "tensor_wide"
    same = check_beta(fit, ref)
    check_rel(fit["overdispersion"], ref["theta"], _theta_mask(ref["theta"], same), 1e-4, "theta MLE")
    monkeypatch.setenv("DEVIL_TCW_MLE", "0")
    base = gpu_fit(dv, P, "MLE", precision="tc_tf32")
    assert dv.context().engine(2) == "shared"
    check_rel(fit["overdispersion"], base["overdispersion"], _theta_mask(base["overdispersion"], same),
              1e-4, "theta MLE vs the CUDA-core pass")


def test_tcw_switch(dv, monkeypatch):
    """DEVIL_TCW=1 selects the engine at the default precision; DEVIL_TCW=0
    keeps it off even for precision="tc_tf32"; fits through both agree."""
    P = synthetic.make("continuous", seed=5, G=150, n=2000, p=10)
    monkeypatch.setenv("DEVIL_TCW", "1")
    on = gpu_fit(dv, P, "MOM")
    assert dv.context().engine(0) == "tensor_wide"
    monkeypatch.setenv("DEVIL_TCW", "0")
    off = gpu_fit(dv, P, "MOM", precision="tc_tf32")
    assert dv.context().engine(0) == "shared"
    _agree(on, off)


def test_tcw_rescue_of_slow_genes(dv, orc, monkeypatch):
    """Genes the tensor-core engine hands back (here every gene with more
    than DEVIL_TCW_RESCUE = 3 steps; by default a coefficient beyond +-8)
    are fitted again from beta_0 on the CUDA-core engine (FP64 per cell at
    p = 12) and must equal the CUDA-core fit of the same genes."""
    P = synthetic.make("continuous", seed=9, G=256, n=3000, p=12)
    ref = oracle_fit(orc, P, orc.OD_MOM)
    ctx = dv.context()
    monkeypatch.setenv("DEVIL_TCW_RESCUE", "3")
    fit = gpu_fit(dv, P, "MOM")
    nr = ctx.irls_rescued
    slow = fit["iterations"]["beta_iters"] > 3
    assert nr >= int(slow.sum()) and nr > P.G // 2
    assert ctx.engine(0) == "tensor_wide"
    check_beta(fit, ref)
    monkeypatch.setenv("DEVIL_TCW", "0")
    base = gpu_fit(dv, P, "MOM")
    assert ctx.irls_rescued == 0
    np.testing.assert_array_equal(fit["iterations"]["beta_iters"][slow],
                                  base["iterations"]["beta_iters"][slow])
    d = np.abs(fit["beta"][slow] - base["beta"][slow]) / np.maximum(1.0, np.abs(base["beta"][slow]))
    assert d.max() <= 1e-9, d.max()
