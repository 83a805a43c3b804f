"""Regenerates the golden fixtures in this directory.

Each fixture holds a small seeded problem (CSR counts, design, clusters)
and the FP64 oracle's outputs for it: size factors, offsets, theta_0,
beta_0, the fitted beta and IRLS iteration counts, MOM and MLE theta,
bread, clustered sandwich, p-values and BH-adjusted p-values.  The devil
reference cannot run here (no R), so these vectors come from the oracle,
whose formulas are pinned to the reference's own tests
(tests/test_oracle_known_answers.py).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as orc  # noqa: E402
from devil_b200 import synthetic  # noqa: E402

CASES = {
    "plain_small_p2": dict(config="plain_small", seed=101, G=40, n=400, od=orc.OD_MLE,
                           sf="normed_sum", clusters=False),
    "plain_sparse_p4": dict(config="plain_sparse", seed=102, G=160, n=2000, od=orc.OD_MOM,
                            sf="normed_sum", clusters=False),
    "clustered_p12": dict(config="clustered", seed=103, G=400, n=2000, od=orc.OD_MOM,
                          sf="psinorm", clusters=True),
}


def build(name, c):
    P = synthetic.make(c["config"], seed=c["seed"], G=c["G"], n=c["n"])
    Y = P.csr_f64()
    sf = orc.calculate_sf(Y, c["sf"])
    off = orc.offset_vector(0.0, P.n, sf)
    th0 = orc.estimate_dispersion(Y, off)
    b0 = orc.init_beta(Y, P.X, off)
    ends = None
    if c["clusters"]:
        lev, _ = orc.factor_first_appearance(P.clusters)
        ends = orc.cluster_blocks(lev)
    r = orc.cpu_fit(Y, P.X, off, th0, b0, c["od"], 200, 1e-3, ends=ends, theta_mom=True)
    contrast = np.zeros(P.p)
    contrast[1] = 1.0
    pv, pa, lf = orc.test_de(r["beta"], r["bread"], r["sandwich"], P.n, contrast)
    out = dict(rowptr=P.rowptr, col=P.col, val=P.val.astype(np.float64), n=P.n, X=P.X,
               clusters=P.clusters if P.clusters is not None else np.zeros(0, np.int64),
               ends=ends if ends is not None else np.zeros(0, np.int32), od=c["od"],
               sf_method=c["sf"], contrast=contrast, sf=sf, off=off, theta0=th0, beta0=b0,
               beta=r["beta"], iters=r["iters"], theta=r["theta"], theta_mom=r["theta_mom"],
               bread=r["bread"],
               sandwich=r["sandwich"] if r["sandwich"] is not None else np.zeros(0),
               pval=pv, padj=pa, lfc=lf)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


if __name__ == "__main__":
    for name, c in CASES.items():
        build(name, c)
        print("wrote", name)
