"""Seeded synthetic count workloads for devil's NB GLM path.

The reference's vignette datasets (scRNAseq BaronPancreas, RichardTCell, ...)
are not available offline; these generators stand in for them with the
shapes, sparsity and value distributions of the benchmark workloads:

* ``plain_small``  -- G=2,000 genes x n=5,000 cells, dense, p=2
  (intercept + binary condition, 50/50), s_c ~ LogNormal(0, 0.3),
  beta0 ~ N(0, 1.5), beta1 = 0 for 90% of genes and N(0, 1) otherwise,
  theta ~ LogNormal(0, 1).
* ``plain_sparse`` -- G=20,000 x n=100,000, CSR uint16, p=4 (intercept,
  condition, two N(0,1) covariates with gene effects N(0, 0.2)),
  beta0 ~ N(-3, 1.5) which gives ~10% nonzeros.
* ``clustered``    -- G=20,000 x n=500,000 over 40 patients whose sizes are
  round(Dirichlet(1) * n), patient offsets N(0, 0.3) added to eta, p=12
  (intercept, condition, 10 cell-type indicators for 11 types).
* ``wide``         -- G=20,000 x n=1,000,000, p=32 (intercept, condition,
  30 indicators for 31 cell types), gene means LogNormal(-3.8, 2): about 8%
  nonzeros (1.6e9 entries at full size).  The location of the gene means is
  set by that density; with LogNormal(-1, 2) the same model gives about 34%
  nonzeros (``mean_loc=-1.0`` reproduces it).
* ``binary``       -- G=20,000 x n=1,000,000, p=2 (intercept + binary
  condition, 50/50), the model of ``plain_small`` with beta0 ~ N(-3, 1.5):
  about 10% nonzeros, CSR uint16.
* ``continuous``   -- G=20,000 x n=100,000, p=16 (intercept, condition and
  p - 2 N(0, 1) covariates with gene effects N(0, 0.2)), beta0 ~ N(-2, 1),
  CSR uint16: a design without few distinct rows.  ``p`` (2..32) overrides
  the number of columns.
* ``many_problems_shapes`` -- the many-uneven-problems workload: per
  problem n ~ LogUniform(200, 50,000) cells, G ~ U{5,000..20,000} genes,
  p ~ U{2..16} (the ``continuous`` design) and a per-problem dispersion
  scale s ~ LogUniform(0.1, 10) (theta_g ~ LogNormal(log s, 1)).

Counts are NB with Var = mu + theta * mu^2 (theta is the dispersion devil
returns), drawn as a Gamma-Poisson mixture: lambda ~ Gamma(shape=1/theta,
scale=theta*mu), y ~ Poisson(lambda).  Counts are stored as uint16 and a
draw above 65535 (heavy Gamma tails of strongly overdispersed, highly
expressed genes of the ``wide`` config) saturates at 65535; the number of
saturated entries is recorded in ``meta["saturated"]``.

The numpy path (``make``) is exact and reproducible for any size that fits
in host memory; ``make_torch`` draws the same model on a CUDA device for
the full-size benchmark workloads (different random stream).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

CONFIGS = {
    "plain_small": dict(G=2000, n=5000, p=2, b0_loc=0.0, b0_sd=1.5, covariates=0, types=0,
                        patients=1, dense=True),
    "plain_sparse": dict(G=20000, n=100000, p=4, b0_loc=-3.0, b0_sd=1.5, covariates=2, types=0,
                         patients=1, dense=False),
    "clustered": dict(G=20000, n=500000, p=12, b0_loc=-3.0, b0_sd=1.5, covariates=0, types=11,
                      patients=40, dense=False),
    "wide": dict(G=20000, n=1000000, p=32, b0_loc=None, b0_sd=None, mean_loc=-3.8, covariates=0,
                 types=31, patients=1, dense=False),
    "binary": dict(G=20000, n=1000000, p=2, b0_loc=-3.0, b0_sd=1.5, covariates=0, types=0,
                   patients=1, dense=False),
    "continuous": dict(G=20000, n=100000, p=16, b0_loc=-2.0, b0_sd=1.0, covariates=14, types=0,
                       patients=1, dense=False),
}


def config_params(name: str, p: int | None = None) -> dict:
    """The config's parameters; ``p`` sets the column count of a config of
    intercept, condition and covariates only."""
    cfg = dict(CONFIGS[name])
    if p is not None and int(p) != cfg["p"]:
        if cfg["types"] or not 2 <= int(p) <= 32:
            raise ValueError(f"config {name!r} has no p = {p}")
        cfg["p"] = int(p)
        cfg["covariates"] = int(p) - 2
    return cfg


@dataclass
class Problem:
    """One DE problem: counts (CSR, gene-major), design, truth."""
    G: int
    n: int
    p: int
    rowptr: np.ndarray          # int64 [G+1]
    col: np.ndarray             # int32 [nnz]
    val: np.ndarray             # uint16 or float64 [nnz]
    X: np.ndarray               # float64 [n, p]
    sf_true: np.ndarray
    beta_true: np.ndarray
    theta_true: np.ndarray
    clusters: np.ndarray | None = None   # int64 patient id per cell (contiguous)
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def dense(self) -> np.ndarray:
        Y = np.zeros((self.G, self.n), dtype=np.float64)
        rows = np.repeat(np.arange(self.G), np.diff(self.rowptr))
        Y[rows, self.col] = self.val
        return Y

    def csr_f64(self):
        return self.rowptr, self.col, self.val.astype(np.float64), self.n

    def subset_genes(self, genes) -> "Problem":
        genes = np.asarray(genes)
        starts, ends = self.rowptr[genes], self.rowptr[genes + 1]
        lens = ends - starts
        rowptr = np.zeros(len(genes) + 1, np.int64)
        rowptr[1:] = np.cumsum(lens)
        idx = np.concatenate([np.arange(s, e) for s, e in zip(starts, ends)]) if len(genes) else \
            np.zeros(0, np.int64)
        return Problem(len(genes), self.n, self.p, rowptr, self.col[idx], self.val[idx], self.X,
                       self.sf_true, self.beta_true[genes], self.theta_true[genes], self.clusters,
                       dict(self.meta, subset=True))


def design(cfg: dict, n: int, rng: np.random.Generator):
    cols = [np.ones(n), (np.arange(n) % 2).astype(np.float64)]
    for _ in range(cfg["covariates"]):
        cols.append(rng.normal(0.0, 1.0, n))
    if cfg["types"]:
        t = rng.integers(0, cfg["types"], n)
        for k in range(1, cfg["types"]):
            cols.append((t == k).astype(np.float64))
    X = np.stack(cols, 1)
    assert X.shape[1] == cfg["p"], (X.shape, cfg["p"])
    return X


def patient_sizes(n: int, k: int, rng: np.random.Generator):
    if k <= 1:
        return np.array([n])
    w = rng.dirichlet(np.ones(k))
    sizes = np.round(w * n).astype(np.int64)
    sizes = np.maximum(sizes, 1)
    sizes[np.argmax(sizes)] += n - sizes.sum()
    return sizes


def make(config: str = "plain_small", seed: int = 0, G: int | None = None, n: int | None = None,
         chunk_cells: int = 1 << 24, mean_loc: float | None = None, p: int | None = None) -> Problem:
    """Draw one problem with numpy (PCG64).  G / n override the config sizes;
    mean_loc the location of the gene means (configs that draw them); p the
    column count of a covariates-only config."""
    cfg = config_params(config, p)
    if mean_loc is not None:
        cfg["mean_loc"] = float(mean_loc)
    G = cfg["G"] if G is None else int(G)
    n = cfg["n"] if n is None else int(n)
    p = cfg["p"]
    rng = np.random.default_rng(seed)
    X = design(cfg, n, rng)
    sf = rng.lognormal(0.0, 0.3, n)
    theta = rng.lognormal(0.0, 1.0, G)
    beta = np.zeros((G, p))
    if cfg["b0_loc"] is None:
        beta[:, 0] = np.log(rng.lognormal(cfg["mean_loc"], 2.0, G))
    else:
        beta[:, 0] = rng.normal(cfg["b0_loc"], cfg["b0_sd"], G)
    de = rng.random(G) < 0.1
    beta[:, 1] = np.where(de, rng.normal(0.0, 1.0, G), 0.0)
    if cfg["covariates"]:
        beta[:, 2:2 + cfg["covariates"]] = rng.normal(0.0, 0.2, (G, cfg["covariates"]))
    if cfg["types"]:
        nt = cfg["types"] - 1
        beta[:, p - nt:] = rng.normal(0.0, 0.5, (G, nt))
    clusters = None
    pat_eff = None
    if cfg["patients"] > 1:
        sizes = patient_sizes(n, cfg["patients"], rng)
        clusters = np.repeat(np.arange(1, cfg["patients"] + 1), sizes).astype(np.int64)
        pat_eff = rng.normal(0.0, 0.3, (G, cfg["patients"]))
    eta_fixed = X @ beta.T                  # n x G, fine for test sizes
    rows_per = max(1, chunk_cells // max(n, 1))
    rowptr = np.zeros(G + 1, np.int64)
    cols, vals = [], []
    sat = 0
    for g0 in range(0, G, rows_per):
        g1 = min(G, g0 + rows_per)
        eta = eta_fixed[:, g0:g1].T
        if pat_eff is not None:
            eta = eta + pat_eff[g0:g1][:, clusters - 1]
        mu = sf[None, :] * np.exp(eta)
        th = theta[g0:g1, None]
        lam = rng.gamma(1.0 / th, th * mu)
        y = rng.poisson(lam)
        sat += int((y > 65535).sum())
        y = np.minimum(y, 65535)
        nz = y != 0
        r, c = np.nonzero(nz)
        rowptr[g0 + 1:g1 + 1] = rowptr[g0] + np.cumsum(nz.sum(1))
        cols.append(c.astype(np.int32))
        vals.append(y[r, c].astype(np.uint16 if not cfg["dense"] else np.float64))
    col = np.concatenate(cols) if cols else np.zeros(0, np.int32)
    val = np.concatenate(vals) if vals else np.zeros(0, np.uint16)
    return Problem(G, n, p, rowptr, col, val, X, sf, beta, theta, clusters,
                   dict(config=config, seed=seed, dense=cfg["dense"], saturated=sat))


def many_problems_shapes(n_problems: int = 500, seed: int = 0):
    """(G, n, p, theta scale) of each problem of the many-uneven-problems
    workload (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(int(n_problems)):
        n = int(round(np.exp(rng.uniform(np.log(200.0), np.log(50000.0)))))
        G = int(rng.integers(5000, 20001))
        p = int(rng.integers(2, 17))
        scale = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
        out.append((G, n, p, scale))
    return out


def make_torch(config: str = "plain_sparse", seed: int = 0, G: int | None = None,
               n: int | None = None, device="cuda", chunk_cells: int = 1 << 27,
               mean_loc: float | None = None, p: int | None = None, theta_scale: float = 1.0):
    """Draw the same model on a torch device (full-size benchmark inputs).

    Returns a dict of device tensors: rowptr (int64), col (int32), val
    (int16 holding uint16 bits), X (float64 n x p, row-major), plus host
    copies of the truth and the design."""
    import torch

    cfg = config_params(config, p)
    if mean_loc is not None:
        cfg["mean_loc"] = float(mean_loc)
    G = cfg["G"] if G is None else int(G)
    n = cfg["n"] if n is None else int(n)
    p = cfg["p"]
    rng = np.random.default_rng(seed)
    X = design(cfg, n, rng)
    sf = rng.lognormal(0.0, 0.3, n)
    theta = rng.lognormal(0.0, 1.0, G) * float(theta_scale)
    beta = np.zeros((G, p))
    if cfg["b0_loc"] is None:
        beta[:, 0] = np.log(rng.lognormal(cfg["mean_loc"], 2.0, G))
    else:
        beta[:, 0] = rng.normal(cfg["b0_loc"], cfg["b0_sd"], G)
    de = rng.random(G) < 0.1
    beta[:, 1] = np.where(de, rng.normal(0.0, 1.0, G), 0.0)
    if cfg["covariates"]:
        beta[:, 2:2 + cfg["covariates"]] = rng.normal(0.0, 0.2, (G, cfg["covariates"]))
    if cfg["types"]:
        nt = cfg["types"] - 1
        beta[:, p - nt:] = rng.normal(0.0, 0.5, (G, nt))
    clusters = None
    pat_eff = None
    if cfg["patients"] > 1:
        sizes = patient_sizes(n, cfg["patients"], rng)
        clusters = np.repeat(np.arange(1, cfg["patients"] + 1), sizes).astype(np.int64)
        pat_eff = rng.normal(0.0, 0.3, (G, cfg["patients"]))

    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    Xd = torch.tensor(X, dtype=torch.float32, device=device)
    sfd = torch.tensor(sf, dtype=torch.float32, device=device)
    bd = torch.tensor(beta, dtype=torch.float32, device=device)
    thd = torch.tensor(theta, dtype=torch.float32, device=device)
    cld = None if clusters is None else torch.tensor(clusters - 1, device=device)
    ped = None if pat_eff is None else torch.tensor(pat_eff, dtype=torch.float32, device=device)
    rows_per = max(1, chunk_cells // n)
    counts, cols, vals = [], [], []
    sat = 0
    for g0 in range(0, G, rows_per):
        g1 = min(G, g0 + rows_per)
        eta = bd[g0:g1] @ Xd.T
        if ped is not None:
            eta = eta + ped[g0:g1][:, cld]
        mu = sfd[None, :] * torch.exp(eta)
        th = thd[g0:g1, None]
        shape = (1.0 / th).expand_as(mu).contiguous()
        lam = torch._standard_gamma(shape, generator=gen) * (th * mu)
        y = torch.poisson(lam, generator=gen)
        sat += int((y > 65535).sum().item())
        y = torch.clamp(y, max=65535.0)
        nz = y != 0
        counts.append(nz.sum(1))
        r, c = torch.nonzero(nz, as_tuple=True)
        cols.append(c.to(torch.int32))
        vals.append(y[r, c].to(torch.int32).to(torch.int16))
        del eta, mu, shape, lam, y, nz, r, c
    cnt = torch.cat(counts)
    rowptr = torch.zeros(G + 1, dtype=torch.int64, device=device)
    rowptr[1:] = torch.cumsum(cnt, 0)
    return dict(G=G, n=n, p=p, rowptr=rowptr, col=torch.cat(cols), val=torch.cat(vals),
                X=X, sf_true=sf, beta_true=beta, theta_true=theta, clusters=clusters,
                config=config, seed=seed, saturated=sat)
