#!/usr/bin/env python
"""Benchmark of devil's NB GLM path on B200: genes/sec for the whole fit
(size factors, theta_0, beta_0, IRLS) + theta (MOM and MLE with Cox-Reid)
+ bread + Wald/t test with BH adjustment.

Default workload ("wide"): G=20,000 genes x n=1,000,000 cells, CSR uint16
counts at ~8% nonzeros (1.6e9 entries, 9.6 GB), design p=32 (intercept,
condition, 30 one-hot cell types), normed_sum size factors, MLE theta.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--config wide|binary|plain_sparse|clustered|plain_small]

One JSON line on rank 0:
  value        genes/s of the chosen form with the counts resident in HBM
               (devil_fit_device + devil_test_de_device), all ranks' genes
               over the max-over-ranks time
  e2e          the same through the host-buffer C ABI (devil_fit +
               devil_test_de) from pinned host memory, copies included
  plain        the plain comparison form (DEVIL_FORM_PLAIN: per-cell FP32
               SIMT passes, no design grouping) timed in the same run on a
               random gene sample with the workload's size factors;
               chosen_vs_plain = chosen genes/s / plain genes/s
  roofline     the pass kernel with the largest share of the step
  cpu_baseline the FP64 oracle on a bounded random gene sample (host cores)
  parity       the timed fit (and the plain form) against the oracle on
               that sample, with the absolute |d beta| bar of 1e-5
Multi-GPU (torchrun): every rank fits its own gene shard (weak scaling);
the only exchange is the all-gather of p-values for the global BH step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("genes/sec fit+theta+sandwich+Wald, chosen vs plain GPU at |Δβ|≤1e-5; "
          "%HBM/TC peak")
FALLBACK_HBM_GBS = 6650.0
BETA_BAR = 1e-5        # absolute |d beta| on genes converging in both
THETA_BAR = 1e-4       # relative d theta
SAMPLE_SEED = 123      # gene sample shared by the CPU baseline, the reference arm and the plain form


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="wide")
    ap.add_argument("--genes", type=int, default=None)
    ap.add_argument("--cells", type=int, default=None)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=20.0,
                    help="CPU-baseline sample budget (our arm)")
    ap.add_argument("--ref-step-seconds", type=float, default=4.0,
                    help="per-step sample budget of the reference arm")
    ap.add_argument("--plain-seconds", type=float, default=3.0,
                    help="per-step budget of the plain form's gene sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--p", type=int, default=None,
                    help="design columns of a covariates-only config (continuous)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "tc_tf32"],
                    help="arithmetic of the Hessian contractions (DEVIL_PREC_*)")
    ap.add_argument("--problems", type=int, default=40,
                    help="--config many: the first K problems of the seeded 500-problem draw")
    ap.add_argument("--workers", type=int, default=4, help="--config many: concurrent streams")
    return ap.parse_args()


def workload_config(cfg_name, G, n, p, nnz):
    """The workload's identity, the same in both arms."""
    return {"workload": f"{cfg_name}: G={G} genes x n={n} cells, p={p}, CSR uint16 counts "
                        f"(NB Gamma-Poisson, seeded); normed_sum size factors, QR beta_0, "
                        f"IRLS (tol 1e-3, max_iter 200), MOM + MLE (Cox-Reid) theta, bread, "
                        f"Wald/t on the condition coefficient + BH",
            "genes": G, "cells": n, "p": p, "nnz": int(nnz), "nnz_frac": round(nnz / (G * n), 4),
            "l2": "inputs exceed L2 (CSR of all genes, re-read every pass)"}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def sample_order(G):
    return np.random.default_rng(SAMPLE_SEED).permutation(G)


# ----------------------------------------------------------------------
# inputs
# ----------------------------------------------------------------------
def make_inputs(args, rank, device):
    from devil_b200 import synthetic

    return synthetic.make_torch(args.config, seed=args.seed + rank, G=args.genes, n=args.cells,
                                device=device, p=args.p)


def normed_sum_offsets(rowptr, col, val, n):
    """log of normed_sum size factors (R/size_factors.R:75-88) with torch:
    input preparation of the reference arm, which times the CPU path only."""
    import torch

    colsum = torch.zeros(n, dtype=torch.float64, device=col.device)
    step = 1 << 27
    for a in range(0, col.numel(), step):
        b = min(col.numel(), a + step)
        colsum.index_add_(0, col[a:b].long(), val[a:b].to(torch.int32).bitwise_and(0xFFFF).double())
    ls = torch.log(colsum)
    return (ls - ls.mean()).cpu().numpy()


def host_rows(rowptr_np, col_np, val_np, genes):
    """CSR rows of `genes` (host numpy), in the given order."""
    genes = np.asarray(genes)
    starts, ends = rowptr_np[genes], rowptr_np[genes + 1]
    rp = np.zeros(len(genes) + 1, np.int64)
    rp[1:] = np.cumsum(ends - starts)
    sel = np.concatenate([np.arange(s, e) for s, e in zip(starts, ends)]) if len(genes) else \
        np.zeros(0, np.int64)
    return rp, col_np[sel], val_np[sel]


def device_rows(rowptr, col, val, genes_t):
    """CSR rows of the genes in genes_t (device tensors)."""
    import torch

    starts = rowptr[genes_t]
    lens = rowptr[genes_t + 1] - starts
    rp = torch.zeros(genes_t.numel() + 1, dtype=torch.int64, device=rowptr.device)
    rp[1:] = torch.cumsum(lens, 0)
    total = int(rp[-1].item())
    base = torch.repeat_interleave(starts - rp[:-1], lens, output_size=total)
    pos = base + torch.arange(total, device=rowptr.device)
    return rp, col[pos].contiguous(), val[pos].contiguous()


# ----------------------------------------------------------------------
# the oracle (CPU baseline, parity, reference arm)
# ----------------------------------------------------------------------
def oracle_step(orc, rowptr, col, val, n, X, off, c):
    Y = (rowptr, col, val.astype(np.float64), n)
    th0 = orc.estimate_dispersion(Y, off)
    b0 = orc.init_beta(Y, X, off)
    r = orc.cpu_fit(Y, X, off, th0, b0, orc.OD_MLE, 200, 1e-3, theta_mom=True)
    r["pval"] = orc.test_de(r["beta"], r["bread"], None, n, c)[0]
    return r


def parity_summary(beta, iters, theta, ref, beta_tol=BETA_BAR):
    """Agreement of a GPU fit with the FP64 oracle on the same genes, with
    the bars of the parity tests: iteration counts, absolute |d beta| and
    relative d theta (1e-3 < theta < 1e3) on genes that converge in both
    with the same iteration count."""
    beta, ref_beta = np.asarray(beta, float), np.asarray(ref["beta"], float)
    iters, ref_it = np.asarray(iters), np.asarray(ref["iters"])
    same = iters == ref_it
    conv = same & (ref_it < 200)
    db = np.abs(beta - ref_beta)
    th, ref_th = np.asarray(theta, float), np.asarray(ref["theta"], float)
    tm = conv & (ref_th > 1e-3) & (ref_th < 1e3)
    dth = np.abs(th - ref_th) / np.maximum(np.abs(ref_th), 1e-300)
    max_db = float(np.nanmax(db[conv])) if conv.any() else None
    return {"genes": int(len(iters)), "iters_agree": round(float(same.mean()), 4),
            "converged_compared": int(conv.sum()), "max_abs_dbeta": max_db,
            "max_rel_dtheta": float(np.nanmax(dth[tm])) if tm.any() else None,
            "bar_abs_dbeta": beta_tol,
            "within_bar": bool(max_db is not None and max_db <= beta_tol)}


# ----------------------------------------------------------------------
# reference arm: devil's CPU path (the FP64 restatement of cpu_fit +
# test_de) on the host cores, on the same workload and gene sample
# ----------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    orc.lib()
    # the same draw as rank 0 of our arm; the device only generates inputs
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    data = make_inputs(args, 0, dev)
    G, n, p = data["G"], data["n"], data["p"]
    nnz = int(data["rowptr"][-1].item())
    off = normed_sum_offsets(data["rowptr"], data["col"], data["val"], n)
    order = sample_order(G)
    need = min(G, 4096)
    # rows of the first `need` sample genes only, in sample order
    gt = torch.as_tensor(order[:need], dtype=torch.int64, device=data["rowptr"].device)
    rp_t, cl_t, vl_t = device_rows(data["rowptr"], data["col"], data["val"], gt)
    sub_rp, sub_col = rp_t.cpu().numpy(), cl_t.cpu().numpy()
    sub_val = vl_t.cpu().numpy().view(np.uint16)
    Xh = data["X"]
    del data, rp_t, cl_t, vl_t, gt
    c = np.zeros(p)
    c[1] = 1.0

    cursor = [0]

    def take(k):
        idx = (np.arange(cursor[0], cursor[0] + k)) % need
        cursor[0] += k
        return host_rows(sub_rp, sub_col, sub_val, idx)

    # warm-up steps: the first one (one gene) sizes the per-step sample
    k_step = 1
    for w in range(max(1, args.warmup)):
        rp, cl, vl = take(k_step)
        t0 = time.perf_counter()
        oracle_step(orc, rp, cl, vl, n, Xh, off, c)
        dt = time.perf_counter() - t0
        if w == 0:
            k_step = int(max(1, min(512, args.ref_step_seconds / max(dt, 1e-6))))
    times = []
    for _ in range(args.steps):
        rp, cl, vl = take(k_step)
        t0 = time.perf_counter()
        oracle_step(orc, rp, cl, vl, n, Xh, off, c)
        times.append(time.perf_counter() - t0)
    total = float(np.sum(times))
    gps = k_step * args.steps / total
    cores = orc.num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": gps, "unit": "genes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": max(1, args.warmup),
        "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.config, G, n, p, nnz),
        "cpu_baseline": {"value": gps, "unit": "genes/s", "cores": cores, "kind": "port",
                         "sample": f"each step fits {k_step} gene(s) of the workload (full n={n}, "
                                   f"the normed_sum offsets of all {G} genes), drawn in the "
                                   f"random order of the GPU arm's CPU-baseline sample; "
                                   f"FP64 restatement of cpu_fit + test_de on {cores} threads"},
        "e2e": {"value": gps, "unit": "genes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "genes_per_step": k_step,
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------
# clocks sampler
# ----------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"devil_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def read_bf16_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def read_traffic_ratio(name):
    """DRAM bytes per algorithmic byte of a pass kernel, from its committed
    ncu summary (line dram_per_alg_byte=...)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for ln in open(path):
            if ln.startswith("dram_per_alg_byte="):
                return float(ln.split("=", 1)[1])
    except Exception:
        pass
    return None


KERNELS = {"register": ("reg_pass_kernel<P={p},{pass},uint16> (register tiles)",
                        "irls_pass_traffic.txt"),
           "tensor": ("tc_irls_kernel<P={p},uint16> (tcgen05 kind::tf32 Hessian)", None),
           "tensor_wide": ("tcw_irls_kernel<XS,uint16> (tcgen05 kind::tf32 Hessian, p={p})", None),
           "shared": ("gen_pass_kernel<{pass},uint16> (shared-memory tiles, p={p})", None),
           "groups": ("grp_slices_kernel<{pass},uint16> (design groups, slice-major, p={p})",
                      "irls_grp_pass_traffic.txt")}
PASS_NAMES = ["irls", "mom", "mle", "bread_meat"]
PASS_TRAITS = ["PassIRLS", "PassMOM", "PassMLE", "PassSandwich"]


# ----------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------
class Fit:
    """Device buffers and C-ABI arguments of one fit + test_de on a CSR."""

    def __init__(self, L, lib, ctx, dev, rowptr, col, val, X, p, n, opts, contrast):
        import torch

        self.L, self.lib, self.ctx = L, lib, ctx
        G = rowptr.numel() - 1
        self.G, self.p, self.n = G, p, n
        f64 = dict(dtype=torch.float64, device=dev)
        i32 = dict(dtype=torch.int32, device=dev)
        self.keep = (rowptr, col, val, X)
        self.out = dict(beta=torch.empty(G * p, **f64), theta=torch.empty(G, **f64),
                        iters=torch.empty(G, **i32), bread=torch.empty(G * p * p, **f64),
                        theta_mom=torch.empty(G, **f64), status=torch.empty(G, **i32),
                        sf=torch.empty(n, **f64), off=torch.empty(n, **f64),
                        pval=torch.empty(G, **f64), padj=torch.empty(G, **f64),
                        lfc=torch.empty(G, **f64))
        o = self.out
        self.counts = L.Counts()
        self.counts.format = L.COUNTS_CSR_U16
        self.counts.n_genes, self.counts.n_cells, self.counts.nnz = G, n, int(rowptr[-1].item())
        self.counts.values, self.counts.ptr, self.counts.idx = (val.data_ptr(), rowptr.data_ptr(),
                                                                col.data_ptr())
        self.opts = opts
        self.X = X
        self.res = L.FitResult(ptr(o["beta"]), ptr(o["theta"]), ptr(o["iters"]), None,
                               ptr(o["bread"]), None, ptr(o["theta_mom"]), ptr(o["status"]),
                               ptr(o["sf"]), ptr(o["off"]), None)
        self.contrast = np.ascontiguousarray(contrast, np.float64)

    def fit(self):
        self.ctx.check(self.lib.devil_fit_device(self.ctx.h, C.byref(self.counts), ptr(self.X),
                                                 self.p, None, 0, C.byref(self.opts),
                                                 C.byref(self.res)))

    def test(self, adjust=True):
        L, o = self.L, self.out
        self.ctx.check(self.lib.devil_test_de_device(
            self.ctx.h, self.G, self.p, ptr(o["beta"]), ptr(o["bread"]), None, self.n,
            self.contrast.ctypes.data_as(C.c_void_p), L.ADJ_BH if adjust else L.ADJ_NONE, 10.0,
            ptr(o["pval"]), ptr(o["padj"]), ptr(o["lfc"])))


def ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def time_plain(args, L, lib, ctx, dev, ext, data, X, p, n, sf_dev, opts_chosen, contrast, G):
    """The plain form (and, for reference, the chosen form) on a random gene
    sample with the workload's size factors: genes/s and the fitted values."""
    import torch

    order = sample_order(G)

    def run(form, k, steps):
        genes = np.sort(order[:k])
        gt = torch.as_tensor(genes, dtype=torch.int64, device=dev)
        rp, cl, vl = device_rows(data["rowptr"], data["col"], data["val"], gt)
        o = L.FitOpts()
        C.memmove(C.byref(o), C.byref(opts_chosen), C.sizeof(o))
        o.form = form
        o.size_factors = L.SF_GIVEN
        o.size_factor_values = sf_dev.data_ptr()  # device pointer (device-buffer entry)
        f = Fit(L, lib, ctx, dev, rp, cl, vl, X, p, n, o, contrast)
        f.fit()  # untimed: workspace growth and first-launch costs
        f.test(adjust=False)
        ctx.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        for _ in range(steps):
            f.fit()
            f.test(adjust=False)
        e1.record(ext)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        return genes, f, ms

    # size the sample from a small probe so that a step takes ~plain_seconds
    k0 = min(G, 32)
    _, _, ms0 = run(L.FORM_PLAIN, k0, 1)
    per_gene = ms0 / k0
    k = int(max(k0, min(G, 2048, args.plain_seconds * 1e3 / max(per_gene, 1e-6))))
    steps = 2
    genes, fp, ms_plain = run(L.FORM_PLAIN, k, steps)
    _, fc, ms_chosen = run(L.FORM_CHOSEN, k, steps)
    o, oc = fp.out, fc.out
    res = {"genes": int(k), "steps": steps, "ms_per_step": ms_plain,
           "value": k / (ms_plain / 1e3), "unit": "genes/s",
           "chosen_same_sample": {"ms_per_step": ms_chosen, "value": k / (ms_chosen / 1e3)},
           "engines": {nm: ctx.engine(i) for i, nm in enumerate(PASS_NAMES)},
           "sample": f"{k} random genes of the workload (full n={n}), the workload's "
                     f"normed_sum size factors given; fit + theta + bread + Wald per step"}
    fitted = {"genes": genes,
              "plain": (o["beta"].view(k, p).cpu().numpy(), o["iters"].cpu().numpy(),
                        o["theta"].cpu().numpy()),
              "chosen": (oc["beta"].view(k, p).cpu().numpy(), oc["iters"].cpu().numpy(),
                         oc["theta"].cpu().numpy())}
    return res, fitted


def run_many(args):
    """Many uneven problems (one fit_devil per problem in the reference,
    R/main.R:164-273): the first K problems of the seeded 500-problem draw
    (n ~ LogUniform(200, 5e4), G ~ U{5000..20000}, p ~ U{2..16}, continuous
    designs, per-problem dispersion scale), fitted through the host-buffer
    C ABI (H2D copies of the counts and design, D2H of the results inside the
    timed region) as (a) one devil_fit_batch call on --workers concurrent
    streams and (b) one devil_fit call per problem.  Both are synchronous
    calls timed by the host clock (the batch spreads over several streams).
    fit + MOM and MLE theta + bread per problem."""
    import torch

    import devil_b200 as dv
    from devil_b200 import _lib as L
    from devil_b200 import synthetic

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    shapes = synthetic.many_problems_shapes(500, seed=args.seed)[: args.problems]
    dev = torch.device("cuda:0")
    keep, probs = [], (L.Problem * len(shapes))()
    res = (L.FitResult * len(shapes))()
    genes = cells = nnz_tot = 0
    for i, (G, n, p, sc) in enumerate(shapes):
        d = synthetic.make_torch("continuous", seed=args.seed + 1000 + i, G=G, n=n, p=p,
                                 theta_scale=sc, device=dev)
        rp = d["rowptr"].cpu().numpy()
        cl = d["col"].cpu().numpy()
        vl = d["val"].cpu().numpy().view(np.uint16)
        X = np.asfortranarray(d["X"]).ravel(order="F").astype(np.float64)
        out = {k: np.empty(sz, dt) for k, sz, dt in [
            ("beta", G * p, np.float64), ("theta", G, np.float64), ("iters", G, np.int32),
            ("bread", G * p * p, np.float64), ("theta_mom", G, np.float64), ("status", G, np.int32)]}
        keep.append((rp, cl, vl, X, out))
        c = probs[i].counts
        c.format = L.COUNTS_CSR_U16
        c.n_genes, c.n_cells, c.nnz = G, n, int(rp[-1])
        c.values, c.ptr, c.idx = vl.ctypes.data, rp.ctypes.data, cl.ctypes.data
        probs[i].X = X.ctypes.data
        probs[i].p = p
        probs[i].cluster_ends = None
        probs[i].n_clusters = 0
        res[i] = L.FitResult(out["beta"].ctypes.data, out["theta"].ctypes.data, out["iters"].ctypes.data,
                             None, out["bread"].ctypes.data, None, out["theta_mom"].ctypes.data,
                             out["status"].ctypes.data, None, None, None)
        genes += G
        cells += n
        nnz_tot += int(rp[-1])
        del d
    torch.cuda.empty_cache()
    ctx = dv.context(0)
    lib = L.load()
    opts = L.FitOpts()
    lib.devil_fit_opts_default(C.byref(opts))
    opts.overdispersion = L.OD_MLE
    opts.size_factors = L.SF_NORMED_SUM
    opts.compute_theta_mom = 1
    opts.precision = {"fp32": L.PREC_FP32, "tc_tf32": L.PREC_TC_TF32}[args.precision]
    K = len(shapes)

    def batch():
        ctx.check(lib.devil_fit_batch(ctx.h, K, probs, C.byref(opts), res, int(args.workers)))

    def loop():
        for i in range(K):
            ctx.check(lib.devil_fit(ctx.h, C.byref(probs[i].counts), C.c_void_p(probs[i].X), probs[i].p,
                                    None, 0, C.byref(opts), C.byref(res[i])))

    for _ in range(max(1, args.warmup)):
        batch()
    loop()
    clocks = Clocks(0)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        batch()
    tb = (time.perf_counter() - t0) / args.steps
    t0 = time.perf_counter()
    for _ in range(args.steps):
        loop()
    tl = (time.perf_counter() - t0) / args.steps
    clk = clocks.stop()
    conv = float(np.mean(np.concatenate([k[4]["status"] for k in keep]) == L.GENE_CONVERGED))
    line = {
        "metric": METRIC, "value": genes / tb, "unit": "genes/s", "n_gpus": 1, "steps": args.steps,
        "warmup": max(1, args.warmup), "ms_per_step": tb * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/tf32x3", "data": "synthetic",
        "config": {"workload": f"many uneven problems: the first {K} of a seeded draw of 500 "
                               f"(n ~ LogUniform(200, 5e4), G ~ U{{5000..20000}}, p ~ U{{2..16}}, "
                               f"continuous designs, per-problem dispersion scale), CSR uint16; "
                               f"normed_sum size factors, IRLS, MOM + MLE theta, bread per problem",
                   "problems": K, "genes": genes, "cells": cells, "nnz": nnz_tot,
                   "timing": "host clock around synchronous host-buffer calls (copies included)"},
        "many": {"batch": {"workers": args.workers, "ms": tb * 1e3, "problems_per_s": K / tb,
                           "genes_per_s": genes / tb},
                 "one_call_per_problem": {"ms": tl * 1e3, "problems_per_s": K / tl, "genes_per_s": genes / tl},
                 "batch_vs_loop": tl / tb, "converged_frac": round(conv, 4)},
        "clocks": clk, "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.config == "many":
        run_many(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)

    import devil_b200 as dv
    from devil_b200 import _lib as L
    from devil_b200 import distributed as D

    dev = torch.device(f"cuda:{local}")
    data = make_inputs(args, rank, dev)
    G, n, p = data["G"], data["n"], data["p"]
    nnz = int(data["rowptr"][-1].item())
    X = torch.tensor(np.asfortranarray(data["X"]).ravel(order="F"), dtype=torch.float64, device=dev)
    if data["clusters"] is not None:
        raise SystemExit("bench.py times unclustered workloads")
    ctx = dv.context(local)
    lib = L.load()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)
    opts = L.FitOpts()
    lib.devil_fit_opts_default(C.byref(opts))
    opts.overdispersion = L.OD_MLE
    opts.size_factors = L.SF_NORMED_SUM
    opts.compute_theta_mom = 1
    opts.form = L.FORM_CHOSEN
    opts.precision = {"fp32": L.PREC_FP32, "tc_tf32": L.PREC_TC_TF32}[args.precision]
    contrast = np.zeros(p)
    contrast[1] = 1.0
    main_fit = Fit(L, lib, ctx, dev, data["rowptr"], data["col"], data["val"], X, p, n, opts,
                   contrast)
    out = main_fit.out

    def dev_adjust(full, method):
        res = torch.empty_like(full)
        ctx.check(lib.devil_p_adjust_device(ctx.h, full.numel(), ptr(full), L.ADJ_BH, ptr(res)))
        return res

    sizes = [G] * world  # equal shards per rank (weak scaling)

    def step_device():
        main_fit.fit()
        main_fit.test(adjust=world == 1)
        if world > 1:
            # the one exchange: global BH needs every rank's p-values
            with torch.cuda.stream(ext):
                out["padj"].copy_(D.global_adjust_tensor(out["pval"], "BH", dev_adjust,
                                                         sizes=sizes))

    for _ in range(args.warmup):
        step_device()
    ctx.synchronize()
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ctx.synchronize()
    ctx.set_profiling(True)
    l0 = ctx.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(args.steps):
        step_device()
    e1.record(ext)
    e1.synchronize()
    ctx.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    launches = ctx.launches - l0
    prof = {k: ctx.profile(k) for k in range(4)}
    tc_flops = ctx.profile_tc_flops(0)
    rescued = ctx.irls_rescued
    ctx.set_profiling(False)
    clk = clocks.stop()
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * G / (ms / 1e3)
    engines = {name: ctx.engine(k) for k, name in enumerate(PASS_NAMES)}
    fitted_main = (out["beta"].view(G, p).cpu().numpy(), out["iters"].cpu().numpy(),
                   out["theta"].cpu().numpy())
    off_np = out["off"].cpu().numpy()
    sf_dev = out["sf"].clone()

    # ---- e2e through the host-buffer C ABI (pinned host inputs) ----
    e2e = None
    if not args.no_e2e:
        h_rowptr = data["rowptr"].cpu().pin_memory()
        h_col = data["col"].cpu().pin_memory()
        h_val = data["val"].cpu().pin_memory()
        h_X = X.cpu().pin_memory()
        hc = L.Counts()
        hc.format = L.COUNTS_CSR_U16
        hc.n_genes, hc.n_cells, hc.nnz = G, n, nnz
        hc.values, hc.ptr, hc.idx = h_val.data_ptr(), h_rowptr.data_ptr(), h_col.data_ptr()
        hb = {k: torch.empty(sz, dtype=dt).pin_memory() for k, sz, dt in [
            ("beta", G * p, torch.float64), ("theta", G, torch.float64),
            ("iters", G, torch.int32), ("bread", G * p * p, torch.float64),
            ("theta_mom", G, torch.float64), ("status", G, torch.int32),
            ("sf", n, torch.float64), ("off", n, torch.float64), ("pval", G, torch.float64),
            ("padj", G, torch.float64), ("lfc", G, torch.float64)]}
        hres = L.FitResult(ptr(hb["beta"]), ptr(hb["theta"]), ptr(hb["iters"]), None,
                           ptr(hb["bread"]), None, ptr(hb["theta_mom"]), ptr(hb["status"]),
                           ptr(hb["sf"]), ptr(hb["off"]), None)
        gathered_dev = torch.empty(G, dtype=torch.float64, device=dev)

        def step_host():
            ctx.check(lib.devil_fit(ctx.h, C.byref(hc), ptr(h_X), p, None, 0, C.byref(opts),
                                    C.byref(hres)))
            ctx.check(lib.devil_test_de(ctx.h, G, p, ptr(hb["beta"]), ptr(hb["bread"]), None, n,
                                        contrast.ctypes.data_as(C.c_void_p),
                                        L.ADJ_BH if world == 1 else L.ADJ_NONE, 10.0,
                                        ptr(hb["pval"]), ptr(hb["padj"]), ptr(hb["lfc"])))
            if world > 1:
                # global BH over every rank's p-values, as in the device step
                with torch.cuda.stream(ext):
                    gathered_dev.copy_(hb["pval"], non_blocking=True)
                    adj = D.global_adjust_tensor(gathered_dev, "BH", dev_adjust, sizes=sizes)
                    hb["padj"].copy_(adj, non_blocking=True)
                ctx.synchronize()

        step_host()  # workspace growth happens here, outside the timed region
        ctx.synchronize()
        if world > 1:
            dist.barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(ext)
        for _ in range(args.steps):
            step_host()
        f1.record(ext)
        f1.synchronize()
        ems = f0.elapsed_time(f1) / args.steps
        if world > 1:
            t = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        h2d = (G + 1) * 8 + nnz * 4 + nnz * 2 + n * p * 8
        d2h = (G * p * 8 + G * 8 * 2 + G * 4 * 2 + G * p * p * 8 + n * 16  # fit results
               + G * 8 * 3)                                                # pval, padj, lfc
        if world > 1:  # p-values up for the gather, globally adjusted slice back
            h2d += G * 8
            d2h += G * 8
        e2e = {"value": world * G / (ems / 1e3), "unit": "genes/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems}
        del h_rowptr, h_col, h_val

    # ---- the plain comparison form on a gene sample (rank 0) ----
    plain, fitted = None, None
    if rank == 0 and not args.no_plain:
        plain, fitted = time_plain(args, L, lib, ctx, dev, ext, data, X, p, n, sf_dev, opts,
                                   contrast, G)
        plain["chosen_vs_plain"] = value / world / plain["value"]
        plain["chosen_vs_plain_same_sample"] = plain["chosen_same_sample"]["value"] / plain["value"]
    if world > 1:
        dist.barrier()

    # ---- roofline of the pass kernel with the largest share ----
    peak, peak_kind = read_peaks()
    dom = max(range(4), key=lambda k: prof[k][1])
    n_l, t_ms, bytes_ = prof[dom]
    eng = engines[PASS_NAMES[dom]]
    kname, tfile = KERNELS.get(eng, (eng, None))
    kname = kname.format(p=p, **{"pass": PASS_TRAITS[dom]})
    roof = None
    if n_l > 0 and t_ms > 0:
        per_launch_s = t_ms / 1e3 / n_l
        alg_per_launch = bytes_ / n_l
        achieved = alg_per_launch / per_launch_s / 1e9
        # DRAM bytes per algorithmic byte from the committed ncu summary of
        # this kernel (IRLS pass of the same engine)
        ratio = read_traffic_ratio(tfile) if (tfile and dom == 0) else None
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": None if ratio is None else round(ratio * alg_per_launch, 1),
                "peak_source": f"{peak_kind} hbm_gbs", "kernel": kname,
                "launches": n_l, "avg_launch_ms": round(t_ms / n_l, 4),
                "alg_bytes_per_launch": round(alg_per_launch, 1),
                "share_of_step": round(t_ms / args.steps / ms, 4)}
        if eng == "tensor_wide" and tc_flops > 0:
            # the Hessian MMAs are the kernel's bound: FLOPs issued (3 split
            # TF32 products, padding included) against the TF32 tensor rate,
            # half the measured dense BF16 rate
            bf16, bf16_kind = read_bf16_peak()
            tf32_peak = bf16 / 2.0
            achieved_tf = tc_flops / (t_ms / 1e3) / 1e12
            roof = {"bound": "tensor", "achieved": round(achieved_tf, 1), "peak": round(tf32_peak, 1),
                    "unit": "TFLOP/s", "frac": round(achieved_tf / tf32_peak, 4), "traffic": None,
                    "peak_source": f"half the {bf16_kind} bf16_tflops (TF32 MMA rate)",
                    "kernel": kname, "launches": n_l, "avg_launch_ms": round(t_ms / n_l, 4),
                    "tc_flops_per_launch": round(tc_flops / n_l, 1),
                    "hbm_achieved_gbs": round(achieved, 1), "hbm_frac": round(achieved / peak, 4),
                    "share_of_step": round(t_ms / args.steps / ms, 4)}
        if eng == "groups":
            roof["tensor_note"] = (
                "no dense contraction left for the tensor cores: the design has few distinct rows, "
                "so the p x p terms are assembled from per-(gene, design row) sums, "
                "U*p^2 FLOPs per gene-pass against 4 B per nonzero read (slice-ordered copy)")
    passes = {name: {"launches": prof[k][0], "ms_per_step": round(prof[k][1] / args.steps, 3)}
              for k, name in enumerate(PASS_NAMES)}
    passes["other"] = {"ms_per_step": round(ms - sum(prof[k][1] for k in range(4)) / args.steps, 3),
                       "what": "validation, design copies, size factors, theta_0, grouping, "
                               "beta_0, finalize kernels, test_de"}

    # ---- CPU baseline: the oracle on a random gene sample of this workload ----
    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc

        orc.lib()
        rowptr_np = data["rowptr"].cpu().numpy()
        col_np = data["col"].cpu().numpy()
        val_np = data["val"].cpu().numpy().view(np.uint16)
        order = sample_order(G)
        # size the sample from one gene so the timed sample takes ~cpu_seconds
        rp, cl, vl = host_rows(rowptr_np, col_np, val_np, order[:1])
        t0 = time.perf_counter()
        oracle_step(orc, rp, cl, vl, n, data["X"], off_np, contrast)
        per_gene = time.perf_counter() - t0
        k = int(max(1, min(G, 2048, args.cpu_seconds / max(per_gene, 1e-6))))
        idx = order[:k]
        rp, cl, vl = host_rows(rowptr_np, col_np, val_np, idx)
        t0 = time.perf_counter()
        ref = oracle_step(orc, rp, cl, vl, n, data["X"], off_np, contrast)
        dt = time.perf_counter() - t0
        cpu = {"value": k / dt, "unit": "genes/s", "cores": orc.num_threads(), "kind": "port",
               "sample": f"{k} random genes of this workload (full n={n}, the fit's normed_sum "
                         f"offsets): the FP64 restatement of cpu_fit + test_de, OpenMP over "
                         f"genes or, for few genes, over cells; genes/s"}
        try:
            parity = parity_summary(fitted_main[0][idx], fitted_main[1][idx], fitted_main[2][idx],
                                    ref)
            parity["reference"] = "FP64 oracle on the CPU-baseline sample (same genes, offsets)"
            if fitted is not None:
                pos = {g: i for i, g in enumerate(fitted["genes"])}
                common = [i for i, g in enumerate(idx) if g in pos]
                if common:
                    sel = np.array([pos[idx[i]] for i in common])
                    refc = {kk: np.asarray(ref[kk])[common] for kk in ("beta", "iters", "theta")}
                    pb, pi, pt = fitted["plain"]
                    parity["plain_form"] = parity_summary(pb[sel], pi[sel], pt[sel], refc)
        except Exception as ex:  # the measurement stands without it
            parity = {"error": f"{type(ex).__name__}: {ex}"}

    line = {
        "metric": METRIC, "value": value, "unit": "genes/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        # per-cell arithmetic of the IRLS pass: FP32 in the register engine,
        # FP64 in the shared-memory and design-group engines
        "dtype": {"register": "f32", "tensor": "tf32x3", "tensor_wide": "tf32x3"}.get(engines["irls"], "f64"),
        "data": "synthetic",
        "config": workload_config(args.config, G, n, p, nnz),
        "chosen_vs_plain": None if plain is None else round(plain["chosen_vs_plain"], 2),
        "plain": plain,
        "roofline": roof, "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "clocks": clk,
        "gpu_launches": int(launches),
        "breakdown": {"form": "chosen", "engines": engines, "passes": passes,
                      "irls_rescued_genes": rescued,
                      "parallelism": f"genes sharded over {world} rank(s), no exchange during "
                                     f"the fit; p-values all-gathered for BH",
                      "saturated_counts": int(data.get("saturated", 0)),
                      "converged_frac": float((out["status"] == 0).float().mean().item()),
                      "mean_irls_iters": float(out["iters"].float().mean().item())},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
