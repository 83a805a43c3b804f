#!/usr/bin/env python
"""Benchmark of devil's NB GLM path on B200: genes/sec for
fit (size factors, theta_0, beta_0, IRLS) + theta (MOM and MLE) + bread +
Wald/t test with BH, on the sparse plain workload (G=20,000 genes x
n=100,000 cells, CSR uint16, ~10% nonzeros, p=4).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--form plain] [--config plain_sparse|plain_small|clustered|wide]

One JSON line on rank 0.  value = genes/s with inputs resident in HBM
(devil_fit_device + devil_test_de_device); e2e = the same through the
host-buffer C ABI (devil_fit + devil_test_de) with pinned host inputs.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="chosen", choices=["chosen", "plain"])
    ap.add_argument("--config", default="plain_sparse")
    ap.add_argument("--genes", type=int, default=None)
    ap.add_argument("--cells", type=int, default=None)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def workload_desc(cfg, G, n, p, nnz=None):
    d = {"workload": f"{cfg}: G={G} genes x n={n} cells, p={p}, CSR uint16 counts "
                     f"(NB Gamma-Poisson, seeded); normed_sum size factors, QR beta_0, "
                     f"IRLS (tol 1e-3, max_iter 200), MOM + MLE (Cox-Reid) theta, bread, "
                     f"Wald/t on the condition coefficient + BH",
         "genes": G, "cells": n, "p": p}
    if nnz is not None:
        d["nnz"] = int(nnz)
        d["nnz_frac"] = round(nnz / (G * n), 4)
    return d


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ----------------------------------------------------------------------
# CPU baseline / reference arm: the FP64 oracle (OpenMP over genes)
# ----------------------------------------------------------------------
def oracle_step(orc, rowptr, col, val, n, X, off, c):
    Y = (rowptr, col, val.astype(np.float64), n)
    th0 = orc.estimate_dispersion(Y, off)
    b0 = orc.init_beta(Y, X, off)
    r = orc.cpu_fit(Y, X, off, th0, b0, orc.OD_MLE, 200, 1e-3, theta_mom=True)
    r["pval"] = orc.test_de(r["beta"], r["bread"], None, n, c)[0]
    return r


def parity_summary(beta, iters, theta, ref, beta_tol=1e-5):
    """Agreement of the GPU fit with the FP64 oracle on the same genes, with
    the bars of the parity tests: iteration counts, |d beta| (absolute for
    |beta| <= 1, relative above) and relative d theta on genes that converge
    in both with the same count (theta resolvable: 1e-3 < theta < 1e3)."""
    beta, ref_beta = np.asarray(beta, float), np.asarray(ref["beta"], float)
    iters, ref_it = np.asarray(iters), np.asarray(ref["iters"])
    same = iters == ref_it
    conv = same & (ref_it < 200)
    db = np.abs(beta - ref_beta) / np.maximum(1.0, np.abs(ref_beta))
    th, ref_th = np.asarray(theta, float), np.asarray(ref["theta"], float)
    tm = conv & (ref_th > 1e-3) & (ref_th < 1e3)
    dth = np.abs(th - ref_th) / np.maximum(np.abs(ref_th), 1e-300)
    max_db = float(np.nanmax(db[conv])) if conv.any() else None
    return {"genes": int(len(iters)), "iters_agree": round(float(same.mean()), 4),
            "converged_compared": int(conv.sum()), "max_dbeta": max_db,
            "max_rel_dtheta": float(np.nanmax(dth[tm])) if tm.any() else None,
            "bar_dbeta": beta_tol,
            "within_bar": bool(max_db is not None and max_db <= beta_tol)}


def timed_oracle(orc, prob_rows, n, X, off, c, target_s):
    """Time the oracle on a gene sample sized to about target_s seconds.
    prob_rows(k) -> (rowptr, col, val) of the first k sample genes."""
    k = 8
    rp, cl, vl = prob_rows(k)
    t0 = time.perf_counter()
    oracle_step(orc, rp, cl, vl, n, X, off, c)
    dt = time.perf_counter() - t0
    per_gene = dt / k
    k2 = int(max(8, min(2048, target_s / max(per_gene, 1e-6))))
    rp, cl, vl = prob_rows(k2)
    t0 = time.perf_counter()
    r = oracle_step(orc, rp, cl, vl, n, X, off, c)
    dt = time.perf_counter() - t0
    return k2, dt, r


def run_reference(args):
    """--impl reference: devil's CPU path (R/main.R cpu_fit), restated in
    FP64 C with OpenMP over genes (the R package itself cannot run here),
    timed on the host cores on bounded samples of the workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from devil_b200 import synthetic

    orc.lib()
    cfg = synthetic.CONFIGS[args.config]
    G = args.genes or cfg["G"]
    n = args.cells or cfg["n"]
    per_step = max(4.0, args.cpu_seconds / 2)
    # sample genes drawn from the same model at full cell count
    k_probe = 8
    P = synthetic.make(args.config, seed=args.seed + 1000, G=k_probe, n=n)
    off = np.log(P.sf_true)
    c = np.zeros(P.p)
    c[1] = 1.0
    t0 = time.perf_counter()
    oracle_step(orc, P.rowptr, P.col, P.val, n, P.X, off, c)
    per_gene = (time.perf_counter() - t0) / k_probe
    k = int(max(8, min(2048, per_step / max(per_gene, 1e-6))))
    S = synthetic.make(args.config, seed=args.seed + 1001, G=k, n=n)
    off = np.log(S.sf_true)
    for _ in range(args.warmup):
        pass  # the oracle has no warm-up state; untimed steps would only repeat the work
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle_step(orc, S.rowptr, S.col, S.val, n, S.X, off, c)
        times.append(time.perf_counter() - t0)
    dt = float(np.mean(times))
    gps = k / dt
    cores = orc.num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": gps, "unit": "genes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3 * (G / k), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload_desc(args.config, G, n, cfg["p"]), form="cpu reference"),
        "cpu_baseline": {"value": gps, "unit": "genes/s", "cores": cores, "kind": "port",
                         "sample": f"{k} genes x {n} cells per step drawn from the same model "
                                   f"(given size factors), genes/s extrapolated to G={G}"},
        "e2e": {"value": gps, "unit": "genes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
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


def read_traffic_ratio():
    """DRAM bytes per algorithmic byte of the IRLS pass kernel, from the
    committed ncu summary (key dram_per_alg_byte=...)."""
    path = os.path.join(ROOT, "profiles", "irls_pass_traffic.txt")
    try:
        for ln in open(path):
            if ln.startswith("dram_per_alg_byte="):
                return float(ln.split("=", 1)[1])
    except Exception:
        pass
    return None


# ----------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------
def main():
    args = parse()
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
    from devil_b200 import synthetic

    cfg = synthetic.CONFIGS[args.config]
    data = synthetic.make_torch(args.config, seed=args.seed + rank, G=args.genes, n=args.cells,
                                device=f"cuda:{local}")
    G, n, p = data["G"], data["n"], data["p"]
    nnz = int(data["rowptr"][-1].item())
    dev = torch.device(f"cuda:{local}")
    X = torch.tensor(np.asfortranarray(data["X"]).ravel(order="F"), dtype=torch.float64, device=dev)
    rowptr, col, val = data["rowptr"], data["col"], data["val"]
    clusters = data["clusters"]
    ends = None
    if clusters is not None:
        _, ends = dv.cluster_blocks(clusters)
    ctx = dv.context(local)
    lib = L.load()
    ext = torch.cuda.ExternalStream(ctx.stream, device=dev)

    f64 = dict(dtype=torch.float64, device=dev)
    i32 = dict(dtype=torch.int32, device=dev)
    out = dict(beta=torch.empty(G * p, **f64), theta=torch.empty(G, **f64),
               iters=torch.empty(G, **i32), bread=torch.empty(G * p * p, **f64),
               theta_mom=torch.empty(G, **f64), status=torch.empty(G, **i32),
               sf=torch.empty(n, **f64), off=torch.empty(n, **f64),
               sw=torch.empty(G * p * p, **f64) if ends is not None else None,
               pval=torch.empty(G, **f64), padj=torch.empty(G, **f64), lfc=torch.empty(G, **f64))
    counts = L.Counts()
    counts.format = L.COUNTS_CSR_U16
    counts.n_genes, counts.n_cells, counts.nnz = G, n, nnz
    counts.values, counts.ptr, counts.idx = val.data_ptr(), rowptr.data_ptr(), col.data_ptr()
    opts = L.FitOpts()
    lib.devil_fit_opts_default(C.byref(opts))
    opts.overdispersion = L.OD_MLE
    opts.size_factors = L.SF_NORMED_SUM
    opts.compute_theta_mom = 1
    opts.form = L.FORM_PLAIN if args.form == "plain" else L.FORM_CHOSEN
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    res = L.FitResult(ptr(out["beta"]), ptr(out["theta"]), ptr(out["iters"]), None,
                      ptr(out["bread"]), ptr(out["sw"]), ptr(out["theta_mom"]),
                      ptr(out["status"]), ptr(out["sf"]), ptr(out["off"]), None)
    contrast = np.zeros(p)
    contrast[1] = 1.0
    ends_np = None if ends is None else np.ascontiguousarray(ends, np.int32)
    gathered = torch.empty(G * world, **f64) if world > 1 else None
    gadj = torch.empty(G * world, **f64) if world > 1 else None

    def step_device():
        ctx.check(lib.devil_fit_device(ctx.h, C.byref(counts), ptr(X), p,
                                       None if ends_np is None else ends_np.ctypes.data_as(C.c_void_p),
                                       0 if ends_np is None else len(ends_np), C.byref(opts),
                                       C.byref(res)))
        ctx.check(lib.devil_test_de_device(
            ctx.h, G, p, ptr(out["beta"]), ptr(out["bread"]), ptr(out["sw"]), n,
            contrast.ctypes.data_as(C.c_void_p), L.ADJ_BH, 10.0, ptr(out["pval"]),
            ptr(out["padj"]), ptr(out["lfc"])))
        if world > 1:
            # the one exchange: global BH needs every rank's p-values
            with torch.cuda.stream(ext):
                dist.all_gather_into_tensor(gathered, out["pval"])
            ctx.check(lib.devil_p_adjust_device(ctx.h, G * world, ptr(gathered), L.ADJ_BH,
                                                ptr(gadj)))

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
    ctx.set_profiling(False)
    clk = clocks.stop()
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * G / (ms / 1e3)

    # ---- e2e through the host-buffer C ABI (pinned host inputs) ----
    e2e = None
    if not args.no_e2e:
        h_rowptr = rowptr.cpu().pin_memory()
        h_col = col.cpu().pin_memory()
        h_val = val.cpu().pin_memory()
        h_X = torch.tensor(np.asfortranarray(data["X"]).ravel(order="F"),
                           dtype=torch.float64).pin_memory()
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

        def step_host():
            ctx.check(lib.devil_fit(ctx.h, C.byref(hc), ptr(h_X), p, None, 0, C.byref(opts),
                                    C.byref(hres)))
            ctx.check(lib.devil_test_de(ctx.h, G, p, ptr(hb["beta"]), ptr(hb["bread"]), None, n,
                                        contrast.ctypes.data_as(C.c_void_p), L.ADJ_BH, 10.0,
                                        ptr(hb["pval"]), ptr(hb["padj"]), ptr(hb["lfc"])))
            if world > 1:
                # global BH over every rank's p-values, as in the device step
                with torch.cuda.stream(ext):
                    dist.all_gather_into_tensor(gathered, hb["pval"].to(dev, non_blocking=True))
                ctx.check(lib.devil_p_adjust_device(ctx.h, G * world, ptr(gathered), L.ADJ_BH,
                                                    ptr(gadj)))
                with torch.cuda.stream(ext):
                    hb["padj"].copy_(gadj[rank * G:(rank + 1) * G], non_blocking=True)
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
        h2d = (G + 1) * 8 + nnz * 4 + nnz * 2 + n * p * 8 + G * p * 8 + G * p * p * 8
        d2h = G * p * 8 + G * 8 * 2 + G * 4 * 2 + G * p * p * 8 + n * 16 + G * 8 * 3
        if world > 1:  # p-values up for the gather, globally adjusted slice back
            h2d += G * 8
            d2h += G * 8
        e2e = {"value": world * G / (ems / 1e3), "unit": "genes/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems}

    # ---- roofline of the dominant kernel (IRLS cell pass) ----
    engines = {name: ctx.engine(k) for k, name in enumerate(["irls", "mom", "mle", "bread_meat"])}
    kernel = {"register": f"reg_pass_kernel<P={p},PassIRLS,uint16> (register tiles)",
              "tensor": f"tc_irls_kernel<P={p},uint16> (tcgen05 kind::tf32 Hessian, 128-gene tiles)",
              "shared": f"gen_pass_kernel<PassIRLS,uint16> (shared-memory tiles, p={p})",
              "groups": f"grp_pass_kernel<PassIRLS,uint16> (design groups, p={p})"}.get(
                  engines["irls"], engines["irls"])
    n_l, t_ms, bytes_ = prof[0]
    peak, peak_kind = read_peaks()
    roof = None
    if n_l > 0 and t_ms > 0:
        per_launch_s = t_ms / 1e3 / n_l
        alg_per_launch = bytes_ / n_l
        achieved = alg_per_launch / per_launch_s / 1e9
        # the committed DRAM/algorithmic ratio was measured on the register engine
        ratio = read_traffic_ratio() if engines["irls"] == "register" else None
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": None if ratio is None else round(ratio * alg_per_launch, 1),
                "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": kernel,
                "launches": n_l, "avg_launch_ms": round(t_ms / n_l, 4),
                "alg_bytes_per_launch": round(alg_per_launch, 1),
                "share_of_step": round(t_ms / args.steps / ms, 4)}

    # The IRLS cell pass is bound on the SM side, not by HBM: per active
    # gene and cell it evaluates exp2 and a reciprocal on the special
    # function units (16 results per clock per SM, nominal) besides the
    # FMAs (register engine) or the TF32 MMAs (tensor engine).  Report its
    # gene-cell rate against that SFU ceiling as well.
    if roof is not None and engines["irls"] in ("register", "tensor") and t_ms > 0:
        gene_cells = float(out["iters"].double().sum().item()) * n * args.steps
        sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
        ceiling = 148 * 16 * sm_mhz * 1e6 / 2.0  # two SFU results per gene-cell
        achieved_gc = gene_cells / (t_ms / 1e3)
        roof["compute"] = {"unit": "gene-cells/s", "achieved": round(achieved_gc, -6),
                           "sfu_ceiling": round(ceiling, -6), "frac": round(achieved_gc / ceiling, 4),
                           "note": "nominal SFU rate at the sampled SM clock; 2 SFU ops per gene-cell"}

    passes = {name: {"launches": prof[k][0], "ms_per_step": round(prof[k][1] / args.steps, 3)}
              for k, name in enumerate(["irls", "mom", "mle", "bread_meat"])}

    # ---- CPU baseline: the oracle on a sample of this workload ----
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc

        orc.lib()
        h_rowptr_np = rowptr.cpu().numpy()
        h_col_np = col.cpu().numpy()
        h_val_np = val.cpu().numpy().view(np.uint16)
        off_np = out["off"].cpu().numpy()
        rng = np.random.default_rng(123)
        order = rng.permutation(G)

        def rows(k):
            idx = order[:k]
            starts, ends_ = h_rowptr_np[idx], h_rowptr_np[idx + 1]
            rp = np.zeros(k + 1, np.int64)
            rp[1:] = np.cumsum(ends_ - starts)
            sel = np.concatenate([np.arange(s, e) for s, e in zip(starts, ends_)])
            return rp, h_col_np[sel], h_val_np[sel]

        k, dt, ref = timed_oracle(orc, rows, n, data["X"], off_np, contrast, args.cpu_seconds)
        cpu = {"value": k / dt, "unit": "genes/s", "cores": orc.num_threads(), "kind": "port",
               "sample": f"{k} randomly chosen genes of this workload (full n={n}), the FP64 "
                         f"restatement of cpu_fit + test_de with OpenMP over genes; genes/s"}
        # the same genes of the timed GPU fit against the oracle's results
        try:
            idx = order[:k]
            parity = parity_summary(out["beta"].view(G, p).cpu().numpy()[idx],
                                    out["iters"].cpu().numpy()[idx],
                                    out["theta"].cpu().numpy()[idx], ref)
            parity["reference"] = "FP64 oracle on the CPU-baseline sample (same genes, offsets)"
        except Exception as ex:  # the measurement stands without it
            parity = {"error": f"{type(ex).__name__}: {ex}"}

    line = {
        "metric": METRIC, "value": value, "unit": "genes/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        # per-cell arithmetic of the IRLS pass: FP32 in the register engine,
        # FP64 in the shared-memory and design-group engines
        "dtype": "f32" if engines["irls"] in ("register", "tensor") else "f64", "data": "synthetic",
        "config": dict(workload_desc(args.config, G, n, p, nnz), form=args.form,
                       l2="inputs exceed L2 (CSR of all genes, re-read every IRLS pass)",
                       parallelism=f"genes sharded over {world} rank(s), no exchange during "
                                   f"the fit; p-values all-gathered for BH",
                       passes=passes, engines=engines,
                       saturated_counts=int(data.get("saturated", 0)),
                       converged_frac=float((out["status"] == 0).float().mean().item()),
                       mean_irls_iters=float(out["iters"].float().mean().item())),
        "roofline": roof, "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "clocks": clk,
        "gpu_launches": int(launches),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
