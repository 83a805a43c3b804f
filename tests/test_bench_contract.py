"""bench.py's reference arm on CPU: one JSON line with the keys and types of
the benchmark contract (the arm times the FP64 oracle on the host cores), and
nothing but a clean exit on ranks other than 0."""
import json
import os
import subprocess
import sys

from conftest import ROOT

ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "1", "--genes", "200",
        "--cells", "2000", "--cpu-seconds", "1"]


def _run(env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + ARGS, cwd=ROOT,
                          env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key, typ in [("metric", str), ("value", float), ("unit", str), ("n_gpus", int),
                     ("steps", int), ("warmup", int), ("ms_per_step", float),
                     ("higher_is_better", bool), ("scaling", str), ("dtype", str), ("data", str),
                     ("config", dict), ("cpu_baseline", dict), ("e2e", dict)]:
        assert isinstance(d[key], typ), key
    assert d["value"] > 0 and d["unit"] == "genes/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["vs_baseline"] is None
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert isinstance(cb["sample"], str) and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_parity_summary_applies_the_test_bars():
    import importlib.util
    import numpy as np

    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    ref = {"beta": np.array([[0.5, -2.0], [3.0, 0.1], [-1.0, 0.0], [9.0, 9.0]]),
           "iters": np.array([5, 7, 200, 4]), "theta": np.array([0.5, 2e-4, 1.0, 10.0])}
    beta = ref["beta"] + np.array([[2e-6, 0.0], [0.0, 0.0], [0.5, 0.5], [0.0, 0.0]])
    beta[1, 0] = 3.0 + 4e-6
    iters = np.array([5, 7, 200, 5])  # gene 3 differs by one step: not compared
    theta = ref["theta"] * np.array([1 + 1e-5, 5.0, 1.0, 1.0])  # gene 1: theta < 1e-3, ignored
    s = bench.parity_summary(beta, iters, theta, ref)
    assert s["genes"] == 4 and s["iters_agree"] == 0.75 and s["converged_compared"] == 2
    assert abs(s["max_abs_dbeta"] - 4e-6) < 1e-12 and s["within_bar"]
    assert abs(s["max_rel_dtheta"] - 1e-5) < 1e-12
    # the bar is absolute: 2e-5 on |beta| = 2 fails it
    beta[0, 1] += 2e-5
    assert not bench.parity_summary(beta, iters, theta, ref)["within_bar"]
