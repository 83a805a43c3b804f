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
