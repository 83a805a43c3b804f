"""World-size-2 gloo test of the multi-rank host logic: genes sharded across
ranks, p-values all-gathered, BH applied globally.  The per-gene numbers
come from the oracle, so no GPU is needed; the result must
equal the single-process BH of the whole gene set exactly."""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, pvals, out_path):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist

    import oracle
    from devil_b200 import distributed as D

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rowptr = np.arange(0, 11 * (len(pvals) + 1), 11)[: len(pvals) + 1]
        b, e = D.shard_ranges(rowptr, world, n_cells=100)[rank]
        local = pvals[b:e]
        adj = D.global_adjust(local, "BH", adjust=lambda p, m: oracle.p_adjust(p, m))
        # the tensor form the multi-GPU benchmark step runs (device tensors
        # under NCCL; CPU tensors here), with the same adjuster
        import torch
        adj_t = D.global_adjust_tensor(
            torch.as_tensor(local, dtype=torch.float64), "BH",
            adjust=lambda full, m: torch.as_tensor(oracle.p_adjust(full.numpy(), m)))
        np.testing.assert_array_equal(adj_t.numpy(), adj)
        np.save(out_path + f".{rank}.npy", np.concatenate([[b, e], adj]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_global_bh_matches_single_process(tmp_path, orc, world):
    import torch.multiprocessing as mp

    rng = np.random.default_rng(0)
    p = rng.uniform(size=101) ** 3
    p[[3, 50]] = np.nan
    out = str(tmp_path / "adj")
    mp.start_processes(_worker, args=(world, _free_port(), p, out), nprocs=world, join=True,
                       start_method="spawn")
    full = np.full(len(p), -1.0)
    for r in range(world):
        a = np.load(out + f".{r}.npy")
        b, e = int(a[0]), int(a[1])
        full[b:e] = a[2:]
    expect = orc.p_adjust(p, "BH")
    np.testing.assert_array_equal(np.isnan(full), np.isnan(expect))
    np.testing.assert_array_equal(full[~np.isnan(full)], expect[~np.isnan(expect)])


def test_shard_ranges_cover_and_balance():
    from devil_b200.distributed import shard_ranges

    rng = np.random.default_rng(1)
    nnz = rng.integers(0, 5000, 1000)
    rowptr = np.concatenate([[0], np.cumsum(nnz)])
    for world in (1, 2, 3, 8):
        r = shard_ranges(rowptr, world, n_cells=2000)
        assert r[0][0] == 0 and r[-1][1] == 1000
        assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
        cost = [(nnz[b:e] + 2000).sum() for b, e in r]
        assert max(cost) - min(cost) <= 2 * (5000 + 2000)
