"""The device-pointer entry points: devil_fit_device (context stream) and
devil_fit_async (the caller's stream) on CSR uint16 counts already in GPU
memory give exactly the results of devil_fit on host buffers (the same
kernels in the same order; every reduction has a fixed order)."""
import ctypes as C

import numpy as np
import pytest

from devil_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    return synthetic.make("plain_sparse", seed=23, G=200, n=5000)


def _device_fit(dv, P, stream=None):
    import torch
    from devil_b200 import _lib as L

    lib = L.load()
    ctx = dv.context()
    dev = torch.device("cuda:0")
    rp = torch.tensor(P.rowptr, dtype=torch.int64, device=dev)
    col = torch.tensor(P.col, dtype=torch.int32, device=dev)
    val = torch.tensor(P.val.astype(np.uint16).view(np.int16), device=dev)  # uint16 bits
    X = torch.tensor(np.asfortranarray(P.X).ravel(order="F"), dtype=torch.float64, device=dev)
    G, n, p = P.G, P.n, P.p
    out = {k: torch.full((sz,), -7, dtype=dt, device=dev) for k, sz, dt in [
        ("beta", G * p, torch.float64), ("theta", G, torch.float64), ("iters", G, torch.int32),
        ("bread", G * p * p, torch.float64), ("status", G, torch.int32)]}
    counts = L.Counts()
    counts.format = L.COUNTS_CSR_U16
    counts.n_genes, counts.n_cells, counts.nnz = G, n, int(P.rowptr[-1])
    counts.values, counts.ptr, counts.idx = val.data_ptr(), rp.data_ptr(), col.data_ptr()
    opts = L.FitOpts()
    lib.devil_fit_opts_default(C.byref(opts))
    opts.overdispersion = L.OD_MLE
    opts.size_factors = L.SF_NORMED_SUM
    ptr = lambda t: C.c_void_p(t.data_ptr())
    res = L.FitResult(ptr(out["beta"]), ptr(out["theta"]), ptr(out["iters"]), None,
                      ptr(out["bread"]), None, None, ptr(out["status"]), None, None, None)
    torch.cuda.synchronize()
    if stream is None:
        rc = lib.devil_fit_device(ctx.h, C.byref(counts), ptr(X), p, None, 0, C.byref(opts),
                                  C.byref(res))
        ctx.check(rc)
        ctx.synchronize()
    else:
        own = lib.devil_ctx_stream(ctx.h)
        rc = lib.devil_fit_async(ctx.h, C.c_void_p(stream.cuda_stream), C.byref(counts), ptr(X),
                                 p, None, 0, C.byref(opts), C.byref(res))
        ctx.check(rc)
        assert lib.devil_ctx_stream(ctx.h) == own  # the context's stream is back
        stream.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def test_device_and_async_entries_match_host_fit(dv, problem):
    import torch

    P = problem
    host = dv.fit_devil((P.rowptr, P.col, P.val, P.n), P.X, overdispersion="MLE",
                        size_factors="normed_sum")
    d = _device_fit(dv, P)
    s = torch.cuda.Stream()
    a = _device_fit(dv, P, stream=s)
    G, p = P.G, P.p
    for r in (d, a):
        np.testing.assert_array_equal(r["beta"].reshape(G, p), host["beta"])
        np.testing.assert_array_equal(r["theta"], host["overdispersion"])
        np.testing.assert_array_equal(r["iters"], host["iterations"]["beta_iters"])
        np.testing.assert_array_equal(r["bread"].reshape(G, p, p).transpose(0, 2, 1),
                                      host["beta_sandwiches_null"])
