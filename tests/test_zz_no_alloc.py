"""devil_p_adjust_device_static: the p-value adjustment for callers that
cannot allocate device memory (their HBM is held by another allocator, or
they cannot afford the device-wide synchronisation of cudaFree), checked
against devil_p_adjust_device on the same device buffers.

Two calls in a row (different inputs and methods) must each equal the
context-based entry point bit for bit, free device memory must not change
across a call once the first call on the device has set up, and m above the
static limit must be rejected with a message.  This file is collected last
(pytest collects files in name order) and also passes on its own."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 16
DEVIL_ERR_ARG = 1


def _inputs(m, seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.0, 1.0, m) ** 3
    p[rng.random(m) < 0.05] = np.nan  # NA: excluded from n
    p[:3] = [0.0, 1.0, 0.5]
    return p


def _reference(dv, pd, method):
    from devil_b200 import _lib as L
    ctx = dv.context()
    import torch
    torch.cuda.synchronize()
    ref = torch.empty_like(pd)
    ctx.check(L.load().devil_p_adjust_device(ctx.h, pd.numel(), C.c_void_p(pd.data_ptr()), method,
                                             C.c_void_p(ref.data_ptr())))
    ctx.synchronize()
    return ref.cpu().numpy()


def _static(pd, out, method):
    import torch
    from devil_b200 import _lib as L
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.load().devil_p_adjust_device_static(pd.numel(), C.c_void_p(pd.data_ptr()), method,
                                               C.c_void_p(out.data_ptr()), C.c_void_p(stream),
                                               err, 256)
    torch.cuda.synchronize()
    return rc, err.value.decode()


@pytest.mark.parametrize("m", [5000, LIMIT])
def test_static_matches_context_entry_twice(dv, m):
    import torch
    calls = [(_inputs(m, 1), 1), (_inputs(m, 2), 5)]  # BH, then BY on new inputs
    for k, (p, method) in enumerate(calls):
        pd = torch.tensor(p, dtype=torch.float64, device="cuda")
        ref = _reference(dv, pd, method)
        out = torch.full_like(pd, -1.0)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc, msg = _static(pd, out, method)
        free1 = torch.cuda.mem_get_info()[0]
        assert rc == 0, msg
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
        if k == 1:  # the first call has set up: nothing is allocated
            assert free1 == free0


def test_static_all_methods(dv):
    import torch
    pd = torch.tensor(_inputs(3000, 3), dtype=torch.float64, device="cuda")
    for method in range(6):
        out = torch.full_like(pd, -1.0)
        rc, msg = _static(pd, out, method)
        assert rc == 0, msg
        np.testing.assert_array_equal(out.cpu().numpy(), _reference(dv, pd, method))


def test_static_rejects_oversize(dv):
    import torch
    pd = torch.zeros(LIMIT + 1, dtype=torch.float64, device="cuda")
    out = torch.zeros_like(pd)
    rc, msg = _static(pd, out, 1)
    assert rc == DEVIL_ERR_ARG
    assert "exceeds the static limit" in msg
