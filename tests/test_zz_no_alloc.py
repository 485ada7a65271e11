"""The pair sum for callers that cannot allocate device memory.

Such callers (hosts that hand over only their own buffers, loops that must
never call cudaMalloc mid-run) use f3d_pair_sum_noalloc, whose scratch is a
fixed device array inside the library.  These tests call it through the C
ABI and check it against f3d_pair_sum with a caller workspace, on two calls
in a row (the array keeps the previous call's contents, so the second call
shows that what must start at zero is cleared).  This file is collected
last so that a stop-at-first-failure run has run every other test first.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _inputs(ns, nt, seed):
    rng = np.random.default_rng(seed)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
    return (t(rng.random((ns, 3))), t(rng.random((nt, 3))), t(rng.normal(size=(ns, 3))),
            t(rng.normal(size=(ns, 3))))


def _with_workspace(lib, kernel, prec, rs, rt, d, n, out):
    nb = ctypes.c_size_t(0)
    assert lib.f3d_pair_workspace_bytes(kernel, prec, rs.shape[0], rt.shape[0], None, ctypes.byref(nb)) == 0
    ws = torch.zeros(max(nb.value, 256), dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.f3d_pair_sum(kernel, prec, 0, rs.data_ptr(), rt.data_ptr(), d.data_ptr(), n.data_ptr(), None,
                          None, out.data_ptr(), rs.shape[0], rt.shape[0], 1.0, 5e-3, 1e-5, 0, None,
                          ws.data_ptr(), ws.numel(), st)
    assert rc == 0


def _noalloc(lib, kernel, prec, rs, rt, d, n, out):
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.f3d_pair_sum_noalloc(kernel, prec, 0, rs.data_ptr(), rt.data_ptr(), d.data_ptr(), n.data_ptr(),
                                  None, None, out.data_ptr(), rs.shape[0], rt.shape[0], 1.0, 5e-3, 1e-5, 0,
                                  st)
    assert rc == 0


@pytest.mark.parametrize("kernel,prec", [(1, 0), (0, 0), (1, 1)])
def test_noalloc_matches_workspace_entry_point_twice(kernel, prec):
    from fiber3d_b200 import _lib
    lib = _lib.lib()
    rs, rt, d, n = _inputs(3000, 2000, 11)      # 2000 targets: the sum is split, scratch is used
    ref = torch.empty(3 * 2000, dtype=torch.float64, device="cuda")
    _with_workspace(lib, kernel, prec, rs, rt, d, n, ref)
    for call in range(2):
        out = torch.full((3 * 2000,), float("nan"), dtype=torch.float64, device="cuda")
        _noalloc(lib, kernel, prec, rs, rt, d, n, out)
        torch.cuda.synchronize()
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < TOL64, f"call {call}"
    # a different size in between still leaves nothing behind for the next call
    rs2, rt2, d2, n2 = _inputs(700, 5000, 12)
    out2 = torch.empty(3 * 5000, dtype=torch.float64, device="cuda")
    _noalloc(lib, kernel, prec, rs2, rt2, d2, n2, out2)
    out = torch.empty_like(ref)
    _noalloc(lib, kernel, prec, rs, rt, d, n, out)
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < TOL64
    assert lib.f3d_get_device_error(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from fiber3d_b200 import _lib
    lib = _lib.lib()
    # FP32C packs 48 bytes per source: 10^6 sources need more than the 32 MiB array
    rc = lib.f3d_pair_sum_noalloc(0, 1, 0, None, None, None, None, None, None, None, 1_000_000, 64, 1.0,
                                  5e-3, 1e-5, 0, None)
    assert rc == 10  # F3D_ERR_TOO_LARGE
