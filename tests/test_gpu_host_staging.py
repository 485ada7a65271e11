"""The host entry point (f3d_pair_sum_host) with every kind of host memory:
page-locked inputs read by the staging kernel (16-byte and only 8-byte
aligned, odd sizes whose last double is copied on its own), pageable inputs
copied with cudaMemcpyAsync, a mix of both, and outputs written by the pair
kernel straight into page-locked memory or copied back into pageable memory.
Every variant agrees bit for bit with the device-resident sum and with the C
oracle to 1e-12."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import pairs_c

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def K():
    torch.cuda.set_device(0)
    from fiber3d_b200 import kernels
    return kernels


def pinned(a: np.ndarray, offset: int = 0) -> torch.Tensor:
    """A page-locked copy of a, starting `offset` doubles into its buffer
    (offset 1: 8-byte but not 16-byte aligned)."""
    flat = torch.empty(a.size + offset, dtype=torch.float64, pin_memory=True)
    view = flat[offset:].view(a.shape)
    view.copy_(torch.as_tensor(a))
    assert view.data_ptr() % 16 == (8 if offset % 2 else 0)
    return view


def host_call(L, kind, mode, rs, rt, d, n, out, ns, nt, shape=None):
    """f3d_pair_sum_host on raw host pointers with its own buffers."""
    from fiber3d_b200 import _lib
    k, m = _lib.KERNEL[kind], _lib.SELF_MODE[mode]
    same = rs == rt
    hb, wb = ctypes.c_size_t(0), ctypes.c_size_t(0)
    _lib.call("f3d_pair_host_bytes", k, ns, nt, int(same), ctypes.byref(hb))
    _lib.call("f3d_pair_workspace_bytes", k, 0, ns, nt, shape, ctypes.byref(wb))
    stage = torch.empty(hb.value, dtype=torch.uint8, device="cuda")
    ws = torch.zeros(max(wb.value, 1), dtype=torch.uint8, device="cuda")
    st = _lib.lib().f3d_pair_sum_host(k, 0, m, rs, rt, d, n, out, ns, nt, 1.0, 5e-3, 1e-5, shape,
                                      stage.data_ptr(), stage.numel(), ws.data_ptr(), ws.numel(),
                                      torch.cuda.current_stream().cuda_stream)
    _lib.check("f3d_pair_sum_host", st)


@pytest.mark.parametrize("ns,nt", [(1001, 777), (128, 4096), (3, 5)])
@pytest.mark.parametrize("offset", [0, 1])
def test_pinned_inputs_staged_by_kernel(K, ns, nt, offset):
    rng = np.random.default_rng(ns + nt + offset)
    rs, rt = rng.random((ns, 3)) * 4, rng.random((nt, 3)) * 4
    d, n = rng.normal(size=(ns, 3)), rng.normal(size=(ns, 3))
    ref = pairs_c.pair_sum("stresslet", rs, rt, d, n)
    dev = K.pair_sum("stresslet", torch.as_tensor(rs, device="cuda"), torch.as_tensor(rt, device="cuda"),
                     torch.as_tensor(d, device="cuda"), torch.as_tensor(n, device="cuda"),
                     shape=K._lib.PairShape(1, 1, 0, 0)).cpu().numpy()
    u_np = K.stresslet_kernel_source_target_numba(rs, rt, n, d, shape=K._lib.PairShape(1, 1, 0, 0))
    u_pin = K.stresslet_kernel_source_target_numba(pinned(rs, offset), pinned(rt, offset), pinned(n, offset),
                                                   pinned(d, offset), shape=K._lib.PairShape(1, 1, 0, 0))
    mixed = K.stresslet_kernel_source_target_numba(pinned(rs, offset), rt, pinned(n, offset), d,
                                                   shape=K._lib.PairShape(1, 1, 0, 0))
    assert rel_err(u_pin, ref) < 1e-12
    assert np.array_equal(u_pin, u_np) and np.array_equal(mixed, u_np)
    assert np.array_equal(u_pin.reshape(-1), dev)


@pytest.mark.parametrize("n", [12000, 1537])
def test_pinned_self_sum_symmetric_form(K, n):
    """The symmetric self-sum on page-locked inputs: its last-arriving
    reductions write the page-locked output directly."""
    from fiber3d_b200 import geometry
    rng = np.random.default_rng(n)
    nrm = geometry.uniform_directions(rng, n)
    x = 10.0 * nrm
    q = rng.normal(size=(n, 3))
    ref = pairs_c.pair_sum("stresslet", x, x, q, nrm, self_mode="skip_index")
    sym = K._lib.PairShape(1, -1, 0, -1)
    u_np = K.stresslet_kernel_times_normal_times_density_numba(x, nrm, q, shape=sym)
    u_pin = K.stresslet_kernel_times_normal_times_density_numba(pinned(x), pinned(nrm), pinned(q), shape=sym)
    assert rel_err(u_pin, ref) < 1e-12
    assert np.array_equal(u_pin, u_np)


def test_outputs_pinned_pageable_and_unaligned(K):
    """The raw entry point: a page-locked `out` is written by the kernel, a
    pageable one (numpy) receives a copy, and one that is not 8-byte
    aligned is copied too; all three hold the same numbers."""
    from fiber3d_b200 import _lib
    rng = np.random.default_rng(3)
    ns, nt = 700, 515
    rs, rt = pinned(rng.random((ns, 3))), pinned(rng.random((nt, 3)))
    d = pinned(rng.normal(size=(ns, 3)))
    ref = pairs_c.pair_sum("oseen", rs.numpy(), rt.numpy(), d.numpy())
    out_pin = torch.empty(3 * nt, dtype=torch.float64, pin_memory=True)
    out_np = np.zeros(3 * nt)
    raw = torch.zeros(3 * nt * 8 + 4, dtype=torch.uint8, pin_memory=True)
    out_odd = raw.data_ptr() + 4
    for out in (out_pin.data_ptr(), out_np.ctypes.data, out_odd):
        host_call(_lib, "oseen", "regularise", rs.data_ptr(), rt.data_ptr(), d.data_ptr(), None, out, ns, nt)
    odd = np.frombuffer(raw.numpy()[4:].tobytes(), dtype=np.float64)
    assert rel_err(out_pin.numpy(), ref.reshape(-1)) < 1e-12
    assert np.array_equal(out_pin.numpy(), out_np) and np.array_equal(out_np, odd)


def test_pinned_traction_and_empty_sources(K):
    """The traction sum stages the target normals (nt of them); with no
    sources a page-locked output is cleared, not left as it was."""
    from fiber3d_b200 import _lib
    from oracle import kernels_np as O
    rng = np.random.default_rng(4)
    x, n, d = rng.random((333, 3)) * 3, rng.normal(size=(333, 3)), rng.normal(size=(333, 3))
    ref = O.traction_kernel_times_normal_times_density(x, n, d)
    v = K.traction_kernel_times_normal_times_density_numba(pinned(x), pinned(n), pinned(d),
                                                           shape=K._lib.PairShape(1, 1, 0, 0))
    assert rel_err(v, ref) < 1e-12
    out = torch.full((3 * 10,), 7.0, dtype=torch.float64, pin_memory=True)
    rt = pinned(rng.random((10, 3)))
    host_call(_lib, "oseen", "regularise", None, rt.data_ptr(), None, None, out.data_ptr(), 0, 10)
    assert torch.count_nonzero(out).item() == 0
