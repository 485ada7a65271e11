"""GPU parity of the all-pairs sums (A1-A6) and the dense builders against
fiber3d's golden vectors and the CPU oracle.

FP64 bar: 1e-12 norm-wise relative (max|a-b| / max|b|).
FP32C bar: 2e-6 norm-wise relative against the FP64 result.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import kernels_np as O
from oracle import pairs_c

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


@pytest.fixture(scope="module")
def K():
    from fiber3d_b200 import kernels
    return kernels


@pytest.fixture(scope="module")
def L():
    from fiber3d_b200 import _lib
    return _lib


@pytest.mark.parametrize("tag", ["a", "b", "c", "d"])
def test_oseen_source_target_golden(K, golden_kernels, tag):
    g = golden_kernels
    u = K.oseen_kernel_source_target_numba(g[f"ost_{tag}_rs"], g[f"ost_{tag}_rt"], g[f"ost_{tag}_f"])
    assert isinstance(u, np.ndarray) and u.shape == g[f"ost_{tag}_u"].shape
    assert rel_err(u, g[f"ost_{tag}_u"]) < TOL64


def test_oseen_params_golden(K, golden_kernels):
    g = golden_kernels
    u = K.oseen_kernel_source_target_numba(g["ostp_rs"], g["ostp_rt"], g["ostp_f"], 2.5, 1e-2, 1e-4)
    assert rel_err(u, g["ostp_u"]) < TOL64
    u = K.oseen_kernel_source_target_numba(g["ostp_rs"], g["ostp_rt"], g["ostp_f"], eta=2.5,
                                           reg=1e-2, epsilon_distance=1e-4)
    assert rel_err(u, g["ostp_u"]) < TOL64


def test_times_density_golden(K, golden_kernels):
    g = golden_kernels
    assert rel_err(K.oseen_kernel_times_density_numba(g["otd_r"], g["otd_f"]), g["otd_u"]) < TOL64
    v = K.stresslet_kernel_times_normal_times_density_numba(g["stnd_r"], g["stnd_n"], g["stnd_d"])
    assert rel_err(v, g["stnd_v"]) < TOL64
    v = K.stresslet_kernel_times_normal_times_density_numba(g["stnd_r"], g["stnd_n"], g["stnd_d"], 3.0)
    assert rel_err(v, g["stnd_v_eta"]) < TOL64


def test_rotlet_stresslet_golden(K, golden_kernels):
    g = golden_kernels
    assert rel_err(K.rotlet_kernel_source_target_numba(g["rot_rs"], g["rot_rt"], g["rot_t"]), g["rot_u"]) < TOL64
    v = K.stresslet_kernel_source_target_numba(g["sst_rs"], g["sst_rt"], g["sst_n"], g["sst_d"])
    assert rel_err(v, g["sst_v"]) < TOL64


def test_dense_golden(K, golden_kernels):
    g = golden_kernels
    assert rel_err(K.stresslet_kernel_times_normal_numba(g["stn_r"], g["stn_n"]), g["stn_M"]) < TOL64
    assert rel_err(K.oseen_tensor(g["ot_r"]), g["ot_G"]) < TOL64
    assert rel_err(K.oseen_tensor(g["ot_r"].T.flatten(), input_format='xyz'), g["ot_Gxyz"]) < TOL64
    assert rel_err(K.oseen_tensor_source_target(g["otst_rs"], g["otst_rt"]), g["otst_G"]) < TOL64
    assert rel_err(K.complementary_kernel(None, g["comp_n"]), g["comp_C"]) < TOL64


def test_config1_golden(K, golden_config1):
    g = golden_config1
    u = K.oseen_kernel_times_density_numba(g["x"], g["f"])
    assert rel_err(u, g["u"]) < TOL64


SHAPES = [(1, 1, 0, 0), (2, 1, 0, 0), (1, 8, 0, 0), (1, 32, 0, 0), (1, 1, 1, 0), (1, 1, 5, 0),
          (1, 1, 3, -1), (2, 1, 0, -1), (1, 32, 7, -1), (1, 1, 19, -1), (2, 1, 38, -1), (4, 1, 0, 0),
          (4, 1, 9, -1)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kind", ["oseen", "stresslet", "rotlet"])
@pytest.mark.parametrize("ns,nt", [(1, 1), (127, 129), (128, 3), (129, 1000), (1000, 257)])
def test_launch_shapes_against_oracle(K, L, kind, shape, ns, nt):
    rng = np.random.default_rng(ns * 1000 + nt)
    xs = rng.random((ns, 3))
    xt = rng.random((nt, 3))
    xt[: min(2, ns, nt)] = xs[: min(2, ns, nt)]
    d = rng.normal(size=(ns, 3))
    n = rng.normal(size=(ns, 3))
    ref = pairs_c.pair_sum(kind, xs, xt, d, n if kind == "stresslet" else None)
    u = K.pair_sum(kind, xs, xt, d, n if kind == "stresslet" else None, shape=L.PairShape(*shape))
    assert rel_err(u.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("kind", ["oseen", "stresslet"])
@pytest.mark.parametrize("shape", [(1, 1, 0, 0), (1, 8, 4, 0), (1, 32, 0, -1)])
def test_skip_index_shapes(K, L, kind, shape):
    rng = np.random.default_rng(7)
    x = rng.random((300, 3)); x[10] = x[11]
    d = rng.normal(size=(300, 3)); n = rng.normal(size=(300, 3))
    ref = pairs_c.pair_sum(kind, x, x, d, n if kind == "stresslet" else None, self_mode="skip_index")
    u = K.pair_sum(kind, x, x, d, n if kind == "stresslet" else None, self_mode="skip_index",
                   shape=L.PairShape(*shape))
    assert rel_err(u.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("shape", [(1, 1, 0, 0), (2, 1, 3, 0), (1, 8, 0, -1)])
def test_skip_group(K, L, shape):
    from fiber3d_b200 import geometry
    rng = np.random.default_rng(11)
    x = np.concatenate(geometry.perturbed_fibers(rng, 20, 32, 2.0, 3.0))
    grp = np.repeat(np.arange(20), 32).astype(np.int32)
    f = rng.normal(size=x.shape)
    ref = pairs_c.pair_sum("oseen", x, x, f, self_mode="skip_group", src_group=grp, trg_group=grp)
    u = K.pair_sum("oseen", x, x, f, self_mode="skip_group", src_group=grp, trg_group=grp,
                   shape=L.PairShape(*shape))
    assert rel_err(u.cpu().numpy(), ref) < TOL64
    # and equal to the reference's add-then-subtract order
    full = O.oseen_kernel_source_target(x, x, f)
    for k in range(20):
        s = slice(32 * k, 32 * (k + 1))
        full[3 * s.start:3 * s.stop] -= O.oseen_tensor(x[s]) @ f[s].reshape(-1)
    assert rel_err(u.cpu().numpy(), full) < TOL64


@pytest.mark.parametrize("kind", ["oseen", "stresslet", "rotlet"])
def test_fp32c_accuracy(K, kind):
    from fiber3d_b200 import geometry
    nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=3, n=3000, n_vol=1000)
    q = mu * w[:, None]
    args = (nodes, vol, q, normals if kind == "stresslet" else None)
    u64 = K.pair_sum(kind, *args).cpu().numpy()
    u32 = K.pair_sum(kind, *args, precision="fp32c").cpu().numpy()
    assert rel_err(u32, u64) < TOL32


def test_accumulate_and_torch_inputs(K):
    rng = np.random.default_rng(3)
    xs = torch.tensor(rng.random((500, 3)), device="cuda")
    xt = torch.tensor(rng.random((400, 3)), device="cuda")
    f = torch.tensor(rng.normal(size=(500, 3)), device="cuda")
    u = K.oseen_kernel_source_target_numba(xs, xt, f)
    assert isinstance(u, torch.Tensor) and u.is_cuda and u.shape == (1200,)
    out = torch.ones(1200, dtype=torch.float64, device="cuda")
    K.pair_sum("oseen", xs, xt, f, out=out, accumulate=True)
    assert rel_err((out - 1.0).cpu().numpy(), u.cpu().numpy()) < 1e-14
    # strided (non-contiguous) numpy input is copied, not misread
    big = rng.random((500, 6))
    fs = big[:, ::2]
    u1 = K.oseen_kernel_source_target_numba(xs.cpu().numpy(), xt.cpu().numpy(), fs)
    u2 = K.oseen_kernel_source_target_numba(xs.cpu().numpy(), xt.cpu().numpy(), np.ascontiguousarray(fs))
    np.testing.assert_array_equal(u1, u2)


def test_empty_inputs(K):
    z = np.zeros((0, 3))
    x = np.random.default_rng(0).random((5, 3))
    assert K.oseen_kernel_source_target_numba(x, z, x).shape == (0,)
    np.testing.assert_array_equal(K.oseen_kernel_source_target_numba(z, x, z), np.zeros(15))
    np.testing.assert_array_equal(K.stresslet_kernel_source_target_numba(z, x, z, z), np.zeros(15))


def test_deterministic_and_error_word_clean(K, L):
    from fiber3d_b200 import geometry
    nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=4, n=2000, n_vol=300)
    a = K.stresslet_kernel_source_target_numba(nodes, vol, normals, mu)
    b = K.stresslet_kernel_source_target_numba(nodes, vol, normals, mu)
    np.testing.assert_array_equal(a, b)   # split partials are summed in a fixed order
    torch.cuda.synchronize()
    assert L.device_error() == 0


def test_config2_full_size_against_c_oracle(K):
    """12000 sphere nodes -> themselves (A4) and -> 4096 ball points (A3)."""
    from fiber3d_b200 import geometry
    nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=2)
    q = mu * w[:, None]
    v_self = K.stresslet_kernel_times_normal_times_density_numba(nodes, normals, q)
    v_vol = K.stresslet_kernel_source_target_numba(nodes, vol, normals, q)
    ref_vol = pairs_c.pair_sum("stresslet", nodes, vol, q, normals)
    assert rel_err(v_vol, ref_vol) < TOL64
    # the self sum is checked on a strided sample of targets by the numpy oracle
    idx = np.arange(0, 12000, 97)
    ref_self = O.stresslet_kernel_source_target(nodes, nodes[idx], normals, q)
    # remove the j == i pair from the sampled rows: it contributes exactly 0
    assert rel_err(v_self.reshape(-1, 3)[idx], ref_self.reshape(-1, 3)) < TOL64
    # linearity at full size: S(a q1 + b q2) = a S(q1) + b S(q2)
    q2 = np.random.default_rng(9).normal(size=q.shape) * w[:, None]
    lhs = K.stresslet_kernel_source_target_numba(nodes, vol, normals, 2.0 * q - 0.5 * q2)
    rhs = 2.0 * v_vol - 0.5 * K.stresslet_kernel_source_target_numba(nodes, vol, normals, q2)
    assert rel_err(lhs, rhs) < 1e-13


def test_workspace_reuse_across_shapes(K, L):
    """A call that writes split partials, then a call with more target blocks
    on the same workspace: the split counters must still start at zero."""
    rng = np.random.default_rng(21)
    xs = rng.random((1000, 3)); d = rng.normal(size=(1000, 3))
    K.pair_sum("oseen", xs, rng.random((300, 3)), d, shape=L.PairShape(1, 1, 7, 0))
    x = rng.random((700, 3)); f = rng.normal(size=(700, 3))
    for shape in [(1, 32, 0, -1), (1, 32, 0, 0), (1, 8, 3, 0)]:
        u = K.pair_sum("oseen", x, x, f, self_mode="skip_index", shape=L.PairShape(*shape))
        ref = pairs_c.pair_sum("oseen", x, x, f, self_mode="skip_index")
        assert rel_err(u.cpu().numpy(), ref) < TOL64


FP32_SHAPES = [(1, 1, 0, 0), (2, 1, 0, 0), (1, 8, 0, 0), (1, 32, 0, 0), (2, 1, 38, -1),
               (1, 1, 19, -1), (2, 1, 5, 0), (1, 8, 9, -1)]


@pytest.mark.parametrize("shape", FP32_SHAPES)
@pytest.mark.parametrize("mode", ["regularise", "skip_group"])
def test_fp32c_shapes(K, L, shape, mode):
    """Every FP32C launch shape the autotuner may pick gives the FP64 result
    to FP32C accuracy (finite everywhere)."""
    from fiber3d_b200 import geometry
    nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=5, n=3000, n_vol=777)
    q = mu * w[:, None]
    trg = np.concatenate([nodes, vol])
    gs = np.arange(3000, dtype=np.int32)
    gt = np.concatenate([gs, -np.ones(777, np.int32)]).astype(np.int32)
    kw = dict(self_mode=mode, src_group=gs, trg_group=gt) if mode == "skip_group" else {}
    u64 = K.pair_sum("stresslet", nodes, trg, q, normals, **kw).cpu().numpy()
    u32 = K.pair_sum("stresslet", nodes, trg, q, normals, precision="fp32c", shape=L.PairShape(*shape),
                     **kw).cpu().numpy()
    assert np.all(np.isfinite(u32))
    assert rel_err(u32, u64) < TOL32


def test_fp32c_single_split_keeps_shared_counters(K, L):
    """One workspace serves calls of every shape: an FP32C call with a single
    split (which packs its sources in the workspace) must leave the split
    counters of later multi-split calls untouched."""
    rng = np.random.default_rng(31)
    x = rng.random((3000, 3)) * 4.0
    y = rng.random((2000, 3)) * 4.0
    n = rng.normal(size=(3000, 3))
    d = rng.normal(size=(3000, 3))
    ref = pairs_c.pair_sum("stresslet", x, y, d, n)
    for _ in range(2):
        K.pair_sum("stresslet", x, y, d, n, precision="fp32c", shape=L.PairShape(1, 8, 1, -1))
        u = K.pair_sum("stresslet", x, y, d, n, shape=L.PairShape(1, 1, 7, -1)).cpu().numpy()
        assert rel_err(u, ref) < TOL64
        u = K.pair_sum("stresslet", x, y, d, n, precision="fp32c",
                       shape=L.PairShape(2, 1, 5, 0)).cpu().numpy()
        assert rel_err(u, ref) < TOL32


@pytest.mark.parametrize("shape", [(1, 1, 0, 0), (2, 1, 5, -1), (1, 8, 3, 0), (1, 32, 0, -1), (2, 1, 1, 0),
                                   (4, 1, 3, -1), (4, 1, 0, 0)])
@pytest.mark.parametrize("mode", ["regularise", "skip_group"])
def test_oseen_dual_equals_two_sums(L, shape, mode):
    """f3d_oseen_dual gives, bit for bit, the two FP64 Oseen sums it fuses."""
    import ctypes
    import torch
    from fiber3d_b200 import kernels as K
    rng = np.random.default_rng(41)
    xs = torch.tensor(rng.random((2000, 3)) * 4.0, device="cuda")
    xt = torch.tensor(rng.random((1500, 3)) * 4.0, device="cuda")
    d1 = torch.tensor(rng.normal(size=(2000, 3)), device="cuda")
    d2 = torch.tensor(rng.normal(size=(2000, 3)), device="cuda")
    gs = torch.tensor(np.arange(2000) // 20, dtype=torch.int32, device="cuda")
    gt = torch.tensor(np.arange(1500) // 20, dtype=torch.int32, device="cuda")
    kw = dict(self_mode=mode, src_group=gs, trg_group=gt) if mode == "skip_group" else {}
    shp = L.PairShape(*shape)
    r1 = K.pair_sum("oseen", xs, xt, d1, shape=shp, **kw).clone()
    r2 = K.pair_sum("oseen", xs, xt, d2, shape=shp, **kw).clone()
    nb = ctypes.c_size_t(0)
    L.call("f3d_oseen_dual_workspace_bytes", 2000, 1500, ctypes.byref(shp), ctypes.byref(nb))
    ws = torch.zeros(max(nb.value, 256), dtype=torch.uint8, device="cuda")
    o1 = torch.empty_like(r1)
    o2 = torch.empty_like(r2)
    for _ in range(2):  # the split counters return to zero between calls
        L.call("f3d_oseen_dual", L.SELF_MODE[mode], L.ptr(xs), L.ptr(xt), L.ptr(d1), L.ptr(d2), L.ptr(gs),
               L.ptr(gt), L.ptr(o1), L.ptr(o2), 2000, 1500, 1.0, 5e-3, 1e-5, 0, ctypes.byref(shp), L.ptr(ws),
               ws.numel(), L.stream_handle())
        assert torch.equal(o1, r1) and torch.equal(o2, r2)


@pytest.mark.parametrize("mode", ["skip_index", "skip_group"])
@pytest.mark.parametrize("ns,nt", [(2000, 2000), (2000, 3500), (130, 131)])
def test_symmetric_oseen_dual_equals_two_sums(L, mode, ns, nt):
    """The two-density form of the symmetric Oseen sum (sources = the first ns
    of nt points) gives, bit for bit, the two symmetric sums it fuses."""
    import ctypes
    import torch
    from fiber3d_b200 import kernels as K
    rng = np.random.default_rng(43 + nt)
    x = torch.tensor(rng.random((nt, 3)) * 4.0, device="cuda")
    d1 = torch.tensor(rng.normal(size=(ns, 3)), device="cuda")
    d2 = torch.tensor(rng.normal(size=(ns, 3)), device="cuda")
    g = torch.tensor(np.arange(nt) // 20, dtype=torch.int32, device="cuda")
    kw = dict(self_mode=mode, src_group=g[:ns], trg_group=g) if mode == "skip_group" else dict(self_mode=mode)
    shp = L.PairShape(*SYM)
    r1 = K.pair_sum("oseen", x[:ns], x, d1, shape=shp, **kw).clone()
    r2 = K.pair_sum("oseen", x[:ns], x, d2, shape=shp, **kw).clone()
    ref = pairs_c.pair_sum("oseen", x[:ns].cpu().numpy(), x.cpu().numpy(), d1.cpu().numpy(), self_mode=mode,
                           src_group=g[:ns].cpu().numpy() if mode == "skip_group" else None,
                           trg_group=g.cpu().numpy() if mode == "skip_group" else None)
    assert rel_err(r1.cpu().numpy(), ref) < TOL64
    nb = ctypes.c_size_t(0)
    L.call("f3d_oseen_dual_workspace_bytes", ns, nt, ctypes.byref(shp), ctypes.byref(nb))
    ws = torch.zeros(max(nb.value, 256), dtype=torch.uint8, device="cuda")
    o1, o2 = torch.empty_like(r1), torch.empty_like(r2)
    for _ in range(2):  # the tile counters return to zero between calls
        L.call("f3d_oseen_dual", L.SELF_MODE[mode], L.ptr(x), L.ptr(x), L.ptr(d1), L.ptr(d2), L.ptr(g),
               L.ptr(g), L.ptr(o1), L.ptr(o2), ns, nt, 1.0, 5e-3, 1e-5, 0, ctypes.byref(shp), L.ptr(ws),
               ws.numel(), L.stream_handle())
        assert torch.equal(o1, r1) and torch.equal(o2, r2)


@pytest.mark.parametrize("ns", [1, 129, 2999])
@pytest.mark.parametrize("kind", ["oseen", "stresslet", "rotlet"])
@pytest.mark.parametrize("mode", ["regularise", "skip_index", "skip_group"])
def test_fp32c_odd_source_counts(K, ns, kind, mode):
    """FP32C takes sources in pairs; an odd count ends on a padding source
    whose terms are exactly zero, in every kernel and self mode, in a full
    tile or a partial one, alone or not."""
    rng = np.random.default_rng(ns)
    xs = rng.uniform(-2.0, 2.0, size=(ns, 3))
    d = rng.normal(size=(ns, 3))
    n = rng.normal(size=(ns, 3)) if kind == "stresslet" else None
    if mode == "skip_index":
        xt = xs
    else:
        xt = rng.uniform(-2.0, 2.0, size=(ns + 37, 3))
    kw = {"self_mode": mode}
    if mode == "skip_group":
        kw.update(src_group=np.arange(ns, dtype=np.int32) // 3,
                  trg_group=(np.arange(xt.shape[0], dtype=np.int32) // 5).astype(np.int32))
    u64 = K.pair_sum(kind, xs, xt, d, n, **kw).cpu().numpy()
    u32 = K.pair_sum(kind, xs, xt, d, n, precision="fp32c", **kw).cpu().numpy()
    assert np.all(np.isfinite(u32))
    if np.abs(u64).max() == 0.0:
        assert np.abs(u32).max() == 0.0
    else:
        assert rel_err(u32, u64) < TOL32


@pytest.mark.parametrize("shape", [(1, 1, 0, 0), (2, 1, 0, 0), (1, 8, 4, 0), (1, 32, 0, -1), (1, 1, 7, -1)])
@pytest.mark.parametrize("n", [1, 129, 700])
def test_traction_shapes(K, L, shape, n):
    """Traction (normal of the target, j == i skipped) at every launch shape."""
    rng = np.random.default_rng(n + 31)
    x = rng.random((n, 3))
    if n > 20:
        x[10] = x[11]
    d = rng.normal(size=(n, 3)); nr = rng.normal(size=(n, 3))
    ref = O.traction_kernel_times_normal_times_density(x, nr, d)
    u = K.pair_sum("traction", x, x, d, nr, self_mode="skip_index", shape=L.PairShape(*shape))
    assert rel_err(u.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("shape", [(1, 1, 0, 0), (2, 1, 3, 0), (1, 8, 0, -1), (1, 32, 5, 0)])
@pytest.mark.parametrize("kind", ["oseen", "stresslet"])
def test_skip_close_shapes(K, L, shape, kind):
    """Pairs closer than eps contribute zero (coincident ones included), at
    every launch shape, FP64 against the oracle."""
    rng = np.random.default_rng(99)
    xs = rng.random((400, 3)); xt = rng.random((333, 3))
    xt[:5] = xs[:5]
    xt[5:9] = xs[5:9] + 2e-6 * rng.normal(size=(4, 3))
    d = rng.normal(size=(400, 3)); nr = rng.normal(size=(400, 3))
    if kind == "oseen":
        ref = O.oseen_kernel_source_target_skip_close(xs, xt, d, epsilon_distance=1e-5)
        u = K.pair_sum("oseen", xs, xt, d, self_mode="skip_close", epsilon_distance=1e-5, shape=L.PairShape(*shape))
    else:
        ref = O.stresslet_kernel_source_target_skip_close(xs, xt, nr, d, epsilon_distance=1e-5)
        u = K.pair_sum("stresslet", xs, xt, d, nr, self_mode="skip_close", epsilon_distance=1e-5,
                       shape=L.PairShape(*shape))
    assert rel_err(u.cpu().numpy(), ref) < TOL64


def test_occupancy_query(L):
    from fiber3d_b200 import autotune
    for kind in ("oseen", "stresslet", "traction"):
        for tpt, sl in ((1, 1), (2, 1), (1, 8), (1, 32)):
            n = autotune.occupancy(kind, "fp64", "skip_group", tpt, sl)
            assert 1 <= n <= 16


@pytest.mark.parametrize("kind,mode", [("stresslet", "skip_index"), ("oseen", "regularise"),
                                       ("traction", "skip_index"), ("rotlet", "regularise")])
def test_host_entry_matches_device_entry(L, kind, mode):
    """f3d_pair_sum_host (host buffers in and out, one call) equals
    f3d_pair_sum on device copies of the same inputs, bit for bit."""
    import ctypes
    rng = np.random.default_rng(5)
    n = 900
    x = rng.random((n, 3)) * 3
    xt = x if mode == "skip_index" else rng.random((700, 3)) * 3
    d = rng.normal(size=(n, 3))
    nr = rng.normal(size=(xt.shape[0] if kind == "traction" else n, 3)) if kind in ("stresslet", "traction") else None
    from fiber3d_b200 import kernels as K
    ref = K.pair_sum(kind, x, xt, d, nr, self_mode=mode).cpu().numpy()
    k, p, m = L.KERNEL[kind], L.PRECISION["fp64"], L.SELF_MODE[mode]
    nt = xt.shape[0]
    out = np.empty(3 * nt)
    hb = ctypes.c_size_t(0)
    L.call("f3d_pair_host_bytes", k, n, nt, int(xt is x), ctypes.byref(hb))
    stage = torch.empty(hb.value, dtype=torch.uint8, device="cuda")
    wb = ctypes.c_size_t(0)
    L.call("f3d_pair_workspace_bytes", k, p, n, nt, None, ctypes.byref(wb))
    ws = torch.zeros(max(wb.value, 1), dtype=torch.uint8, device="cuda")
    ptr = lambda a: a.ctypes.data if a is not None else None
    L.call("f3d_pair_sum_host", k, p, m, ptr(x), ptr(xt), ptr(d), ptr(nr), ptr(out), n, nt, 1.0, 5e-3, 1e-5,
           None, stage.data_ptr(), stage.numel(), ws.data_ptr(), ws.numel(), L.stream_handle())
    assert np.array_equal(out, ref)


def test_drop_in_host_fast_path_repeatable(K):
    """The second call of a size bucket takes the one-call host path; it
    gives the oracle's sum like the first."""
    rng = np.random.default_rng(6)
    x = rng.random((1500, 3)) * 4
    nr = rng.normal(size=(1500, 3))
    d = rng.normal(size=(1500, 3))
    ref = O.stresslet_kernel_times_normal_times_density(x, nr, d)
    a = K.stresslet_kernel_times_normal_times_density_numba(x, nr, d)
    b = K.stresslet_kernel_times_normal_times_density_numba(x, nr, d)
    assert rel_err(a, ref) < TOL64 and rel_err(b, ref) < TOL64
    assert isinstance(b, np.ndarray) and b.shape == (4500,)


def test_drop_in_host_fast_path_cpu_tensors(K):
    """The one-call host path also takes CPU (and page-locked) torch tensors."""
    rng = np.random.default_rng(7)
    x = rng.random((1300, 3)) * 4
    f = rng.normal(size=(1300, 3))
    ref = O.oseen_kernel_times_density(x, f)
    for pin in (False, True):
        xt, ft = torch.as_tensor(x), torch.as_tensor(f)
        if pin:
            xt, ft = xt.pin_memory(), ft.pin_memory()
        for _ in range(2):
            u = K.oseen_kernel_times_density_numba(xt, ft)
            assert isinstance(u, np.ndarray) and rel_err(u, ref) < TOL64


SYM = (1, -1, 0, -1)


@pytest.mark.parametrize("kind", ["oseen", "stresslet"])
@pytest.mark.parametrize("n", [1, 127, 128, 129, 300, 1000, 5000])
def test_symmetric_self_sum_skip_index(K, L, kind, n):
    """The symmetric form (each unordered pair once) against the C oracle,
    with a duplicated point and a sub-epsilon pair (the careful redo)."""
    rng = np.random.default_rng(n + 13)
    x = rng.random((n, 3)) * 3
    if n > 40:
        x[10] = x[11]
        x[30] = x[31] + 3e-6
    d = rng.normal(size=(n, 3)); nr = rng.normal(size=(n, 3))
    ref = pairs_c.pair_sum(kind, x, x, d, nr if kind == "stresslet" else None, self_mode="skip_index")
    xt = torch.as_tensor(x, device="cuda")
    u = K.pair_sum(kind, xt, xt, d, nr if kind == "stresslet" else None, self_mode="skip_index",
                   shape=L.PairShape(*SYM))
    assert rel_err(u.cpu().numpy(), ref) < TOL64
    # deterministic, and accumulate adds to what is there
    u2 = K.pair_sum(kind, xt, xt, d, nr if kind == "stresslet" else None, self_mode="skip_index",
                    shape=L.PairShape(*SYM))
    assert torch.equal(u, u2)
    K.pair_sum(kind, xt, xt, d, nr if kind == "stresslet" else None, self_mode="skip_index",
               shape=L.PairShape(*SYM), out=u2, accumulate=True)
    assert rel_err(u2.cpu().numpy(), 2 * ref) < TOL64


@pytest.mark.parametrize("kind", ["oseen", "stresslet"])
@pytest.mark.parametrize("nfib,npts", [(20, 32), (70, 32), (9, 24)])
def test_symmetric_self_sum_skip_group(K, L, kind, nfib, npts):
    """Fibers: pairs within one fiber skipped, in the symmetric form."""
    from fiber3d_b200 import geometry
    rng = np.random.default_rng(nfib * 7 + npts)
    x = np.concatenate(geometry.perturbed_fibers(rng, nfib, npts, 2.0, 3.0))
    grp = np.repeat(np.arange(nfib), npts).astype(np.int32)
    d = rng.normal(size=x.shape); nr = rng.normal(size=x.shape)
    ref = pairs_c.pair_sum(kind, x, x, d, nr if kind == "stresslet" else None, self_mode="skip_group",
                           src_group=grp, trg_group=grp)
    xt = torch.as_tensor(x, device="cuda")
    g = torch.as_tensor(grp, device="cuda")
    u = K.pair_sum(kind, xt, xt, d, nr if kind == "stresslet" else None, self_mode="skip_group", src_group=g,
                   trg_group=g, shape=L.PairShape(*SYM))
    assert rel_err(u.cpu().numpy(), ref) < TOL64


def test_symmetric_config2_self_sum(K, L):
    """The 12000-node sphere's double-layer self-sum in the symmetric form
    against the regular kernel (full size) and sampled C-oracle rows."""
    from fiber3d_b200 import geometry
    nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=2)
    q = mu * w[:, None]
    xt = torch.as_tensor(nodes, device="cuda")
    a = K.pair_sum("stresslet", xt, xt, q, normals, self_mode="skip_index", shape=L.PairShape(*SYM))
    b = K.pair_sum("stresslet", xt, xt, q, normals, self_mode="skip_index", shape=L.PairShape(1, 1, 0, 0))
    assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < 1e-13


@pytest.mark.parametrize("kind", ["oseen", "stresslet"])
@pytest.mark.parametrize("mode", ["skip_index", "skip_group"])
@pytest.mark.parametrize("n,m", [(127, 1), (300, 129), (1000, 700), (129, 300)])
def test_symmetric_with_further_targets(K, L, kind, mode, n, m):
    """Sources as the first n of n + m targets: the symmetric launch sums the
    further m targets one-sided in the same launch.  Against the C oracle and
    the regular kernel, with coincident and sub-epsilon pairs among the
    sources, between a further target and a source, and (skip_group)
    further targets in a source's group."""
    rng = np.random.default_rng(n * 31 + m)
    x = rng.random((n + m, 3)) * 3
    x[n] = x[5]                    # a further target on a source: regularised
    if m > 2:
        x[n + 2] = x[7] + 4e-6     # and one within eps of a source
    if n > 40:
        x[10] = x[11]
        x[30] = x[31] + 3e-6
    d = rng.normal(size=(n, 3)); nr = rng.normal(size=(n, 3))
    nrm = nr if kind == "stresslet" else None
    kw = {}
    if mode == "skip_group":
        grp = (np.arange(n + m) // 16).astype(np.int32)
        grp[n + 1:] = rng.integers(0, n // 16 + 1, size=m - 1) if m > 1 else grp[n + 1:]
        kw = dict(src_group=grp[:n], trg_group=grp)
    ref = pairs_c.pair_sum(kind, x[:n], x, d, nrm, self_mode=mode, **kw)
    xt = torch.as_tensor(x, device="cuda")
    if mode == "skip_group":
        g = torch.as_tensor(grp, device="cuda")
        kw = dict(src_group=g[:n], trg_group=g)
    u = K.pair_sum(kind, xt[:n], xt, d, nrm, self_mode=mode, shape=L.PairShape(*SYM), **kw)
    assert rel_err(u.cpu().numpy(), ref) < TOL64
    v = K.pair_sum(kind, xt[:n], xt, d, nrm, self_mode=mode, shape=L.PairShape(1, 1, 0, 0), **kw)
    assert rel_err(v.cpu().numpy(), ref) < TOL64
    u2 = K.pair_sum(kind, xt[:n], xt, d, nrm, self_mode=mode, shape=L.PairShape(*SYM), **kw)
    assert torch.equal(u, u2)


def test_symmetric_config2_step(K, L):
    """The 12000-node sphere's double layer on its own nodes (j != i) and on
    4096 ball points, as one symmetric launch over one array, against the
    regular kernel over the same array (full size)."""
    from fiber3d_b200 import geometry
    nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=2)
    q = mu * w[:, None]
    xt = torch.as_tensor(np.concatenate([nodes, vol]), device="cuda")
    n = nodes.shape[0]
    a = K.pair_sum("stresslet", xt[:n], xt, q, normals, self_mode="skip_index", shape=L.PairShape(*SYM))
    b = K.pair_sum("stresslet", xt[:n], xt, q, normals, self_mode="skip_index", shape=L.PairShape(1, 1, 0, 0))
    assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < 1e-13
    idx = np.r_[0:50, n - 50:n + 50, xt.shape[0] - 50:xt.shape[0]]
    ref = pairs_c.pair_sum("stresslet", nodes, xt.cpu().numpy()[idx], q, normals)
    # the sampled rows: j == i skipped for the sphere nodes among them
    for r, i in enumerate(idx):
        if i < n:
            ref[3 * r:3 * r + 3] = pairs_c.pair_sum("stresslet", np.delete(nodes, i, 0), nodes[i:i + 1],
                                                    np.delete(q, i, 0), np.delete(normals, i, 0))
    got = a.cpu().numpy().reshape(-1, 3)[idx].reshape(-1)
    assert rel_err(got, ref) < 1e-12


def test_symmetric_largest_step_sum(K, L):
    """The largest time step's fiber Oseen sum (2000 fibers x 32 points onto
    the 85600 points of fibers, bodies and periphery, pairs within a fiber
    skipped): 500 source tiles, 1 GB of partial sums; the symmetric form
    against the regular kernel at full size, single and two-density."""
    import ctypes
    from fiber3d_b200 import geometry
    P = geometry.hydro_step_problem(seed=3, nfib=2000, nshell=20000, shell_radius=12.0, fiber_ball=8.0,
                                    body_shell=9.5)
    fib = np.concatenate(P.fibers)
    rest = np.concatenate([b.nodes for b in P.bodies]
                          + [P.shell.nodes])
    x = torch.as_tensor(np.concatenate([fib, rest]), device="cuda")
    n = fib.shape[0]
    g = torch.as_tensor(np.concatenate([np.repeat(np.arange(2000), 32), -1 - np.arange(rest.shape[0])])
                        .astype(np.int32), device="cuda")
    rng = np.random.default_rng(1)
    f1 = torch.as_tensor(rng.normal(size=(n, 3)), device="cuda")
    f2 = torch.as_tensor(rng.normal(size=(n, 3)), device="cuda")
    kw = dict(self_mode="skip_group", src_group=g[:n], trg_group=g)
    a = K.pair_sum("oseen", x[:n], x, f1, shape=L.PairShape(*SYM), **kw)
    b = K.pair_sum("oseen", x[:n], x, f1, shape=L.PairShape(4, 1, 0, -1), **kw)
    assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < 1e-13
    shp = L.PairShape(*SYM)
    nb = ctypes.c_size_t(0)
    L.call("f3d_oseen_dual_workspace_bytes", n, x.shape[0], ctypes.byref(shp), ctypes.byref(nb))
    ws = torch.zeros(nb.value, dtype=torch.uint8, device="cuda")
    o1, o2 = torch.empty_like(a), torch.empty_like(a)
    L.call("f3d_oseen_dual", L.SELF_MODE["skip_group"], L.ptr(x), L.ptr(x), L.ptr(f1), L.ptr(f2), L.ptr(g),
           L.ptr(g), L.ptr(o1), L.ptr(o2), n, x.shape[0], 1.0, 5e-3, 1e-5, 0, ctypes.byref(shp), L.ptr(ws),
           ws.numel(), L.stream_handle())
    assert torch.equal(o1, a)
    c = K.pair_sum("oseen", x[:n], x, f2, shape=shp, **kw)
    assert torch.equal(o2, c)


def test_symmetric_rejects_other_sums(K, L):
    rng = np.random.default_rng(3)
    x = rng.random((200, 3)); y = rng.random((200, 3)); d = rng.normal(size=(200, 3))
    with pytest.raises(L.F3DError):   # two point sets
        K.pair_sum("oseen", x, y, d, self_mode="skip_index", shape=L.PairShape(*SYM))
    with pytest.raises(L.F3DError):   # FP32C
        xt = torch.as_tensor(x, device="cuda")
        K.pair_sum("oseen", xt, xt, d, self_mode="skip_index", precision="fp32c", shape=L.PairShape(*SYM))
    big = torch.zeros((1024 * 128 + 1, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(L.F3DError) as e:
        K.pair_sum("oseen", big, big, big, self_mode="skip_index", shape=L.PairShape(*SYM))
    assert e.value.status == 10


TILE = (1, -2, 0, -1)


@pytest.mark.parametrize("sub", [0, 1, 2])
@pytest.mark.parametrize("kind", ["oseen", "stresslet"])
@pytest.mark.parametrize("ns,nt", [(1, 1), (127, 129), (128, 3), (1000, 257), (3000, 4097)])
def test_tile_form_source_target(K, L, kind, ns, nt, sub):
    """The tile form of a source -> target sum (sl = -2; nsplit 1 or 2:
    128- or 64-point source tiles, 0: chosen from the size) against the C
    oracle, with a target on a source (coincident: regularised) and a
    sub-epsilon pair (the careful redo); deterministic; accumulate adds to
    the output."""
    rng = np.random.default_rng(ns * 7 + nt)
    xs, xt = rng.random((ns, 3)) * 3, rng.random((nt, 3)) * 3
    if ns > 40 and nt > 40:
        xt[5] = xs[7]
        xt[20] = xs[30] + 3e-6
    d, nr = rng.normal(size=(ns, 3)), rng.normal(size=(ns, 3))
    n_arg = nr if kind == "stresslet" else None
    ref = pairs_c.pair_sum(kind, xs, xt, d, n_arg)
    s, t = torch.as_tensor(xs, device="cuda"), torch.as_tensor(xt, device="cuda")
    shp = L.PairShape(1, -2, sub, -1)
    u = K.pair_sum(kind, s, t, d, n_arg, shape=shp)
    assert rel_err(u.cpu().numpy(), ref) < TOL64
    u2 = K.pair_sum(kind, s, t, d, n_arg, shape=shp)
    assert torch.equal(u, u2)
    K.pair_sum(kind, s, t, d, n_arg, shape=shp, out=u2, accumulate=True)
    assert rel_err(u2.cpu().numpy(), 2 * ref) < TOL64


def test_tile_form_config2_ball_targets(K, L):
    """fiber3d's second config-2 call (the 12000-node double layer onto the
    4096 ball points) in the tile form: equal to the regular kernel to
    rounding, sampled rows against the C oracle; the host entry point takes
    the same shape."""
    from fiber3d_b200 import geometry
    nodes, normals, w, mu, vol = geometry.stresslet_sphere_workload(seed=2)
    q = mu * w[:, None]
    s, t = torch.as_tensor(nodes, device="cuda"), torch.as_tensor(vol, device="cuda")
    a = K.pair_sum("stresslet", s, t, q, normals, shape=L.PairShape(*TILE))
    b = K.pair_sum("stresslet", s, t, q, normals, shape=L.PairShape(1, 1, 0, 0))
    assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < TOL64
    for sub in (1, 2):
        c = K.pair_sum("stresslet", s, t, q, normals, shape=L.PairShape(1, -2, sub, -1))
        assert rel_err(c.cpu().numpy(), b.cpu().numpy()) < TOL64
    ref = pairs_c.pair_sum("stresslet", nodes, vol[:300], q, normals)
    assert rel_err(a.cpu().numpy()[:900], ref) < TOL64
    h = K.stresslet_kernel_source_target_numba(nodes, vol, normals, q, shape=L.PairShape(*TILE))
    assert np.array_equal(np.asarray(h).reshape(-1), a.cpu().numpy())


@pytest.mark.parametrize("sub", [1, 2])
@pytest.mark.parametrize("ns,nt", [(300, 700), (5000, 129)])
def test_tile_form_oseen_dual_equals_two_sums(L, ns, nt, sub):
    """The two-density Oseen pass in the tile form gives, bit for bit, the two
    tile-form sums it fuses."""
    import ctypes
    from fiber3d_b200 import kernels as K
    rng = np.random.default_rng(ns + nt)
    s = torch.tensor(rng.random((ns, 3)) * 4.0, device="cuda")
    t = torch.tensor(rng.random((nt, 3)) * 4.0, device="cuda")
    d1, d2 = (torch.tensor(rng.normal(size=(ns, 3)), device="cuda") for _ in range(2))
    shp = L.PairShape(1, -2, sub, -1)
    r1 = K.pair_sum("oseen", s, t, d1, shape=shp).clone()
    r2 = K.pair_sum("oseen", s, t, d2, shape=shp).clone()
    nb = ctypes.c_size_t(0)
    L.call("f3d_oseen_dual_workspace_bytes", ns, nt, ctypes.byref(shp), ctypes.byref(nb))
    ws = torch.zeros(max(nb.value, 256), dtype=torch.uint8, device="cuda")
    o1, o2 = torch.empty_like(r1), torch.empty_like(r2)
    for _ in range(2):  # the tile counters return to zero between calls
        L.call("f3d_oseen_dual", L.SELF_MODE["regularise"], L.ptr(s), L.ptr(t), L.ptr(d1), L.ptr(d2), None, None,
               L.ptr(o1), L.ptr(o2), ns, nt, 1.0, 5e-3, 1e-5, 0, ctypes.byref(shp), L.ptr(ws), ws.numel(),
               L.stream_handle())
        assert torch.equal(o1, r1) and torch.equal(o2, r2)


def test_tile_form_rejects_other_rules(K, L):
    s = torch.rand(200, 3, dtype=torch.float64, device="cuda")
    d = torch.rand(200, 3, dtype=torch.float64, device="cuda")
    for mode in ("skip_index", "skip_close"):
        with pytest.raises(L.F3DError):
            K.pair_sum("oseen", s, s, d, self_mode=mode, shape=L.PairShape(*TILE))
    with pytest.raises(L.F3DError):
        K.pair_sum("rotlet", s, s, d, shape=L.PairShape(*TILE))
