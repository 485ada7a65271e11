"""Drop-in replacement for fiber3d's ``kernels.kernels`` module on one B200.

Every function keeps the name, positional/keyword signature, defaults and
return convention of the fiber3d function it replaces
(``python/kernels/kernels.py``), so ``sys.modules['kernels.kernels']`` can
point at this module and the unmodified time stepper runs on the GPU.

* Inputs may be numpy arrays (any shape whose size is 3N, any strides; they
  are copied host->device) or torch tensors (CUDA tensors are used in place).
* Outputs follow the inputs: a new flat float64 numpy array of length 3*Nt
  when any point array came from the host, else a flat CUDA float64 tensor.
* Inputs are never modified.
* The work runs on the current CUDA stream through the C ABI of
  ``libfiber3d_b200.so``; there is no CPU path.

Keyword-only extensions (not in fiber3d): ``precision`` ('fp64' default or
'fp32c') and ``shape`` (a :class:`fiber3d_b200._lib.PairShape` launch shape).
Without ``shape`` the pair-sum drop-ins take the launch shape
:mod:`fiber3d_b200.autotune` found for the sum's kernel, mode and size
bucket, timing the candidates on the first call of a bucket (tens of
milliseconds, once per bucket and GPU model; cached on disk) while
``AUTOTUNE`` is true, else the library's default shape.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

__all__ = [
    "oseen_kernel_source_target_numba", "oseen_kernel_times_density_numba",
    "rotlet_kernel_source_target_numba", "stresslet_kernel_source_target_numba",
    "stresslet_kernel_times_normal_times_density_numba", "stresslet_kernel_times_normal_numba",
    "traction_kernel_times_normal_times_density_numba", "stresslet_kernel",
    "stresslet_kernel_times_normal", "oseen_tensor", "oseen_tensor_source_target",
    "complementary_kernel", "complementary_kernel_times_density_numba",
    "oseen_kernel_source_target_pycuda", "oseen_kernel_source_target_stkfmm",
    "stresslet_kernel_source_target_stkfmm", "single_double_layer_kernel_source_target_stkfmm",
    "pair_sum",
]

# The FMM-backed functions (STKFMM) leave out a source that coincides with
# the target; the direct sums that stand in for them drop pairs closer than
# this distance (squared: 1e-300, a normal double) and regularise nothing.
COINCIDENT = 1e-150


# Launch shapes of the pair-sum drop-ins come from the autotuner (see above).
AUTOTUNE = True


# ------------------------------------------------------------------ helpers --
def _device() -> torch.device:
    _lib.lib()  # raises if no CUDA device or no library
    return torch.device("cuda", torch.cuda.current_device())


def _to_dev(x, dev: torch.device, name: str) -> torch.Tensor:
    """(N,3) contiguous float64 CUDA tensor from a numpy array or torch tensor."""
    if isinstance(x, torch.Tensor):
        t = x.detach()
        if t.device != dev or t.dtype != torch.float64:
            # from page-locked memory the copy is queued on the stream like
            # the kernel that reads it; the result comes back synchronously
            t = t.to(device=dev, dtype=torch.float64, non_blocking=t.device.type == "cpu" and t.is_pinned())
    else:
        a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
        t = torch.from_numpy(a).to(dev)
    if t.numel() % 3 != 0:
        raise ValueError(f"{name}: size {t.numel()} is not a multiple of 3")
    return t.reshape(-1, 3).contiguous()


def _any_host(*xs) -> bool:
    return any(not (isinstance(x, torch.Tensor) and x.is_cuda) for x in xs if x is not None)


def _out(u: torch.Tensor, host: bool, what: str = "kernels"):
    """The result as the caller wants it.  For host callers it is copied into
    a new page-locked array on the stream together with the device error
    word, and one wait covers both: a bounded wait that ran out in this call's
    kernels raises here instead of returning numbers."""
    u = u.reshape(-1)
    if not host:
        return u
    h = torch.empty(u.shape, dtype=u.dtype, pin_memory=True)
    h.copy_(u, non_blocking=True)
    word = _lib.ErrorPeek.queue(u.device)
    torch.cuda.current_stream(u.device).synchronize()
    if int(word[0]) != 0:
        _lib.check_device_error(what, u.device)
    return h.numpy()


def _resolve_precision(precision) -> int:
    if isinstance(precision, int):
        return precision
    try:
        return _lib.PRECISION[precision]
    except KeyError as e:
        raise ValueError(f"precision must be one of {list(_lib.PRECISION)}") from e


def pair_sum(kernel: str, r_source, r_target, density, normal=None, *, eta=1.0, reg=5e-3,
             epsilon_distance=1e-5, self_mode: str = "regularise", src_group=None,
             trg_group=None, precision="fp64", shape: _lib.PairShape | None = None,
             out: torch.Tensor | None = None, accumulate: bool = False):
    """General all-pairs sum on CUDA tensors (the building block of the drop-ins).

    Returns a flat CUDA float64 tensor of length 3*Nt (``out`` if given).
    """
    dev = _device()
    rs = _to_dev(r_source, dev, "r_source")
    rt = rs if r_target is r_source else _to_dev(r_target, dev, "r_target")
    d = _to_dev(density, dev, "density")
    if d.shape[0] != rs.shape[0]:
        raise ValueError(f"density has {d.shape[0]} points, r_source has {rs.shape[0]}")
    n = None
    if kernel in ("stresslet", "traction"):
        if normal is None:
            raise ValueError(f"{kernel} needs normals")
        n = _to_dev(normal, dev, "normal")
        # the stresslet takes the sources' normals, the traction the targets'
        want, who = (rs.shape[0], "r_source") if kernel == "stresslet" else (rt.shape[0], "r_target")
        if n.shape[0] != want:
            raise ValueError(f"normal has {n.shape[0]} points, {who} has {want}")
    gs = gt = None
    if self_mode == "skip_group":
        gs = torch.as_tensor(src_group, dtype=torch.int32, device=dev).contiguous()
        gt = gs if trg_group is src_group else torch.as_tensor(trg_group, dtype=torch.int32, device=dev).contiguous()
        if gs.numel() != rs.shape[0] or gt.numel() != rt.shape[0]:
            raise ValueError("group id arrays must have one entry per point")
    ns, nt = rs.shape[0], rt.shape[0]
    if out is None:
        out = torch.empty(3 * nt, dtype=torch.float64, device=dev)
    elif out.numel() != 3 * nt or out.dtype != torch.float64 or not out.is_contiguous():
        raise ValueError("out must be a contiguous float64 tensor of length 3*Nt")
    _launch(dev, _lib.KERNEL[kernel], _resolve_precision(precision), _lib.SELF_MODE[self_mode], rs, rt, d, n,
            gs, gt, out, float(eta), float(reg), float(epsilon_distance), accumulate, shape)
    return out


_ws_bytes: dict = {}
_host_bytes: dict = {}  # (kernel, ns, nt, one point set) -> f3d_pair_host_bytes
_tuned: dict = {}  # host fast path: (device, sum, sizes, one point set) -> tuned launch shape


def _launch(dev, k: int, p: int, m: int, rs, rt, d, n, gs, gt, out, eta: float, reg: float, eps: float,
            accumulate: bool, shape) -> None:
    """One f3d_pair_sum on validated device tensors (the workspace size of a
    (kernel, precision, sizes, shape) is asked of the library once)."""
    ns, nt = rs.shape[0], rt.shape[0]
    shp = ctypes.byref(shape) if shape is not None else None
    key = (k, p, ns, nt, None if shape is None else (shape.tpt, shape.sl, shape.nsplit, shape.use_tma))
    nbytes = _ws_bytes.get(key)
    if nbytes is None:
        nb = ctypes.c_size_t(0)
        _lib.call("f3d_pair_workspace_bytes", k, p, ns, nt, shp, ctypes.byref(nb))
        nbytes = _ws_bytes[key] = nb.value
    ws_ptr, ws_len = _lib.Workspace.get(dev).ensure(nbytes)
    _lib.call("f3d_pair_sum", k, p, m, _lib.ptr(rs), _lib.ptr(rt), _lib.ptr(d), _lib.ptr(n),
              _lib.ptr(gs), _lib.ptr(gt), _lib.ptr(out), ns, nt, eta, reg, eps, int(bool(accumulate)), shp,
              ws_ptr, ws_len, _lib.stream_handle(dev))


def _host_points(x, name: str):
    """A host (N, 3) float64 array (numpy or CPU tensor) -> (contiguous array
    or tensor kept alive, its address, N)."""
    if isinstance(x, torch.Tensor):
        t = x
        if t.dtype != torch.float64 or not t.is_contiguous():
            t = t.detach().to(torch.float64).contiguous()
        n = t.numel()
        ptr = t.data_ptr()
    else:
        t = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
        n = t.size
        ptr = t.ctypes.data
    if n % 3 != 0:
        raise ValueError(f"{name}: size {n} is not a multiple of 3")
    return t, ptr, n // 3


def _drop_in_host(kernel, r_source, r_target, density, normal, self_mode, eta, reg, epsilon_distance,
                  precision, shape, dev):
    """All inputs on the host and the launch shape known: one library call
    stages the inputs, runs the sum, copies the result back and waits
    (f3d_pair_sum_host)."""
    rs, p_rs, ns = _host_points(r_source, "r_source")
    if r_target is r_source:
        rt, p_rt, nt = rs, p_rs, ns
    else:
        rt, p_rt, nt = _host_points(r_target, "r_target")
    d, p_d, nd = _host_points(density, "density")
    p_n, nn = None, None
    if normal is not None:
        nrm, p_n, nn = _host_points(normal, "normal")
    if nd != ns or (nn is not None and nn != (nt if kernel == "traction" else ns)):
        raise ValueError("density / normal point counts do not match the points")
    k, p, m = _lib.KERNEL[kernel], _resolve_precision(precision), _lib.SELF_MODE[self_mode]
    out = torch.empty(3 * nt, dtype=torch.float64, pin_memory=True)
    if nt == 0:
        return out.numpy()
    shp = ctypes.byref(shape) if shape is not None else None
    key = (k, p, ns, nt, None if shape is None else (shape.tpt, shape.sl, shape.nsplit, shape.use_tma))
    nbytes = _ws_bytes.get(key)
    if nbytes is None:
        nb = ctypes.c_size_t(0)
        _lib.call("f3d_pair_workspace_bytes", k, p, ns, nt, shp, ctypes.byref(nb))
        nbytes = _ws_bytes[key] = nb.value
    ws_ptr, ws_len = _lib.Workspace.get(dev).ensure(nbytes)
    hkey = (k, ns, nt, p_rs == p_rt)
    hbytes = _host_bytes.get(hkey)
    if hbytes is None:
        hb = ctypes.c_size_t(0)
        _lib.call("f3d_pair_host_bytes", k, ns, nt, int(p_rs == p_rt), ctypes.byref(hb))
        hbytes = _host_bytes[hkey] = hb.value
    st_ptr, st_len = _lib.Staging.get(dev).ensure(hbytes)
    status = _lib.lib().f3d_pair_sum_host(k, p, m, p_rs, p_rt, p_d, p_n, out.data_ptr(), ns, nt, float(eta),
                                          float(reg), float(epsilon_distance), shp, st_ptr, st_len, ws_ptr, ws_len,
                                          _lib.stream_handle(dev))
    if status != _lib.F3D_OK:
        if status == _lib.F3D_ERR_TIMEOUT:
            _lib.Workspace.reset_all()
        _lib.check("f3d_pair_sum_host", status)
    return out.numpy()


def _drop_in(kernel, r_source, r_target, density, normal, self_mode, eta, reg, epsilon_distance,
             precision, shape):
    """A pair-sum drop-in: inputs to the device once, the autotuned launch
    shape unless one is given, the sum, the output back like the inputs.
    With every input on the host and the shape known (given, tuned earlier
    for this size bucket, or the library default when tuning is off), one
    library call does it all."""
    host = _any_host(r_source, r_target, density, normal)
    dev = _device()
    if host and not any(isinstance(x, torch.Tensor) and x.is_cuda for x in (r_source, r_target, density, normal)):
        if shape is None and AUTOTUNE:
            size = lambda a: a.numel() if isinstance(a, torch.Tensor) else np.size(a)
            key = (dev.index, kernel, precision, self_mode, size(r_source) // 3, size(r_target) // 3,
                   r_target is r_source)
            shp = _tuned.get(key)
            if shp is None:
                from . import autotune
                shp = autotune.cached(kernel, precision, self_mode, key[4], key[5], same=key[6])
                if shp is not None:
                    _tuned[key] = shp
            if shp is not None:
                return _drop_in_host(kernel, r_source, r_target, density, normal, self_mode, eta, reg,
                                     epsilon_distance, precision, shp, dev)
        else:
            return _drop_in_host(kernel, r_source, r_target, density, normal, self_mode, eta, reg,
                                 epsilon_distance, precision, shape, dev)
    rs = _to_dev(r_source, dev, "r_source")
    rt = rs if r_target is r_source else _to_dev(r_target, dev, "r_target")
    d = _to_dev(density, dev, "density")
    n = _to_dev(normal, dev, "normal") if normal is not None else None
    if d.shape[0] != rs.shape[0] or (n is not None and n.shape[0] != (rt if kernel == "traction" else rs).shape[0]):
        raise ValueError("density / normal point counts do not match the points")
    if shape is None and AUTOTUNE and rs.shape[0] and rt.shape[0]:
        from . import autotune
        shape = autotune.tune(kernel, rs, rt, d, n, self_mode=self_mode, precision=precision, eta=eta,
                              reg=reg, epsilon_distance=epsilon_distance)
    u = torch.empty(3 * rt.shape[0], dtype=torch.float64, device=dev)
    _launch(dev, _lib.KERNEL[kernel], _resolve_precision(precision), _lib.SELF_MODE[self_mode], rs, rt, d, n,
            None, None, u, float(eta), float(reg), float(epsilon_distance), False, shape)
    return _out(u, host, kernel)


# ------------------------------------------------------------ pair sums ----
def oseen_kernel_source_target_numba(r_source, r_target, density, eta=1.0, reg=5e-3,
                                     epsilon_distance=1e-5, *, precision="fp64", shape=None):
    """u_t = 1/(8 pi eta) sum_s [f_s/r + (r.f_s) r/r^3], r = x_t - x_s; pairs with
    r < epsilon_distance use sqrt(r^2 + reg^2).  fiber3d kernels.py:794-846."""
    return _drop_in("oseen", r_source, r_target, density, None, "regularise", eta, reg, epsilon_distance,
                    precision, shape)


def oseen_kernel_times_density_numba(r_vectors, density, eta=1.0, reg=5e-3,
                                     epsilon_distance=1e-5, *, precision="fp64", shape=None):
    """Oseen sum over one point set with the pair j == i skipped (other close
    pairs regularised).  fiber3d kernels.py:214-287."""
    return _drop_in("oseen", r_vectors, r_vectors, density, None, "skip_index", eta, reg, epsilon_distance,
                    precision, shape)


def rotlet_kernel_source_target_numba(r_source, r_target, density, eta=1.0, reg=5e-3,
                                      epsilon_distance=1e-5, *, precision="fp64", shape=None):
    """u_t = 1/(8 pi eta) sum_s tau_s x r / r^3.  fiber3d kernels.py:856-908."""
    return _drop_in("rotlet", r_source, r_target, density, None, "regularise", eta, reg, epsilon_distance,
                    precision, shape)


def stresslet_kernel_source_target_numba(r_source, r_target, normal, density, eta=1.0,
                                         reg=5e-3, epsilon_distance=1e-5, *, precision="fp64",
                                         shape=None):
    """v_t = -3/(4 pi eta) sum_s (r.d_s)(r.n_s) r / r^5.  fiber3d kernels.py:1186-1217."""
    return _drop_in("stresslet", r_source, r_target, density, normal, "regularise", eta, reg,
                    epsilon_distance, precision, shape)


def stresslet_kernel_times_normal_times_density_numba(r_vectors, normal, density, eta=1.0,
                                                      reg=5e-3, epsilon_distance=1e-5, *,
                                                      precision="fp64", shape=None):
    """Stresslet sum over one point set, j == i skipped.  fiber3d kernels.py:1123-1183."""
    return _drop_in("stresslet", r_vectors, r_vectors, density, normal, "skip_index", eta, reg,
                    epsilon_distance, precision, shape)


def traction_kernel_times_normal_times_density_numba(r_vectors, normal, density, eta=1.0,
                                                     reg=5e-3, epsilon_distance=1e-5, *,
                                                     precision="fp64", shape=None):
    """t_i = -3/(4 pi eta) sum_{j != i} (r.d_j)(r.n_i) r / r^5, r = x_i - x_j:
    the stresslet contracted with the normal of the TARGET (the traction of
    the single layer).  fiber3d kernels.py:1221-1264; its ``eta = 1.0`` at
    :1232 comes after the prefactor is formed, so the eta passed in is the
    one that counts."""
    return _drop_in("traction", r_vectors, r_vectors, density, normal, "skip_index", eta, reg,
                    epsilon_distance, precision, shape)


def oseen_kernel_source_target_pycuda(r_source, r_target, density, eta=1.0, epsilon_distance=1e-5):
    """Oseen source -> target sum in which pairs closer than epsilon_distance
    contribute nothing (no regularisation): the semantics of fiber3d's PyCUDA
    kernel (kernels.py:849 -> kernels_pycuda.py:22-66, which skips a pair
    when 1/|r| > 1/epsilon_distance).  The output starts from zero."""
    return _drop_in("oseen", r_source, r_target, density, None, "skip_close", eta, 0.0,
                    epsilon_distance, "fp64", None)


def _fmm_handle(kwargs):
    """The package FMM behind a ``fmm_PVel`` argument (a ``stkfmm.STKFMM`` of
    this package, or an ``fmm.FMM``), else None: any other handle (one of the
    external STKFMM library, say) is accepted and left unused, and the sum is
    then the exact direct one."""
    h = kwargs.get("fmm_PVel")
    if h is None:
        return None
    from . import fmm as F, stkfmm as S
    if isinstance(h, S.STKFMM):
        return h.fmm
    if isinstance(h, F.FMM):
        return h
    return None


def _fmm_sum(fmm, r_sl, r_dl, r_target, f_sl, normal, dens_dl, eta, host):
    """The FMM evaluation of the reference's *_stkfmm functions: the tree is
    rebuilt only when the sources or targets changed (kernels.py:1328-1352),
    its box the bounding cube with a 10 % margin (:1339-1348)."""
    dev = fmm.device
    pts = [None if a is None else _to_dev(a, dev, name) for a, name in
           ((r_sl, "r_source_SL"), (r_dl, "r_source_DL"), (r_target, "r_target"))]
    pts = [None if p is None or p.shape[0] == 0 else p for p in pts]
    last = getattr(fmm, "_drop_in_points", None)
    same = last is not None and all(
        (a is None and b is None) or (a is not None and b is not None and a.shape == b.shape and torch.equal(a, b))
        for a, b in zip(pts, last))
    if not same:
        fmm.set_points(*pts)
        fmm._drop_in_points = [None if p is None else p.clone() for p in pts]
    u = fmm.evaluate(sl_density=None if pts[0] is None else _to_dev(f_sl, dev, "density_SL"),
                     dl_normal=None if pts[1] is None else _to_dev(normal, dev, "normal"),
                     dl_density=None if pts[1] is None else _to_dev(dens_dl, dev, "density_DL"), eta=eta)
    return _out(u, host, "fmm")


def oseen_kernel_source_target_stkfmm(r_source, r_target, density, eta=1.0, reg=5e-3,
                                      epsilon_distance=1e-5, *args, **kwargs):
    """fiber3d's STKFMM Stokeslet (kernels.py:1298-1364):
    u_t = 1/(8 pi eta) sum_s [f/r + (r.f) r/r^3], nothing regularised,
    coincident source-target pairs left out.  With ``fmm_PVel`` (this
    package's ``stkfmm.STKFMM`` or ``fmm.FMM``) by the GPU FMM, accurate to
    its expansion order, the tree kept while the points do not change; without
    it by direct summation on the GPU (exact).  ``reg`` and
    ``epsilon_distance`` are accepted and unused, as in fiber3d."""
    fmm = _fmm_handle(kwargs)
    if fmm is not None:
        return _fmm_sum(fmm, r_source, None, r_target, density, None, None, eta,
                        _any_host(r_source, r_target, density))
    return _drop_in("oseen", r_source, r_target, density, None, "skip_close", eta, 0.0,
                    COINCIDENT, "fp64", None)


def stresslet_kernel_source_target_stkfmm(r_source, r_target, normal, density, eta=1.0, reg=5e-3,
                                          epsilon_distance=1e-5, *args, **kwargs):
    """fiber3d's STKFMM double layer (kernels.py:1367-1419):
    v_t = -3/(4 pi eta) sum_s (r.n_s)(r.d_s) r / r^5.  fiber3d hands the FMM
    the double-layer tensor 2 (n (x) d) (:1410) because STKFMM's double-layer
    kernel carries half of fiber3d's prefactor; the product is this stresslet
    sum, the one fiber3d checks the FMM against (kernels/test_stkfmm.py).
    Coincident pairs are left out, nothing is regularised.  By the GPU FMM
    with ``fmm_PVel``, else by direct summation."""
    fmm = _fmm_handle(kwargs)
    if fmm is not None:
        return _fmm_sum(fmm, None, r_source, r_target, None, normal, density, eta,
                        _any_host(r_source, r_target, normal, density))
    return _drop_in("stresslet", r_source, r_target, density, normal, "skip_close", eta, 0.0,
                    COINCIDENT, "fp64", None)


def single_double_layer_kernel_source_target_stkfmm(r_source_SL, r_source_DL, r_target, normal,
                                                    density_SL, density_DL, eta=1.0, reg=5e-3,
                                                    epsilon_distance=1e-5, *args, **kwargs):
    """fiber3d's combined STKFMM evaluation (kernels.py:1422-1485): the
    Stokeslet sum of density_SL at r_source_SL plus the double layer of
    (normal, density_DL) at r_source_DL (fiber3d's 2 (n (x) d) tensor, :1476),
    on the same targets; coincident pairs left out.  By the GPU FMM with
    ``fmm_PVel``, else by direct summation."""
    host = _any_host(r_source_SL, r_source_DL, r_target, normal, density_SL, density_DL)
    fmm = _fmm_handle(kwargs)
    if fmm is not None:
        return _fmm_sum(fmm, r_source_SL, r_source_DL, r_target, density_SL, normal, density_DL, eta, host)
    dev = _device()
    rt = _to_dev(r_target, dev, "r_target")
    u = torch.zeros(3 * rt.shape[0], dtype=torch.float64, device=dev)
    rsl = _to_dev(r_source_SL, dev, "r_source_SL")
    if rsl.shape[0]:
        pair_sum("oseen", rsl, rt, _to_dev(density_SL, dev, "density_SL"), eta=eta, reg=0.0,
                 epsilon_distance=COINCIDENT, self_mode="skip_close", out=u, accumulate=True)
    rdl = _to_dev(r_source_DL, dev, "r_source_DL")
    if rdl.shape[0]:
        pair_sum("stresslet", rdl, rt, _to_dev(density_DL, dev, "density_DL"), _to_dev(normal, dev, "normal"),
                 eta=eta, reg=0.0, epsilon_distance=COINCIDENT, self_mode="skip_close", out=u,
                 accumulate=True)
    return _out(u, host, "single_double_layer")


def complementary_kernel_times_density_numba(r_vectors, normal, density):
    """u_i = n_i sum_j n_j . d_j (rank-one).  fiber3d kernels.py:1267-1283.

    The reference spends O(N^2) on this O(N) product; here it is one reduction
    and one scaling on the device.
    """
    dev = _device()
    n = _to_dev(normal, dev, "normal")
    d = _to_dev(density, dev, "density")
    s = (n * d).sum()
    u = n * s
    return _out(u, _any_host(r_vectors, normal, density))


# ------------------------------------------------------- dense operators ---
def _dense_out(nrows: int, ncols: int, dev) -> torch.Tensor:
    return torch.empty((nrows, ncols), dtype=torch.float64, device=dev)


def stresslet_kernel_times_normal_numba(r_vectors, normal, eta=1.0, reg=5e-3,
                                        epsilon_distance=1e-5):
    """Dense 3N x 3N double-layer matrix, block S_ij = -3/(4 pi eta) (r.n_j)/r^5 r r^T,
    r = x_i - x_j, zero diagonal blocks.  fiber3d kernels.py:1063-1120."""
    dev = _device()
    x = _to_dev(r_vectors, dev, "r_vectors")
    n = _to_dev(normal, dev, "normal")
    N = x.shape[0]
    M = _dense_out(3 * N, 3 * N, dev)
    _lib.call("f3d_stresslet_times_normal_dense", _lib.ptr(x), _lib.ptr(n), _lib.ptr(M), N, 3 * N,
              float(eta), float(reg), float(epsilon_distance), _lib.stream_handle(dev))
    return M.cpu().numpy() if _any_host(r_vectors, normal) else M


def stresslet_kernel_times_normal(r_vectors, normal, eta=1.0, reg=5e-3, epsilon_distance=1e-5):
    """Dense 3N x 3N stresslet contracted with the source normals: block
    (i, j) = 3/(4 pi eta) (dr.n_j) dr dr^T / dr^5 with dr = x_j - x_i, which
    is the same matrix as stresslet_kernel_times_normal_numba (r = -dr), zero
    diagonal blocks; pairs closer than epsilon_distance regularised.  fiber3d
    kernels.py:995-1060 (numpy form)."""
    return stresslet_kernel_times_normal_numba(r_vectors, normal, eta, reg, epsilon_distance)


def stresslet_kernel(r_vectors, eta=1.0, reg=5e-3, epsilon_distance=1e-5, input_format='r'):
    """Dense 3-index stresslet tensor, (3N) x (3N) x 3: S[3i+a, 3j+b, c] =
    fr dr_a dr_b dr_c, dr = x_j - x_i, fr = -3/(4 pi eta dr^5) (dr <=
    epsilon_distance: (dr^2 + reg^2)^(5/2) in place of dr^5), zero diagonal
    blocks.  input_format 'r' ((N, 3) points) or 'xyz' (x_all, y_all, z_all).
    fiber3d kernels.py:911-992."""
    dev = _device()
    host = _any_host(r_vectors)
    size = r_vectors.numel() if isinstance(r_vectors, torch.Tensor) else np.size(r_vectors)
    N = size // 3
    xin = _xyz_to_r(r_vectors, N) if input_format != 'r' else r_vectors
    x = _to_dev(xin, dev, "r_vectors")
    S = torch.empty((3 * N, 3 * N, 3), dtype=torch.float64, device=dev)
    _lib.call("f3d_stresslet_tensor_dense", _lib.ptr(x), _lib.ptr(S), N, float(eta), float(reg),
              float(epsilon_distance), _lib.stream_handle(dev))
    return S.cpu().numpy() if host else S


def _xyz_to_r(x, N):
    """'xyz' layout (x_all, y_all, z_all) -> (N, 3)."""
    if isinstance(x, torch.Tensor):
        return x.reshape(3, N).t().contiguous()
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(3, N).T)


def _perm_r_to_xyz(N: int) -> np.ndarray:
    # row/col index in 'xyz' order -> index in 'r' (interleaved) order
    return (np.arange(3)[:, None] + 3 * np.arange(N)[None, :]).reshape(-1)


def oseen_tensor(r_vectors, eta=1.0, reg=5e-3, epsilon_distance=1e-5, input_format='r'):
    """Dense 3N x 3N Oseen tensor; r <= epsilon_distance regularised (so the
    diagonal block is I/(8 pi eta reg)).  fiber3d kernels.py:31-116."""
    dev = _device()
    host = _any_host(r_vectors)
    size = r_vectors.numel() if isinstance(r_vectors, torch.Tensor) else np.size(r_vectors)
    N = size // 3
    xin = _xyz_to_r(r_vectors, N) if input_format != 'r' else r_vectors
    x = _to_dev(xin, dev, "r_vectors")
    G = _dense_out(3 * N, 3 * N, dev)
    _lib.call("f3d_oseen_tensor_dense", _lib.ptr(x), _lib.ptr(G), N, 3 * N, float(eta),
              float(reg), float(epsilon_distance), _lib.stream_handle(dev))
    if input_format != 'r':
        p = torch.as_tensor(_perm_r_to_xyz(N), device=dev)
        G = G[p][:, p].contiguous()
    return G.cpu().numpy() if host else G


def oseen_tensor_source_target(r_source, r_target, eta=1.0, reg=5e-3, epsilon_distance=1e-5,
                               input_format='r'):
    """Dense 3Nt x 3Ns Oseen tensor.  fiber3d kernels.py:119-211."""
    dev = _device()
    host = _any_host(r_source, r_target)
    sz = lambda a: a.numel() if isinstance(a, torch.Tensor) else np.size(a)
    Ns, Nt = sz(r_source) // 3, sz(r_target) // 3
    if input_format != 'r':
        r_source, r_target = _xyz_to_r(r_source, Ns), _xyz_to_r(r_target, Nt)
    xs = _to_dev(r_source, dev, "r_source")
    xt = _to_dev(r_target, dev, "r_target")
    G = _dense_out(3 * Nt, 3 * Ns, dev)
    _lib.call("f3d_oseen_tensor_source_target_dense", _lib.ptr(xs), _lib.ptr(xt), _lib.ptr(G),
              Ns, Nt, 3 * Ns, float(eta), float(reg), float(epsilon_distance),
              _lib.stream_handle(dev))
    if input_format != 'r':
        pt = torch.as_tensor(_perm_r_to_xyz(Nt), device=dev)
        ps = torch.as_tensor(_perm_r_to_xyz(Ns), device=dev)
        G = G[pt][:, ps].contiguous()
    return G.cpu().numpy() if host else G


def complementary_kernel(r_vectors, normal):
    """Dense outer(normal.flat, normal.flat).  fiber3d kernels.py:1286-1295."""
    dev = _device()
    n = _to_dev(normal, dev, "normal")
    N = n.shape[0]
    C = _dense_out(3 * N, 3 * N, dev)
    _lib.call("f3d_complementary_dense", _lib.ptr(n), _lib.ptr(C), N, 3 * N,
              _lib.stream_handle(dev))
    return C.cpu().numpy() if _any_host(normal) else C
