"""ctypes binding of ``libfiber3d_b200.so`` (the C ABI in include/fiber3d_b200.h).

The library is loaded from ``fiber3d_b200/_lib/`` (built in-tree by
``fiber3d_b200.build``).  There is no CPU fallback: if the library or a CUDA
device is missing, :func:`lib` raises.  Device memory, streams and the
workspace come from PyTorch; every call goes through the C ABI with plain
pointers.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import torch

LIBPATH = Path(__file__).resolve().parent / "_lib" / "libfiber3d_b200.so"

# status codes (f3d_status)
F3D_OK = 0
F3D_ERR_TIMEOUT = 8
F3D_ERR_SINGULAR = 9

# enums
KERNEL = {"oseen": 0, "stresslet": 1, "rotlet": 2, "traction": 3}
SELF_MODE = {"regularise": 0, "skip_index": 1, "skip_group": 2, "skip_close": 3}
PRECISION = {"fp64": 0, "fp32c": 1}


class F3DError(RuntimeError):
    """A C-ABI call returned a non-zero f3d_status."""

    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn}: status {status} ({msg})")
        self.status = status


class PairShape(ctypes.Structure):
    _fields_ = [("tpt", ctypes.c_int32), ("sl", ctypes.c_int32),
                ("nsplit", ctypes.c_int32), ("use_tma", ctypes.c_int32)]


class FiberSetC(ctypes.Structure):
    """f3d_fiber_set (device pointers)."""
    _fields_ = [("nfib", ctypes.c_int32), ("n", ctypes.c_void_p), ("pt_off", ctypes.c_void_p),
                ("mat_off", ctypes.c_void_p), ("res_off", ctypes.c_void_p),
                ("length", ctypes.c_void_p), ("bc", ctypes.c_void_p), ("pt_fib", ctypes.c_void_p),
                ("mats", ctypes.c_void_p), ("band", ctypes.c_int32)]


_lock = threading.Lock()
_lib = None

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double
_I = ctypes.c_int
_SZ = ctypes.c_size_t

# name -> argtypes; every function returns int (f3d_status) unless listed in _RESTYPE.
SIGNATURES: dict[str, list] = {
    "f3d_version": [],
    "f3d_status_string": [_I],
    "f3d_get_device_error": [_P],
    "f3d_peek_device_error_async": [_P, _P],
    "f3d_set_wait_limit_ns": [ctypes.c_uint64],
    "f3d_wait_limit_ns": [],
    "f3d_selftest_bounded_wait": [ctypes.c_uint64, _P],
    "f3d_probe_fma": [_I, _I, _P, ctypes.POINTER(_D), _P],
    "f3d_pair_workspace_bytes": [_I, _I, _I64, _I64, ctypes.POINTER(PairShape), ctypes.POINTER(_SZ)],
    "f3d_pair_sum": [_I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _I64, _I64, _D, _D, _D, _I,
                     ctypes.POINTER(PairShape), _P, _SZ, _P],
    "f3d_oseen_dual_workspace_bytes": [_I64, _I64, ctypes.POINTER(PairShape), ctypes.POINTER(_SZ)],
    "f3d_oseen_dual": [_I, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _I64, _D, _D, _D, _I, ctypes.POINTER(PairShape), _P,
                       _SZ, _P],
    "f3d_pair_host_bytes": [_I, _I64, _I64, _I, ctypes.POINTER(_SZ)],
    "f3d_pair_sum_host": [_I, _I, _I, _P, _P, _P, _P, _P, _I64, _I64, _D, _D, _D, ctypes.POINTER(PairShape), _P,
                          _SZ, _P, _SZ, _P],
    "f3d_pair_occupancy": [_I, _I, _I, _I, ctypes.POINTER(PairShape), ctypes.POINTER(_I)],
    "f3d_pair_sum_noalloc": [_I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _I64, _I64, _D, _D, _D, _I, _P],
    "f3d_oseen_source_target": [_P, _P, _P, _P, _I64, _I64, _D, _D, _D, _I, _P, _SZ, _P],
    "f3d_oseen_times_density": [_P, _P, _P, _I64, _D, _D, _D, _I, _P, _SZ, _P],
    "f3d_rotlet_source_target": [_P, _P, _P, _P, _I64, _I64, _D, _D, _D, _I, _P, _SZ, _P],
    "f3d_stresslet_source_target": [_P, _P, _P, _P, _P, _I64, _I64, _D, _D, _D, _I, _P, _SZ, _P],
    "f3d_stresslet_times_normal_times_density": [_P, _P, _P, _P, _I64, _D, _D, _D, _I, _P, _SZ, _P],
    "f3d_stresslet_times_normal_dense": [_P, _P, _P, _I64, _I64, _D, _D, _D, _P],
    "f3d_oseen_tensor_dense": [_P, _P, _I64, _I64, _D, _D, _D, _P],
    "f3d_oseen_tensor_source_target_dense": [_P, _P, _P, _I64, _I64, _I64, _D, _D, _D, _P],
    "f3d_complementary_dense": [_P, _P, _I64, _I64, _P],
    "f3d_stresslet_tensor_dense": [_P, _P, _I64, _D, _D, _D, _P],
    "f3d_batched_lu_workspace_bytes": [ctypes.POINTER(_SZ)],
    "f3d_singularity_vectors_workspace_bytes": [_I64, ctypes.POINTER(_SZ)],
    "f3d_singularity_vectors": [_P, _P, _P, _P, _I64, _D, _D, _D, _P, _SZ, _P],
    "f3d_shell_residual": [_P, _P, _P, _P, _P, _P, _I64, _P, _P],
    "f3d_block3_gemv": [_P, _P, _P, _I64, _P],
    "f3d_shell_block_inverse": [_P, _P, _P, _P, _I64, _P, _P],
    "f3d_fmm_create": [_I, _I, _P, _P, _P, _P],
    "f3d_fmm_destroy": [_P],
    "f3d_fmm_set_box": [_P, _P, _D],
    "f3d_fmm_set_points": [_P, _I64, _P, _I64, _P, _I64, _P, _P],
    "f3d_fmm_evaluate": [_P, _P, _P, _P, _P, _P, _D, _P],
    "f3d_fmm_tree_info": [_P, _P, _P, _P, _P, _P],
    "f3d_fmm_last_launches": [_P, _P],
    "f3d_body_residual": [ctypes.c_int32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "f3d_surface_dense": [_I, _P, _P, _P, _P, _P, _P, _I64, _I64, _D, _D, _D, _P],
    "f3d_rotate_blocks": [_P, _P, _P, _P, ctypes.c_int32, _I, _P],
    "f3d_body_advance": [_P, _P, ctypes.c_int32, _D, _P, _P, _P, _P],
    "f3d_gemv_batched": [_P, _P, _P, _P, _P, ctypes.c_int32, _I64, _I, _P, _P, _P],
    "f3d_fiber_self_flow_up": [_P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P, ctypes.c_int32, _D, _D,
                               _D, _P, _P],
    "f3d_grid_near_fiber": [_P, _I64, _P, _P, ctypes.c_int32, _P, _D, _P, _P],
    "f3d_grid_rigid_override": [_P, _I64, _P, _P, _D, _P, _P],
    "f3d_surface_quadrature_workspace_bytes": [_I64, _I64, ctypes.POINTER(_SZ)],
    "f3d_surface_quadrature": [_P, _I64, _P, _I64, _P, _P, _P, _P, _SZ, _P],
    "f3d_rigid_body_update": [_P, _P, _P, _P, _P, _P, _I64, _P, _P, _P, _P],
    "f3d_gather_segments": [_P, _P, _P, _P, _P, ctypes.c_int32, _I64, _P],
    "f3d_krylov_workspace_bytes": [_I64, ctypes.c_int32, ctypes.POINTER(_SZ)],
    "f3d_krylov_multidot": [_P, _I64, _P, _P, ctypes.c_int32, _P, _I64, _I, _P, _SZ, _P],
    "f3d_krylov_multiaxpy": [_P, _I64, _P, _P, _P, _I64, _P],
    "f3d_krylov_combine": [_P, _I64, _P, ctypes.c_int32, _P, _I64, _I, _P],
    "f3d_krylov_norm": [_P, _I64, _P, _P, _P, _P, _SZ, _P],
    "f3d_krylov_scale_into": [_P, _P, _P, _P, _I64, _I64, _I, _P, _P],
    "f3d_krylov_store": [_P, _P, ctypes.c_int32, _P, _I64, _I64, _P],
    "f3d_gemv": [_I, _P, _I64, _P, _P, _I64, _I64, _P],
    "f3d_cast_to_float": [_P, _P, _I64, _P],
    "f3d_gemm_bf16": [_P, _I64, _I64, _P, _I64, _I64, _P, _I64, ctypes.c_int32, ctypes.c_int32,
                      ctypes.c_int32, _P, _I, _P, _I64, _P, ctypes.c_float, _I, _P],
    "f3d_colsum": [_P, _I64, ctypes.c_int32, ctypes.c_int32, _P, _I, _P],
    "f3d_adam": [_P, _P, _P, _P, _I64, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                 ctypes.c_int32, _P],
    "f3d_mse_grad": [_P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P],
    "f3d_fiber_geometry": [ctypes.POINTER(FiberSetC), _P, _P, _I64, _P],
    "f3d_fiber_assemble": [ctypes.POINTER(FiberSetC), _D, _D, _D, _D, _D, _P, _P, _P, _P, _P, _P, _P,
                           ctypes.c_int32, _P],
    "f3d_fiber_forces": [ctypes.POINTER(FiberSetC), _D, _P, _P, _P, _I64, _I, _P],
    "f3d_fiber_weight": [ctypes.POINTER(FiberSetC), _P, _P, _I64, _P],
    "f3d_fiber_residual": [ctypes.POINTER(FiberSetC), _P, _P, _P, _P, _P, ctypes.c_int32, _P],
    "f3d_batched_lu_factor": [_P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _SZ, _P],
    "f3d_batched_lu_factor_panel": [_P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P,
                                    _P, _SZ, _P],
    "f3d_batched_lu_solve": [_P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _SZ, _P],
    "f3d_quantize_rows_f16": [_P, _I64, _I64, _I64, ctypes.c_int32, _P, _I64, _P, _P, _P],
    "f3d_gemv_f16": [_P, _I64, _P, _P, ctypes.c_int32, _P, _P, _I64, _I64, _P],
    "f3d_warmstart_features": [_P, _P, _P, _P, _I64, _I64, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P, _P,
                               _P],
    "f3d_warmstart_guess": [_P, _P, _P, _I64, _I64, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P, _P],
    "f3d_batched_inverse": [_P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P],
    "f3d_dense_inverse_workspace_bytes": [_I64, _I64, _P],
    "f3d_dense_inverse": [_P, _I64, _I64, _P, _SZ, _P],
    "f3d_block_gemv": [_I, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P, _P],
}
_RESTYPE = {"f3d_version": ctypes.c_char_p, "f3d_status_string": ctypes.c_char_p,
            "f3d_wait_limit_ns": ctypes.c_uint64}


def load_library(path: Path | str = LIBPATH) -> ctypes.CDLL:
    """Load the shared library and attach prototypes (no CUDA device needed)."""
    path = Path(path)
    if not path.exists():
        raise ImportError(
            f"fiber3d_b200 CUDA library not found at {path}; build it with "
            "`python -m fiber3d_b200.build` (there is no CPU fallback)")
    dll = ctypes.CDLL(str(path))
    for name, argtypes in SIGNATURES.items():
        fn = getattr(dll, name)
        fn.argtypes = argtypes
        fn.restype = _RESTYPE.get(name, ctypes.c_int)
    return dll


def lib() -> ctypes.CDLL:
    """The loaded library; requires a CUDA device (the product path is GPU-only)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not torch.cuda.is_available():
                    raise RuntimeError("fiber3d_b200 needs a CUDA device; none is visible "
                                       "(there is no CPU fallback)")
                _lib = load_library()
    return _lib


def check(fn: str, status: int) -> None:
    if status != F3D_OK:
        msg = lib().f3d_status_string(status).decode()
        raise F3DError(fn, status, msg)


def call(fn: str, *args) -> None:
    check(fn, getattr(lib(), fn)(*args))


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_handle(device: torch.device | None = None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class Workspace:
    """Per-device zero-initialised scratch buffer, grown on demand.

    Kernels that use it return its counter words to zero, so it is zeroed only
    when (re)allocated, or after a device-side timeout.  Calls that share a
    workspace must be ordered on one stream.
    """

    _per_device: dict[int, "Workspace"] = {}

    def __init__(self, device: torch.device):
        self.device = device
        self.buf = torch.zeros(0, dtype=torch.uint8, device=device)

    @classmethod
    def get(cls, device: torch.device) -> "Workspace":
        idx = device.index if device.index is not None else torch.cuda.current_device()
        ws = cls._per_device.get(idx)
        if ws is None:
            ws = cls(torch.device("cuda", idx))
            cls._per_device[idx] = ws
        return ws

    def ensure(self, nbytes: int) -> tuple[int, int]:
        if nbytes > self.buf.numel():
            self.buf = torch.zeros(max(nbytes, 2 * self.buf.numel()), dtype=torch.uint8,
                                   device=self.device)
        if self.buf.numel() == 0:
            return 0, 0
        return self.buf.data_ptr(), self.buf.numel()

    def reset(self) -> None:
        self.buf.zero_()

    @classmethod
    def reset_all(cls) -> None:
        for ws in cls._per_device.values():
            ws.reset()


def device_error(device: torch.device | None = None) -> int:
    """Read and clear the device error word (F3D_OK, or the first failing status a kernel
    recorded: F3D_ERR_TIMEOUT, F3D_ERR_ARG, F3D_ERR_SINGULAR, F3D_ERR_TOO_LARGE)."""
    return lib().f3d_get_device_error(stream_handle(device))


def check_device_error(what: str, device: torch.device | None = None, on_error=None) -> None:
    """Raise F3DError if a kernel recorded a failure since the last read.

    A kernel whose bounded wait ran out returns early and may leave the split
    counters of a workspace non-zero, which would make later sums wrong; so
    on any recorded failure every shared pair workspace is zeroed (and
    ``on_error``, e.g. a solver's own workspace reset, is called) before the
    error is raised.  The next call then starts from a clean state.
    """
    status = device_error(device)
    if status != F3D_OK:
        Workspace.reset_all()
        if on_error is not None:
            on_error()
        raise F3DError(what, status, lib().f3d_status_string(status).decode())


class Staging(Workspace):
    """Per-device buffer that host-side sums stage their inputs and result
    in (f3d_pair_sum_host); grown on demand, never needs zeroing."""

    _per_device: dict[int, "Staging"] = {}

    def ensure(self, nbytes: int) -> tuple[int, int]:
        if nbytes > self.buf.numel():
            self.buf = torch.empty(max(nbytes, 2 * self.buf.numel()), dtype=torch.uint8, device=self.device)
        return (self.buf.data_ptr(), self.buf.numel()) if self.buf.numel() else (0, 0)


class ErrorPeek:
    """A page-locked word per device into which the device error word is
    copied on the stream (f3d_peek_device_error_async), so that a caller that
    waits for its results anyway learns of a failed kernel in the same wait."""

    _per_device: dict[int, torch.Tensor] = {}

    @classmethod
    def queue(cls, device: torch.device) -> torch.Tensor:
        idx = device.index if device.index is not None else torch.cuda.current_device()
        word = cls._per_device.get(idx)
        if word is None:
            word = cls._per_device[idx] = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        call("f3d_peek_device_error_async", word.data_ptr(), stream_handle(device))
        return word


def set_wait_limit_ns(limit_ns: int) -> None:
    """Limit (ns) of the kernels' bounded waits for later calls; 0 restores 2 s."""
    lib().f3d_set_wait_limit_ns(int(limit_ns))


def wait_limit_ns() -> int:
    return int(lib().f3d_wait_limit_ns())
