"""One implicit hydrodynamic time step of fiber3d, device-resident.

Mirrors ``tstep.time_step_hydro`` (python/tstep/tstep.py:628-1458) for free
fibers, rigid bodies and a confining periphery:

* unknown layout (tstep_utils.get_num_particles_and_offsets :906-931)
  ``[shell q (3 Nsh) | body k: lambda (3 Nb_k), U, Omega | fiber k: X_x, X_y, X_z, T]``;
* right-hand side: explicit flows of the external fiber forces
  (tstep.py:789-846) and the fiber systems (tstep_utils.py:1238-1338);
* matvec ``A_body_fiber_hyd`` (tstep.py:1003-1178);
* block preconditioner ``P_inv`` (tstep.py:950-994): explicit inverse of the
  dense periphery operator (computed once per periphery), batched LU of the
  body and fiber blocks.

All sums run in the library's pair kernels.  The matvec is two pair launches
— Oseen from the fiber points (pairs within one fiber skipped, which fuses
``flow_fibers`` and ``self_flow_fibers``) and one stresslet launch from the
body and periphery nodes together — onto every point, then three row
kernels (periphery, bodies, fibers).  ``precision='fp32c'`` runs both pair
launches in compensated FP32 for the inner solves of mixed precision.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .blocklu import BlockLU
from .fibers import FiberSet


@dataclass
class Body:
    """Rigid body surface: reference nodes/normals rotated by `rotation` and
    shifted to `location`; quadrature `weights`."""
    location: np.ndarray
    rotation: np.ndarray
    ref_nodes: np.ndarray
    ref_normals: np.ndarray
    weights: np.ndarray

    @property
    def nodes(self):
        return np.asarray(self.ref_nodes) @ np.asarray(self.rotation).T + np.asarray(self.location)

    @property
    def normals(self):
        return np.asarray(self.ref_normals) @ np.asarray(self.rotation).T


@dataclass
class Shell:
    nodes: np.ndarray
    normals: np.ndarray
    weights: np.ndarray


@dataclass
class Problem:
    """Inputs of one time step (fiber3d defaults: epsilon 1e-3, penalty 500,
    reg 5e-3, epsilon_distance 1e-5)."""
    fibers: list
    lengths: list
    E: float
    dt: float
    eta: float = 1.0
    bodies: list = field(default_factory=list)
    shell: Shell | None = None
    force_fibers: np.ndarray | None = None
    epsilon: float = 1e-3
    penalty: float = 500.0
    reg: float = 5e-3
    eps_dist: float = 1e-5

    def mobility(self):
        c0 = -np.log(np.e * self.epsilon ** 2) / (8.0 * np.pi * self.eta)
        c1 = 2.0 / (8.0 * np.pi * self.eta)
        return c0, c1


def quaternion_rotation(q) -> np.ndarray:
    """Rotation matrix of the unit quaternion (s, p1, p2, p3)."""
    s, p = float(q[0]), np.asarray(q[1:4], dtype=np.float64)
    d = s * s - 0.5
    return 2.0 * np.array([[p[0] ** 2 + d, p[0] * p[1] - s * p[2], p[0] * p[2] + s * p[1]],
                           [p[1] * p[0] + s * p[2], p[1] ** 2 + d, p[1] * p[2] - s * p[0]],
                           [p[2] * p[0] - s * p[1], p[2] * p[1] + s * p[0], p[2] ** 2 + d]])


def quaternion_from_rotation(phi) -> np.ndarray:
    """Unit quaternion of a rotation by |phi| about phi (quaternion.py:14-26)."""
    phi = np.asarray(phi, dtype=np.float64)
    a = float(np.linalg.norm(phi))
    if a == 0.0:
        return np.array([1.0, 0.0, 0.0, 0.0])
    return np.concatenate([[np.cos(a / 2.0)], np.sin(a / 2.0) * phi / a])


def quaternion_multiply(q, r) -> np.ndarray:
    """q r (quaternion.py:29-38)."""
    s = q[0] * r[0] - np.dot(q[1:], r[1:])
    p = q[0] * np.asarray(r[1:]) + r[0] * np.asarray(q[1:]) + np.cross(q[1:], r[1:])
    return np.concatenate([[s], p])


def rotation_to_quaternion(R) -> np.ndarray:
    """Unit quaternion of a rotation matrix (inverse of quaternion_rotation)."""
    R = np.asarray(R, dtype=np.float64)
    t = np.trace(R)
    if t > 0:
        s = np.sqrt(t + 1.0) * 2.0
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    elif R[0, 0] > R[1, 1] and R[0, 0] > R[2, 2]:
        s = np.sqrt(1.0 + R[0, 0] - R[1, 1] - R[2, 2]) * 2.0
        q = [(R[2, 1] - R[1, 2]) / s, 0.25 * s, (R[0, 1] + R[1, 0]) / s, (R[0, 2] + R[2, 0]) / s]
    elif R[1, 1] > R[2, 2]:
        s = np.sqrt(1.0 + R[1, 1] - R[0, 0] - R[2, 2]) * 2.0
        q = [(R[0, 2] - R[2, 0]) / s, (R[0, 1] + R[1, 0]) / s, 0.25 * s, (R[1, 2] + R[2, 1]) / s]
    else:
        s = np.sqrt(1.0 + R[2, 2] - R[0, 0] - R[1, 1]) * 2.0
        q = [(R[1, 0] - R[0, 1]) / s, (R[0, 2] + R[2, 0]) / s, (R[1, 2] + R[2, 1]) / s, 0.25 * s]
    q = np.asarray(q)
    return q / np.linalg.norm(q)


class PhaseTimers:
    """Named phase timers on CUDA events (the phases of fiber3d's
    utils/timer.py table: Build_linear_system_fibers, Build_PC_fibers, GMRES, ...)."""

    def __init__(self):
        self.open, self.done = {}, []

    def start(self, name):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.open[name] = e

    def stop(self, name):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.done.append((name, self.open.pop(name), e))

    def report(self) -> dict:
        torch.cuda.synchronize()
        out = {}
        for name, a, b in self.done:
            out[name] = out.get(name, 0.0) + a.elapsed_time(b)
        self.done.clear()
        return out


class ShellOperator:
    """Device data of a periphery: nodes, normals, weights, singularity
    vectors E and its preconditioner, built once per periphery.

    pc="dense" (fiber3d's choice, the LU of the dense shell operator,
    tstep.py:327-348): the explicit inverse of that operator in FP64, with
    FP32 and row-scaled FP16 copies for the inner solves of mixed precision;
    O(N^2) memory (10.4 + 5.2 + 2.6 GB at 12000 nodes).
    pc="block": the inverses of its 3 x 3 diagonal blocks,
    B_i = -(E_i + I) / w_i + n_i n_i^T (the double layer's own diagonal block
    is zero), O(N) memory and no factorisation; GMRES then resolves the
    periphery's nonlocal coupling itself (more iterations, same answer)."""

    def __init__(self, shell: Shell, eta=1.0, reg=5e-3, eps_dist=1e-5, device=None,
                 build_inverse=True, pc: str = "dense"):
        if pc not in ("dense", "block"):
            raise ValueError("pc must be 'dense' or 'block'")
        self.pc = pc
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        self.nodes = t(np.asarray(shell.nodes).reshape(-1, 3))
        self.normals = t(np.asarray(shell.normals).reshape(-1, 3))
        self.weights = t(np.asarray(shell.weights).reshape(-1))
        self.n = self.nodes.shape[0]
        self.eta, self.reg, self.eps = eta, reg, eps_dist
        self.E = singularity_vectors(self.nodes, self.normals, self.weights, eta, reg, eps_dist)
        self.inv64 = None
        self.inv32 = None
        self.inv16 = None
        self.block_inv = None
        self.ld = 3 * self.n
        if pc == "block":
            self.build_block_inverse()
        elif build_inverse:
            self.build_inverse()

    def build_block_inverse(self):
        """Inverses of the dense operator's 3 x 3 diagonal blocks
        (f3d_shell_block_inverse, on the device)."""
        self.block_inv = torch.empty((self.n, 9), dtype=torch.float64, device=self.device)
        info = torch.zeros(1, dtype=torch.int32, device=self.device)
        _lib.call("f3d_shell_block_inverse", _lib.ptr(self.E), _lib.ptr(self.weights), _lib.ptr(self.normals),
                  _lib.ptr(self.block_inv), self.n, _lib.ptr(info), _lib.stream_handle(self.device))
        bad = int(info.item())
        if bad:
            raise _lib.F3DError("f3d_shell_block_inverse", _lib.F3D_ERR_SINGULAR,
                                f"{bad} singular 3 x 3 periphery blocks")

    def dense(self) -> torch.Tensor:
        m = 3 * self.n
        M = torch.empty((m, m), dtype=torch.float64, device=self.device)
        _lib.call("f3d_surface_dense", 0, _lib.ptr(self.nodes), _lib.ptr(self.normals), _lib.ptr(self.E),
                  _lib.ptr(self.weights), None, _lib.ptr(M), self.n, m, self.eta, self.reg, self.eps,
                  _lib.stream_handle(self.device))
        return M

    def build_inverse(self):
        """Explicit inverse of the dense shell operator (one-time set-up):
        the operator is written into a buffer padded to a multiple of 128
        rows and inverted in place there (f3d_dense_inverse); inv64 and inv32
        are the top-left 3n x 3n views, row stride self.ld."""
        m = 3 * self.n
        self.ld = ld = dense_inverse_ld(m)
        full = torch.empty((ld, ld), dtype=torch.float64, device=self.device)
        _lib.call("f3d_surface_dense", 0, _lib.ptr(self.nodes), _lib.ptr(self.normals), _lib.ptr(self.E),
                  _lib.ptr(self.weights), None, _lib.ptr(full), self.n, ld, self.eta, self.reg, self.eps,
                  _lib.stream_handle(self.device))
        dense_inverse(full, m)
        self.inv64 = full[:m, :m]
        full32 = torch.empty((ld, ld), dtype=torch.float32, device=self.device)
        _lib.call("f3d_cast_to_float", _lib.ptr(full), _lib.ptr(full32), full.numel(),
                  _lib.stream_handle(self.device))
        self.inv32 = full32[:m, :m]
        # FP16 rows scaled by powers of two, the 3x3 node blocks on the
        # diagonal kept in FP64 (the inverse of this second-kind operator is
        # dominated by them; the rest spans a few decades per row)
        self.inv16 = torch.empty((m, m), dtype=torch.float16, device=self.device)
        self.scale16 = torch.empty(m, dtype=torch.float32, device=self.device)
        self.diag16 = torch.empty((m, 3), dtype=torch.float64, device=self.device)
        _lib.call("f3d_quantize_rows_f16", _lib.ptr(self.inv64), ld, m, m, 3, _lib.ptr(self.inv16), m,
                  _lib.ptr(self.scale16), _lib.ptr(self.diag16), _lib.stream_handle(self.device))

    def apply(self, x: torch.Tensor, y: torch.Tensor, storage: str = "fp64") -> torch.Tensor:
        """y = P_shell^-1 x from the FP64, FP32 or FP16 copy of the inverse
        (pc="block": the 3 x 3 block inverses, in FP64 whatever `storage`)."""
        m = 3 * self.n
        st = _lib.stream_handle(self.device)
        if self.pc == "block":
            _lib.call("f3d_block3_gemv", _lib.ptr(self.block_inv), _lib.ptr(x), _lib.ptr(y), self.n, st)
            return y
        if storage == "fp16":
            _lib.call("f3d_gemv_f16", _lib.ptr(self.inv16), m, _lib.ptr(self.scale16), _lib.ptr(self.diag16), 3,
                      _lib.ptr(x), _lib.ptr(y), m, m, st)
        else:
            M = self.inv64 if storage == "fp64" else self.inv32
            _lib.call("f3d_gemv", _lib.PRECISION["fp64" if storage == "fp64" else "fp32c"], _lib.ptr(M), self.ld,
                      _lib.ptr(x), _lib.ptr(y), m, m, st)
        return y


def dense_inverse_ld(m: int) -> int:
    """Rows (and row stride) of the buffer f3d_dense_inverse inverts an
    m x m matrix in: m rounded up to a multiple of 128."""
    return -(-m // 128) * 128


def dense_inverse(A: torch.Tensor, m: int) -> torch.Tensor:
    """Inverts the m x m top-left corner of the square FP64 device buffer A
    (dense_inverse_ld(m) rows or more, row stride A.shape[1]) in place
    (f3d_dense_inverse: blocked Gauss-Jordan elimination on the device);
    the padding becomes the identity.  Raises on a singular pivot block."""
    if A.dtype != torch.float64 or not A.is_cuda or not A.is_contiguous() or A.dim() != 2:
        raise ValueError("A must be a contiguous 2-D float64 CUDA tensor")
    ld = A.shape[1]
    if A.shape[0] < dense_inverse_ld(m) or ld < dense_inverse_ld(m):
        raise ValueError(f"A must have at least {dense_inverse_ld(m)} rows and columns for m = {m}")
    nb = ctypes.c_size_t(0)
    _lib.call("f3d_dense_inverse_workspace_bytes", m, ld, ctypes.byref(nb))
    ws = torch.empty(max(nb.value, 1), dtype=torch.uint8, device=A.device)
    _lib.call("f3d_dense_inverse", _lib.ptr(A), m, ld, _lib.ptr(ws), ws.numel(), _lib.stream_handle(A.device))
    return A


def singularity_vectors(nodes, normals, weights, eta, reg, eps) -> torch.Tensor:
    n = nodes.shape[0]
    E = torch.empty((n, 9), dtype=torch.float64, device=nodes.device)
    nb = ctypes.c_size_t(0)
    _lib.call("f3d_singularity_vectors_workspace_bytes", n, ctypes.byref(nb))
    ws = torch.zeros(max(nb.value, 1), dtype=torch.uint8, device=nodes.device)
    _lib.call("f3d_singularity_vectors", _lib.ptr(nodes), _lib.ptr(normals), _lib.ptr(weights),
              _lib.ptr(E), n, eta, reg, eps, _lib.ptr(ws), ws.numel(), _lib.stream_handle(nodes.device))
    return E


class _PairCall:
    """A pre-planned pair-sum launch with fixed device pointers (so that it
    can be captured in a CUDA graph)."""

    def __init__(self, kernel, mode, src, trg, dens, nrm, gs, gt, out, eta, reg, eps, shape=None):
        self.args = dict(kernel=kernel, mode=mode, src=src, trg=trg, dens=dens, nrm=nrm, gs=gs, gt=gt,
                         out=out, eta=eta, reg=reg, eps=eps)
        self.shape = {p: shape for p in ("fp64", "fp32c")}
        self.ws = {}

    def set_shape(self, precision, shape):
        self.shape[precision] = shape

    def _ws(self, precision):
        a = self.args
        key = precision
        shp = self.shape.get(precision)
        nb = ctypes.c_size_t(0)
        _lib.call("f3d_pair_workspace_bytes", _lib.KERNEL[a["kernel"]], _lib.PRECISION[precision],
                  a["src"].shape[0], a["trg"].shape[0], ctypes.byref(shp) if shp else None, ctypes.byref(nb))
        cur = self.ws.get(key)
        if cur is None or cur.numel() < nb.value:
            cur = torch.zeros(max(nb.value, 256), dtype=torch.uint8, device=a["out"].device)
            self.ws[key] = cur
        return cur

    def __call__(self, precision="fp64", accumulate=False):
        a = self.args
        ws = self._ws(precision)
        shp = self.shape.get(precision)
        _lib.call("f3d_pair_sum", _lib.KERNEL[a["kernel"]], _lib.PRECISION[precision],
                  _lib.SELF_MODE[a["mode"]], _lib.ptr(a["src"]), _lib.ptr(a["trg"]), _lib.ptr(a["dens"]),
                  _lib.ptr(a["nrm"]), _lib.ptr(a["gs"]), _lib.ptr(a["gt"]), _lib.ptr(a["out"]),
                  a["src"].shape[0], a["trg"].shape[0], a["eta"], a["reg"], a["eps"], int(accumulate),
                  ctypes.byref(shp) if shp else None, _lib.ptr(ws), ws.numel(),
                  _lib.stream_handle(a["out"].device))


class HydroSystem:
    """Device linear system of one time step: ``rhs``, :meth:`matvec`,
    :meth:`pc` (the right preconditioner P^-1) and :meth:`solve`."""

    PC_AUTO_MARGIN = 0.5   # pc_refresh="auto": rebuild after a solve that ended above this * tol
    PC_AUTO_MAX_AGE = 8    # ... and at least every this many steps

    def __init__(self, problem: Problem, shell_op: ShellOperator | None = None, device=None,
                 tune: bool = False, fiber_pc: str = "auto", inner_shell_pc: str = "fp16",
                 pc_refresh: int | str = 1, shell_pc: str = "dense"):
        self.p = problem
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        st = lambda: _lib.stream_handle(dev)
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        P = problem
        self.c0, self.c1 = P.mobility()
        # ---- fibers
        self.fs = FiberSet(P.fibers, P.lengths, device=dev)
        nF = self.fs.total
        self.nF = nF
        x_fib0 = np.concatenate(P.fibers) if P.fibers else np.zeros((0, 3))
        ff = P.force_fibers if P.force_fibers is not None else np.zeros((nF, 3))
        self.force = f64(np.asarray(ff).reshape(-1, 3))
        self.has_force = bool(np.any(ff))
        self.geo = torch.empty((max(nF, 1), 9), dtype=torch.float64, device=dev)
        self.timers = PhaseTimers()
        self.v_gain = self._flow_to_residual_gain(P.lengths)
        # ---- bodies (device state: location, orientation quaternion, nodes, normals, E)
        self.nbody = len(P.bodies)
        nb = [np.asarray(b.ref_nodes).reshape(-1, 3).shape[0] for b in P.bodies]
        self.nb = nb
        self.body_node_off_h = np.concatenate([[0], np.cumsum(nb)]).astype(np.int64)
        nB = int(self.body_node_off_h[-1])
        self.nB = nB
        self.body_ref = [np.asarray(b.ref_nodes, dtype=np.float64).reshape(-1, 3) for b in P.bodies]
        self.body_ref_n = [np.asarray(b.ref_normals, dtype=np.float64).reshape(-1, 3) for b in P.bodies]
        # ---- shell
        if P.shell is not None:
            self.shell = shell_op or ShellOperator(P.shell, P.eta, P.reg, P.eps_dist, dev, pc=shell_pc)
            nS = self.shell.n
        else:
            self.shell = None
            nS = 0
        self.nS = nS
        # ---- layout
        self.o_body = [3 * nS + 3 * int(self.body_node_off_h[k]) + 6 * k for k in range(self.nbody)]
        self.o_fib = 3 * nS + 3 * nB + 6 * self.nbody
        self.size = self.o_fib + 4 * nF
        self.x_off_body = torch.as_tensor(np.array(self.o_body, dtype=np.int64), device=dev) if self.nbody else None
        self.body_node_off = torch.as_tensor(self.body_node_off_h, device=dev)
        # ---- positions, one buffer: targets [fibers; bodies; shell].  The
        # fiber points (the Oseen sources), the body nodes and the stresslet
        # sources [bodies; shell] are views of it, so moving the geometry in
        # place moves every sum's sources and targets together.
        self.trg = torch.empty((nF + nB + nS, 3), dtype=torch.float64, device=dev)
        self.x_fib = self.trg[:nF]
        self.x_fib.copy_(f64(x_fib0.reshape(-1, 3)))
        if nS:
            self.trg[nF + nB:].copy_(self.shell.nodes)
        # fiber point p0 + i, coordinate c is entry o_fib + 4 p0 + c n + i of a solution
        gat = np.empty((nF, 3), dtype=np.int64)
        for f in range(self.fs.nfib):
            n, p0 = int(self.fs.npts[f]), int(self.fs.pt_off_h[f])
            gat[p0:p0 + n] = self.o_fib + 4 * p0 + np.arange(3)[None, :] * n + np.arange(n)[:, None]
        self._x_fib_from_sol = torch.as_tensor(gat.reshape(-1), device=dev)
        if self.nbody:
            self.body_nodes = self.trg[nF:nF + nB]
            self.stress_normals = torch.zeros((nB + nS, 3), dtype=torch.float64, device=dev)
            self.body_normals = self.stress_normals[:nB]
            self.body_w = f64(np.concatenate([np.asarray(b.weights).reshape(-1) for b in P.bodies]))
            self.body_E = torch.empty((nB, 9), dtype=torch.float64, device=dev)
            self.body_R = torch.zeros((self.nbody, 9), dtype=torch.float64, device=dev)
            self.body_centers = f64(np.array([np.asarray(b.location, dtype=np.float64)
                                              for b in P.bodies]).reshape(-1, 3))
            self.body_quat = f64(np.array([rotation_to_quaternion(b.rotation)
                                           for b in P.bodies]).reshape(-1, 4))
            self._vel_off = torch.as_tensor(np.array([self.o_body[k] + 3 * nb[k] for k in range(self.nbody)],
                                                     dtype=np.int64), device=dev)
            # body node i of body k -> rows o_body[k] + 3 (i - first node of k) .. +3
            self._rhs_body_idx = torch.as_tensor(np.concatenate(
                [self.o_body[k] + np.arange(3 * nb[k]) for k in range(self.nbody)]).astype(np.int64), device=dev)
            self._load_bodies()
        self.ntrg = self.trg.shape[0]
        grp = np.concatenate([np.repeat(np.arange(self.fs.nfib), self.fs.npts),
                              -np.ones(self.ntrg - nF)]).astype(np.int32)
        self.trg_grp = torch.as_tensor(grp, device=dev)
        self.src_grp = self.trg_grp[:nF].contiguous()
        # stresslet sources: [body nodes; shell nodes] (a view of the targets)
        self.nstress = nB + nS
        if self.nstress:
            self.stress_nodes = self.trg[nF:]
            if not self.nbody:
                self.stress_normals = torch.zeros((nS, 3), dtype=torch.float64, device=dev)
            if nS:
                self.stress_normals[nB:].copy_(self.shell.normals)
            self.stress_dens = torch.zeros((self.nstress, 3), dtype=torch.float64, device=dev)
            seg_src, seg_dst, seg_len = [], [], []
            for k in range(self.nbody):
                seg_src.append(self.o_body[k]); seg_dst.append(3 * int(self.body_node_off_h[k])); seg_len.append(3 * nb[k])
            if nS:
                seg_src.append(0); seg_dst.append(3 * nB); seg_len.append(3 * nS)
            self.seg = [torch.as_tensor(np.array(a, dtype=np.int64), device=dev) for a in (seg_src, seg_dst, seg_len)]
            self.seg_max = max(seg_len)
        # ---- work buffers
        self.v = torch.zeros(3 * self.ntrg, dtype=torch.float64, device=dev)
        self.fw = torch.zeros((max(nF, 1), 3), dtype=torch.float64, device=dev)
        # the fiber forces of a guess x0 and their Oseen flow, summed in the
        # same pass as the explicit flow (update(x0)); used by the solve's
        # first residual
        self.fw2 = torch.zeros((max(nF, 1), 3), dtype=torch.float64, device=dev)
        self.v2 = torch.zeros(3 * self.ntrg, dtype=torch.float64, device=dev)
        self._pending_x0 = None
        self._dual_ws = None
        self.scratch = torch.zeros(4, dtype=torch.float64, device=dev)
        self.oseen = _PairCall("oseen", "skip_group", self.x_fib, self.trg, self.fw, None, self.src_grp,
                               self.trg_grp, self.v, P.eta, P.reg, P.eps_dist) if nF else None
        self.stress = _PairCall("stresslet", "regularise", self.stress_nodes, self.trg, self.stress_dens,
                                self.stress_normals, None, None, self.v, P.eta, P.reg, P.eps_dist) \
            if self.nstress else None
        # the same sum split by target block (fibers | bodies and periphery),
        # for residuals that take the two blocks in different precisions
        self.stress_fib = self.stress_rest = None
        if self.nstress and nF:
            self.stress_fib = _PairCall("stresslet", "regularise", self.stress_nodes, self.trg[:nF],
                                        self.stress_dens, self.stress_normals, None, None, self.v[:3 * nF],
                                        P.eta, P.reg, P.eps_dist)
            if nB + nS:
                self.stress_rest = _PairCall("stresslet", "regularise", self.stress_nodes, self.trg[nF:],
                                             self.stress_dens, self.stress_normals, None, None, self.v[3 * nF:],
                                             P.eta, P.reg, P.eps_dist)
        if tune:
            self.autotune()
        # ---- right-hand side and preconditioner blocks
        self.rhs = torch.zeros(self.size, dtype=torch.float64, device=dev)
        self.lu = BlockLU(list(4 * self.fs.npts), device=dev)
        # fiber blocks of the preconditioner: explicit inverses applied as a
        # block GEMV (blocks up to 128), else LU factors and substitution
        if fiber_pc == "auto":
            fiber_pc = "inverse" if self.lu.max_n <= 128 else "lu"
        if fiber_pc not in ("inverse", "lu"):
            raise ValueError("fiber_pc must be 'auto', 'inverse' or 'lu'")
        self.fiber_pc = fiber_pc
        # storage of the periphery inverse read by the FP32-class preconditioner
        if inner_shell_pc not in ("fp32", "fp16"):
            raise ValueError("inner_shell_pc must be 'fp32' or 'fp16'")
        self.inner_shell_pc = inner_shell_pc
        # the fiber blocks of the preconditioner are rebuilt every pc_refresh
        # steps (fiber3d: every step); in between the last ones are kept --
        # still a fixed operator within each solve, of a geometry at most
        # pc_refresh - 1 steps old.  "auto": rebuilt for the next step when
        # the last solve needed more than one GMRES iteration or ended above
        # PC_AUTO_MARGIN * tol, and at least every PC_AUTO_MAX_AGE steps.
        if pc_refresh != "auto" and (isinstance(pc_refresh, str) or int(pc_refresh) < 1):
            raise ValueError("pc_refresh must be >= 1 or 'auto'")
        self.pc_refresh = pc_refresh if pc_refresh == "auto" else int(pc_refresh)
        self._pc_age = None
        self._pc_stale = False  # set by solve() under pc_refresh="auto"
        self.A_fib = torch.zeros(max(self.fs.mat_total, 1), dtype=torch.float64, device=dev)
        self.flow_ext = torch.zeros((max(nF, 1), 3), dtype=torch.float64, device=dev)
        self._body_blocks()
        self.update()

    def _flow_to_residual_gain(self, lengths) -> float:
        """Bound on |d(matvec)| / |d v| for a change d v of the pair sums v at
        the targets: 1 on periphery and body rows; on a fiber's rows v enters
        as P_X v (positions) and P_T (x_s . (2/L) D1 v) (tensions), whose
        2-norm is at most sqrt(|P_X|^2 + ((2/L) |P_T| |D1|)^2) (|x_s| = 1)."""
        g = 1.0
        lengths = np.asarray(lengths, dtype=np.float64).reshape(-1)
        for n, res in self.fs.resolutions.items():
            Lmin = float(lengths[self.fs.npts == n].min()) if lengths.size else 1.0
            nx = np.linalg.norm(res.PX, 2)
            nt = np.linalg.norm(res.PT, 2)
            nd = np.linalg.norm(res.D0[0], 2)
            g = max(g, float(np.sqrt(nx ** 2 + (2.0 / Lmin * nt * nd) ** 2)))
        return g

    # ------------------------------------------------------------------------
    def _load_bodies(self):
        """Body nodes, normals and singularity vectors at the initial
        location/orientation, on the device.  A rigid body's singularity
        vectors are those of its reference surface rotated with it: the
        3 x 3 map E_i (unit density -> velocity at node i) of the rotated
        surface is R E_i^ref R^T (the stresslet sum is rotation-equivariant
        and translation-invariant), so the pair sum runs once per body, at
        set-up, not every step."""
        dev = self.device
        self._body_of = torch.as_tensor(np.repeat(np.arange(self.nbody), self.nb).astype(np.int32), device=dev)
        self._ref_nodes = torch.as_tensor(np.concatenate(self.body_ref), device=dev)
        self._ref_normals = torch.as_tensor(np.concatenate(self.body_ref_n), device=dev)
        P = self.p
        E = []
        for k in range(self.nbody):
            a, b = int(self.body_node_off_h[k]), int(self.body_node_off_h[k + 1])
            E.append(singularity_vectors(self._ref_nodes[a:b], self._ref_normals[a:b], self.body_w[a:b],
                                         P.eta, P.reg, P.eps_dist))
        self._ref_E = torch.cat(E).contiguous()
        R = np.stack([quaternion_rotation(q).reshape(9) for q in self.body_quat.cpu().numpy()])
        self.body_R.copy_(torch.as_tensor(R, device=dev))
        self._place_bodies()

    def _place_bodies(self):
        """Nodes, normals and E of every body from body_R / body_centers (one kernel)."""
        _lib.call("f3d_rigid_body_update", _lib.ptr(self._body_of), _lib.ptr(self.body_R), _lib.ptr(self.body_centers),
                  _lib.ptr(self._ref_nodes), _lib.ptr(self._ref_normals), _lib.ptr(self._ref_E), self.nB,
                  _lib.ptr(self.body_nodes), _lib.ptr(self.body_normals), _lib.ptr(self.body_E),
                  _lib.stream_handle(self.device))

    def _body_blocks(self):
        """Body preconditioner blocks in each body's own frame (location 0,
        orientation identity), inverted once.  A rigid body's block only
        rotates with the body, so P_b^-1 x = Q A_ref^-1 Q^T x with Q the
        body rotation on every 3-vector — fiber3d's precompute_body_PC path
        (A_inv_bodies, tstep.py:227-252 and 966-981)."""
        self.body_inv = []
        if not self.nbody:
            return
        P = self.p
        st = _lib.stream_handle(self.device)
        origin = torch.zeros(3, dtype=torch.float64, device=self.device)
        self.rot_off = torch.as_tensor(np.array([o - 3 * self.nS for o in self.o_body], dtype=np.int64),
                                       device=self.device)
        self.rot_nvec = torch.as_tensor(np.array([n + 2 for n in self.nb], dtype=np.int32), device=self.device)
        self.body_tmp = torch.zeros(self.o_fib - 3 * self.nS, dtype=torch.float64, device=self.device)
        for k in range(self.nbody):
            ref = torch.as_tensor(self.body_ref[k], device=self.device)
            refn = torch.as_tensor(self.body_ref_n[k], device=self.device)
            a, b = int(self.body_node_off_h[k]), int(self.body_node_off_h[k + 1])
            w = self.body_w[a:b].contiguous()
            E = singularity_vectors(ref, refn, w, P.eta, P.reg, P.eps_dist)
            n = b - a
            mb = 3 * n + 6
            ldb = dense_inverse_ld(mb)
            A = torch.empty((ldb, ldb), dtype=torch.float64, device=self.device)
            _lib.call("f3d_surface_dense", 1, _lib.ptr(ref), _lib.ptr(refn), _lib.ptr(E), _lib.ptr(w),
                      _lib.ptr(origin), _lib.ptr(A), n, ldb, P.eta, P.reg, P.eps_dist, st)
            dense_inverse(A, mb)
            self.body_inv.append(A[:mb, :mb].contiguous())
            del A
        # all body inverses back to back, applied by one batched GEMV
        m = np.array([3 * n + 6 for n in self.nb], dtype=np.int64)
        moff = np.concatenate([[0], np.cumsum(m * m)[:-1]]).astype(np.int64)
        self.body_inv_all = torch.cat([bi.reshape(-1) for bi in self.body_inv]).contiguous()
        self._binv = [torch.as_tensor(a, device=self.device) for a in
                      (moff, m, np.array([o - 3 * self.nS for o in self.o_body], dtype=np.int64))]
        self._binv_max = int(m.max())
        self._binv_vec = int(bool(np.all(m % 2 == 0)) and bool(np.all(moff % 2 == 0)))

    def update(self, x0: torch.Tensor | None = None):
        """Recompute everything that depends on the current geometry (fiber
        derivatives, body surfaces and singularity vectors, explicit flows,
        right-hand side, fiber/body blocks and their LU) in place, so that
        device pointers — and CUDA graphs captured on them — stay valid.

        With the initial guess `x0` of the coming solve, the Oseen flow of
        x0's fiber forces is summed in the same pass over the fiber pairs as
        the explicit flow of the external forces (``f3d_oseen_dual``); a
        :meth:`solve` given this same tensor, unmodified, starts from it
        instead of a fresh Oseen sum (the residual is bit-for-bit the same)."""
        st = _lib.stream_handle(self.device)
        if self.nF:
            _lib.call("f3d_fiber_geometry", ctypes.byref(self.fs.c), _lib.ptr(self.x_fib), _lib.ptr(self.geo),
                      self.nF, st)
        self._assemble(x0)

    def advance(self, sol: torch.Tensor, x0: torch.Tensor | None = None):
        """Move the geometry one step with solution `sol` (tstep.py:1392-1407:
        fibers take their new positions; bodies x += dt U and
        q <- q(Omega dt) q), then :meth:`update` (with the next guess x0).
        Everything stays on the device: one gather for the fiber points, one
        kernel for the body states and one for their surfaces."""
        if sol.dtype != torch.float64 or not sol.is_contiguous() or sol.numel() != self.size:
            raise ValueError(f"solution must be a contiguous float64 vector of {self.size} entries")
        if self.nF:
            torch.index_select(sol, 0, self._x_fib_from_sol, out=self.x_fib.view(-1))
        if self.nbody:
            _lib.call("f3d_body_advance", _lib.ptr(sol), _lib.ptr(self._vel_off), self.nbody, self.p.dt,
                      _lib.ptr(self.body_centers), _lib.ptr(self.body_quat), _lib.ptr(self.body_R),
                      _lib.stream_handle(self.device))
            self._place_bodies()
        self.update(x0)

    def body_state(self):
        """(locations (nbody, 3), quaternions (nbody, 4)) of the bodies, on the host."""
        if not self.nbody:
            return np.zeros((0, 3)), np.zeros((0, 4))
        return self.body_centers.cpu().numpy(), self.body_quat.cpu().numpy()

    # ------------------------------------------------------------------------
    def autotune(self):
        from . import autotune as at
        P = self.p
        for call, kind, precs in ((self.oseen, "oseen", ("fp64", "fp32c")),
                                  (self.stress, "stresslet", ("fp64", "fp32c")),
                                  (self.stress_fib, "stresslet", ("fp64",)),
                                  (self.stress_rest, "stresslet", ("fp32c",))):
            if call is None:
                continue
            a = call.args
            for prec in precs:
                shp = at.tune(kind, a["src"], a["trg"], a["dens"], a["nrm"], self_mode=a["mode"],
                              src_group=a["gs"], trg_group=a["gt"], precision=prec, eta=P.eta,
                              reg=P.reg, epsilon_distance=P.eps_dist)
                call.set_shape(prec, shp)

    def _oseen_dual(self):
        """v = Oseen flow of fw (external forces), v2 = that of fw2, one pass;
        the FP64 Oseen call's launch shape, so that each equals its single
        sum bit for bit."""
        a = self.oseen.args
        shp = self.oseen.shape.get("fp64")
        nb = ctypes.c_size_t(0)
        _lib.call("f3d_oseen_dual_workspace_bytes", a["src"].shape[0], a["trg"].shape[0],
                  ctypes.byref(shp) if shp else None, ctypes.byref(nb))
        if self._dual_ws is None or self._dual_ws.numel() < nb.value:
            self._dual_ws = torch.zeros(max(nb.value, 256), dtype=torch.uint8, device=self.device)
        _lib.call("f3d_oseen_dual", _lib.SELF_MODE[a["mode"]], _lib.ptr(a["src"]), _lib.ptr(a["trg"]),
                  _lib.ptr(self.fw), _lib.ptr(self.fw2), _lib.ptr(a["gs"]), _lib.ptr(a["gt"]), _lib.ptr(self.v),
                  _lib.ptr(self.v2), a["src"].shape[0], a["trg"].shape[0], a["eta"], a["reg"], a["eps"], 0,
                  ctypes.byref(shp) if shp else None, _lib.ptr(self._dual_ws), self._dual_ws.numel(),
                  _lib.stream_handle(self.device))

    def pending_oseen(self, x: torch.Tensor) -> bool:
        """Whether update() already summed the Oseen flow of x's fiber forces."""
        return self._pending_x0 is not None and x is self._pending_x0

    def _assemble(self, x0=None):
        P = self.p
        dev = self.device
        st = _lib.stream_handle(dev)
        nF, nB, nS = self.nF, self.nB, self.nS
        # explicit flow of the external fiber forces (tstep.py:789-821)
        self.timers.start("fiber2all_explicit_interactions")
        self._pending_x0 = None
        if not (nF and self.has_force):
            self.v.zero_()  # no explicit flow (else the pass below overwrites v)
        if nF and self.has_force:
            _lib.call("f3d_fiber_weight", ctypes.byref(self.fs.c), _lib.ptr(self.force), _lib.ptr(self.fw), nF, st)
            if x0 is not None:
                _lib.call("f3d_fiber_forces", ctypes.byref(self.fs.c), P.E, _lib.ptr(self.geo),
                          _lib.ptr(x0[self.o_fib:]), _lib.ptr(self.fw2), nF, 1, st)
                self._oseen_dual()
                self._pending_x0 = x0
            else:
                self.oseen("fp64")
        self.timers.stop("fiber2all_explicit_interactions")
        v = self.v.view(-1, 3)
        if nF:
            self.flow_ext.copy_(v[:nF])
        if nS:
            torch.neg(v[nF + nB:].reshape(-1), out=self.rhs[:3 * nS])
        if self.nbody:
            self.rhs.index_copy_(0, self._rhs_body_idx, v[nF:nF + nB].reshape(-1).neg())
        flow = self.flow_ext
        # fiber blocks into A_fib and (a copy) into the LU buffer
        if self.pc_refresh == "auto":
            refresh = self._pc_age is None or self._pc_stale or self._pc_age >= self.PC_AUTO_MAX_AGE - 1
        else:
            refresh = self._pc_age is None or self._pc_age >= self.pc_refresh - 1
        self.timers.start("Build_linear_system_fibers")
        if nF:
            A_copy = self.lu.A.data_ptr() if refresh else None
            _lib.call("f3d_fiber_assemble", ctypes.byref(self.fs.c), P.E, P.dt, self.c0, self.c1, P.penalty,
                      _lib.ptr(self.x_fib), _lib.ptr(self.geo), _lib.ptr(flow), _lib.ptr(self.force),
                      _lib.ptr(self.A_fib), A_copy, _lib.ptr(self.rhs[self.o_fib:]), self.fs.max_n, st)
        self.timers.stop("Build_linear_system_fibers")
        if refresh:
            self.timers.start("Build_PC_fibers")
            if self.fiber_pc == "inverse":
                self.lu.invert(fp32=True)
            else:
                self.lu.factor()
            self.timers.stop("Build_PC_fibers")
            self._pc_age = 0
        else:
            self._pc_age += 1

    # ------------------------------------------------------------------------
    def matvec(self, x: torch.Tensor, y: torch.Tensor, precision: str = "fp64",
               oseen_done: bool = False) -> torch.Tensor:
        """y = A x (tstep.py:1003-1178).  With `oseen_done` the FP64 Oseen
        flow of x's fiber forces is the one update(x) summed (see
        :meth:`pending_oseen`).  precision "split": FP64 pair sums on the
        fiber targets, FP32C stresslet sums on the body and periphery
        targets (whose rows take the flow with gain 1)."""
        st = _lib.stream_handle(self.device)
        nF, nB, nS = self.nF, self.nB, self.nS
        XT = x[self.o_fib:]
        split = precision == "split"
        first = True
        if nF:
            if oseen_done:
                self.v.copy_(self.v2)
            else:
                _lib.call("f3d_fiber_forces", ctypes.byref(self.fs.c), self.p.E, _lib.ptr(self.geo),
                          _lib.ptr(XT), _lib.ptr(self.fw), nF, 1, st)
                self.oseen("fp64" if split else precision, accumulate=False)
            first = False
        if self.nstress:
            _lib.call("f3d_gather_segments", _lib.ptr(x), _lib.ptr(self.stress_dens), _lib.ptr(self.seg[0]),
                      _lib.ptr(self.seg[1]), _lib.ptr(self.seg[2]), self.seg[0].numel(), self.seg_max, st)
            if split and self.stress_fib is not None:
                if first:
                    self.v.zero_()
                self.stress_fib("fp64", accumulate=True)
                if self.stress_rest is not None:
                    self.stress_rest("fp32c", accumulate=True)
            else:
                self.stress("fp32c" if split else precision, accumulate=not first)
            first = False
        if first:
            self.v.zero_()
        v = self.v
        if nS:
            _lib.call("f3d_shell_residual", _lib.ptr(v[3 * (nF + nB):]), _lib.ptr(self.shell.E),
                      _lib.ptr(self.shell.weights), _lib.ptr(self.shell.normals), _lib.ptr(x), _lib.ptr(y),
                      nS, _lib.ptr(self.scratch), st)
        if self.nbody:
            _lib.call("f3d_body_residual", self.nbody, _lib.ptr(self.body_node_off), _lib.ptr(self.x_off_body),
                      _lib.ptr(self.body_nodes), _lib.ptr(self.body_centers), _lib.ptr(self.body_E),
                      _lib.ptr(self.body_w), _lib.ptr(v[3 * nF:]), _lib.ptr(x), _lib.ptr(y), st)
        if nF:
            _lib.call("f3d_fiber_residual", ctypes.byref(self.fs.c), _lib.ptr(self.A_fib), _lib.ptr(self.geo),
                      _lib.ptr(XT), _lib.ptr(v), _lib.ptr(y[self.o_fib:]), self.fs.max_n, st)
        return y

    def pc(self, x: torch.Tensor, y: torch.Tensor, precision: str = "fp64") -> torch.Tensor:
        """y = P^-1 x (tstep.py:950-994)."""
        st = _lib.stream_handle(self.device)
        nS = self.nS
        if nS:
            self.shell.apply(x, y, "fp64" if precision == "fp64" else self.inner_shell_pc)
        if self.nbody:
            tb = self.body_tmp
            tb.copy_(x[3 * nS:self.o_fib])
            _lib.call("f3d_rotate_blocks", _lib.ptr(tb), _lib.ptr(self.rot_off), _lib.ptr(self.rot_nvec),
                      _lib.ptr(self.body_R), self.nbody, 1, st)
            moff, m, off = self._binv
            _lib.call("f3d_gemv_batched", _lib.ptr(self.body_inv_all), _lib.ptr(moff), _lib.ptr(m), _lib.ptr(off),
                      _lib.ptr(off), self.nbody, self._binv_max, self._binv_vec, _lib.ptr(tb),
                      _lib.ptr(y[3 * nS:]), st)
            _lib.call("f3d_rotate_blocks", _lib.ptr(y[3 * nS:]), _lib.ptr(self.rot_off), _lib.ptr(self.rot_nvec),
                      _lib.ptr(self.body_R), self.nbody, 0, st)
        if self.nF:
            if self.fiber_pc == "inverse":
                self.lu.apply(x[self.o_fib:], y[self.o_fib:], precision)
            else:
                rest = y[self.o_fib:]
                rest.copy_(x[self.o_fib:])
                self.lu.solve(rest)
        return y

    def reset_workspaces(self) -> None:
        """Zero every pair-sum workspace of this system (their split counters
        must start at zero; a kernel that gave up on a bounded wait may have
        left some set)."""
        for name in ("oseen", "stress", "stress_fib", "stress_rest"):
            call = getattr(self, name, None)
            for t in (call.ws.values() if call is not None else ()):
                t.zero_()
        for name in ("_dual_ws", "_grid_ws"):
            t = getattr(self, name, None)
            if t is not None:
                t.zero_()

    def solve(self, tol=1e-8, restart=100, maxiter=200, x0=None, mixed=False, **kw):
        from .gmres import solve_system
        res = solve_system(self, tol=tol, restart=restart, maxiter=maxiter, x0=x0, mixed=mixed, **kw)
        # a kernel whose bounded wait ran out has returned early: its sums are
        # incomplete, so the solve is not trusted (raises F3DError after
        # zeroing the workspaces)
        _lib.check_device_error("HydroSystem.solve", self.device, on_error=self.reset_workspaces)
        if self.pc_refresh == "auto":
            self._pc_stale = res["iterations"] > 1 or res["history"][-1] > self.PC_AUTO_MARGIN * tol
        return res

    # --------------------------------------------------------- grid velocity --
    def grid_velocity(self, sol: torch.Tensor, grid_points, body0_radius: float | None = None,
                      near: float = 0.2, uprate: int = 2) -> torch.Tensor:
        """Velocity field (ngrid, 3) at grid points for the solution `sol` of
        the current step, as fiber3d's time step evaluates it before moving
        the geometry (compute_velocity, tstep.py:1273-1381, and
        tstep.py:1414-1448); free fibers, no fiber-body links, no external
        body forces:
          * periphery and body double layers of their densities in sol
            (stresslet source -> target);
          * the fibers' Oseen flow of their implicit forces (force operator
            of sol, trapezoid-weighted; flow_fibers, tstep_utils.py:653-700),
            where a grid point within `near` of a fiber node takes instead
            that fiber's self-flow at its nearest node, with `uprate`-fold
            upsampled quadrature (f3d_fiber_self_flow_up,
            f3d_grid_near_fiber); the last such fiber in fiber order wins;
          * the Oseen flow of the external fiber forces;
          * with body0_radius, rigid motion U + W x (g - c) inside the first
            body, moved to c = location + dt U (f3d_grid_rigid_override)."""
        from . import kernels as K
        dev = self.device
        P = self.p
        st = _lib.stream_handle(dev)
        if sol.dtype != torch.float64 or not sol.is_contiguous() or sol.numel() != self.size:
            raise ValueError(f"solution must be a contiguous float64 vector of {self.size} entries")
        g = torch.as_tensor(grid_points, dtype=torch.float64, device=dev).reshape(-1, 3).contiguous()
        ng = g.shape[0]
        kw = dict(eta=P.eta, reg=P.reg, epsilon_distance=P.eps_dist, self_mode="regularise")
        v = torch.zeros(3 * ng, dtype=torch.float64, device=dev)
        if ng == 0:
            return v.view(0, 3)
        nF, nS = self.nF, self.nS
        if nS:
            K.pair_sum("stresslet", self.shell.nodes, g, sol[:3 * nS].view(-1, 3), self.shell.normals,
                       out=v, accumulate=True, **kw)
        if self.nbody:
            dens = torch.cat([sol[self.o_body[k]:self.o_body[k] + 3 * self.nb[k]] for k in range(self.nbody)])
            K.pair_sum("stresslet", self.body_nodes, g, dens.view(-1, 3), self.body_normals, out=v,
                       accumulate=True, **kw)
        if nF:
            f = torch.empty((nF, 3), dtype=torch.float64, device=dev)
            _lib.call("f3d_fiber_forces", ctypes.byref(self.fs.c), P.E, _lib.ptr(self.geo),
                      _lib.ptr(sol[self.o_fib:]), _lib.ptr(f), nF, 0, st)
            fw = torch.empty_like(f)
            _lib.call("f3d_fiber_weight", ctypes.byref(self.fs.c), _lib.ptr(f), _lib.ptr(fw), nF, st)
            vfib = torch.empty(3 * ng, dtype=torch.float64, device=dev)
            vext = None
            if self.has_force:
                # the implicit- and external-force flows over the same pairs: one dual pass
                fe = torch.empty_like(f)
                _lib.call("f3d_fiber_weight", ctypes.byref(self.fs.c), _lib.ptr(self.force), _lib.ptr(fe), nF, st)
                vext = torch.empty_like(vfib)
                nb = ctypes.c_size_t(0)
                _lib.call("f3d_oseen_dual_workspace_bytes", nF, ng, None, ctypes.byref(nb))
                ws = getattr(self, "_grid_ws", None)
                if ws is None or ws.numel() < nb.value:
                    # zeroed: the split-sum counters at its start must be zero on entry
                    ws = self._grid_ws = torch.zeros(max(nb.value, 256), dtype=torch.uint8, device=dev)
                _lib.call("f3d_oseen_dual", _lib.SELF_MODE["regularise"], _lib.ptr(self.x_fib), _lib.ptr(g),
                          _lib.ptr(fw), _lib.ptr(fe), None, None, _lib.ptr(vfib), _lib.ptr(vext), nF, ng, P.eta,
                          P.reg, P.eps_dist, 0, None, _lib.ptr(ws), ws.numel(), st)
            else:
                K.pair_sum("oseen", self.x_fib, g, fw, out=vfib, **kw)
            up, up_off = self.fs.upsampling(uprate)
            vself = torch.empty((nF, 3), dtype=torch.float64, device=dev)
            _lib.call("f3d_fiber_self_flow_up", _lib.ptr(self.fs.n), _lib.ptr(self.fs.pt_off),
                      _lib.ptr(self.fs.length), self.fs.nfib, self.fs.max_n, _lib.ptr(self.x_fib), _lib.ptr(f),
                      _lib.ptr(up), _lib.ptr(up_off), uprate, P.eta, P.reg, P.eps_dist, _lib.ptr(vself), st)
            _lib.call("f3d_grid_near_fiber", _lib.ptr(g), ng, _lib.ptr(self.x_fib), _lib.ptr(self.fs.pt_off),
                      self.fs.nfib, _lib.ptr(vself), near, _lib.ptr(vfib), st)
            v += vfib
            if vext is not None:
                v += vext
        if self.nbody and body0_radius is not None:
            o = self.o_body[0] + 3 * self.nb[0]
            uw = sol[o:o + 6].contiguous()
            center = (self.body_centers[0] + uw[:3] * P.dt).contiguous()
            _lib.call("f3d_grid_rigid_override", _lib.ptr(g), ng, _lib.ptr(center), _lib.ptr(uw),
                      float(body0_radius), _lib.ptr(v), st)
        return v.view(ng, 3)

    # ---------------------------------------------------------------- layout --
    def split(self, sol: torch.Tensor):
        """Solution blocks: shell density, per body (lambda, U, Omega), per
        fiber (X (N,3), T (N,))."""
        out = {"shell": sol[:3 * self.nS].view(-1, 3) if self.nS else None, "bodies": [], "fibers": []}
        for k in range(self.nbody):
            o, n = self.o_body[k], self.nb[k]
            out["bodies"].append((sol[o:o + 3 * n].view(-1, 3), sol[o + 3 * n:o + 3 * n + 3], sol[o + 3 * n + 3:o + 3 * n + 6]))
        for k in range(self.fs.nfib):
            n = int(self.fs.npts[k])
            o = self.o_fib + 4 * int(self.fs.pt_off_h[k])
            blk = sol[o:o + 4 * n]
            out["fibers"].append((blk[:3 * n].view(3, n).t(), blk[3 * n:]))
        return out
