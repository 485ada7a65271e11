"""CPU restatement of one fiber3d hydrodynamic step's linear system (test
oracle): unknown layout, right-hand side, the GMRES matvec, the block
preconditioner and right-preconditioned GMRES.

Follows python/tstep/tstep.py (fiber3d):
  layout / offsets      tstep_utils.get_num_particles_and_offsets :906-931
  explicit flows, RHS   tstep.py:745-846, tstep_utils.get_fibers_and_bodies_matrices :1238-1338
  matvec                A_body_fiber_hyd, tstep.py:1003-1178
  preconditioner        P_inv, tstep.py:950-994; body blocks tstep_utils.py:1341-1386;
                        fiber blocks tstep_utils.py:1405-1419; shell tstep.py:327-351
  GMRES                 bpm_utilities/gmres.py:94-111 (right preconditioning)
Fibers are free (force/torque-free ends, no fiber-body links); bodies are
rigid with singularity subtraction; the periphery is a sphere-like shell.
Test infrastructure only.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
import scipy.sparse.linalg as spla

from . import fiber_ops as F
from . import kernels_np as KN
from . import pairs_c


def quaternion_rotation(q) -> np.ndarray:
    """Rotation matrix of unit quaternion (s, p) (quaternion.py:41-50)."""
    s, p = q[0], np.asarray(q[1:4])
    d = s * s - 0.5
    return 2.0 * np.array([[p[0] ** 2 + d, p[0] * p[1] - s * p[2], p[0] * p[2] + s * p[1]],
                           [p[1] * p[0] + s * p[2], p[1] ** 2 + d, p[1] * p[2] - s * p[0]],
                           [p[2] * p[0] - s * p[1], p[2] * p[1] + s * p[0], p[2] ** 2 + d]])


@dataclass
class Body:
    location: np.ndarray
    rotation: np.ndarray
    ref_nodes: np.ndarray
    ref_normals: np.ndarray
    weights: np.ndarray

    @property
    def nodes(self):
        return self.ref_nodes @ self.rotation.T + self.location

    @property
    def normals(self):
        return self.ref_normals @ self.rotation.T

    def K(self):
        """K = [J, rot] (body.py:180-193): block i maps (U, W) to U + W x r_i."""
        r = self.nodes - self.location
        n = r.shape[0]
        K = np.zeros((3 * n, 6))
        for i in range(n):
            K[3 * i:3 * i + 3, 0:3] = np.eye(3)
            x, y, z = r[i]
            K[3 * i:3 * i + 3, 3:6] = [[0.0, z, -y], [-z, 0.0, x], [y, -x, 0.0]]
        return K


@dataclass
class Shell:
    nodes: np.ndarray
    normals: np.ndarray
    weights: np.ndarray


def singularity_vectors(nodes, normals, weights, eta):
    """e_c(i) = sum_{j != i} S_ij w_j e_c, c = x, y, z (periphery.py:75-98,
    body.py:325-346).  Returns E with E[i, :, c] = e_c(i)."""
    n = nodes.shape[0]
    E = np.zeros((n, 3, 3))
    for c in range(3):
        e = np.zeros((n, 3))
        e[:, c] = weights
        E[:, :, c] = pairs_c.pair_sum("stresslet", nodes, nodes, e, normals, eta=eta,
                                      self_mode="skip_index").reshape(n, 3)
    return E


@dataclass
class HydroSystem:
    fibers: list                     # list of (N, 3) arrays (positions)
    lengths: list
    E: float
    dt: float
    eta: float
    bodies: list = field(default_factory=list)
    shell: Shell | None = None
    force_fibers: np.ndarray | None = None   # (sum N, 3) external force per point
    epsilon: float = 1e-3
    penalty: float = 500.0
    # False: no dense shell matrix and no LU of it (36000^2 at 12000 nodes);
    # the shell block of pc() is then unavailable and shell_pc_residual()
    # checks a preconditioned vector against the matrix-free operator
    dense_shell: bool = True

    def __post_init__(self):
        self.c0, self.c1 = F.mobility_constants(self.epsilon, self.eta)
        self.npts = [x.shape[0] for x in self.fibers]
        self.off_f = np.concatenate([[0], np.cumsum(self.npts)]).astype(int)
        self.nb = [b.ref_nodes.shape[0] for b in self.bodies]
        self.off_b = np.concatenate([[0], np.cumsum(self.nb)]).astype(int)
        self.nshell = 0 if self.shell is None else self.shell.nodes.shape[0]
        self.size = 3 * self.nshell + 3 * self.off_b[-1] + 6 * len(self.bodies) + 4 * self.off_f[-1]
        self.fms = {}
        for n in set(self.npts):
            self.fms[n] = F.FiberMatrices(n)
        self.trg_fib = np.concatenate(self.fibers) if self.fibers else np.zeros((0, 3))
        self.trg_bdy = np.concatenate([b.nodes for b in self.bodies]) if self.bodies else np.zeros((0, 3))
        self.nrm_bdy = np.concatenate([b.normals for b in self.bodies]) if self.bodies else np.zeros((0, 3))
        parts = [self.trg_fib, self.trg_bdy] + ([self.shell.nodes] if self.shell is not None else [])
        self.trg_all = np.concatenate(parts)
        self.grp_fib = np.repeat(np.arange(len(self.fibers)), self.npts).astype(np.int32)
        if self.force_fibers is None:
            self.force_fibers = np.zeros((self.off_f[-1], 3))
        self._assemble()

    # ------------------------------------------------------------ offsets --
    @property
    def o_body(self):
        return 3 * self.nshell

    def o_body_k(self, k):
        return 3 * self.nshell + 3 * self.off_b[k] + 6 * k

    @property
    def o_fib(self):
        return 3 * self.nshell + 3 * self.off_b[-1] + 6 * len(self.bodies)

    # ------------------------------------------------------------ kernels --
    def fiber_flow(self, f):
        """Velocity on all targets due to fiber forces f (per point), with
        each fiber's own contribution removed (flow_fibers + self_flow_fibers)."""
        fw = np.concatenate([f[self.off_f[k]:self.off_f[k + 1]] * self.fms[n].weights(self.lengths[k])[:, None]
                             for k, n in enumerate(self.npts)])
        v = pairs_c.pair_sum("oseen", self.trg_fib, self.trg_all, fw, eta=self.eta)
        for k in range(len(self.fibers)):
            a, b = self.off_f[k], self.off_f[k + 1]
            G = KN.oseen_tensor(self.fibers[k], eta=self.eta)
            v[3 * a:3 * b] -= G @ fw[a:b].reshape(-1)
        return v

    # ------------------------------------------------------------ assembly --
    def _assemble(self):
        eta = self.eta
        nF = self.off_f[-1]
        nB = self.off_b[-1]
        # body geometry, singularity vectors
        self.E_bdy = [singularity_vectors(b.nodes, b.normals, b.weights, eta) for b in self.bodies]
        self.K_bdy = [b.K() for b in self.bodies]
        if self.shell is not None:
            s = self.shell
            self.E_shell = singularity_vectors(s.nodes, s.normals, s.weights, eta)
        # explicit flows from external fiber forces (tstep.py:789-821)
        if self.fibers and np.any(self.force_fibers):
            v = self.fiber_flow(self.force_fibers)
        else:
            v = np.zeros(3 * self.trg_all.shape[0])
        vfib = v[:3 * nF].reshape(-1, 3)
        vbdy = v[3 * nF:3 * (nF + nB)]
        vshell = v[3 * (nF + nB):]
        self.rhs = np.zeros(self.size)
        if self.shell is not None:
            self.rhs[:3 * self.nshell] = -vshell
        for k in range(len(self.bodies)):
            i0 = self.o_body_k(k)
            self.rhs[i0:i0 + 3 * self.nb[k]] = -vbdy[3 * self.off_b[k]:3 * self.off_b[k + 1]]
        # per-fiber operators
        self.A_fib, self.Fop, self.xs = [], [], []
        ff = self.force_fibers if np.any(self.force_fibers) else None
        for k, x in enumerate(self.fibers):
            n, L = self.npts[k], self.lengths[k]
            fm = self.fms[n]
            a, b = self.off_f[k], self.off_f[k + 1]
            fk = None if ff is None else ff[a:b]
            flow = vfib[a:b]
            A = F.linear_operator(fm, x, L, self.E, self.dt, self.c0, self.c1, self.penalty)
            R = F.rhs(fm, x, L, self.dt, self.c0, self.c1, force=fk, flow=flow, penalty=self.penalty)
            B, r = F.bc_rows(fm, x, L, self.E, self.dt, self.c0,
                             end_vec0=(fk[-1] if fk is not None else None),
                             v_on_fiber=flow, force_on_fiber=fk)
            AA, RR = F.apply_bc_rectangular(fm, A, R, B, r)
            self.A_fib.append(AA)
            self.Fop.append(F.force_operator(fm, x, L, self.E))
            self.xs.append(F.derivatives(fm, x, L)[0])
            i0 = self.o_fib + 4 * a
            self.rhs[i0:i0 + 4 * n] = RR
        # preconditioner factors
        self.lu_fib = [sla.lu_factor(A, check_finite=False) for A in self.A_fib]
        self.lu_bdy = []
        for k, bd in enumerate(self.bodies):
            M = KN.stresslet_kernel_times_normal_dense(bd.nodes, bd.normals, eta=eta)
            nb = self.nb[k]
            I = np.zeros((3 * nb, 3 * nb))
            for i in range(nb):
                I[3 * i:3 * i + 3, 3 * i:3 * i + 3] = self.E_bdy[k][i] / bd.weights[i]
            A = np.zeros((3 * nb + 6, 3 * nb + 6))
            A[:3 * nb, :3 * nb] = M - I
            A[:3 * nb, 3 * nb:] = -self.K_bdy[k]
            A[3 * nb:, :3 * nb] = -self.K_bdy[k].T
            A[3 * nb:, 3 * nb:] = np.eye(6)
            self.lu_bdy.append(sla.lu_factor(A))
        if self.shell is not None and self.dense_shell:
            self.M_shell = self.shell_dense()
            self.lu_shell = sla.lu_factor(self.M_shell)

    def shell_dense(self):
        """Shell self operator + complementary (tstep.py:327-347)."""
        s = self.shell
        n = self.nshell
        M = KN.stresslet_kernel_times_normal_dense(s.nodes, s.normals, eta=self.eta)
        for i in range(n):
            M[3 * i:3 * i + 3, 3 * i:3 * i + 3] -= self.E_shell[i] / s.weights[i] + np.eye(3) / s.weights[i]
        M += KN.complementary_kernel(None, s.normals)
        return M

    def shell_apply(self, q):
        """Matrix-free shell_stresslet @ q + shell_complementary @ q."""
        s = self.shell
        n = self.nshell
        qq = q.reshape(n, 3)
        v = pairs_c.pair_sum("stresslet", s.nodes, s.nodes, qq, s.normals, eta=self.eta,
                             self_mode="skip_index").reshape(n, 3)
        mu = qq / s.weights[:, None]
        v -= np.einsum("iac,ic->ia", self.E_shell, mu) + mu
        v += s.normals * np.sum(s.normals * qq)
        return v.reshape(-1)

    # -------------------------------------------------------------- matvec --
    def matvec(self, x):
        """A_body_fiber_hyd (tstep.py:1003-1178), free fibers."""
        eta = self.eta
        nF, nB = self.off_f[-1], self.off_b[-1]
        res = np.zeros_like(x)
        q = x[:3 * self.nshell]
        dens = np.zeros((nB, 3))
        vel = np.zeros((len(self.bodies), 6))
        for k in range(len(self.bodies)):
            i0 = self.o_body_k(k)
            dens[self.off_b[k]:self.off_b[k + 1]] = x[i0:i0 + 3 * self.nb[k]].reshape(-1, 3)
            vel[k] = x[i0 + 3 * self.nb[k]:i0 + 3 * self.nb[k] + 6]
        XT = x[self.o_fib:]
        ntrg = self.trg_all.shape[0]
        v = np.zeros(3 * ntrg)
        # fibers -> all (implicit forces)
        if self.fibers:
            f = np.concatenate([(self.Fop[k] @ XT[4 * self.off_f[k]:4 * self.off_f[k + 1]]).reshape(3, -1).T
                                for k in range(len(self.fibers))])
            v += self.fiber_flow(f)
        # bodies -> all (double layer)
        if self.bodies:
            v += pairs_c.pair_sum("stresslet", self.trg_bdy, self.trg_all, dens, self.nrm_bdy, eta=eta)
        # shell
        if self.shell is not None:
            res[:3 * self.nshell] = self.shell_apply(q) + v[3 * (nF + nB):]
            v[:3 * (nF + nB)] += pairs_c.pair_sum("stresslet", self.shell.nodes, self.trg_all[:nF + nB], q.reshape(-1, 3),
                                                  self.shell.normals, eta=eta)
        # bodies
        for k, bd in enumerate(self.bodies):
            i0 = self.o_body_k(k)
            nb = self.nb[k]
            d = dens[self.off_b[k]:self.off_b[k + 1]]
            mu = d / bd.weights[:, None]
            KU = self.K_bdy[k] @ vel[k]
            r = -np.einsum("iac,ic->ia", self.E_bdy[k], mu).reshape(-1) - KU
            r += v[3 * (nF + self.off_b[k]):3 * (nF + self.off_b[k + 1])]
            res[i0:i0 + 3 * nb] = r
            res[i0 + 3 * nb:i0 + 3 * nb + 6] = -self.K_bdy[k].T @ d.reshape(-1) + vel[k]
        # fibers
        for k in range(len(self.fibers)):
            n, L = self.npts[k], self.lengths[k]
            fm = self.fms[n]
            a, b = self.off_f[k], self.off_f[k + 1]
            vk = v[3 * a:3 * b].reshape(-1, 3)
            D1 = fm.D(L)[0]
            vT = np.concatenate([vk[:, 0], vk[:, 1], vk[:, 2], np.sum(self.xs[k] * (D1 @ vk), axis=1)])
            vT_in = np.zeros(4 * n)
            vT_in[:4 * n - 14] = fm.Pcheb @ vT
            i0 = self.o_fib + 4 * a
            res[i0:i0 + 4 * n] = self.A_fib[k] @ XT[4 * a:4 * b] - vT_in
        return res

    # ----------------------------------------------------- grid velocity --
    def grid_velocity(self, x_all, grid_points, body0_radius=None, near=2e-1, uprate=2):
        """Velocity field at grid points for the solution x_all, as fiber3d's
        time step evaluates it (compute_velocity, tstep.py:1273-1381, and the
        post-processing at tstep.py:1414-1448), free fibers, no fiber-body
        links, no external body forces:
          periphery and body double layers (stresslet source->target of
          their densities), the fibers' Oseen flow of their implicit forces
          (force operator of x_all, trapezoid-weighted, flow_fibers
          tstep_utils.py:653-700), where each grid point within `near` of a
          fiber's node takes instead the fiber's self-flow at its nearest
          node, evaluated with `uprate`-fold upsampled quadrature
          (fiber_matrices.py:84-92: P_kerUp, weights_0_up), the last such
          fiber in fiber order winning; plus the Oseen flow of the external
          fiber forces; and, with body0_radius, rigid motion U + W x (g - c)
          at grid points inside the first body moved to c = loc + dt U."""
        eta = self.eta
        g = np.asarray(grid_points, dtype=np.float64).reshape(-1, 3)
        nB = self.off_b[-1]
        vgrid = np.zeros_like(g)
        if self.shell is not None:
            q = x_all[:3 * self.nshell].reshape(-1, 3)
            vgrid += KN.stresslet_kernel_source_target(self.shell.nodes, g, self.shell.normals, q,
                                                       eta=eta).reshape(-1, 3)
        vel = np.zeros((len(self.bodies), 6))
        if self.bodies:
            dens = np.zeros((nB, 3))
            for k in range(len(self.bodies)):
                i0 = self.o_body_k(k)
                dens[self.off_b[k]:self.off_b[k + 1]] = x_all[i0:i0 + 3 * self.nb[k]].reshape(-1, 3)
                vel[k] = x_all[i0 + 3 * self.nb[k]:i0 + 3 * self.nb[k] + 6]
            vgrid += KN.stresslet_kernel_source_target(self.trg_bdy, g, self.nrm_bdy, dens,
                                                       eta=eta).reshape(-1, 3)
        if self.fibers:
            XT = x_all[self.o_fib:]
            f = np.concatenate([(self.Fop[k] @ XT[4 * self.off_f[k]:4 * self.off_f[k + 1]]).reshape(3, -1).T
                                for k in range(len(self.fibers))])
            fw = np.concatenate([f[self.off_f[k]:self.off_f[k + 1]] * self.fms[n].weights(self.lengths[k])[:, None]
                                 for k, n in enumerate(self.npts)])
            vfib = KN.oseen_kernel_source_target(self.trg_fib, g, fw, eta=eta).reshape(-1, 3)
            for i in range(g.shape[0]):
                for k, xk in enumerate(self.fibers):
                    dist = np.sqrt((g[i, 0] - xk[:, 0]) ** 2 + (g[i, 1] - xk[:, 1]) ** 2 + (g[i, 2] - xk[:, 2]) ** 2)
                    if (dist <= near).any():
                        n, L = self.npts[k], self.lengths[k]
                        a_up = np.linspace(-1.0, 1.0, uprate * n)
                        P_up = F.barycentric_matrix(self.fms[n].alpha, a_up)
                        w_up = np.full(uprate * n, 2.0)
                        w_up[0] = w_up[-1] = 1.0
                        w_up *= (L / 2.0) / (uprate * n - 1)
                        fup = (P_up @ f[self.off_f[k]:self.off_f[k + 1]]) * w_up[:, None]
                        G = KN.oseen_tensor_source_target(P_up @ xk, xk, eta=eta)
                        vself = (G @ fup.reshape(-1)).reshape(-1, 3)
                        vfib[i] = vself[np.argmin(dist)]
            vgrid += vfib
            if np.any(self.force_fibers):
                fe = np.concatenate([self.force_fibers[self.off_f[k]:self.off_f[k + 1]]
                                     * self.fms[n].weights(self.lengths[k])[:, None]
                                     for k, n in enumerate(self.npts)])
                vgrid += KN.oseen_kernel_source_target(self.trg_fib, g, fe, eta=eta).reshape(-1, 3)
        if self.bodies and body0_radius is not None:
            U, W = vel[0, :3], vel[0, 3:]
            c = self.bodies[0].location + U * self.dt
            ids = (g[:, 0] - c[0]) ** 2 + (c[1] - g[:, 1]) ** 2 + (c[2] - g[:, 2]) ** 2 <= body0_radius ** 2
            vgrid[ids] = U
            r = g[ids] - c
            vgrid[ids, 0] += W[1] * r[:, 2] - W[2] * r[:, 1]
            vgrid[ids, 1] += W[2] * r[:, 0] - W[0] * r[:, 2]
            vgrid[ids, 2] += W[0] * r[:, 1] - W[1] * r[:, 0]
        return vgrid

    # ------------------------------------------------------ preconditioner --
    def shell_pc_residual(self, y_shell, x_shell):
        """||M_shell y - x|| / ||x||: how well y solves the shell block of the
        preconditioner (tstep.py:327-351, the LU of M_shell applied to x),
        measured with the matrix-free operator, so no dense matrix is needed."""
        r = self.shell_apply(np.asarray(y_shell)) - np.asarray(x_shell)
        return float(np.linalg.norm(r) / np.linalg.norm(x_shell))

    def shell_block_pc(self, x_shell):
        """Block-Jacobi alternative to the shell LU: each node's 3 x 3 diagonal
        block of the dense operator of tstep.py:327-347 (the double layer
        skips i == j, so the block is -(E_i + I) / w_i + n_i n_i^T) solved
        on its own."""
        s = self.shell
        B = -(self.E_shell + np.eye(3)) / s.weights[:, None, None] + s.normals[:, :, None] * s.normals[:, None, :]
        return np.linalg.solve(B, np.asarray(x_shell).reshape(-1, 3, 1)).reshape(-1)

    def pc(self, x):
        """P_inv (tstep.py:950-994).  Without the dense shell the shell block
        of the result is NaN (use shell_pc_residual for it)."""
        y = np.empty_like(x)
        if self.shell is not None and self.dense_shell:
            y[:3 * self.nshell] = sla.lu_solve(self.lu_shell, x[:3 * self.nshell])
        elif self.shell is not None:
            y[:3 * self.nshell] = np.nan
        for k in range(len(self.bodies)):
            i0 = self.o_body_k(k)
            i1 = i0 + 3 * self.nb[k] + 6
            y[i0:i1] = sla.lu_solve(self.lu_bdy[k], x[i0:i1])
        for k in range(len(self.fibers)):
            i0 = self.o_fib + 4 * self.off_f[k]
            i1 = self.o_fib + 4 * self.off_f[k + 1]
            y[i0:i1] = sla.lu_solve(self.lu_fib[k], x[i0:i1], check_finite=False)
        return y

    # --------------------------------------------------------------- solve --
    def true_residual(self, x):
        """||b - A x|| / ||b|| with this oracle's matvec and right-hand side."""
        return float(np.linalg.norm(self.rhs - self.matvec(np.asarray(x))) / np.linalg.norm(self.rhs))

    def solve(self, tol=1e-8, restart=150, maxiter=200):
        """Right-preconditioned GMRES (bpm_utilities/gmres.py:94-111)."""
        n = self.size
        APinv = spla.LinearOperator((n, n), matvec=lambda y: self.matvec(self.pc(y)), dtype=np.float64)
        its = [0]

        def cb(_):
            its[0] += 1

        y, info = spla.gmres(APinv, self.rhs, rtol=tol, atol=0.0, restart=restart, maxiter=maxiter,
                             callback=cb, callback_type="pr_norm")
        return self.pc(y), info, its[0]


def system_at(problem, fibers, body_locations=None, body_rotations=None, dense_shell=False) -> HydroSystem:
    """The oracle's system for `problem` (any object with the fields of a step
    problem: lengths, E, dt, eta, bodies with ref_nodes / ref_normals /
    weights, shell with nodes / normals / weights, force_fibers, epsilon,
    penalty) at the given fiber positions and body poses (defaults: the
    problem's own).  Without the dense shell (the default) it stays
    matrix-free at any periphery size."""
    bodies = []
    for k, b in enumerate(problem.bodies or []):
        loc = b.location if body_locations is None else body_locations[k]
        rot = b.rotation if body_rotations is None else body_rotations[k]
        bodies.append(Body(np.asarray(loc, dtype=np.float64), np.asarray(rot, dtype=np.float64),
                           np.asarray(b.ref_nodes).reshape(-1, 3), np.asarray(b.ref_normals).reshape(-1, 3),
                           np.asarray(b.weights).reshape(-1)))
    shell = None
    if problem.shell is not None:
        sh = problem.shell
        shell = Shell(np.asarray(sh.nodes).reshape(-1, 3), np.asarray(sh.normals).reshape(-1, 3),
                      np.asarray(sh.weights).reshape(-1))
    ff = problem.force_fibers
    return HydroSystem([np.asarray(f, dtype=np.float64).reshape(-1, 3) for f in fibers], list(problem.lengths),
                       problem.E, problem.dt, problem.eta, bodies, shell,
                       None if ff is None else np.asarray(ff, dtype=np.float64).reshape(-1, 3),
                       getattr(problem, "epsilon", 1e-3), getattr(problem, "penalty", 500.0),
                       dense_shell=dense_shell)
