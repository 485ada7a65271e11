"""Generate golden vectors by running fiber3d's own code (needs the fiber3d
sources; set FIBER3D_REFERENCE to their ``python/`` folder).

    python tests/golden/make_golden.py

Writes compressed .npz fixtures next to this file.  Inputs are seeded
(numpy default_rng); outputs are whatever fiber3d's functions return, so
the fixtures pin the oracle and the GPU path to the reference itself.

Fixtures
  kernels_small.npz   every kernels.kernels function on small seeded inputs,
                      with coincident / sub-epsilon pairs and tile tails
  config1.npz         the Oseen fiber workload (1024 points) and its sum
  sphere.npz          shape_gallery('sphere') nodes/normals, the periphery
                      singularity-subtraction vectors and the dense shell
                      operator (tstep.py:327-347) applied to seeded vectors
  fiber_ops.npz       fiber_matrices for N in {16,24,32,48,64} and, for two
                      fibers, the operator / RHS / BC rows / force operator
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

import refshim  # noqa: E402

refshim.install()

from kernels import kernels as K  # noqa: E402  (fiber3d)
from shape_gallery import shape_gallery  # noqa: E402
from periphery import periphery  # noqa: E402
from quaternion import quaternion  # noqa: E402
from fiber import fiber as fiber_mod  # noqa: E402
from tstep import fiber_matrices  # noqa: E402

from fiber3d_b200 import geometry  # noqa: E402


def with_close_pairs(rng, xs, nt, ncoinc=3, nclose=2):
    """Targets: random points, some coinciding with sources exactly, some at
    a distance below epsilon_distance = 1e-5."""
    xt = rng.random((nt, 3))
    xt[:ncoinc] = xs[:ncoinc]
    for k in range(nclose):
        xt[ncoinc + k] = xs[ncoinc + k] + 3e-6 * rng.normal(size=3) / np.sqrt(3)
    return xt


def kernels_small(rng):
    out = {}
    # A1 Oseen source-target, sizes straddling a 128-point tile
    for tag, ns, nt in (("a", 150, 120), ("b", 129, 257), ("c", 1, 1), ("d", 7, 300)):
        xs = rng.random((ns, 3))
        xt = with_close_pairs(rng, xs, nt, ncoinc=min(3, ns, nt), nclose=min(2, max(ns - 3, 0), max(nt - 3, 0)))
        f = rng.normal(size=(ns, 3))
        out[f"ost_{tag}_rs"], out[f"ost_{tag}_rt"], out[f"ost_{tag}_f"] = xs, xt, f
        out[f"ost_{tag}_u"] = K.oseen_kernel_source_target_numba(xs, xt, f)
    # A1 with non-default eta/reg/eps
    xs = rng.random((90, 3)); xt = with_close_pairs(rng, xs, 70); f = rng.normal(size=(90, 3))
    out["ostp_rs"], out["ostp_rt"], out["ostp_f"] = xs, xt, f
    out["ostp_u"] = K.oseen_kernel_source_target_numba(xs, xt, f, 2.5, 1e-2, 1e-4)
    # A2 Oseen times density: duplicated point at a different index is regularised
    x = rng.random((160, 3)); x[10] = x[20]; x[30] = x[31] + 2e-6
    f = rng.normal(size=(160, 3))
    out["otd_r"], out["otd_f"] = x, f
    out["otd_u"] = K.oseen_kernel_times_density_numba(x, f)
    # A6 rotlet
    xs = rng.random((130, 3)); xt = with_close_pairs(rng, xs, 110); t = rng.normal(size=(130, 3))
    out["rot_rs"], out["rot_rt"], out["rot_t"] = xs, xt, t
    out["rot_u"] = K.rotlet_kernel_source_target_numba(xs, xt, t)
    # A3 stresslet source-target
    xs = rng.random((140, 3)); xt = with_close_pairs(rng, xs, 125)
    n = geometry.uniform_directions(rng, 140); d = rng.normal(size=(140, 3))
    out["sst_rs"], out["sst_rt"], out["sst_n"], out["sst_d"] = xs, xt, n, d
    out["sst_v"] = K.stresslet_kernel_source_target_numba(xs, xt, n, d)
    # A4 stresslet times normal times density
    x = rng.random((150, 3)); x[5] = x[6]
    n = geometry.uniform_directions(rng, 150); d = rng.normal(size=(150, 3))
    out["stnd_r"], out["stnd_n"], out["stnd_d"] = x, n, d
    out["stnd_v"] = K.stresslet_kernel_times_normal_times_density_numba(x, n, d)
    out["stnd_v_eta"] = K.stresslet_kernel_times_normal_times_density_numba(x, n, d, 3.0)
    # A5 dense stresslet times normal
    x = rng.random((40, 3)); n = geometry.uniform_directions(rng, 40)
    out["stn_r"], out["stn_n"] = x, n
    out["stn_M"] = K.stresslet_kernel_times_normal_numba(x, n)
    # oseen_tensor / oseen_tensor_source_target / complementary
    x = rng.random((30, 3)); x[3] = x[4]
    out["ot_r"] = x
    out["ot_G"] = K.oseen_tensor(x)
    out["ot_Gxyz"] = K.oseen_tensor(x.T.flatten(), input_format='xyz')
    xs = rng.random((20, 3)); xt = rng.random((15, 3)); xt[0] = xs[0]
    out["otst_rs"], out["otst_rt"] = xs, xt
    out["otst_G"] = K.oseen_tensor_source_target(xs, xt)
    n = geometry.uniform_directions(rng, 20)
    out["comp_n"] = n
    out["comp_C"] = K.complementary_kernel(rng.random((20, 3)), n)
    d = rng.normal(size=(20, 3))
    out["compd_d"] = d
    out["compd_u"] = K.complementary_kernel_times_density_numba(rng.random((20, 3)), n, d)
    return out


def config1():
    x, f = geometry.oseen_fiber_workload(seed=1)
    return {"x": x, "f": f, "u": K.oseen_kernel_times_density_numba(x, f)}


def sphere(rng):
    out = {}
    for n in (100, 101, 600):
        nodes, normals, _, _ = shape_gallery.shape_gallery('sphere', n, radius=10.0)
        out[f"nodes_{n}"], out[f"normals_{n}"] = nodes, normals
    # periphery operator at N = 300, equal weights (config-2 style), inward normals
    N, R = 300, 10.0
    nodes, normals, _, _ = shape_gallery.shape_gallery('sphere', N, radius=R)
    normals = -normals
    w = np.full(N, 4 * np.pi * R**2 / N)
    shell = periphery.Periphery(np.zeros(3), quaternion.Quaternion([1.0, 0.0, 0.0, 0.0]), nodes, normals, w)
    shell.get_singularity_subtraction_vectors(eta=1.0)
    out["shell_nodes"], out["shell_normals"], out["shell_w"] = nodes, normals, w
    out["shell_ex"], out["shell_ey"], out["shell_ez"] = shell.ex, shell.ey, shell.ez
    # tstep.py:327-347 (dense shell operator, then + complementary)
    M = K.stresslet_kernel_times_normal_numba(nodes, normals, eta=1.0)
    I = np.zeros((3 * N, 3 * N))
    for i in range(N):
        I[3 * i:3 * (i + 1), 3 * i + 0] = shell.ex[3 * i:3 * (i + 1)] / w[i]
        I[3 * i:3 * (i + 1), 3 * i + 1] = shell.ey[3 * i:3 * (i + 1)] / w[i]
        I[3 * i:3 * (i + 1), 3 * i + 2] = shell.ez[3 * i:3 * (i + 1)] / w[i]
    I_vec = np.ones(N * 3)
    I_vec[0::3] /= w; I_vec[1::3] /= w; I_vec[2::3] /= w
    M += -I - np.diag(I_vec)
    C = K.complementary_kernel(nodes, normals)
    q = rng.normal(size=(4, 3 * N))
    out["shell_q"] = q
    out["shell_stresslet_q"] = q @ M.T          # shell_stresslet @ q
    out["shell_full_q"] = q @ (M + C).T         # (shell_stresslet + complementary) @ q
    out["shell_pc_q"] = np.linalg.solve(M + C, q.T).T   # LU preconditioner apply
    return out


def fiber_ops(rng):
    out = {}
    for N in (16, 24, 32, 48, 64):
        fm = fiber_matrices.fiber_matrices(num_points=N, num_points_finite_diff=4)
        fm.compute_matrices()
        out[f"fm{N}_D1"], out[f"fm{N}_D2"] = fm.D_1_0, fm.D_2_0
        out[f"fm{N}_D3"], out[f"fm{N}_D4"] = fm.D_3_0, fm.D_4_0
        out[f"fm{N}_PX"], out[f"fm{N}_PT"] = fm.P_X, fm.P_T
        out[f"fm{N}_Pcheb"] = fm.P_cheb_representations_all_dof
        out[f"fm{N}_w"] = fm.weights_0
    cases = [(32, 2.0, 0.0025, 1e-3, "force", "torque", "force", "torque"),
             (24, 1.5, 0.01, 5e-3, "velocity", "angular_velocity", "velocity", "torque")]
    for c, (N, L, E, dt, b0, b1, e0, e1) in enumerate(cases):
        fm = fiber_matrices.fiber_matrices(num_points=N, num_points_finite_diff=4)
        fm.compute_matrices()
        fib = fiber_mod.fiber(num_points=N, num_points_finite_diff=4, dt=dt, E=E, length=L,
                              epsilon=1e-3, viscosity=1.0)
        x = geometry.perturbed_fibers(rng, 1, N, L, 3.0)[0]
        fib.x = x.copy()
        D1, D2, D3, D4 = fm.get_matrices(fib.length, fib.num_points_up, 'Ds')
        fib.xs, fib.xss, fib.xsss, fib.xssss = D1 @ x, D2 @ x, D3 @ x, D4 @ x
        flow = rng.normal(size=(N, 3))
        force = rng.normal(size=(N, 3)) * 0.1
        fib.set_BC(BC_start_0=b0, BC_start_1=b1, BC_end_0=e0, BC_end_1=e1,
                   BC_end_vec_0=force[-1] if e0 == "force" else np.zeros(3))
        A = fib.form_linear_operator(fm)
        RHS = fib.compute_RHS(fib_mat=fm, force_external=force, flow=flow)
        AA, RR = fib.apply_BC_rectangular(A.copy(), RHS.copy(), fm, flow, force)
        out[f"fib{c}_N"], out[f"fib{c}_L"], out[f"fib{c}_E"], out[f"fib{c}_dt"] = N, L, E, dt
        out[f"fib{c}_bc"] = np.array([b0, b1, e0, e1])
        out[f"fib{c}_x"], out[f"fib{c}_flow"], out[f"fib{c}_force"] = x, flow, force
        out[f"fib{c}_A"], out[f"fib{c}_RHS"] = A, RHS
        out[f"fib{c}_Abc"], out[f"fib{c}_RHSbc"] = AA, RR
        out[f"fib{c}_Fop"] = fib.force_operator(fm)
        out[f"fib{c}_c0"], out[f"fib{c}_c1"] = fib.c_0, fib.c_1
    return out


def main():
    rng = np.random.default_rng(20261203)
    np.savez_compressed(HERE / "kernels_small.npz", **kernels_small(rng))
    np.savez_compressed(HERE / "config1.npz", **config1())
    np.savez_compressed(HERE / "sphere.npz", **sphere(rng))
    np.savez_compressed(HERE / "fiber_ops.npz", **fiber_ops(rng))
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
