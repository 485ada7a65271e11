"""GPU hydrodynamic step (RHS, matvec, block preconditioner, GMRES) against
fiber3d's own time step (tests/golden/step_small.npz: 6 fibers of 16/24/32
points, 2 rigid spheres of 80 nodes, a 240-node periphery), and against the
CPU oracle on a larger seeded system."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu


def problem_from_golden(g):
    from fiber3d_b200 import hydro as H
    npts = [int(n) for n in g["npts"]]
    fibers = [g[f"fib{k}_x"] for k in range(len(npts))]
    ff = np.concatenate([np.tile(g["fext"][k], (npts[k], 1)) for k in range(len(npts))])
    bodies = []
    k = 0
    while f"body{k}_loc" in g:
        bodies.append(H.Body(g[f"body{k}_loc"], H.quaternion_rotation(g[f"body{k}_quat"]),
                             g[f"body{k}_ref_nodes"], g[f"body{k}_ref_normals"], g[f"body{k}_w"]))
        k += 1
    shell = H.Shell(g["shell_nodes"].reshape(-1, 3), g["shell_normals"].reshape(-1, 3), g["shell_w"])
    return H.Problem(fibers, [float(g["L"])] * len(npts), float(g["E"]), float(g["dt"]), float(g["eta"]),
                     bodies, shell, ff)


@pytest.fixture(scope="module")
def golden_step():
    return load_golden("step_small.npz")


@pytest.fixture(scope="module")
def system(golden_step):
    from fiber3d_b200.hydro import HydroSystem
    return HydroSystem(problem_from_golden(golden_step))


def test_rhs(system, golden_step):
    assert system.size == golden_step["rhs"].size
    assert rel_err(system.rhs.cpu().numpy(), golden_step["rhs"]) < 1e-12


def test_matvec(system, golden_step):
    y = torch.empty(system.size, dtype=torch.float64, device="cuda")
    for x, ax in zip(golden_step["probe_x"], golden_step["probe_Ax"]):
        system.matvec(torch.tensor(x, device="cuda"), y)
        assert rel_err(y.cpu().numpy(), ax) < 1e-12


def test_matvec_fp32c(system, golden_step):
    y = torch.empty(system.size, dtype=torch.float64, device="cuda")
    for x, ax in zip(golden_step["probe_x"], golden_step["probe_Ax"]):
        system.matvec(torch.tensor(x, device="cuda"), y, "fp32c")
        assert rel_err(y.cpu().numpy(), ax) < 1e-5


def test_preconditioner(system, golden_step):
    y = torch.empty(system.size, dtype=torch.float64, device="cuda")
    for x, px in zip(golden_step["probe_x"], golden_step["probe_Px"]):
        system.pc(torch.tensor(x, device="cuda"), y)
        assert rel_err(y.cpu().numpy(), px) < 1e-9


def test_preconditioner_lu_path(golden_step):
    """The LU-factor/substitution evaluation of the fiber blocks (fiber3d's
    own, used for blocks above 128) gives the same preconditioner."""
    from fiber3d_b200.hydro import HydroSystem
    s = HydroSystem(problem_from_golden(golden_step), fiber_pc="lu")
    assert s.fiber_pc == "lu"
    y = torch.empty(s.size, dtype=torch.float64, device="cuda")
    for x, px in zip(golden_step["probe_x"], golden_step["probe_Px"]):
        s.pc(torch.tensor(x, device="cuda"), y)
        assert rel_err(y.cpu().numpy(), px) < 1e-9


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_preconditioner_inner_precision(golden_step, storage):
    """The FP32-class preconditioner of the inner solves (FP32 inverses of the
    fiber blocks; FP32 or row-scaled FP16 periphery inverse) stays close to
    fiber3d's P^-1 x."""
    from fiber3d_b200.hydro import HydroSystem
    s = HydroSystem(problem_from_golden(golden_step), inner_shell_pc=storage)
    y = torch.empty(s.size, dtype=torch.float64, device="cuda")
    tol = 1e-5 if storage == "fp32" else 2e-3
    for x, px in zip(golden_step["probe_x"], golden_step["probe_Px"]):
        s.pc(torch.tensor(x, device="cuda"), y, "fp32c")
        assert rel_err(y.cpu().numpy(), px) < tol


@pytest.mark.parametrize("m", [3 * 700, 3 * 704, 3 * 2000])
def test_gemv_f16_row_scaled(m):
    """FP16 rows scaled by powers of two plus FP64 3x3 diagonal blocks, against
    an FP64 product, on a matrix whose rows span several decades (2100
    columns: the element-wise kernel; 2112 and 6000: 16-byte rows, x staged
    whole)."""
    from fiber3d_b200 import _lib
    g = torch.Generator(device="cpu").manual_seed(5)
    M = torch.randn((m, m), generator=g, dtype=torch.float64) * 1e-4
    M *= torch.logspace(-3, 3, m, dtype=torch.float64)[:, None]
    for i in range(0, m, 3):
        M[i:i + 3, i:i + 3] += torch.randn((3, 3), generator=g, dtype=torch.float64) * 1e3
    M = M.cuda()
    x = torch.randn(m, generator=g, dtype=torch.float64).cuda()
    M16 = torch.empty((m, m), dtype=torch.float16, device="cuda")
    sc = torch.empty(m, dtype=torch.float32, device="cuda")
    dg = torch.empty((m, 3), dtype=torch.float64, device="cuda")
    st = _lib.stream_handle()
    _lib.call("f3d_quantize_rows_f16", _lib.ptr(M), m, m, m, 3, _lib.ptr(M16), m, _lib.ptr(sc), _lib.ptr(dg), st)
    y = torch.empty(m, dtype=torch.float64, device="cuda")
    _lib.call("f3d_gemv_f16", _lib.ptr(M16), m, _lib.ptr(sc), _lib.ptr(dg), 3, _lib.ptr(x), _lib.ptr(y), m, m, st)
    ref = M @ x
    off = M.clone()
    for i in range(0, m, 3):
        off[i:i + 3, i:i + 3] = 0
    # the diagonal blocks are exact; the rest carries FP16 rounding per entry
    err = (y - ref).abs().cpu()
    bound = 2e-3 * (off.abs() @ x.abs()).cpu() + 1e-12 * ref.abs().cpu()
    assert bool((err <= bound).all())
    assert bool(torch.all(torch.log2(sc.cpu()) == torch.round(torch.log2(sc.cpu()))))


@pytest.mark.parametrize("use_graph", [False, True])
def test_solve_fp64(system, golden_step, use_graph):
    res = system.solve(tol=1e-10, use_graph=use_graph)
    assert res["info"] == 0
    x = res["x"]
    y = torch.empty_like(x)
    system.matvec(x, y)
    rr = float(torch.linalg.vector_norm(y - system.rhs) / torch.linalg.vector_norm(system.rhs))
    assert rr < 1e-10
    assert rel_err(x.cpu().numpy(), golden_step["sol"]) < 1e-7
    # fiber3d needed 11 iterations at 1e-10 on this system
    assert res["iterations"] <= 16


def test_solve_mixed(system, golden_step):
    res = system.solve(tol=1e-10, mixed=True)
    assert res["info"] == 0
    x = res["x"]
    y = torch.empty_like(x)
    system.matvec(x, y)
    rr = float(torch.linalg.vector_norm(y - system.rhs) / torch.linalg.vector_norm(system.rhs))
    assert rr < 1e-10
    assert rel_err(x.cpu().numpy(), golden_step["sol"]) < 1e-7


def test_fp32c_pair_error_bound(system, golden_step):
    """The FP32C pair sums of the matvec stay within the relative error the
    mixed solver assumes when it tests convergence on FP32C residuals."""
    from fiber3d_b200.gmres import FP32C_PAIR_REL_ERR
    y = torch.empty(system.size, dtype=torch.float64, device="cuda")
    for x in golden_step["probe_x"]:
        xd = torch.tensor(x, device="cuda")
        system.matvec(xd, y, "fp64")
        v64 = system.v.clone()
        y64 = y.clone()
        system.matvec(xd, y, "fp32c")
        err = float(torch.linalg.vector_norm(system.v - v64) / torch.linalg.vector_norm(v64))
        assert err < 0.25 * FP32C_PAIR_REL_ERR
        # the matvec itself moves by at most eps G |v| (G = system.v_gain)
        dy = float(torch.linalg.vector_norm(y - y64))
        assert dy <= FP32C_PAIR_REL_ERR * system.v_gain * float(torch.linalg.vector_norm(v64))


def test_split_residual_bound(system, golden_step):
    """matvec(precision="split") (FP64 sums on the fiber targets, FP32C
    stresslet sums on the body and periphery targets) moves the matvec by at
    most FP32C_PAIR_REL_ERR times the stresslet flow on those targets (their
    rows take the flow with gain 1) -- the bound the mixed solver uses for
    its first residual -- with a factor 4 to spare."""
    from fiber3d_b200.gmres import FP32C_PAIR_REL_ERR
    nf3 = 3 * system.nF
    y64 = torch.empty(system.size, dtype=torch.float64, device="cuda")
    ys = torch.empty_like(y64)
    for x in golden_step["probe_x"]:
        xd = torch.tensor(x, device="cuda")
        system.matvec(xd, y64, "fp64")
        system.matvec(xd, ys, "split")
        xs = xd.clone()
        xs[system.o_fib:] = 0.0  # no fiber forces: v is the stresslet flow alone
        system.matvec(xs, torch.empty_like(y64), "fp64")
        vs_rest = float(torch.linalg.vector_norm(system.v[nf3:]))
        assert vs_rest > 0.0
        dy = float(torch.linalg.vector_norm(ys - y64))
        assert dy <= 0.25 * FP32C_PAIR_REL_ERR * vs_rest
        # the fiber rows see FP64 sums only (split into a launch of their
        # own, so equal to rounding)
        assert rel_err(ys[system.o_fib:].cpu().numpy(), y64[system.o_fib:].cpu().numpy()) < 1e-12


def test_norm_of_vectors_of_any_length(system):
    """The GMRES workspace's norm reads exactly the vector it is given (the
    mixed solver takes the norm of the pair sums, which are shorter than the
    unknown vector)."""
    from fiber3d_b200.gmres import DeviceGMRES
    g = DeviceGMRES(system.size, 10)
    beta = torch.zeros(1, dtype=torch.float64, device="cuda")
    for n in (1, 7, 1000, system.size - 3, system.size):
        w = torch.randn(n, dtype=torch.float64, device="cuda")
        g._norm(w, beta)
        assert abs(float(beta) - float(torch.linalg.vector_norm(w))) <= 1e-14 * float(torch.linalg.vector_norm(w))


@pytest.mark.parametrize("mixed", [False, True])
def test_guess_flow_summed_in_update(golden_step, mixed):
    """update(x0) sums the Oseen flow of the guess with the explicit flow in
    one pass; the FP64 solve that starts from it returns exactly what it
    returns when it sums that flow itself, and the mixed one (whose first
    residual then adds only an FP32C stresslet flow) reaches the same
    tolerance."""
    from fiber3d_b200.hydro import HydroSystem
    P = problem_from_golden(golden_step)
    a, b = HydroSystem(P), HydroSystem(P)
    x0 = torch.tensor(golden_step["probe_x"][0], device="cuda") * 1e-3 + torch.tensor(golden_step["sol"],
                                                                                     device="cuda")
    a.update(x0)
    assert a.pending_oseen(x0)
    assert torch.equal(a.rhs, b.rhs)
    ra = a.solve(tol=1e-10, x0=x0, mixed=mixed)
    rb = b.solve(tol=1e-10, x0=x0, mixed=mixed)
    assert not a.pending_oseen(x0)
    if not mixed:
        assert torch.equal(ra["x"], rb["x"]) and ra["iterations"] == rb["iterations"]
    else:
        y = torch.empty_like(ra["x"])
        for r, s in ((ra, a), (rb, b)):
            s.matvec(r["x"], y)
            assert float(torch.linalg.vector_norm(y - s.rhs) / torch.linalg.vector_norm(s.rhs)) <= 1e-10
        assert rel_err(ra["x"].cpu().numpy(), rb["x"].cpu().numpy()) < 1e-7


def test_advance_equals_fresh_system(golden_step):
    """A system moved by advance(sol) equals one built from scratch at the
    moved geometry (fibers at the positions in sol; bodies moved by
    tstep.py:1403-1407 on the host): the right-hand side and the matvec at
    1e-12, the bodies' states at 1e-14.  The step is exaggerated (fiber
    points shifted by up to 0.02, bodies translated by 0.05 and turned by
    0.1 rad) so that any sum left at the old geometry shows."""
    from fiber3d_b200 import hydro as H
    P = problem_from_golden(golden_step)
    s = H.HydroSystem(P)
    rng = np.random.default_rng(7)
    sol = golden_step["sol"].copy()
    dt = P.dt
    for k in range(s.nbody):
        o = s.o_body[k] + 3 * s.nb[k]
        u = rng.normal(size=3)
        w = rng.normal(size=3)
        sol[o:o + 3] = 0.05 / dt * u / np.linalg.norm(u)
        sol[o + 3:o + 6] = 0.1 / dt * w / np.linalg.norm(w)
    fibers = []
    for f in range(s.fs.nfib):
        n, p0 = int(s.fs.npts[f]), int(s.fs.pt_off_h[f])
        o = s.o_fib + 4 * p0
        sol[o:o + 3 * n] += rng.uniform(-0.02, 0.02, size=3 * n)
        fibers.append(sol[o:o + 3 * n].reshape(3, n).T.copy())
    loc0, q0 = s.body_state()
    s.advance(torch.tensor(sol, device="cuda"))
    bodies = []
    for k, b in enumerate(P.bodies):
        o = s.o_body[k] + 3 * s.nb[k]
        loc = loc0[k] + dt * sol[o:o + 3]
        q = H.quaternion_multiply(H.quaternion_from_rotation(sol[o + 3:o + 6] * dt), q0[k])
        bodies.append(H.Body(loc, H.quaternion_rotation(q), b.ref_nodes, b.ref_normals, b.weights))
        loc_d, q_d = s.body_state()
        assert np.max(np.abs(loc_d[k] - loc)) < 1e-14 and np.max(np.abs(q_d[k] - q)) < 1e-14
    moved = H.Problem(fibers, P.lengths, P.E, P.dt, P.eta, bodies, P.shell, P.force_fibers)
    fresh = H.HydroSystem(moved)
    assert rel_err(s.rhs.cpu().numpy(), fresh.rhs.cpu().numpy()) < 1e-12
    assert rel_err(s.rhs.cpu().numpy(), H.HydroSystem(P).rhs.cpu().numpy()) > 1e-6
    y, z = (torch.empty(s.size, dtype=torch.float64, device="cuda") for _ in range(2))
    for x in golden_step["probe_x"]:
        xt = torch.tensor(x, device="cuda")
        s.matvec(xt, y)
        fresh.matvec(xt, z)
        assert rel_err(y.cpu().numpy(), z.cpu().numpy()) < 1e-12


def test_pc_refresh_auto(golden_step):
    """pc_refresh="auto" keeps the fiber-block inverses while solves end in
    one iteration with margin, rebuilds them after any other solve, and
    every step still reaches the tolerance in FP64."""
    from fiber3d_b200 import hydro as H, warmstart as W
    P = problem_from_golden(golden_step)
    for bad in (0, "sometimes"):
        with pytest.raises(ValueError):
            H.HydroSystem(P, pc_refresh=bad)
    s = H.HydroSystem(P, pc_refresh="auto")
    history, rebuilt = [], []
    y = torch.empty(s.size, dtype=torch.float64, device="cuda")
    for step in range(6):
        x0 = W.extrapolate(history)
        stale, age = s._pc_stale, s._pc_age
        if history:
            s.advance(history[-1], x0=x0)
            expect = stale or age + 1 >= s.PC_AUTO_MAX_AGE
            assert s._pc_age == (0 if expect else age + 1)
        rebuilt.append(s._pc_age == 0)
        res = s.solve(tol=1e-9, x0=x0, mixed=True)
        assert res["info"] == 0
        assert s._pc_stale == (res["iterations"] > 1 or res["history"][-1] > s.PC_AUTO_MARGIN * 1e-9)
        s.matvec(res["x"], y)
        assert float(torch.linalg.vector_norm(y - s.rhs) / torch.linalg.vector_norm(s.rhs)) <= 1e-9
        history = (history + [res["x"]])[-3:]
    assert rebuilt[0]


def test_speculative_first_inner_step_is_exact(golden_step):
    """Launching the inner solve's first Arnoldi step before the host reads
    the first residual's norm changes the order of host reads only: the
    solution is bit-for-bit the one of the plain order."""
    from fiber3d_b200.hydro import HydroSystem
    P = problem_from_golden(golden_step)
    x0 = torch.tensor(golden_step["probe_x"][0], device="cuda") * 1e-3 + torch.tensor(golden_step["sol"],
                                                                                     device="cuda")
    out = []
    for spec in (False, True):
        s = HydroSystem(P)
        s.update(x0)
        s._spec_first = spec
        res = s.solve(tol=1e-10, x0=x0, mixed=True)
        assert res["info"] == 0 and res["iterations"] >= 1
        out.append(res)
    assert torch.equal(out[0]["x"], out[1]["x"])
    assert out[0]["iterations"] == out[1]["iterations"] and out[0]["history"] == out[1]["history"]


def test_graph_and_eager_agree(system):
    a = system.solve(tol=1e-9, use_graph=False)["x"]
    b = system.solve(tol=1e-9, use_graph=True)["x"]
    assert torch.equal(a, b)


def test_larger_system_against_oracle():
    """48 fibers of uneven resolution (16..64 points), 2 bodies, 600-node
    periphery: device matvec / preconditioner / RHS equal the oracle's."""
    from fiber3d_b200 import geometry, hydro as H
    from oracle import system as S
    rng = np.random.default_rng(77)
    npts = list(rng.choice([16, 24, 32, 48, 64], size=48))
    fibers = geometry.perturbed_fibers(rng, 48, npts, 2.0, 4.0)
    ff = np.concatenate([np.tile(rng.normal(scale=0.1, size=3), (n, 1)) for n in npts])
    nodes, normals = geometry.fibonacci_sphere(80, 0.5)
    w = np.full(80, 4 * np.pi * 0.25 / 80)
    bl = [geometry.uniform_ball(rng, 1, 4.0)[0] for _ in range(2)]
    qs = [rng.normal(size=4) for _ in range(2)]
    qs = [q / np.linalg.norm(q) for q in qs]
    snodes, snormals = geometry.fibonacci_sphere(600, 8.0)
    sw = np.full(600, 4 * np.pi * 64.0 / 600)
    gp = H.Problem(fibers, [2.0] * 48, 0.0025, 1e-3, 1.0,
                   [H.Body(bl[k], H.quaternion_rotation(qs[k]), nodes, normals, w) for k in range(2)],
                   H.Shell(snodes, -snormals, sw), ff)
    op = S.HydroSystem(fibers, [2.0] * 48, 0.0025, 1e-3, 1.0,
                       [S.Body(bl[k], S.quaternion_rotation(qs[k]), nodes, normals, w) for k in range(2)],
                       S.Shell(snodes, -snormals, sw), ff)
    dev = H.HydroSystem(gp)
    assert rel_err(dev.rhs.cpu().numpy(), op.rhs) < 1e-12
    x = rng.normal(size=op.size)
    y = torch.empty(op.size, dtype=torch.float64, device="cuda")
    dev.matvec(torch.tensor(x, device="cuda"), y)
    # 1e-10 here: at N = 64 the third derivative xsss = D3 x carries ~1e-9
    # of FP64 rounding (|D3| ~ 2e6), which the tension rows multiply by
    # 6 c0 E D3 ~ 2e4; any two FP64 evaluation orders differ by that much.
    assert rel_err(y.cpu().numpy(), op.matvec(x)) < 1e-10
    dev.pc(torch.tensor(x, device="cuda"), y)
    assert rel_err(y.cpu().numpy(), op.pc(x)) < 1e-9


def test_output_records_from_marched_system(golden_step, tmp_path):
    """A step marched on the device is written in fiber3d's layout: the
    fibers file holds the solution's positions and tensions, the velocity
    file the bodies' U and Omega, the clones file the advanced poses."""
    from fiber3d_b200 import hydro as H
    from fiber3d_b200.output import OutputWriter, records_from_solution
    P = problem_from_golden(golden_step)
    s = H.HydroSystem(P)
    sol = golden_step["sol"].copy()
    s.advance(torch.tensor(sol, device="cuda"))
    fibers, bodies = records_from_solution(s, sol, P.E, P.lengths, body_radius=[0.5] * s.nbody)
    out = str(tmp_path / "run")
    with OutputWriter(out, True, P.dt, 1) as w:
        w.write(P.dt, 1, 0, fibers, bodies)
    rows = np.loadtxt(out + "_one_fibers.txt")
    r = 1
    for f in range(s.fs.nfib):
        n, p0 = int(s.fs.npts[f]), int(s.fs.pt_off_h[f])
        blk = sol[s.o_fib + 4 * p0:s.o_fib + 4 * (p0 + n)].reshape(4, n)
        assert rows[r][0] == n and rows[r][1] == P.E
        assert np.array_equal(rows[r + 1:r + 1 + n], blk.T)
        r += 1 + n
    vel = np.loadtxt(out + "_onevelocity_clones.txt")[1:]
    locs, quats = s.body_state()
    clones = np.loadtxt(out + "_one_clones.txt")[1:].reshape(s.nbody, 2, 7)
    for k in range(s.nbody):
        o = s.o_body[k] + 3 * s.nb[k]
        assert np.array_equal(vel[k], sol[o:o + 6])
        assert np.array_equal(clones[k, 1], np.concatenate([locs[k], quats[k]]))
