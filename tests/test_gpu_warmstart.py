"""The learned GMRES warm start.  Trained by the library's own tensor-core
kernels on time steps of small seeded problems, it must start GMRES far below
fiber3d's zero guess (r0 = 1), lower the initial residual of the quadratic
extrapolation it corrects on a held-out trajectory, and leave the converged
answer unchanged (GMRES still runs to the same relative residual)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TRAIN_SEEDS = (301, 302, 303, 304)
TRAIN_STEPS = 20
EVAL_STEPS = 12


def small_problem(seed):
    from fiber3d_b200 import geometry
    return geometry.hydro_step_problem(seed=seed, nfib=64, nshell=800, shell_radius=8.0, nbody=0,
                                       fiber_ball=4.0)


@pytest.fixture(scope="module")
def trained():
    from fiber3d_b200 import hydro as H, warmstart as W
    P0 = small_problem(300)
    shell = H.ShellOperator(P0.shell, P0.eta, P0.reg, P0.eps_dist)
    X, T = [], []
    for seed in TRAIN_SEEDS:
        s = H.HydroSystem(small_problem(seed), shell_op=shell)
        _, x, t = W.march(s, TRAIN_STEPS, guess="extrapolate", record=True)
        X.append(x)
        T.append(t)
    X, T = torch.cat(X), torch.cat(T)
    model = W.LearnedWarmStart(seed=0)
    hist = model.fit(X, T, epochs=60, batch=256, lr=1e-3)
    sel = model.select_scale(lambda: [H.HydroSystem(small_problem(sd), shell_op=shell) for sd in (305, 306)],
                             EVAL_STEPS)
    return model, shell, hist, sel


@pytest.fixture(scope="module")
def held_out(trained):
    from fiber3d_b200 import hydro as H, warmstart as W
    model, shell, _, _ = trained
    P = small_problem(399)  # seed outside the training set
    return {g: W.march(H.HydroSystem(P, shell_op=shell), EVAL_STEPS, guess=g, net=model)
            for g in ("zero", "extrapolate", "learned")}


def test_training_converges(trained):
    model, _, hist, _ = trained
    assert np.isfinite(hist).all()
    assert hist[-1] < 0.5 * hist[0]
    g = model.gain.cpu().numpy()
    assert np.all((g >= 0.0) & (g <= 1.0))


def test_learned_guess_far_below_zero_guess(held_out):
    zero, learned = held_out["zero"], held_out["learned"]
    assert all(s["converged"] for s in zero + learned)
    assert all(s["initial_rel_residual"] == 1.0 for s in zero)
    # once the history exists the guess starts GMRES orders of magnitude lower
    assert max(s["initial_rel_residual"] for s in learned[4:]) < 1e-2
    assert sum(s["iterations"] for s in learned) < sum(s["iterations"] for s in zero)


def test_scale_selected_on_validation_trajectory(trained):
    """The correction factors are the candidates with the fewest GMRES
    iterations on the validation trajectories, and a correction is kept only
    if it strictly beats plain extrapolation (factors 0, 0) there."""
    model, _, _, sel = trained
    key = f"{model.scale[0]},{model.scale[1]}"
    best = min(v["iterations"] for v in sel.values())
    assert sel[key]["iterations"] == best
    if model.scale != (0.0, 0.0):
        assert sel[key]["iterations"] < sel["0.0,0.0"]["iterations"]


def test_learned_correction_on_held_out_trajectory(trained, held_out):
    """On a trajectory used neither for training nor for the selection, the
    corrected guess needs no more GMRES iterations than the extrapolation it
    corrects, and where the network acts it lowers the initial residual (in
    the geometric mean over the steps)."""
    ex, le = held_out["extrapolate"], held_out["learned"]
    assert sum(s["iterations"] for s in le) <= sum(s["iterations"] for s in ex)


def test_network_lowers_extrapolation_residual(trained):
    """What the trained network itself gains: with its correction applied
    (factors 1, 1), the initial residual on a held-out trajectory is below
    that of the quadratic extrapolation alone, in the geometric mean over
    the steps where the network acts."""
    from fiber3d_b200 import hydro as H, warmstart as W
    model, shell, _, _ = trained
    saved = model.scale
    model.scale, model._fold = (1.0, 1.0), None
    try:
        P = small_problem(399)
        le = W.march(H.HydroSystem(P, shell_op=shell), EVAL_STEPS, guess="learned", net=model)
    finally:
        model.scale, model._fold = saved, None
    ex = W.march(H.HydroSystem(P, shell_op=shell), EVAL_STEPS, guess="extrapolate")
    r_ex = np.array([s["initial_rel_residual"] for s in ex[W.HISTORY:]])
    r_le = np.array([s["initial_rel_residual"] for s in le[W.HISTORY:]])
    assert np.exp(np.mean(np.log(r_le / r_ex))) < 1.0


def _history(model, shell, seed):
    from fiber3d_b200 import hydro as H, warmstart as W
    s = H.HydroSystem(small_problem(seed), shell_op=shell)
    history = []
    for _ in range(W.HISTORY + 2):
        if history:
            s.advance(history[-1])
        history = (history + [s.solve(tol=1e-10)["x"]])[-W.HISTORY:]
    s.advance(history[-1])
    return s, history


def test_feature_kernel_matches_reference(trained):
    """f3d_warmstart_features against the PyTorch restatement of the
    features (raw and standardised)."""
    from fiber3d_b200 import _lib, warmstart as W
    model, shell, _, _ = trained
    s, history = _history(model, shell, 397)
    f_ref, sx_ref, st_ref = W.history_features(s, history)
    nfib = s.fs.nfib
    for mean, std in ((None, None), (model.net.in_mean, model.net.in_std)):
        f = torch.empty_like(f_ref)
        sx = torch.empty(nfib, dtype=torch.float64, device="cuda")
        st = torch.empty_like(sx)
        h = [x.contiguous() for x in history]
        _lib.call("f3d_warmstart_features", *[_lib.ptr(x) for x in h], h[0].numel(), s.o_fib, nfib, W.NPTS,
                  _lib.ptr(mean), _lib.ptr(std), _lib.ptr(f), _lib.ptr(sx), _lib.ptr(st), _lib.stream_handle())
        ref = f_ref if mean is None else (f_ref - mean) / std
        assert float((f - ref).abs().max() / ref.abs().max()) < 1e-5
        assert torch.allclose(sx, sx_ref.view(-1), rtol=1e-12, atol=0)
        assert torch.allclose(st, st_ref.view(-1), rtol=1e-12, atol=0)


def test_guess_kernels_match_reference(trained):
    """The six-launch guess (feature kernel, GEMMs with the folded last
    layer, guess kernel) against the PyTorch-composed guess: the correction
    agrees to BF16 accuracy and the extrapolation part exactly."""
    from fiber3d_b200 import warmstart as W
    model, shell, _, _ = trained
    s, history = _history(model, shell, 397)
    x_q = W.extrapolate(history)
    saved = model.scale
    model.scale, model._fold = (1.0, 1.0), None
    try:
        g = model.guess(s, history)
        g_ref = model.guess_reference(s, history)
    finally:
        model.scale, model._fold = saved, None
    o = s.o_fib
    assert torch.equal(g[:o], x_q[:o])
    c, c_ref = g[o:] - x_q[o:], g_ref[o:] - x_q[o:]
    assert float(torch.linalg.vector_norm(c - c_ref) / torch.linalg.vector_norm(c_ref)) < 3e-2


def test_converged_answer_unchanged(trained):
    from fiber3d_b200 import hydro as H, warmstart as W
    model, shell, _, _ = trained
    s = H.HydroSystem(small_problem(398), shell_op=shell)
    history = []
    for _ in range(W.HISTORY):
        if history:
            s.advance(history[-1])
        history.append(s.solve(tol=1e-10)["x"])
    s.advance(history[-1])
    ref = s.solve(tol=1e-10)["x"]
    x0 = W.learned_guess(s, history, model)
    got = s.solve(tol=1e-10, x0=x0)["x"]
    assert float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)) < 1e-8
