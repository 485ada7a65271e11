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
    return model, shell, hist


@pytest.fixture(scope="module")
def held_out(trained):
    from fiber3d_b200 import hydro as H, warmstart as W
    model, shell, _ = trained
    P = small_problem(399)  # seed outside the training set
    return {g: W.march(H.HydroSystem(P, shell_op=shell), EVAL_STEPS, guess=g, net=model)
            for g in ("zero", "extrapolate", "learned")}


def test_training_converges(trained):
    model, _, hist = trained
    assert np.isfinite(hist).all()
    assert hist[-1] < 0.5 * hist[0]
    g = model.gain.cpu().numpy()
    assert np.all((g >= 0.0) & (g <= 1.0))


def test_learned_guess_far_below_zero_guess(held_out):
    zero, learned = held_out["zero"], held_out["learned"]
    assert all(s["converged"] for s in zero + learned)
    assert all(s["initial_rel_residual"] == 1.0 for s in zero)
    # once the history exists the guess starts GMRES orders of magnitude lower
    assert max(s["initial_rel_residual"] for s in learned[4:]) < 1e-3
    assert sum(s["iterations"] for s in learned) < sum(s["iterations"] for s in zero)


def test_learned_correction_lowers_extrapolation_residual(held_out):
    """Where the network acts (four solutions known) the corrected guess has
    a lower initial residual than the quadratic extrapolation alone, in the
    geometric mean over the held-out steps."""
    ex = np.array([s["initial_rel_residual"] for s in held_out["extrapolate"][4:]])
    le = np.array([s["initial_rel_residual"] for s in held_out["learned"][4:]])
    assert np.exp(np.mean(np.log(le / ex))) < 0.9


def test_converged_answer_unchanged(trained):
    from fiber3d_b200 import hydro as H, warmstart as W
    model, shell, _ = trained
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
