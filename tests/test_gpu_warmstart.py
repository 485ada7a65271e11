"""The learned GMRES warm start: trained by the library's own tensor-core
kernels on the plain solver's time steps, it must start GMRES closer to the
solution than fiber3d's zero guess, need fewer iterations over a held-out
trajectory, and leave the converged answer unchanged (GMRES still runs to the
same relative residual)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


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
    for seed in (301, 302, 303, 304):
        s = H.HydroSystem(small_problem(seed), shell_op=shell)
        _, x, t = W.march(s, 15, guess="previous", record=True)
        X.append(x)
        T.append(t)
    X, T = torch.cat(X), torch.cat(T)
    net = W.FiberMLP(seed=0)
    net.set_normalisation(X, T)
    hist = net.train(X, T, epochs=60, batch=256, lr=1e-3)
    return net, shell, hist


def test_training_converges(trained):
    net, shell, hist = trained
    assert np.isfinite(hist).all()
    assert hist[-1] < 0.5 * hist[0]


def test_learned_guess_beats_zero_guess(trained):
    from fiber3d_b200 import hydro as H, warmstart as W
    net, shell, _ = trained
    P = small_problem(399)  # seed outside the training set
    zero = W.march(H.HydroSystem(P, shell_op=shell), 8, guess="zero")
    learned = W.march(H.HydroSystem(P, shell_op=shell), 8, guess="learned", net=net)
    assert all(s["converged"] for s in zero + learned)
    iz = sum(s["iterations"] for s in zero)
    il = sum(s["iterations"] for s in learned)
    assert il < iz, f"learned {il} vs zero {iz} iterations"
    # after the first step the network starts GMRES far below fiber3d's r0 = 1
    assert max(s["initial_rel_residual"] for s in learned[1:]) < 1e-2


def test_converged_answer_unchanged(trained):
    from fiber3d_b200 import hydro as H, warmstart as W
    net, shell, _ = trained
    P = small_problem(398)
    s = H.HydroSystem(P, shell_op=shell)
    ref = s.solve(tol=1e-10)["x"]
    u = W.background_velocity(s, None)
    x0 = W.guess_from_prediction(s, net.predict(W.fiber_features(s.x_fib, u, 32)), u, None)
    got = s.solve(tol=1e-10, x0=x0)["x"]
    assert float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)) < 1e-8
