"""tcgen05 BF16 GEMM and the warm-start network's forward/backward passes.

GEMM numerics are compared with a plain PyTorch FP32 product of the same
BF16-rounded operands (tolerance 1e-4 relative: FP32 accumulation order);
the network's loss and gradients with the CPU oracle (oracle/mlp.py).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import mlp as OM
from fiber3d_b200.warmstart import LAYERS

pytestmark = pytest.mark.gpu


def _bf(x):
    return x.to(torch.bfloat16).to(torch.float32)


@pytest.mark.parametrize("M,N,K", [(128, 256, 192), (2000, 256, 256), (77, 128, 256), (256, 192, 1000),
                                   (5, 16, 16), (300, 48, 40)])
def test_gemm_matches_fp32_reference(M, N, K):
    from fiber3d_b200.warmstart import gemm
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N)
    A = torch.randn(M, K, generator=g).cuda()
    B = torch.randn(N, K, generator=g).cuda()
    C = gemm(A, B)
    ref = _bf(A) @ _bf(B).T
    assert rel_err(C.cpu().numpy(), ref.cpu().numpy()) < 1e-4


def test_gemm_transposes_bias_relu_mask():
    from fiber3d_b200.warmstart import gemm
    g = torch.Generator(device="cpu").manual_seed(3)
    A = torch.randn(256, 300, generator=g).cuda()     # used as A^T: K=256 x M=300
    B = torch.randn(256, 160, generator=g).cuda()     # used untransposed: K=256 x N=160
    C = gemm(A, B, transpose_a=True, transpose_b=False)
    ref = _bf(A).T @ _bf(B)
    assert rel_err(C.cpu().numpy(), ref.cpu().numpy()) < 1e-4
    X = torch.randn(200, 64, generator=g).cuda()
    W = torch.randn(32, 64, generator=g).cuda()
    bias = torch.randn(32, generator=g).cuda()
    pre = torch.empty(200, 32, device="cuda")
    Y = gemm(X, W, bias=bias, relu=True, pre=pre)
    z = _bf(X) @ _bf(W).T + bias
    assert rel_err(pre.cpu().numpy(), z.cpu().numpy()) < 1e-4
    assert rel_err(Y.cpu().numpy(), torch.relu(z).cpu().numpy()) < 1e-4
    M = gemm(X, W, mask=z)
    assert rel_err(M.cpu().numpy(), ((_bf(X) @ _bf(W).T) * (z > 0)).cpu().numpy()) < 1e-4


def test_mlp_gradients_against_cpu_oracle():
    from fiber3d_b200.warmstart import FiberMLP
    net = FiberMLP(seed=4)
    rng = np.random.default_rng(8)
    X = rng.normal(size=(384, LAYERS[0])).astype(np.float32)
    T = rng.normal(size=(384, LAYERS[-1])).astype(np.float32)
    loss, gr = net.grads(torch.tensor(X, device="cuda"), torch.tensor(T, device="cuda"))
    W = [w.cpu().numpy() for w in net.W]
    b = [x.cpu().numpy() for x in net.b]
    ref_loss, gW, gb = OM.grads(W, b, X, T)
    assert abs(float(loss) - ref_loss) / ref_loss < 1e-3
    for k in range(4):
        assert rel_err(gr[k].cpu().numpy(), gW[k]) < 2e-2, f"dW{k}"
        assert rel_err(gr[4 + k].cpu().numpy(), gb[k]) < 2e-2, f"db{k}"


def test_mlp_training_reduces_loss():
    """A learnable map (targets a fixed random network of the inputs) is
    fitted by the GPU Adam steps."""
    from fiber3d_b200.warmstart import FiberMLP
    teacher = FiberMLP(seed=1)
    g = torch.Generator(device="cpu").manual_seed(2)
    X = torch.randn(4096, LAYERS[0], generator=g).cuda()
    T = teacher.forward(X)
    student = FiberMLP(seed=9)
    student.set_normalisation(X, T)
    hist = student.train(X, T, epochs=15, batch=512, lr=2e-3)
    assert hist[-1] < 0.7 * hist[0]
