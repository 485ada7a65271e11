"""RBF quadrature weights of a smooth closed surface on the GPU.

Drop-in for fiber3d's ``quadratures.Smooth_Closed_Surface_Quadrature_RBF``
(python/quadratures/Smooth_Closed_Surface_Quadrature_RBF.py:3-470), the
set-up step that gives the periphery and the bodies their node weights
(tstep/tstep.py:297-300, body/body.py:104-107).  fiber3d loops over the
triangles in Python (about 5 ms each, 1-2 minutes for a 12000-node shell);
here one call to ``f3d_surface_quadrature`` does every triangle on the device
(csrc/f3d_quadrature.cu).

Install as the module fiber3d imports::

    import sys, fiber3d_b200.quadrature as q
    sys.modules["quadratures.Smooth_Closed_Surface_Quadrature_RBF"] = q
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

N_NEIGHBORS = 80


def _as_device(a, dtype, device) -> torch.Tensor:
    t = a if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a))
    return t.to(device=device, dtype=dtype).contiguous()


def surface_quadrature_weights(nodes, triangles, gradient, device=None, return_neighbors: bool = False):
    """Node weights (n,) float64 on the device.

    nodes (n, 3) and gradient (n, 3) (the level-set gradient at the nodes,
    ``gradh(nodes)``), triangles (ntri, 3) of a closed triangulation;
    numpy arrays or tensors.  With ``return_neighbors`` also returns the
    (ntri, 80) int32 nodes nearest each triangle's midpoint, nearest first.
    Raises ``ValueError`` for fewer than 80 nodes (fiber3d's neighbour
    search needs 80) and ``F3DError`` for a triangulation that is not a closed
    surface or a singular local system.  The device error word is read (and
    cleared) after the call, so an error an earlier kernel left there is
    raised here too rather than lost.
    """
    if device is None:
        device = nodes.device if isinstance(nodes, torch.Tensor) and nodes.is_cuda else torch.device("cuda", 0)
    X = _as_device(nodes, torch.float64, device)
    G = _as_device(gradient, torch.float64, device)
    T = _as_device(triangles, torch.int32, device)
    if X.ndim != 2 or X.shape[1] != 3 or G.shape != X.shape or T.ndim != 2 or T.shape[1] != 3:
        raise ValueError("nodes and gradient must be (n, 3), triangles (ntri, 3)")
    n, ntri = X.shape[0], T.shape[0]
    if n < N_NEIGHBORS:
        raise ValueError(f"Expected n_neighbors <= n_samples_fit, but n_neighbors = {N_NEIGHBORS}, "
                         f"n_samples_fit = {n}")
    nbytes = ctypes.c_size_t(0)
    _lib.call("f3d_surface_quadrature_workspace_bytes", n, ntri, ctypes.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=device)
    w = torch.empty(n, dtype=torch.float64, device=device)
    nni = torch.empty((ntri, N_NEIGHBORS), dtype=torch.int32, device=device) if return_neighbors else None
    with torch.cuda.device(device):
        _lib.call("f3d_surface_quadrature", _lib.ptr(X), n, _lib.ptr(T), ntri, _lib.ptr(G), _lib.ptr(w),
                  _lib.ptr(nni), _lib.ptr(ws), nbytes.value, _lib.stream_handle(device))
        torch.cuda.current_stream(device).synchronize()
        err = _lib.device_error(device)
    if err:
        _lib.check("f3d_surface_quadrature", err)
    return (w, nni) if return_neighbors else w


def Smooth_Closed_Surface_Quadrature_RBF(Quadrature_Nodes, Triangles, *args):  # noqa: N802 (fiber3d's name)
    """fiber3d's signature and return value: an (n, 1) float64 numpy array.

    ``args`` = (h, gradh), the level set and its gradient as callables on
    (n, 3) arrays.  fiber3d warns when h is not near zero at the nodes
    (:62-67); so does this.  The branch without (h, gradh), which fits the
    normals from an RBF interpolant, is not used by any fiber3d caller and is
    not provided.
    """
    if len(args) != 2:
        raise NotImplementedError("only the exact-gradient form Smooth_Closed_Surface_Quadrature_RBF("
                                  "nodes, triangles, h, gradh) is provided (the one every fiber3d caller uses)")
    h, gradh = args
    nodes = np.asarray(Quadrature_Nodes, dtype=np.float64)
    if np.linalg.norm(h(nodes), ord=np.inf) > 100 * np.spacing(1):
        print('')
        print('Warning: h(x,y,z) is not sufficiently close to zero for')
        print('all points in Quadrature_Nodes.')
        print('')
    grad = np.asarray(gradh(nodes), dtype=np.float64)
    w = surface_quadrature_weights(nodes, np.asarray(Triangles), grad)
    return w.cpu().numpy()[:, None]
