"""The drop-in module carries every public function of fiber3d's
kernels.kernels (python/kernels/kernels.py) with fiber3d's parameter names,
so substituting it in sys.modules raises no AttributeError.  No GPU needed
(nothing is called)."""
from __future__ import annotations

import inspect

import pytest

from fiber3d_b200 import kernels

# fiber3d's kernels.kernels: name -> its parameters in order (the effective,
# i.e. later, definition of names defined twice)
FIBER3D = {
    "oseen_tensor": ["r_vectors", "eta", "reg", "epsilon_distance", "input_format"],
    "oseen_tensor_source_target": ["r_source", "r_target", "eta", "reg", "epsilon_distance", "input_format"],
    "oseen_kernel_times_density_numba": ["r_vectors", "density", "eta", "reg", "epsilon_distance"],
    "oseen_kernel_source_target_numba": ["r_source", "r_target", "density", "eta", "reg", "epsilon_distance"],
    "oseen_kernel_source_target_pycuda": ["r_source", "r_target", "density", "eta", "epsilon_distance"],
    "rotlet_kernel_source_target_numba": ["r_source", "r_target", "density", "eta", "reg", "epsilon_distance"],
    "stresslet_kernel": ["r_vectors", "eta", "reg", "epsilon_distance", "input_format"],
    "stresslet_kernel_times_normal": ["r_vectors", "normal", "eta", "reg", "epsilon_distance"],
    "stresslet_kernel_times_normal_numba": ["r_vectors", "normal", "eta", "reg", "epsilon_distance"],
    "stresslet_kernel_times_normal_times_density_numba": ["r_vectors", "normal", "density", "eta", "reg",
                                                          "epsilon_distance"],
    "stresslet_kernel_source_target_numba": ["r_source", "r_target", "normal", "density", "eta", "reg",
                                             "epsilon_distance"],
    "traction_kernel_times_normal_times_density_numba": ["r_vectors", "normal", "density", "eta", "reg",
                                                         "epsilon_distance"],
    "complementary_kernel_times_density_numba": ["r_vectors", "normal", "density"],
    "complementary_kernel": ["r_vectors", "normal"],
    "oseen_kernel_source_target_stkfmm": ["r_source", "r_target", "density", "eta", "reg", "epsilon_distance"],
    "stresslet_kernel_source_target_stkfmm": ["r_source", "r_target", "normal", "density", "eta", "reg",
                                              "epsilon_distance"],
    "single_double_layer_kernel_source_target_stkfmm": ["r_source_SL", "r_source_DL", "r_target", "normal",
                                                        "density_SL", "density_DL", "eta", "reg",
                                                        "epsilon_distance"],
}


@pytest.mark.parametrize("name", sorted(FIBER3D))
def test_function_and_parameters(name):
    fn = getattr(kernels, name)
    params = [p for p in inspect.signature(fn).parameters.values()
              if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)]
    assert [p.name for p in params] == FIBER3D[name]
    assert name in kernels.__all__


def test_stkfmm_accept_fmm_handle():
    for name in ("oseen_kernel_source_target_stkfmm", "stresslet_kernel_source_target_stkfmm",
                 "single_double_layer_kernel_source_target_stkfmm"):
        kinds = {p.kind for p in inspect.signature(getattr(kernels, name)).parameters.values()}
        assert inspect.Parameter.VAR_KEYWORD in kinds and inspect.Parameter.VAR_POSITIONAL in kinds
