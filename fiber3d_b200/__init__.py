"""fiber3d_b200 — the hydrodynamic hot path of fiber3d on one NVIDIA B200.

Modules
  kernels   drop-in replacement of fiber3d's ``kernels.kernels`` (same names
            and signatures), running hand-written sm_100a CUDA through the C
            ABI declared in include/fiber3d_b200.h
  geometry  seeded synthetic geometry (Fibonacci sphere, fibers)
  build     nvcc recipe for the in-tree shared library
"""
__version__ = "0.1.0"
