"""fiber3d_b200 — the hydrodynamic hot path of fiber3d on one NVIDIA B200.

Modules
  kernels       drop-in replacement of fiber3d's ``kernels.kernels`` (all its
                functions, same names and signatures), running hand-written
                sm_100a CUDA through the C ABI of include/fiber3d_b200.h
  _lib          ctypes binding of that C ABI, workspaces, the device error word
  autotune      launch-shape tuner of the pair kernels (cached per GPU)
  hydro         the time step's linear system on the device: RHS, matvec,
                block preconditioner, advance, grid velocity
  gmres         right-preconditioned restarted GMRES on the device, FP64 and
                mixed precision with iterative refinement
  blocklu       batched block factorisations / inverses of the fiber blocks
  fibers        fiber resolutions (finite differences, barycentric matrices)
  warmstart     GMRES initial guess: extrapolation + learned per-fiber correction
  flowstart     the (positions, background velocity) -> (tensions, forces)
                network form of the learned guess
  fmm           GPU fast multipole method for the Stokes single and double
                layer (fiber3d's useFMM path): operators and the device handle
  stkfmm        STKFMM's Python API, as fiber3d calls it, over fmm
  quadrature    drop-in for fiber3d's RBF surface quadrature
  output        fiber3d's output and restart files
  tstep_bridge  solver-level drop-in for fiber3d's tstep (GMRES on the device)
  geometry      seeded synthetic geometry (Fibonacci sphere, fibers, problems)
  replicas      multi-process bookkeeping (barrier, max over ranks)
  build         nvcc recipe for the in-tree shared library
"""
__version__ = "0.2.0"
