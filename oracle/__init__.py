"""CPU oracle for the fiber3d hydrodynamic hot path — TEST INFRASTRUCTURE ONLY.

This package restates, on the CPU, the algorithms of fiber3d's
``python/kernels/kernels.py`` and of the solver pieces that call them
(periphery operator, fiber operators, block preconditioner, GMRES matvec).
It is the checker the GPU path is compared against, and the timed CPU
baseline of ``bench.py``.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference arm may import it; the product
package ``fiber3d_b200`` never does.

Parity pin: the restatements are checked against golden vectors produced by
running fiber3d's own code (``tests/golden/make_golden.py``) — see
``tests/test_oracle_golden.py``.
"""
