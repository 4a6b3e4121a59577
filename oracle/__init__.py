"""CPU oracle for the SpinFEMx demag + LLG hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports, links or
executes this package: it is the checker.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it.

Every function restates the reference algorithm in plain numpy/scipy and
cites the reference file:line (paths relative to the reference project root,
``src/spinfemx/...``) it follows.

Pinning status (how each part was checked against the reference itself):

* Lindholm weights, solid angle, dense B entries, cluster tree, block
  partition, full-pivot ACA and the CPU H-matrix matvec: pinned against the
  reference's own numba/numpy code, imported in the fixture generator
  ``tests/golden/make_golden.py`` and stored as ``tests/golden/*.npz``.
* LLG RHS, Jv, 3x3 block preconditioner and nodal anisotropy: pinned against
  the reference's CUDA-C ElementwiseKernel bodies and the CPU numba Jv kernel,
  extracted from the reference sources as text, compiled with gcc / numba by
  the same generator, and stored as fixtures.
* P1 FEM operators (DOLFINx forms) and the exact FP64 Poisson solves:
  DOLFINx/PETSc are absent here, so these are pinned by known answers only
  (zero row sums, exact gradients of linear fields, B.1 = -1, demag of a
  uniformly magnetised film and of a cube).  Parity for these parts is
  "pinned by known answers", not by reference outputs.
"""
