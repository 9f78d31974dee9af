"""CPU FP64 oracle for the YASPS Newton inner loop.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library imports, links or
executes this package: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` use it, and only
as the checker (or as the timed CPU restatement of the reference), never as
the thing the product computes with.

The package restates, in plain NumPy, the algorithms of the reference
(txstc55/yasps) on the hot path.  Every function cites the reference file and
line it follows; paths are relative to the reference project root, ``PKG``
meaning ``yasps/yasps``.

Parity pins (see ``tests/test_oracle_golden.py``):

* element math: the reference's own float64 PyTorch SNH formulation
  (``examples/backup/pytorch_energy_hessian_and_gradient/stable_neo_hookean.py``)
  and its SymPy check script (``tests/energy/check_stable_neo_hookean.py``),
  both executed in the development container to produce committed fixtures;
* MAS preconditioned CG: the reference's NumPy MAS path
  (``PKG/solver/mas``) run in the development container with the
  chunk-ordering shim described in ``oracle/mas.py``;
* assembly / SpMV / solver: the dense known-answer cases of
  ``tests/differentiator/test_hessian_sparsity_permutation_gpu.py``,
  restated in ``tests/test_oracle_kat.py``.

The eigen-projection follows the reference's published rule (LDL^T PSD
short-circuit, then eigen-decomposition with |lambda| or max(lambda, 0));
the reference delegates the eigen-solve to Eigen's SelfAdjointEigenSolver
(third-party, not vendored, version unpinned), so the oracle uses LAPACK
``eigh`` for it.  The decision rule itself is reproduced operation by
operation.
"""
