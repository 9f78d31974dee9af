"""Vertex-tuple energies (barriers, bending, membranes, friction) on the GPU
against the oracle, through the public scene API and the C ABI.

Tolerances: pattern and lookups bit-exact; FP64 gradient and projected
Hessian 1e-12 relative to the largest magnitude; solves at the stated true
relative residual.
"""

import numpy as np
import pytest

from oracle import solvers
from oracle import pattern as opattern
from tests.vertex_scene import VertexScene

pytestmark = pytest.mark.gpu


def rel(a, b):
  a, b = np.asarray(a), np.asarray(b)
  return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("membrane", ["baraff_witkin", "stvk"])
@pytest.mark.parametrize("method", [1, 2, 0])
def test_assembly_matches_oracle(membrane, method):
  vs = VertexScene(m=6, seed=3, membrane=membrane)
  sc = vs.build(projection_method=method)
  H = sc.minimizer.computeNumericValue()
  pat, values, grad = vs.oracle_assembly(projection_method=method)
  pos = H.block_positions.cpu().numpy().astype(np.int64).reshape(-1, 2)
  assert np.array_equal(pos, pat.positions)
  assert rel(H.gradient.value.cpu().numpy(), grad) <= 1e-12
  assert rel(H.blocks_flattened.cpu().numpy()[:values.size], values) <= 1e-12


def test_projection_changes_indefinite_terms():
  vs = VertexScene(m=6, seed=4)
  _, v_proj, _ = vs.oracle_assembly(projection_method=1)
  _, v_raw, _ = vs.oracle_assembly(projection_method=0)
  assert rel(v_proj, v_raw) > 1e-6, "the scene must exercise the projection"


def test_cloth_contact_solve():
  vs = VertexScene(m=8, seed=5)
  sc = vs.build(projection_method=1)
  sc.minimizer.setSolver("mas", stop_rule="residual")
  segs = sc.minimizeEnergy(tolerance=1e-8, maxIterations=2000)
  x = segs[0].cpu().numpy()
  pat, values, grad = vs.oracle_assembly(projection_method=1)
  matvec = lambda v: opattern.spmv(pat, values, v)
  assert solvers.relative_residual(matvec, grad, x) <= 1e-8
