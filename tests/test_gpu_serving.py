"""Serving form on the GPU: batched solves against the oracle, and the same
result alone and in a mix.

Tolerances: every served solve meets ||g - H x|| <= 1e-6 ||g|| with g and H
assembled by the oracle in FP64 (the matrices agree with the device's to
1e-12); a request's solution is bit-identical alone and in any mix of other
requests (its CTA partition and reduction order do not depend on the mix).
"""

import numpy as np
import pytest

from oracle import solvers
from tests.oracle_scene import OracleCube
from yasps_b200 import _lib as L
from yasps_b200 import scenes, serving

pytestmark = pytest.mark.gpu

CASES = [(6, 5e4, 0.35, 0.01, 1), (9, 2e5, 0.42, 0.01, 2), (12, 1e4, 0.30, 0.008, 3), (7, 1e6, 0.45, 0.01, 4)]


def oracle_residual(case, x):
  side, young, nu, noise, seed = case
  ora = OracleCube(scenes.fem_cube(side, young=young, poisson=nu, noise=noise, seed=seed))
  return solvers.relative_residual(ora.matvec, ora.gradient, x)


def request(case, arrival=0.0):
  side, young, nu, noise, seed = case
  return serving.fem_request(side, young, nu, noise, seed, arrival=arrival, tag=case)


@pytest.fixture(scope="module")
def server():
  s = serving.NewtonServer(max_slots=8, passes=4, memory_budget=4e9)
  s.register(sorted({c[0] for c in CASES}))
  yield s
  s.close()


def test_served_solves_meet_the_fp64_residual(server):
  done = server.run([request(c) for c in CASES])
  assert len(done) == len(CASES)
  for r in done:
    assert r.converged, (r.tag, r.phase)
    assert r.relative_residual <= 1e-6
    assert oracle_residual(r.tag, r.solution) <= 1e-6


def test_result_is_the_same_alone_and_in_a_mix(server):
  alone = {}
  for c in CASES:
    (r,) = server.run([request(c)])
    alone[c] = r.solution
  # all at once, then staggered arrivals (later requests join solves in flight)
  mixes = [[request(c) for c in CASES],
           [request(c, arrival=0.0005 * k) for k, c in enumerate(reversed(CASES))]]
  for mix in mixes:
    for r in server.run(mix):
      assert r.converged
      assert np.array_equal(r.solution, alone[r.tag]), r.tag


def test_serial_fp64_path_matches_the_residual(server):
  done = server.solve_serial_fp64([request(c) for c in CASES[:2]])
  for r in done:
    assert r.phase == L.YS_SERVE_DONE
    assert oracle_residual(r.tag, r.solution) <= 1e-6


def test_slots_are_reused_and_budget_bounds_residency(server):
  before = server.resident_bytes
  server.run([request(CASES[0]) for _ in range(3)])
  assert server.resident_bytes <= server.memory_budget
  assert server.resident_bytes >= before
  assert server.launches > 0
