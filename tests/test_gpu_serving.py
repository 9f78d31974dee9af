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


def test_mixed_stream_of_cloth_scenes_and_fem_cubes():
  """The mixed serving form at small size: cloth + affine-body + contact
  scenes (their own topologies) interleaved with FEM cubes, served together;
  every result meets the residual of its FP64 oracle system and is
  bit-identical to the same request served alone."""
  from oracle import cloth_scene
  wl = serving.mixed_workload(num_scenes=3, num_fem=2, fem_side=10, side_range=(20, 28), body_range=(1, 3),
                              pair_range=(300, 900), fem_young=1e6, fem_poisson=0.45, fem_noise=0.005,
                              mean_spacing=5e-4, seed=7)
  srv = serving.NewtonServer(max_slots=8, passes=4, memory_budget=4e9, max_iterations=5000)
  try:
    for spec in wl.scenes:
      srv.add_topology(serving.cloth_scene_topology(spec))
    srv.register([s.key for s in wl.scenes] + [wl.fem_side], slots_per_side=1)
    alone = {}
    for r in wl.requests(srv):
      (d,) = srv.run([r])
      alone[d.tag] = d.solution
    done = srv.run(wl.requests(srv))
    assert len(done) == len(wl.order)
    for r in done:
      assert r.converged, (r.tag, r.phase)
      assert np.array_equal(r.solution, alone[r.tag]), r.tag
      kind, i = wl.order[r.tag]
      if kind == "cloth":
        cc = srv.topology(wl.scenes[i].key).cloth
        assert cloth_scene.relative_residual(cc, r.solution) <= 1e-6
      else:
        f = wl.fem[i]
        case = (wl.fem_side, f["young"], f["poisson"], f["noise"], f["seed"])
        assert oracle_residual(case, r.solution) <= 1e-6
  finally:
    srv.close()
