"""The c2 scene's affine bodies and body-cloth pairs, on the CPU.

Icospheres: 10 * 4^s + 2 unit vertices, a closed oriented surface (Euler
characteristic 2, every edge in two faces, outward normals).  Bodies rest
on the cloth: every body-cloth point-triangle pair indexes the union
[cloth, abd, obstacle] correctly and has its squared plane distance inside
(0.1, 1) d-hat; the point-triangle total stays at half the pairs.
"""

import numpy as np
import pytest

from yasps_b200 import scenes


@pytest.mark.parametrize("s", [0, 1, 2, 4])
def test_icosphere_is_a_closed_oriented_unit_sphere(s):
  v, f = scenes.icosphere(s)
  assert v.shape == (10 * 4 ** s + 2, 3) and f.shape == (20 * 4 ** s, 3)
  assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-14)
  e = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
  uniq, counts = np.unique(e, axis=0, return_counts=True)
  assert (counts == 2).all()
  assert len(v) - len(uniq) + len(f) == 2
  n = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
  assert (np.einsum("ij,ij->i", n, v[f].mean(axis=1)) > 0).all()


def test_body_cloth_pairs_lie_in_the_distance_window():
  cc = scenes.cloth_contact(48, 20_000, num_bodies=4, body_subdivisions=3, body_radius=0.3)
  nc, nv = len(cc.cloth_position), len(cc.bodies.rest)
  bp = cc.body_pt.astype(np.int64)
  assert len(bp) > 0
  # exactly one side of each pair is on a body, and it is the point or the whole triangle
  on_body = (bp >= nc) & (bp < nc + nv)
  assert ((on_body[:, 0] & ~on_body[:, 1:].any(axis=1)) | (~on_body[:, 0] & on_body[:, 1:].all(axis=1))).all()
  tri_body = cc.bodies.vertex_body[bp[on_body[:, 1], 1] - nc]
  for k in (2, 3):
    assert (cc.bodies.vertex_body[bp[on_body[:, 1], k] - nc] == tri_body).all()
  x = np.concatenate([cc.cloth_position, cc.bodies.positions()])[bp]
  b = np.cross(x[:, 2] - x[:, 1], x[:, 3] - x[:, 1])
  d = np.einsum("ij,ij->i", x[:, 0] - x[:, 1], b) ** 2 / np.einsum("ij,ij->i", b, b)
  assert (d > 0.1 * cc.dhat).all() and (d < cc.dhat).all()
  assert len(cc.pt) + len(bp) == 10_000 and len(cc.ee) == 10_000
  # the bodies are close to rotations (orthogonality energy near its minimum)
  a = cc.bodies.affine.reshape(-1, 3, 3)
  assert np.abs(np.einsum("bki,bkj->bij", a, a) - np.eye(3)).max() < 5e-3
