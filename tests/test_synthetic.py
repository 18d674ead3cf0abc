"""The batched-audit mesh set: seeded, sized as asked, 4-16 UV charts whose
seams duplicate vertices, and 2-manifold with consistent orientation (closed
spheres and tori, heightfields open only at their border)."""
import numpy as np

from blitzremesher_b200 import synthetic as syn


def _edges(m):
    _, inv = np.unique(m.positions.view(np.dtype((np.void, 12))), return_inverse=True)
    f = inv.reshape(-1)[m.indices.reshape(-1, 3)]
    und = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), 1)
    _, cnt = np.unique(und, axis=0, return_counts=True)
    d = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    _, dcnt = np.unique(d, axis=0, return_counts=True)
    return f, cnt, dcnt, int(inv.max() + 1)


def test_generators_are_manifold_with_seams():
    for m, closed in [(syn.seamed_sphere(3000, 5), True), (syn.seamed_torus(3000, 6, 8), True),
                      (syn.seamed_heightfield(3000, 7, 9), False)]:
        f, cnt, dcnt, classes = _edges(m)
        assert 2500 < m.face_count < 3500
        assert (cnt <= 2).all() and (dcnt == 1).all()
        assert (cnt == 1).any() != closed
        assert not ((f[:, 0] == f[:, 1]) | (f[:, 1] == f[:, 2]) | (f[:, 0] == f[:, 2])).any()
        assert classes < m.vertex_count  # seams duplicate vertices
        assert m.uv.dtype == np.float32 and m.uv.shape == (m.vertex_count, 2)
        assert 4 <= m.meta["charts"] <= 16


def test_batched_set_is_seeded_and_log_uniform():
    a = syn.batched_set(12, seed=3)
    b = syn.batched_set(12, seed=3)
    assert all(np.array_equal(x.positions, y.positions) and np.array_equal(x.indices, y.indices)
               for x, y in zip(a, b))
    faces = [m.face_count for m in a]
    assert min(faces) >= 1500 and max(faces) <= 230000
    assert [m.meta["kind"] for m in a[:3]] == ["sphere", "torus", "heightfield"]
