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


def test_ribbons_cards():
    """Ribbon cards: 2,000 cards of 10 x 10 quads = 400,000 triangles; each
    card an open, consistently wound strip with its own uv atlas cell, length
    (arc) 0.5-3% of the scene height; seeded."""
    m = syn.ribbons()
    assert m.face_count == 400_000 and m.vertex_count == 2000 * 121
    assert m.double_sided is not None and m.double_sided[0] == 1
    a = syn.ribbons(50, seed=9)
    assert np.array_equal(a.positions, syn.ribbons(50, seed=9).positions)
    assert not np.array_equal(a.positions, syn.ribbons(50, seed=10).positions)
    f, cnt, dcnt, classes = _edges(a)
    assert (cnt <= 2).all() and (dcnt == 1).all() and (cnt == 1).any()
    tri = a.positions[a.indices.reshape(-1, 3)].astype(np.float64)
    area = np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)
    assert (area > 0).all()
    cards = a.positions.reshape(50, 11, 11, 3).astype(np.float64)
    mid = cards[:, :, 5, :]  # centre line
    arc = np.linalg.norm(np.diff(mid, axis=1), axis=2).sum(1)
    assert (arc > 0.004 * 2.0).all() and (arc < 0.031 * 2.0).all()
    uv = a.uv.reshape(50, 121, 2)
    side = int(np.ceil(np.sqrt(50)))
    cell = np.floor(uv * side).astype(int)
    assert (cell == cell[:, :1, :]).all()  # every card inside one atlas cell
    assert len({tuple(c) for c in cell[:, 0, :]}) == 50


def test_ribbons_oracle_topology():
    """The oracle sees open cards: boundary classes and legal collapses."""
    from oracle.oracle import Oracle

    m = syn.ribbons(3, seed=2)
    O = Oracle()
    geometry, boundary, invalid = O.topology_flags(m)
    assert boundary.any() and not invalid.any()
    assert len(O.actions(m, placement=True, preserve_uv=True)) > 0
