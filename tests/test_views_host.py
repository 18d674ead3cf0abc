"""The library's host-side view set (blitz_mesh_bounds, blitz_view_cameras:
the bounds and cameras every audit projects with) against the oracle and,
when built, the reference's own blitz::bounds / blitz::cameras
(oracle/_ref): bit for bit, field by field. CPU only."""
import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn

MESHES = {
    "icosphere": lambda: syn.noisy_icosphere(3, 7),
    "seamed_sphere": lambda: syn.seamed_sphere(3000, 5),
    "rock": lambda: syn.rock(3, 3),
    "grid": lambda: syn.grid(8, scale=0.37, bend=0.2),
    "ribbons": lambda: syn.ribbons(20, seed=4),
}
VIEW_SETS = [(24.0, (32, 0, 0xB1172026)), (512.0, (6, 6, 0xB1172024)), (100.5, (0, 5, 1)), (7.5, (64, 0, 77))]


def _same_camera(mine, other) -> bool:
    f32 = lambda v: np.asarray(list(v), np.float32).tobytes()
    return (f32(mine.right) == f32(other.right) and f32(mine.up) == f32(other.up)
            and f32(mine.forward) == f32(other.forward)
            and np.float64(mine.distance).tobytes() == np.float64(other.distance).tobytes()
            and np.float64(mine.focal).tobytes() == np.float64(other.focal).tobytes()
            and np.float64(mine.scale).tobytes() == np.float64(other.scale).tobytes()
            and int(mine.perspective) == int(other.perspective))


def _check(ref_like, name):
    mesh = MESHES[name]()
    center, radius = br.mesh_bounds(mesh)
    b = ref_like.bounds(mesh)
    assert np.asarray(list(b.center), np.float32).tobytes() == center.tobytes()
    assert np.float64(b.radius).tobytes() == np.float64(radius).tobytes()
    for screen, views in VIEW_SETS:
        mine = br.view_cameras(center, radius, screen, views)
        other = ref_like.cameras(b, screen, views)
        assert len(mine) == len(other) == views[0] + views[1]
        assert all(_same_camera(m, o) for m, o in zip(mine, other)), (name, screen, views)


@pytest.mark.parametrize("name", sorted(MESHES))
def test_views_match_oracle(oracle, name):
    _check(oracle, name)


@pytest.mark.parametrize("name", ["icosphere", "rock"])
def test_views_match_reference(reference, name):
    _check(reference, name)


def test_view_cameras_reject_bad_arguments():
    with pytest.raises(br.BlitzError):
        br.view_cameras(np.zeros(3, np.float32), 0.0, 24.0, (4, 0, 1))
