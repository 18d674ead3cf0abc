"""Generates the golden fixtures in this folder from the reference itself.

Run in a container that has the reference sources (oracle/Makefile compiles
them into oracle/_ref/libblitz_ref.so):

    python tests/golden/make_golden.py

Fixtures (all produced by the reference's own CPU code):
  precision_masks.npz   packed coverage masks of the grid fixture of the
                        reference test tests/precision.cpp:61-81 (cameras,
                        culling, zero-area faces, clipping, behind-camera)
  precision_distance.npz the 40 random 13x11 mask pairs of
                        tests/precision.cpp:82-91 with coverage_distance
  evaluate_cases.npz    blitz::evaluate Measurements for endpoint-collapse
                        candidates of small noisy icospheres under varied
                        settings (orthographic and perspective views,
                        refinement, area gate, conservative screen)
  actions.npz           the reference CPU executor's legal action set
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from blitzremesher_b200 import synthetic as syn  # noqa: E402
from oracle.oracle import BoMeasurement, Reference, build, settings  # noqa: E402

OUT = Path(__file__).resolve().parent


def measurement_row(m: BoMeasurement) -> np.ndarray:
    return np.frombuffer(bytes(m), dtype=np.uint8).copy()


def precision_masks(R: Reference) -> None:
    grid = syn.grid(4)
    b = R.bounds(grid)
    keys, words, clipped = [], [], []
    for seed in (17, 9381):
        for ss in (1, 2, 4, 8):
            cams = R.cameras(b, 17.25, (8, 4, seed))
            for ci, cam in enumerate(cams):
                for two in (0, 1):
                    w, cl, size = R.rasterize(grid, b, cam, 17.25, ss, bool(two))
                    keys.append((seed, ss, ci, two, size))
                    words.append(w)
                    clipped.append(cl)
    # Special cases of precision.cpp:70-81 on the same grid.
    special = syn.grid(4, two_sided=False)
    special.indices = np.concatenate([special.indices, np.zeros(3, np.uint32)])
    cam = R.cameras(b, 17.25, (1, 1, 99))[-1]
    cases = []
    s1 = special.copy()
    s1.positions[:, 2] += np.float32(0.00001)
    cases.append(("zero_area_culled", s1, cam, False))
    s2 = s1.copy()
    s2.positions[:, 0] += np.float32(100)
    cases.append(("offscreen_clip", s2, cam, True))
    cam3 = R.cameras(b, 17.25, (1, 1, 99))[-1]
    cam3.distance = -100.0
    cases.append(("behind_camera", s2, cam3, True))
    special_words, special_clipped, special_meshes = [], [], {}
    for name, mesh, c, two in cases:
        w, cl, size = R.rasterize(mesh, b, c, 17.25, 2, two)
        special_words.append(w)
        special_clipped.append(cl)
        special_meshes[name + "_positions"] = mesh.positions
        special_meshes[name + "_indices"] = mesh.indices
        special_meshes[name + "_camera"] = np.frombuffer(bytes(c), np.uint8)
    np.savez_compressed(OUT / "precision_masks.npz", keys=np.array(keys, np.int64),
                        offsets=np.cumsum([0] + [w.size for w in words]), words=np.concatenate(words),
                        clipped=np.array(clipped, np.uint8), special_names=np.array([c[0] for c in cases]),
                        special_two=np.array([c[3] for c in cases], np.uint8),
                        special_words=np.stack(special_words), special_clipped=np.array(special_clipped, np.uint8),
                        bounds_center=np.array(list(b.center), np.float32), bounds_radius=np.float64(b.radius),
                        **special_meshes)


def precision_distance(R: Reference) -> None:
    a, b = R.precision_masks(2921, 40)
    expected = np.zeros((40, 3))
    for t in range(40):
        for k, ss in enumerate((1, 2, 8)):
            expected[t, k] = R.coverage_distance(a[t], b[t], 13, 11, ss)
            assert expected[t, k] == R.coverage_distance(a[t], b[t], 13, 11, ss, scalar=False)
    np.savez_compressed(OUT / "precision_distance.npz", a=a, b=b, ss=np.array([1, 2, 8]), expected=expected)


def evaluate_cases(R: Reference) -> None:
    rows = []
    meshes = {}
    configs = [
        # screen, limit, (ortho, persp, seed), ss, max_ss, area, conservative
        (24.0, 1.0, (32, 0, 0xB1172026), 8, 8, 1.0, 0),
        (24.0, 2.0, (16, 8, 0xB1172024), 4, 8, 1.0, 0),
        (24.0, 0.5, (8, 4, 7), 2, 16, 0.05, 0),
        (17.25, 1.0, (6, 6, 99), 1, 8, 1.0, 0),
        (40.0, 1.0, (12, 0, 5), 4, 4, 1.0, 1),
    ]
    for level, seed in ((2, 1), (3, 2)):
        mesh = syn.noisy_icosphere(level, seed)
        b = R.bounds(mesh)
        acts = R.actions(mesh)
        picks = np.linspace(0, len(acts) - 1, 6).astype(int)
        meshes[f"mesh{level}_{seed}_positions"] = mesh.positions
        meshes[f"mesh{level}_{seed}_indices"] = mesh.indices
        for p in picks:
            frm, to = (int(x) for x in acts[p])
            idx = R.trial_endpoint(mesh, frm, to)
            key = f"cand{level}_{seed}_{frm}_{to}"
            meshes[key] = idx
            cand = syn.Mesh(mesh.positions, idx)
            for ci, (screen, limit, views, ss, mss, area, cons) in enumerate(configs):
                s = settings(screen, limit, views, ss, mss, area, False, bool(cons))
                m = R.evaluate(mesh, cand, b, s)
                rows.append((level, seed, frm, to, ci))
                meshes[f"meas_{len(rows) - 1}"] = measurement_row(m)
    np.savez_compressed(OUT / "evaluate_cases.npz", rows=np.array(rows, np.int64),
                        configs=np.array([(c[0], c[1], c[2][0], c[2][1], c[2][2], c[3], c[4], c[5], c[6])
                                          for c in configs], np.float64), **meshes)


def actions(R: Reference) -> None:
    out = {}
    for level, seed in ((2, 1), (3, 2)):
        mesh = syn.noisy_icosphere(level, seed)
        out[f"actions{level}_{seed}"] = R.actions(mesh)
    g = syn.grid(6)
    out["actions_grid6"] = R.actions(g)
    np.savez_compressed(OUT / "actions.npz", **out)


def main() -> None:
    build(ref=True)
    R = Reference()
    precision_masks(R)
    precision_distance(R)
    evaluate_cases(R)
    actions(R)
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
