"""Pins the CPU oracle restatement against the reference's own outputs.

The golden fixtures come from the reference's CPU code (tests/golden/make_golden.py);
when oracle/_ref is present the oracle is also compared live with it.
"""
import numpy as np
import pytest

from blitzremesher_b200 import synthetic as syn
from oracle.oracle import BoBounds, BoCamera, BoEdit, BoMeasurement, settings

from conftest import GOLDEN


def _bounds(center, radius):
    b = BoBounds()
    b.center[:] = [float(x) for x in center]
    b.radius = float(radius)
    return b


def test_precision_masks_match_golden(oracle):
    g = np.load(GOLDEN / "precision_masks.npz")
    grid = syn.grid(4)
    b = oracle.bounds(grid)
    assert list(b.center) == list(g["bounds_center"]) and b.radius == float(g["bounds_radius"])
    keys, offsets, words, clipped = g["keys"], g["offsets"], g["words"], g["clipped"]
    cams = {}
    for i, (seed, ss, ci, two, size) in enumerate(keys):
        if seed not in cams:
            cams[seed] = oracle.cameras(b, 17.25, (8, 4, int(seed)))
        w, cl, sz = oracle.rasterize(grid, b, cams[seed][ci], 17.25, int(ss), bool(two))
        assert sz == size
        assert np.array_equal(w, words[offsets[i]:offsets[i + 1]]), (seed, ss, ci, two)
        assert cl == bool(clipped[i])
        tail = (size * size) % 64
        if tail:
            assert (int(w[-1]) >> tail) == 0


def test_precision_special_cases_match_golden(oracle):
    g = np.load(GOLDEN / "precision_masks.npz")
    b = _bounds(g["bounds_center"], g["bounds_radius"])
    for k, name in enumerate(g["special_names"]):
        mesh = syn.Mesh(g[f"{name}_positions"], g[f"{name}_indices"], double_sided=np.array([0], np.uint8))
        cam = BoCamera.from_buffer_copy(g[f"{name}_camera"].tobytes())
        w, cl, _ = oracle.rasterize(mesh, b, cam, 17.25, 2, bool(g["special_two"][k]))
        assert np.array_equal(w, g["special_words"][k]), name
        assert cl == bool(g["special_clipped"][k]), name


def test_precision_distance_matches_golden(oracle):
    g = np.load(GOLDEN / "precision_distance.npz")
    for t in range(g["a"].shape[0]):
        for k, ss in enumerate(g["ss"]):
            assert oracle.coverage_distance(g["a"][t], g["b"][t], 13, 11, int(ss)) == g["expected"][t, k]


def test_distance_empty_and_one(oracle):
    empty = np.zeros(1, np.uint64)
    one = np.ones(1, np.uint64)
    assert oracle.coverage_distance(empty, empty, 1, 1, 1) == 0
    assert np.isinf(oracle.coverage_distance(empty, one, 1, 1, 1))


def _evaluate_cases():
    g = np.load(GOLDEN / "evaluate_cases.npz")
    return g


def test_evaluate_matches_golden(oracle):
    g = _evaluate_cases()
    configs = g["configs"]
    for r, (level, seed, frm, to, ci) in enumerate(g["rows"]):
        pos = g[f"mesh{level}_{seed}_positions"]
        idx = g[f"mesh{level}_{seed}_indices"]
        cand_idx = g[f"cand{level}_{seed}_{frm}_{to}"]
        mesh, cand = syn.Mesh(pos, idx), syn.Mesh(pos, cand_idx)
        b = oracle.bounds(mesh)
        c = configs[ci]
        s = settings(c[0], c[1], (int(c[2]), int(c[3]), int(c[4])), int(c[5]), int(c[6]), c[7], False, bool(c[8]))
        m = oracle.evaluate(mesh, cand, b, s)
        assert bytes(m) == g[f"meas_{r}"].tobytes(), (r, m.as_dict(),
                                                     BoMeasurement.from_buffer_copy(g[f"meas_{r}"].tobytes()).as_dict())


def test_endpoint_actions_match_golden(oracle):
    g = np.load(GOLDEN / "actions.npz")
    cases = {"actions2_1": syn.noisy_icosphere(2, 1), "actions3_2": syn.noisy_icosphere(3, 2),
             "actions_grid6": syn.grid(6)}
    for key, mesh in cases.items():
        mine = np.array([(e.from_, e.to) for e in oracle.actions(mesh, placement=False)], np.uint32).reshape(-1, 2)
        assert np.array_equal(mine, g[key]), key


def test_bounded_refinement(oracle):
    # graph.cpp:5-18 — 520^2 * 16^2 exceeds 64M samples, 8 fits.
    assert oracle.bounded_refinement(512.0, 8, 32) == 8
    assert oracle.bounded_refinement(24.0, 1, 32) == 32
    assert oracle.bounded_refinement(1024.0, 4, 32) == 4


def test_schedule_matches_reference_semantics(oracle):
    p, t, s = oracle.schedule(1024.0, 32.0, 6, [(0, 1), (1, 3)], 2.0)
    assert np.allclose(p, 1024.0 * (32.0 / 1024.0) ** (np.arange(6) / 5.0))
    assert list(t[1:]) == [1.0, 1.5, 2.0, 2.5, 3.0]
    assert s[1] == 1.0 and all(s[1:] <= 2.0)


@pytest.mark.parametrize("level", [2, 3])
def test_oracle_matches_reference_live(oracle, reference, level):
    mesh = syn.noisy_icosphere(level, 7)
    bo, br = oracle.bounds(mesh), reference.bounds(mesh)
    assert bytes(bo) == bytes(br)
    co = oracle.cameras(bo, 24.0, (6, 6, 0xB1172026))
    cr = reference.cameras(br, 24.0, (6, 6, 0xB1172026))
    assert all(bytes(a) == bytes(b) for a, b in zip(co, cr))
    for cam in co:
        for ss in (1, 4):
            for two in (False, True):
                wo, clo, _ = oracle.rasterize(mesh, bo, cam, 24.0, ss, two)
                wr, clr, _ = reference.rasterize(mesh, bo, cam, 24.0, ss, two)
                assert np.array_equal(wo, wr) and clo == clr
    acts = reference.actions(mesh)
    mine = np.array([(e.from_, e.to) for e in oracle.actions(mesh, placement=False)], np.uint32).reshape(-1, 2)
    assert np.array_equal(mine, acts)
    s = settings(24.0, 1.0, (6, 6, 3), 2, 8, 0.5)
    for frm, to in acts[:: max(1, len(acts) // 5)]:
        idx = reference.trial_endpoint(mesh, int(frm), int(to))
        cand = syn.Mesh(mesh.positions, idx)
        assert bytes(oracle.evaluate(mesh, cand, bo, s)) == bytes(reference.evaluate(mesh, cand, bo, s))


def test_midpoint_trial_properties(oracle):
    """Midpoint placement: every slot of class `to` moves to fl(a+b)*0.5, faces
    containing both classes disappear, face order is preserved."""
    mesh = syn.noisy_icosphere(2, 3)
    edits = oracle.actions(mesh, placement=True)
    assert len(edits) > 0
    for e in edits[:: max(1, len(edits) // 7)]:
        idx, pos, _, valid = oracle.trial_midpoint(mesh, e)
        a, b = mesh.positions[e.from_], mesh.positions[e.to]
        mid = ((a + b).astype(np.float32) * np.float32(0.5)).astype(np.float32)
        assert np.array_equal(pos[e.to], mid)
        assert idx.size // 3 == mesh.face_count - e.removed
        assert not np.any(idx == e.from_)


def test_oracle_matches_reference_live_ribbons(oracle, reference):
    """Two-sided open cards (the ribbon workload's mesh): bounds, cameras,
    masks (the mesh's own double-sided flag and forced two-sided), action sets
    and evaluate Measurements of endpoint trials equal the reference's."""
    mesh = syn.ribbons(40, seed=6)
    bo, br = oracle.bounds(mesh), reference.bounds(mesh)
    assert bytes(bo) == bytes(br)
    co = oracle.cameras(bo, 48.0, (5, 3, 0xB1172026))
    cr = reference.cameras(br, 48.0, (5, 3, 0xB1172026))
    assert all(bytes(a) == bytes(b) for a, b in zip(co, cr))
    covered = 0
    for cam in co:
        for ss in (1, 4):
            for two in (False, True):
                wo, clo, _ = oracle.rasterize(mesh, bo, cam, 48.0, ss, two)
                wr, clr, _ = reference.rasterize(mesh, bo, cam, 48.0, ss, two)
                assert np.array_equal(wo, wr) and clo == clr
                covered += int(np.unpackbits(wo.view(np.uint8)).sum())
    assert covered > 0
    acts = reference.actions(mesh)
    mine = np.array([(e.from_, e.to) for e in oracle.actions(mesh, placement=False)], np.uint32).reshape(-1, 2)
    assert len(acts) > 0 and np.array_equal(mine, acts)
    s = settings(48.0, 1.0, (5, 3, 3), 2, 8, 0.5)
    for frm, to in acts[:: max(1, len(acts) // 6)]:
        idx = reference.trial_endpoint(mesh, int(frm), int(to))
        cand = syn.Mesh(mesh.positions, idx, double_sided=mesh.double_sided)
        assert bytes(oracle.evaluate(mesh, cand, bo, s)) == bytes(reference.evaluate(mesh, cand, bo, s))


@pytest.mark.parametrize("level,seed,screen,limit,batch,budget", [
    (2, 1, 24.0, 1.0, 1, 120), (2, 3, 24.0, 0.6, 8, 100), (3, 2, 24.0, 1.0, 64, 40), (3, 5, 48.0, 0.5, 16, 60)])
def test_endpoint_walk_matches_reference_executor(oracle, reference, level, seed, screen, limit, batch, budget):
    """The oracle's executor walk (rank, disjoint batches, halving on
    rejection, stop reasons), run over endpoint collapses, equals the
    reference's own neural::execute_actions (action.cpp:453-525) with the same
    ShortestEdge ranking and four blitz::evaluate gates: trial count, accepted
    collapses, stop reason and final indices. The GPU executor is compared
    with the same walk over midpoint collapses (tests/test_gpu_executor.py)."""
    mesh = syn.noisy_icosphere(level, seed)
    views = (8, 0, 0xB1172026)
    gates = [settings(screen, 2.0, views, 4, 8, 1.0), settings(screen, limit, views, 4, 8, 1.0),
             settings(screen, 2.0, views, 8, 8, 0.5), settings(screen, limit, views, 8, 8, 0.5)]
    mine = oracle.execute_endpoint(mesh, mesh.face_count // 2, budget, gates, batch)
    ref = reference.execute_actions(mesh, mesh.face_count // 2, budget, gates, batch)
    assert mine["trials"] == ref["trials"] and len(mine["commits"]) == ref["accepted"]
    assert mine["stop"] == ref["stop"]
    assert np.array_equal(mine["indices"], ref["indices"])
    assert ref["accepted"] > 0


PLACEMENT_GOLDEN = GOLDEN / "placement_ref.npz"


@pytest.mark.skipif(not PLACEMENT_GOLDEN.exists(), reason="reference placement fixture absent")
def test_midpoint_trials_match_reference_gpu_placement(oracle):
    """The oracle's midpoint trial (placement, uv transport, validate_placement)
    equals the reference's own GPU path (GpuActionState::trial,
    action_gpu.cu:962-1156, run on a B200 by tests/golden/make_placement_golden.py)
    trial for trial: validity, indices, and every moved slot's position and uv
    bit for bit, on seamed meshes, a rock with 8 uv charts and ribbon cards,
    with and without preserve_uv."""
    import hashlib
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_placement_golden", GOLDEN / "make_placement_golden.py")
    maker = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(maker)
    cases = maker.cases

    g = np.load(PLACEMENT_GOLDEN)
    checked = invalid = 0
    for name, mesh, preserve in cases():
        key = f"{name}_uv{preserve}"
        at = 0
        for row, (frm, to) in enumerate(g[f"{key}_from_to"]):
            e = BoEdit()
            e.from_, e.to = int(frm), int(to)
            idx, pos, uv, valid = oracle.trial_midpoint(mesh, e, preserve_uv=bool(preserve))
            assert int(valid) == int(g[f"{key}_valid"][row]), (key, frm, to)
            if not valid:
                invalid += 1
                continue
            n = int(g[f"{key}_count"][row])
            slots = g[f"{key}_slots"][at:at + n]
            assert idx.size // 3 == g[f"{key}_faces"][row]
            assert hashlib.sha256(idx.astype(np.uint32).tobytes()).hexdigest()[:32] == g[f"{key}_sha"][row]
            moved = np.any(pos.view(np.uint32) != mesh.positions.view(np.uint32), axis=1)
            if mesh.uv is not None:
                moved |= np.any(uv.view(np.uint32) != mesh.uv.view(np.uint32), axis=1)
            assert np.array_equal(np.nonzero(moved)[0], slots), (key, frm, to)
            assert np.array_equal(pos[slots].view(np.uint32), g[f"{key}_positions"][at:at + n].view(np.uint32))
            if mesh.uv is not None:
                assert np.array_equal(uv[slots].view(np.uint32), g[f"{key}_uv"][at:at + n].view(np.uint32))
            at += n
            checked += 1
    assert checked > 200 and invalid > 0
