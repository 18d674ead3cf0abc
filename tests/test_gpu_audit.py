"""GPU parity of the CUDA audit path against the oracle and the golden fixtures.

Bit-exact bar: coverage masks, Measurements (every field), legal action sets
and four-gate verdicts equal the reference CPU semantics on the same inputs.
"""
import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn
from oracle.oracle import BoEdit, BoMeasurement, settings as oracle_settings

from conftest import GOLDEN, measurement_fields

pytestmark = pytest.mark.gpu


def _gpu_settings(cfg):
    screen, limit, ortho, persp, seed, ss, mss, area, cons = cfg
    return br.eval_settings(screen, limit, (int(ortho), int(persp), int(seed)), int(ss), int(mss), area, False,
                            bool(cons))


def test_raster_masks_match_golden(gpu_lib):
    g = np.load(GOLDEN / "precision_masks.npz")
    grid = syn.grid(4)
    with br.AuditSession(grid) as s:
        for i, (seed, ss, ci, two, size) in enumerate(g["keys"]):
            w, cl, sz = s.rasterize(grid, 17.25, int(ss), (8, 4, int(seed)), int(ci), bool(two))
            assert sz == size
            assert np.array_equal(w, g["words"][g["offsets"][i]:g["offsets"][i + 1]]), (seed, ss, ci, two)
            assert cl == bool(g["clipped"][i])


def test_raster_masks_match_oracle_icosphere(gpu_lib, oracle):
    mesh = syn.noisy_icosphere(4, 5)
    b = oracle.bounds(mesh)
    cams = oracle.cameras(b, 24.0, (8, 8, 11))
    with br.AuditSession(mesh) as s:
        for v, cam in enumerate(cams):
            for ss in (1, 3, 8):
                for two in (False, True):
                    w, cl, _ = s.rasterize(mesh, 24.0, ss, (8, 8, 11), v, two)
                    wo, clo, _ = oracle.rasterize(mesh, b, cam, 24.0, ss, two)
                    assert np.array_equal(w, wo) and cl == clo, (v, ss, two)


def test_coverage_distance_matches_golden(gpu_lib):
    """The 40 random 13x11 mask pairs of the reference precision test."""
    g = np.load(GOLDEN / "precision_distance.npz")
    with br.AuditSession(syn.noisy_icosphere(1, 1)) as s:
        for t in range(g["a"].shape[0]):
            for k, ss in enumerate(g["ss"]):
                assert s.coverage_distance(g["a"][t], g["b"][t], 13, 11, int(ss)) == g["expected"][t, k], (t, ss)
        empty, one = np.zeros(1, np.uint64), np.ones(1, np.uint64)
        assert s.coverage_distance(empty, empty, 1, 1, 1) == 0
        assert np.isinf(s.coverage_distance(empty, one, 1, 1, 1))


def _blob_mask(rng, width, height, blobs):
    yy, xx = np.mgrid[0:height, 0:width]
    m = np.zeros((height, width), bool)
    for _ in range(blobs):
        cx, cy, r = rng.uniform(0, width), rng.uniform(0, height), rng.uniform(2, width / 6)
        m |= (xx - cx) ** 2 + (yy - cy) ** 2 < r * r
    bits = np.packbits(m.reshape(-1), bitorder="little")
    bits = np.concatenate([bits, np.zeros((-bits.size) % 8, np.uint8)])
    return bits.view(np.uint64)


def test_coverage_distance_matches_oracle_random(gpu_lib, oracle):
    rng = np.random.default_rng(11)
    with br.AuditSession(syn.noisy_icosphere(1, 1)) as s:
        for width, height in ((257, 190), (64, 64), (1000, 37), (129, 600)):
            for trial in range(3):
                a = _blob_mask(rng, width, height, 3)
                b = _blob_mask(rng, width, height, 2 + trial)
                for ss in (1, 3):
                    want = oracle.coverage_distance(a, b, width, height, ss)
                    assert s.coverage_distance(a, b, width, height, ss) == want, (width, height, trial, ss)


def test_evaluate_matches_golden(gpu_lib):
    g = np.load(GOLDEN / "evaluate_cases.npz")
    sessions = {}
    for r, (level, seed, frm, to, ci) in enumerate(g["rows"]):
        key = (int(level), int(seed))
        mesh = syn.Mesh(g[f"mesh{level}_{seed}_positions"], g[f"mesh{level}_{seed}_indices"])
        if key not in sessions:
            sessions[key] = br.AuditSession(mesh)
        cand = syn.Mesh(mesh.positions, g[f"cand{level}_{seed}_{frm}_{to}"])
        m = sessions[key].evaluate(mesh, cand, _gpu_settings(g["configs"][ci]))
        want = BoMeasurement.from_buffer_copy(g[f"meas_{r}"].tobytes())
        assert measurement_fields(m) == measurement_fields(want), (r, m.as_dict(), want.as_dict())
    for s in sessions.values():
        s.close()


def test_evaluate_identical_and_empty(gpu_lib, oracle):
    mesh = syn.noisy_icosphere(2, 9)
    s = br.eval_settings(24.0, 1.0, (4, 2, 1), 2, 8)
    with br.AuditSession(mesh) as sess:
        m = sess.evaluate(mesh, mesh, s)
        assert m.passed == 1 and m.views_evaluated == 0
        # Candidate moved far away: one view sees nothing of it -> infinite error.
        moved = mesh.copy()
        moved.positions = moved.positions + np.float32(0.5)
        b = oracle.bounds(mesh)
        want = oracle.evaluate(mesh, moved, b, oracle_settings(24.0, 1.0, (4, 2, 1), 2, 8))
        got = sess.evaluate(mesh, moved, s)
        assert measurement_fields(got) == measurement_fields(want)


@pytest.mark.parametrize("case", ["sphere2", "sphere3", "grid6", "sphere5"])
def test_actions_match_oracle(gpu_lib, oracle, case):
    mesh = {"sphere2": lambda: syn.noisy_icosphere(2, 1), "sphere3": lambda: syn.noisy_icosphere(3, 2),
            "grid6": lambda: syn.grid(6), "sphere5": syn.config1_mesh}[case]()
    mesh.uv = None
    want = np.array([(e.from_, e.to) for e in oracle.actions(mesh, placement=True)], np.uint32).reshape(-1, 2)
    with br.AuditSession(mesh) as s:
        got = s.actions()
    assert np.array_equal(np.stack([got["from"], got["to"]], 1), want)


def _oracle_verdict(oracle, mesh, frm, to, b, gates_o):
    e = BoEdit()
    e.from_, e.to = int(frm), int(to)
    return oracle.audit_candidate(mesh, e, mesh, mesh, b, gates_o)


def _check_candidates(oracle, mesh, gates_args, picks=None):
    b = oracle.bounds(mesh)
    gates_o = [oracle_settings(*a) for a in gates_args]
    gates_g = [br.eval_settings(*a) for a in gates_args]
    with br.AuditSession(mesh) as s:
        acts = s.actions()
        cands = br.midpoint_collapses(acts)
        if picks is not None:
            cands = cands[picks]
        verdicts, meas = s.candidates(cands, gates_g, measurements=True)
    accepted = 0
    for i, c in enumerate(cands):
        want = _oracle_verdict(oracle, mesh, c["from"], c["to"], b, gates_o)
        v = verdicts[i]
        assert v["accepted"] == want.accepted, (i, c, v, want.failed_gate)
        assert v["failed_gate"] == want.failed_gate, (i, c, v)
        stop = 4 if want.failed_gate == 0 else (want.failed_gate if want.failed_gate <= 4 else 0)
        for gi in range(stop):
            got = meas[i, gi]
            assert measurement_fields(got) == measurement_fields(want.gates[gi]), (
                i, gi, {k: got[k].item() for k in got.dtype.names if k != "reserved"},
                                                  want.gates[gi].as_dict())
        accepted += int(v["accepted"])
    return accepted, len(cands)


def test_candidates_match_oracle_small(gpu_lib, oracle):
    mesh = syn.noisy_icosphere(3, 4)
    views = (12, 4, 0xB1172026)
    gates = [(24.0, 2.0, views, 8, 8, 1.0), (24.0, 1.0, views, 8, 8, 1.0),
             (24.0, 2.0, views, 8, 8, 0.2), (24.0, 1.0, views, 8, 8, 0.2)]
    accepted, n = _check_candidates(oracle, mesh, gates)
    assert n > 0


def test_candidates_match_oracle_refinement(gpu_lib, oracle):
    """Search gates at ss 2 refine up to 8 through the exact path."""
    mesh = syn.noisy_icosphere(2, 6)
    views = (6, 2, 77)
    gates = [(16.0, 1.5, views, 2, 8, 1.0), (16.0, 1.0, views, 2, 8, 1.0),
             (16.0, 1.5, views, 4, 8, 0.3), (16.0, 1.0, views, 4, 8, 0.3)]
    _check_candidates(oracle, mesh, gates)


def test_candidates_match_oracle_config1_sample(gpu_lib, oracle):
    mesh = syn.config1_mesh()
    views = (32, 0, 0xB1172026)
    gates = [(24.0, 2.0, views, 8, 8, 1.0), (24.0, 1.0, views, 8, 8, 1.0),
             (24.0, 2.0, views, 8, 8, 1.0), (24.0, 1.0, views, 8, 8, 1.0)]
    with br.AuditSession(mesh) as s:
        n = s.actions().size
    picks = np.linspace(0, n - 1, 16).astype(int)
    _check_candidates(oracle, mesh, gates, picks)


def test_candidates_config1_all_deterministic(gpu_lib):
    mesh = syn.config1_mesh()
    views = (32, 0, 0xB1172026)
    gates = [br.eval_settings(24.0, 2.0, views), br.eval_settings(24.0, 1.0, views),
             br.eval_settings(24.0, 2.0, views), br.eval_settings(24.0, 1.0, views)]
    with br.AuditSession(mesh) as s:
        cands = br.midpoint_collapses(s.actions())
        v1 = s.candidates(cands, gates)
        v2 = s.candidates(cands, gates)
    assert cands.size > 50000
    assert np.array_equal(v1, v2)
    assert set(np.unique(v1["failed_gate"])) <= {0, 1, 2, 3, 4, 6}
    assert (v1["accepted"] == (v1["failed_gate"] == 0)).all()
