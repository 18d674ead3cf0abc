"""uv transport on the candidate path (place_vertices, action_gpu.cu:962-1067)
and the uv flip check of validate_placement (action_gpu.cu:1121-1126) against
the oracle: candidate verdicts, executor commits and the final state's uv,
bit for bit, on seamed meshes whose uv carry per-slot jitter (so that some
midpoint placements fold a uv triangle)."""
import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn
from oracle.oracle import BoEdit, settings as oracle_settings

from conftest import measurement_fields

pytestmark = pytest.mark.gpu


def _jittered(mesh, scale, seed):
    rng = np.random.default_rng(seed)
    mesh.uv = (mesh.uv + rng.uniform(-scale, scale, mesh.uv.shape)).astype(np.float32)
    return mesh


MESHES = {
    "torus": lambda: _jittered(syn.seamed_torus(800, 7, 8, amplitude=0.1), 0.015, 1),
    "sphere": lambda: _jittered(syn.seamed_sphere(600, 5, amplitude=0.15), 0.02, 2),
}


def _gates(screen, views, ss):
    return [(screen, 2.0, views, ss, ss, 1.0), (screen, 1.0, views, ss, ss, 1.0),
            (screen, 2.0, views, ss, ss, 0.5), (screen, 1.0, views, ss, ss, 0.5)]


@pytest.mark.parametrize("preserve_uv", [1, 0])
@pytest.mark.parametrize("name", sorted(MESHES))
def test_uv_candidates_match_oracle(gpu_lib, oracle, name, preserve_uv):
    """Every legal midpoint collapse of the source: verdict and every gate
    Measurement equal the oracle's, with and without the uv flip check."""
    mesh = MESHES[name]()
    args = _gates(24.0, (6, 2, 31), 4)
    b = oracle.bounds(mesh)
    with br.AuditSession(mesh, br.neural_options(preserve_uv=preserve_uv)) as s:
        cands = br.midpoint_collapses(s.actions())
        verdicts, meas = s.candidates(cands, [br.eval_settings(*a) for a in args], measurements=True)
    invalid = 0
    for i, c in enumerate(cands):
        e = BoEdit()
        e.from_, e.to = int(c["from"]), int(c["to"])
        want = oracle.audit_candidate(mesh, e, mesh, mesh, b, [oracle_settings(*a) for a in args],
                                      preserve_uv=bool(preserve_uv))
        assert verdicts[i]["accepted"] == want.accepted and verdicts[i]["failed_gate"] == want.failed_gate, i
        invalid += want.failed_gate == 6
        stop = 4 if want.failed_gate == 0 else (want.failed_gate if want.failed_gate <= 4 else 0)
        for g in range(stop):
            assert measurement_fields(meas[i, g]) == measurement_fields(want.gates[g]), (i, g)
    # The jitter makes the uv flip check reject placements; without it none are.
    assert (invalid > 0) == bool(preserve_uv), invalid


@pytest.mark.parametrize("preserve_uv", [1, 0])
@pytest.mark.parametrize("name,batch", [("torus", 1), ("torus", 8), ("sphere", 16)])
def test_uv_executor_matches_oracle(gpu_lib, oracle, name, batch, preserve_uv):
    """The greedy executor on a uv mesh: the same commits, trials, stop
    reason, indices, positions and transported uv as the oracle executor."""
    mesh = MESHES[name]()
    args = _gates(24.0, (6, 2, 31), 4)
    target = mesh.face_count // 2
    want = oracle.execute(mesh, target, 240, [oracle_settings(*a) for a in args], batch=batch,
                          preserve_uv=bool(preserve_uv))
    with br.AuditSession(mesh, br.neural_options(preserve_uv=preserve_uv)) as s:
        got = s.execute(target, 240, [br.eval_settings(*a) for a in args], batch=batch)
        idx, pos = s.state()
        uv = s.state_uv()
        s.reset()
        assert np.array_equal(s.state_uv(), mesh.uv)
    assert len(want["commits"]) > 5
    assert np.array_equal(got["commits"], want["commits"])
    assert got["trials"] == want["trials"] and got["stop"] == want["stop"]
    assert np.array_equal(idx, want["indices"])
    assert np.array_equal(pos, want["positions"])
    assert np.array_equal(uv.view(np.uint32), want["uv"].view(np.uint32))
    # Commits moved uv: the transport ran on the kept slots of each class `to`.
    assert not np.array_equal(uv, mesh.uv)


def test_state_uv_needs_uv(gpu_lib):
    mesh = syn.noisy_icosphere(2, 3)
    with br.AuditSession(mesh) as s:
        with pytest.raises(br.BlitzError) as exc:
            s.state_uv()
    assert exc.value.status == br.BLITZ_INVALID_ARGUMENT
