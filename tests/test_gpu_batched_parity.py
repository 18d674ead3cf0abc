"""Parity on the batched workload itself (512 px x ss 8, 4160 x 4160 samples
per view; seamed spheres, tori and heightfields of 2,028-181,656 faces),
against the oracle's four-gate audit of the same candidates
(tests/golden/batched_512px.npz, made by tests/golden/make_batched_golden.py;
the reference's own blitz::evaluate agreed on its 64-view rows).

The multi-session batch (the benchmark's launch: one persistent audit per
plan slot over all sessions, then replayed from its CUDA graph) must give the
oracle's verdict and failed gate for every candidate, and the per-session
entry point every gate Measurement field by field, bit for bit."""
from pathlib import Path

import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn
from oracle.oracle import BoMeasurement

from conftest import measurement_fields

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "batched_512px.npz"
VIEW_SEED = 0xB1172026
LIMITS = (2.0, 1.0, 2.0, 1.0)


def _gates(views: int):
    return [br.eval_settings(512.0, lim, (views, 0, VIEW_SEED), 8, 8, 1.0) for lim in LIMITS]


def _bench_candidates(session) -> np.ndarray:
    c = br.midpoint_collapses(session.actions())
    return c[np.linspace(0, c.size - 1, min(64, c.size)).astype(np.int64)]


@pytest.fixture(scope="module")
def workload(gpu_lib):
    g = np.load(GOLDEN)
    meshes = syn.batched_set(64, seed=2)
    chosen = sorted(set(int(i) for i in g["mesh"]))
    opts = br.neural_options(device=0, preserve_uv=0)
    sessions = {i: br.AuditSession(meshes[i], opts) for i in chosen}
    yield g, meshes, sessions
    for s in sessions.values():
        s.close()


def _rows(g, views):
    return [r for r in range(g["mesh"].size) if g["views"][r] == views]


def _check_measurements(g, r, got_verdict, got_meas):
    assert got_verdict["accepted"] == g["accepted"][r] and got_verdict["failed_gate"] == g["failed_gate"][r], r
    failed = int(g["failed_gate"][r])
    stop = 4 if failed == 0 else (failed if failed <= 4 else 0)
    for k in range(stop):
        want = BoMeasurement.from_buffer_copy(g["gates"][r, k].tobytes())
        assert measurement_fields(got_meas[k]) == measurement_fields(want), (r, k, want.as_dict())


@pytest.mark.parametrize("views", [16, 64])
def test_batched_workload_matches_oracle(workload, views):
    g, meshes, sessions = workload
    rows = _rows(g, views)
    assert rows
    per_session = {i: [r for r in rows if g["mesh"][r] == i] for i in sorted(sessions)}
    order = [i for i in sorted(sessions) if per_session[i]]
    picks = {i: _bench_candidates(sessions[i]) for i in order}
    cands = []
    for i in order:
        c = np.array([picks[i][g["pick"][r]] for r in per_session[i]], dtype=br.COLLAPSE_DTYPE)
        for r, row in zip(per_session[i], c):
            assert (row["from"], row["to"]) == (g["frm"][r], g["to"][r]), "candidate lists diverged"
        cands.append(c)
    gates = _gates(views)
    batch = br.AuditBatch([sessions[i] for i in order])
    try:
        first = batch.candidates(cands, gates)
        replay = batch.candidates(cands, gates, br.BATCH_GRAPH)
    finally:
        batch.close()
    for i, v1, v2 in zip(order, first, replay):
        assert np.array_equal(v1, v2)
        for r, got in zip(per_session[i], v1):
            assert got["accepted"] == g["accepted"][r] and got["failed_gate"] == g["failed_gate"][r], (i, r)
    for i, c in zip(order, cands):
        verdicts, meas = sessions[i].candidates(c, gates, measurements=True)
        for r, v, m in zip(per_session[i], verdicts, meas):
            _check_measurements(g, r, v, m)

