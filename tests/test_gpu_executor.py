"""GPU greedy executor against the oracle executor, and candidate audits of a
state that differs from its references (the tile-maxima path)."""
import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn
from oracle.oracle import BoEdit, settings as oracle_settings

from conftest import measurement_fields

pytestmark = pytest.mark.gpu

CASES = {
    "sphere2_96": (lambda: syn.noisy_icosphere(2, 3), (6, 2, 5), 16.0, 4, 200),
    "sphere3_256": (lambda: syn.noisy_icosphere(3, 4), (8, 0, 0xB1172026), 24.0, 8, 160),
}


def _gates(screen, views, ss):
    return [(screen, 2.0, views, ss, ss, 1.0), (screen, 1.0, views, ss, ss, 1.0),
            (screen, 2.0, views, ss, ss, 0.5), (screen, 1.0, views, ss, ss, 0.5)]


@pytest.mark.parametrize("case", sorted(CASES))
def test_executor_matches_oracle(gpu_lib, oracle, case):
    make, views, screen, ss, budget = CASES[case]
    mesh = make()
    args = _gates(screen, views, ss)
    target = mesh.face_count // 2
    want = oracle.execute(mesh, target, budget, [oracle_settings(*a) for a in args])
    with br.AuditSession(mesh) as s:
        got = s.execute(target, budget, [br.eval_settings(*a) for a in args])
        idx, pos = s.state()
        # The same walk again from the source gives the same result.
        s.reset()
        again = s.execute(target, budget, [br.eval_settings(*a) for a in args])
    assert len(want["commits"]) > 5
    assert np.array_equal(got["commits"], want["commits"])
    assert got["trials"] == want["trials"] and got["stop"] == want["stop"]
    assert np.array_equal(idx, want["indices"])
    assert np.array_equal(pos, want["positions"])
    assert np.array_equal(again["commits"], got["commits"]) and again["trials"] == got["trials"]


@pytest.mark.parametrize("case,batch", [("sphere2_96", 8), ("sphere2_96", 64), ("sphere3_256", 16)])
def test_batched_executor_matches_oracle(gpu_lib, oracle, case, batch):
    """Batches of independent collapses audited as one combined trial, halved
    on rejection: the same commits, trials and final state as the oracle."""
    make, views, screen, ss, budget = CASES[case]
    mesh = make()
    args = _gates(screen, views, ss)
    target = mesh.face_count // 2
    want = oracle.execute(mesh, target, budget, [oracle_settings(*a) for a in args], batch=batch)
    with br.AuditSession(mesh) as s:
        got = s.execute(target, budget, [br.eval_settings(*a) for a in args], batch=batch)
        idx, pos = s.state()
    assert len(want["commits"]) > 5
    assert np.array_equal(got["commits"], want["commits"])
    assert got["trials"] == want["trials"] and got["stop"] == want["stop"]
    assert np.array_equal(idx, want["indices"])
    assert np.array_equal(pos, want["positions"])


def test_candidates_of_committed_state_match_oracle(gpu_lib, oracle):
    """After commits the state differs from both references: every gate
    Measurement of a candidate sample still equals the oracle's."""
    mesh = syn.noisy_icosphere(3, 9)
    views = (8, 4, 77)
    args = _gates(24.0, views, 8)
    with br.AuditSession(mesh) as s:
        s.execute(mesh.face_count - 60, 400, [br.eval_settings(*a) for a in args])
        idx, pos = s.state()
        cands = br.midpoint_collapses(s.actions())
        picks = cands[:: max(1, cands.size // 40)]
        verdicts, meas = s.candidates(picks, [br.eval_settings(*a) for a in args], measurements=True)
    state = syn.Mesh(pos, idx)
    b = oracle.bounds(mesh)
    for i, c in enumerate(picks):
        e = BoEdit()
        e.from_, e.to = int(c["from"]), int(c["to"])
        want = oracle.audit_candidate(state, e, mesh, mesh, b, [oracle_settings(*a) for a in args])
        assert verdicts[i]["accepted"] == want.accepted and verdicts[i]["failed_gate"] == want.failed_gate, i
        stop = 4 if want.failed_gate == 0 else (want.failed_gate if want.failed_gate <= 4 else 0)
        for g in range(stop):
            assert measurement_fields(meas[i, g]) == measurement_fields(want.gates[g]), (i, g)


def _stacked_sheets(layers: int, seed: int):
    """`layers` parallel 2 x 2-quad sheets facing +z, 0.0005 apart, each with
    its centre vertex jittered: front views see every layer over most samples,
    so more than 255 faces cover a sample."""
    rng = np.random.default_rng(seed)
    g = np.linspace(-1.0, 1.0, 3)
    xs, ys = np.meshgrid(g, g)
    pos, idx = [], []
    for k in range(layers):
        p = np.stack([xs.ravel(), ys.ravel(), np.full(9, 0.0005 * k)], 1)
        p[4, :2] += rng.uniform(-0.3, 0.3, 2)
        pos.append(p)
        for i in range(2):
            for j in range(2):
                a = 9 * k + 3 * i + j
                idx += [a, a + 1, a + 4, a, a + 4, a + 3]
    return syn.Mesh(np.concatenate(pos).astype(np.float32), np.array(idx, np.uint32))


def test_deep_overlap_matches_oracle(gpu_lib, oracle):
    """Samples covered by more than 255 faces: the state counts are held at
    255, which leaves every verdict, Measurement and commit exact (a collapse
    changes at most 48 faces)."""
    mesh = _stacked_sheets(320, 4)
    views = (6, 2, 5)
    args = _gates(16.0, views, 4)
    gates_o = [oracle_settings(*a) for a in args]
    gates_g = [br.eval_settings(*a) for a in args]
    b = oracle.bounds(mesh)
    with br.AuditSession(mesh) as s:
        cands = br.midpoint_collapses(s.actions())
        picks = cands[:: max(1, cands.size // 24)]
        verdicts, meas = s.candidates(picks, gates_g, measurements=True)
        got = s.execute(mesh.face_count - 200, 40, gates_g, batch=8)
        idx, pos = s.state()
    for i, c in enumerate(picks):
        e = BoEdit()
        e.from_, e.to = int(c["from"]), int(c["to"])
        want = oracle.audit_candidate(mesh, e, mesh, mesh, b, gates_o)
        assert verdicts[i]["accepted"] == want.accepted and verdicts[i]["failed_gate"] == want.failed_gate, i
        stop = 4 if want.failed_gate == 0 else (want.failed_gate if want.failed_gate <= 4 else 0)
        for g in range(stop):
            assert measurement_fields(meas[i, g]) == measurement_fields(want.gates[g]), (i, g)
    want = oracle.execute(mesh, mesh.face_count - 200, 40, gates_o, batch=8)
    assert len(want["commits"]) > 0
    assert np.array_equal(got["commits"], want["commits"])
    assert got["trials"] == want["trials"] and got["stop"] == want["stop"]
    assert np.array_equal(idx, want["indices"]) and np.array_equal(pos, want["positions"])


@pytest.mark.parametrize("commit", [False, True])
def test_large_regions_match_oracle(gpu_lib, oracle, commit):
    """Coarse triangles at 64 px x ss 8: most (candidate, view) regions
    overflow the warp tier and go to the large tier; verdicts and every gate
    Measurement still equal the oracle's, and few candidates need the
    full-raster path."""
    mesh = syn.noisy_icosphere(2, 5)
    views = (6, 0, 91)
    args = _gates(64.0, views, 8)
    with br.AuditSession(mesh) as s:
        if commit:
            s.execute(mesh.face_count - 40, 100, [br.eval_settings(*a) for a in args], batch=8)
        idx, pos = s.state()
        cands = br.midpoint_collapses(s.actions())
        picks = cands[:: max(1, cands.size // 36)]
        verdicts, meas = s.candidates(picks, [br.eval_settings(*a) for a in args], measurements=True)
    assert np.mean(verdicts["exact_path"]) < (0.5 if commit else 0.25)
    state = syn.Mesh(pos, idx)
    b = oracle.bounds(mesh)
    for i, c in enumerate(picks):
        e = BoEdit()
        e.from_, e.to = int(c["from"]), int(c["to"])
        want = oracle.audit_candidate(state, e, mesh, mesh, b, [oracle_settings(*a) for a in args])
        assert verdicts[i]["accepted"] == want.accepted and verdicts[i]["failed_gate"] == want.failed_gate, i
        stop = 4 if want.failed_gate == 0 else (want.failed_gate if want.failed_gate <= 4 else 0)
        for g in range(stop):
            assert measurement_fields(meas[i, g]) == measurement_fields(want.gates[g]), (i, g)


@pytest.mark.parametrize("commit", [False, True])
def test_huge_regions_match_oracle(gpu_lib, oracle, commit):
    """An 80-face sphere at 64 px x ss 8: 1-ring regions of about 300 x 300
    samples overflow the large tier and are audited by the huge tier (global
    scratch, the word-row region phase); verdicts and gate Measurements equal
    the oracle's, at LOD0 and after commits (state unlike its references:
    tile maxima, region widened to whole tiles)."""
    mesh = syn.noisy_icosphere(1, 5)
    views = (6, 0, 91)
    args = _gates(64.0, views, 8)
    with br.AuditSession(mesh) as s:
        if commit:  # loose 6 px gates so that a few collapses commit
            s.execute(mesh.face_count - 12, 60, [br.eval_settings(64.0, 6.0, views, 8, 8, 1.0)] * 4, batch=4)
        idx, pos = s.state()
        cands = br.midpoint_collapses(s.actions())
        picks = cands[:: max(1, cands.size // 30)]
        verdicts, meas = s.candidates(picks, [br.eval_settings(*a) for a in args], measurements=True)
    assert np.mean(verdicts["exact_path"]) < (0.5 if commit else 0.25)
    state = syn.Mesh(pos, idx)
    assert not commit or state.face_count < mesh.face_count
    b = oracle.bounds(mesh)
    for i, c in enumerate(picks):
        e = BoEdit()
        e.from_, e.to = int(c["from"]), int(c["to"])
        want = oracle.audit_candidate(state, e, mesh, mesh, b, [oracle_settings(*a) for a in args])
        assert verdicts[i]["accepted"] == want.accepted and verdicts[i]["failed_gate"] == want.failed_gate, i
        stop = 4 if want.failed_gate == 0 else (want.failed_gate if want.failed_gate <= 4 else 0)
        for g in range(stop):
            assert measurement_fields(meas[i, g]) == measurement_fields(want.gates[g]), (i, g)


def test_giant_regions_match_oracle(gpu_lib, oracle):
    """An 80-face sphere at 256 px x ss 8 (2112 x 2112 samples): 1-ring
    regions beyond 1024 samples go to the giant tier; verdicts and gate
    Measurements equal the oracle's."""
    mesh = syn.noisy_icosphere(1, 7)
    views = (4, 0, 93)
    args = _gates(256.0, views, 8)
    with br.AuditSession(mesh) as s:
        cands = br.midpoint_collapses(s.actions())
        picks = cands[:: max(1, cands.size // 10)]
        verdicts, meas = s.candidates(picks, [br.eval_settings(*a) for a in args], measurements=True)
    assert np.mean(verdicts["exact_path"]) < 0.25
    b = oracle.bounds(mesh)
    for i, c in enumerate(picks):
        e = BoEdit()
        e.from_, e.to = int(c["from"]), int(c["to"])
        want = oracle.audit_candidate(mesh, e, mesh, mesh, b, [oracle_settings(*a) for a in args])
        assert verdicts[i]["accepted"] == want.accepted and verdicts[i]["failed_gate"] == want.failed_gate, i
        stop = 4 if want.failed_gate == 0 else (want.failed_gate if want.failed_gate <= 4 else 0)
        for g in range(stop):
            assert measurement_fields(meas[i, g]) == measurement_fields(want.gates[g]), (i, g)


def _oracle_chain(oracle, mesh, levels, base, last, curve, lod0, search, audit, ss, batch, budget):
    p, t, b = oracle.schedule(base, last, levels, [v for xy in curve for v in xy], lod0)
    state, prev, out = None, None, []
    for i in range(1, levels):
        gates = [oracle_settings(p[i], b[i], search, ss, ss, 1.0), oracle_settings(p[i], t[i], search, ss, ss, 1.0),
                 oracle_settings(p[i], b[i], audit, ss, ss, 1.0), oracle_settings(p[i], t[i], audit, ss, ss, 1.0)]
        r = oracle.execute(mesh, 1, budget, gates, previous=prev, batch=batch, start=state)
        state = syn.Mesh(r["positions"], r["indices"])
        prev = state
        out.append(r)
    return out


@pytest.mark.parametrize("batch", [1, 8])
def test_chain_matches_oracle(gpu_lib, oracle, batch):
    """A 4-level chain (48 -> 12 px, transition 1 -> 3 px, LOD0 bound capped at
    2 px): each level's executor against the bound previous level, then the
    confirmation; every emitted level equals the oracle chain's."""
    mesh = syn.noisy_icosphere(3, 21)
    curve, search, audit = ((0.0, 1.0), (1.0, 3.0)), (6, 0, 5), (8, 0, 7)
    want = _oracle_chain(oracle, mesh, 4, 48.0, 12.0, curve, 2.0, search, audit, 4, batch, 120)
    settings = br.chain_settings(4, 48.0, 12.0, curve, 2.0, search, audit, 4, 4, 4, 1.0, batch, 0, 120, 1)
    with br.AuditSession(mesh) as s:
        levels, meshes = s.chain(settings)
    assert len(levels) == 3 and len(meshes) == 3
    p, t, b = oracle.schedule(48.0, 12.0, 4, [v for xy in curve for v in xy], 2.0)
    bounds = oracle.bounds(mesh)
    prev = mesh
    for i, (lv, (idx, pos), w) in enumerate(zip(levels, meshes, want), start=1):
        assert lv["trials"] == w["trials"] and lv["stop_reason"] == w["stop"]
        assert np.array_equal(idx, w["indices"]) and np.array_equal(pos, w["positions"])
        assert lv["confirmed"] == 1
        # the confirmation's Measurements (from the audit plans' resident
        # data) equal the oracle's full evaluation of the emitted level
        level = syn.Mesh(pos, idx)
        src = oracle.evaluate(mesh, level, bounds, oracle_settings(p[i], b[i], audit, 4, 4, 1.0))
        trn = oracle.evaluate(prev, level, bounds, oracle_settings(p[i], t[i], audit, 4, 4, 1.0))
        assert measurement_fields(lv["source_audit"]) == measurement_fields(src), i
        assert measurement_fields(lv["transition_audit"]) == measurement_fields(trn), i
        prev = level
    assert levels[-1]["faces"] < levels[0]["faces"] < mesh.face_count


@pytest.mark.parametrize("ranking,batch", [(4, 1), (4, 8), (1, 8)])
def test_rankings_match_oracle(gpu_lib, oracle, ranking, batch):
    """CurrentPlane (4) and Constant (1) rankings of rank_actions: the same walk
    as the oracle's executor with that ranking."""
    make, views, screen, ss, budget = CASES["sphere2_96"]
    mesh = make()
    args = _gates(screen, views, ss)
    target = mesh.face_count // 2
    want = oracle.execute(mesh, target, budget, [oracle_settings(*a) for a in args], batch=batch, ranking=ranking)
    with br.AuditSession(mesh) as s:
        got = s.execute(target, budget, [br.eval_settings(*a) for a in args], batch=batch, ranking=ranking)
        idx, pos = s.state()
    assert len(want["commits"]) > 5
    assert np.array_equal(got["commits"], want["commits"])
    assert got["trials"] == want["trials"] and got["stop"] == want["stop"]
    assert np.array_equal(idx, want["indices"]) and np.array_equal(pos, want["positions"])


def test_learned_ranking_passes_the_exact_audit(gpu_lib):
    """Learned ranking (the attached surrogate's logits) reorders the walk; the
    exact audit still judges every committed batch."""
    mesh = syn.noisy_icosphere(3, 8)
    args = _gates(64.0, (8, 0, 0xB1172026), 8)
    gates = [br.eval_settings(*a) for a in args]
    with br.AuditSession(mesh) as s:
        s.attach_surrogate(br.Surrogate(seed=3))
        r = s.execute(mesh.face_count // 3, 300, gates, batch=16, ranking=0)
        idx, pos = s.state()
        assert len(r["commits"]) > 0
        for g in gates:
            m = br.evaluate(mesh, syn.Mesh(pos, idx), g, session=s)
            assert m.passed == 1


@pytest.mark.parametrize("level,screen,limits", [(3, 24.0, (1.0, 0.5)), (1, 64.0, (2.0, 1.0)), (2, 96.0, (3.0, 1.5))])
def test_verdict_only_audit_gives_the_exact_verdicts(gpu_lib, level, screen, limits):
    """Without a Measurement buffer the audit stops measuring a view once its
    verdicts are certain (the threshold predicate of evaluate.cu:1034-1169):
    the verdicts and failed gates equal those of the exactly measured audit,
    rejections included, at LOD0 and after commits."""
    mesh = syn.noisy_icosphere(level, 31)
    views = (6, 2, 97)
    gates = [br.eval_settings(screen, limits[0], views, 8, 8, 1.0), br.eval_settings(screen, limits[1], views, 8, 8, 1.0),
             br.eval_settings(screen, limits[0], views, 8, 8, 0.5), br.eval_settings(screen, limits[1], views, 8, 8, 0.5)]
    accepted = rejected = 0
    with br.AuditSession(mesh) as s:
        for commit in (False, True):
            if commit:
                s.execute(mesh.face_count - 8, 40, [br.eval_settings(screen, 6.0, views, 8, 8, 1.0)] * 4, batch=4)
            cands = br.midpoint_collapses(s.actions())
            exact, _ = s.candidates(cands, gates, measurements=True)
            quick = s.candidates(cands, gates)
            assert np.array_equal(exact["accepted"], quick["accepted"])
            assert np.array_equal(exact["failed_gate"], quick["failed_gate"])
            accepted += int(exact["accepted"].sum())
            rejected += int(cands.size - exact["accepted"].sum())
    assert accepted > 0 and rejected > 0
