"""Generates tests/golden/batched_512px.npz: oracle four-gate verdicts and gate
Measurements for a fixed sample of the batched workload's candidates.

Workload: the 64 seeded meshes of `synthetic.batched_set(64, seed=2)` (noisy
spheres, R/r = 3 tori, value-noise heightfields; FP32 UVs with chart seams),
audited at 512 px x ss 8 (4160 x 4160 samples per view) with a 2 px LOD0 and
a 1 px transition limit, midpoint placement, uv not preserved (so uv seams
are welded, as the reference's GPU state does without preserve_uv). Sample: the
smallest mesh, the median one and the three largest (sphere, torus and
heightfield among them); per mesh 4 of the 64 evenly spaced legal collapses
the benchmark audits (positions 0, 21, 42 and 63 of its list), on the first
16 of the Fibonacci views; 2 more candidates (median and largest mesh) on all
64 views. The oracle (oracle/liboracle.so, the reference's CPU audit
restated) computes every row; where oracle/_ref exists, the reference's own
blitz::evaluate re-audits the midpoint trials of the 64-view rows and of the
two smaller meshes' rows, and must agree.

    python tests/golden/make_batched_golden.py   (about 2.5 minutes on 8 cores)
"""
from __future__ import annotations

import multiprocessing as mp
import sys
from concurrent.futures import ProcessPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "batched_512px.npz"
SEED = 2
VIEW_SEED = 0xB1172026
SCREEN, SS = 512.0, 8
LIMITS = (2.0, 1.0, 2.0, 1.0)
PICKS = (0, 21, 42, 63)


def sample_meshes(meshes) -> list:
    order = np.argsort([m.face_count for m in meshes], kind="stable")
    return [int(order[0]), int(order[len(order) // 2])] + [int(i) for i in order[-3:]]


def gate_settings(views: int):
    from oracle.oracle import settings

    return [settings(SCREEN, lim, (views, 0, VIEW_SEED), SS, SS, 1.0) for lim in LIMITS]


def bench_candidates(oracle, mesh) -> list:
    """The benchmark's 64 evenly spaced legal midpoint collapses of a mesh."""
    acts = oracle.actions(mesh, placement=True, preserve_uv=False)
    idx = np.linspace(0, len(acts) - 1, min(64, len(acts))).astype(np.int64)
    return [acts[i] for i in idx]


def _audit(job):
    mesh_index, pick, views, check_reference = job
    sys.path.insert(0, str(ROOT))
    from blitzremesher_b200 import synthetic as syn
    from oracle.oracle import Oracle, Reference

    mesh = syn.batched_set(64, seed=SEED)[mesh_index]
    O = Oracle()
    e = bench_candidates(O, mesh)[pick]
    b = O.bounds(mesh)
    v = O.audit_candidate(mesh, e, mesh, mesh, b, gate_settings(views), preserve_uv=False)
    ref_ok = -1
    if check_reference and Reference.available():
        R = Reference()
        idx, pos, _, valid = O.trial_midpoint(mesh, e, preserve_uv=False)
        cand = syn.Mesh(pos, idx)
        ok = bool(valid)
        if ok:
            for s in gate_settings(views):
                m = R.evaluate(mesh, cand, R.bounds(mesh), s)
                if not (m.complete and m.passed and not m.resource_limited):
                    ok = False
                    break
        ref_ok = int(ok)
    gates = np.frombuffer(b"".join(bytes(g) for g in v.gates), np.uint8).reshape(4, -1).copy()
    return (mesh_index, pick, views, int(e.from_), int(e.to), int(v.accepted), int(v.failed_gate),
            int(v.placement_valid), gates, ref_ok)


def main() -> None:
    from blitzremesher_b200 import synthetic as syn

    meshes = syn.batched_set(64, seed=SEED)
    chosen = sample_meshes(meshes)
    jobs = [(i, p, 16, meshes[i].face_count < 20000) for i in chosen for p in PICKS]
    jobs += [(chosen[1], 21, 64, True), (chosen[-1], 42, 64, True)]
    with ProcessPoolExecutor(max_workers=8, mp_context=mp.get_context("spawn")) as ex:
        rows = list(ex.map(_audit, jobs))
    for r in rows:
        if r[9] >= 0:
            assert r[9] == r[5], f"reference and oracle disagree on mesh {r[0]} pick {r[1]}"
    np.savez_compressed(
        OUT,
        mesh=np.array([r[0] for r in rows], np.int32), pick=np.array([r[1] for r in rows], np.int32),
        views=np.array([r[2] for r in rows], np.int32), frm=np.array([r[3] for r in rows], np.uint32),
        to=np.array([r[4] for r in rows], np.uint32), accepted=np.array([r[5] for r in rows], np.uint8),
        failed_gate=np.array([r[6] for r in rows], np.uint8),
        placement_valid=np.array([r[7] for r in rows], np.uint8),
        gates=np.stack([r[8] for r in rows]), reference_accepted=np.array([r[9] for r in rows], np.int8),
        faces=np.array([meshes[r[0]].face_count for r in rows], np.int64))
    print(f"{len(rows)} rows -> {OUT.name}; accepted {sum(r[5] for r in rows)}; "
          f"meshes {[meshes[i].name for i in chosen]}")


if __name__ == "__main__":
    main()
