"""CPU checks of the batched-workload golden fixture
(tests/golden/batched_512px.npz): it spans the workload's size range and mesh
kinds, its 64-view rows agree with the reference's own blitz::evaluate, and
the oracle reproduces its smallest mesh's rows live, Measurement for
Measurement."""
from pathlib import Path

import numpy as np

from blitzremesher_b200 import synthetic as syn
from oracle.oracle import BoMeasurement, settings

from conftest import measurement_fields

GOLDEN = Path(__file__).resolve().parent / "golden" / "batched_512px.npz"


def test_batched_golden_covers_the_workload():
    g = np.load(GOLDEN)
    meshes = syn.batched_set(64, seed=2)
    kinds = {meshes[int(i)].name.split("-")[0] for i in g["mesh"]}
    assert kinds == {"sphere", "torus", "heightfield"}
    assert g["faces"].min() <= 2100 and g["faces"].max() >= 180_000
    assert int(g["accepted"].sum()) > 0
    ref = g["reference_accepted"]
    assert np.all(ref[g["views"] == 64] >= 0) and np.all(ref[g["faces"] < 20000] >= 0)
    assert int((g["accepted"][ref >= 0] == 0).sum()) > 0  # rejections confirmed by the reference too
    assert np.array_equal(ref[ref >= 0], g["accepted"][ref >= 0])


def test_oracle_reproduces_smallest_mesh_rows(oracle):
    g = np.load(GOLDEN)
    meshes = syn.batched_set(64, seed=2)
    small = int(g["mesh"][np.argmin(g["faces"])])
    mesh = meshes[small]
    acts = oracle.actions(mesh, placement=True, preserve_uv=False)
    picks = np.linspace(0, len(acts) - 1, min(64, len(acts))).astype(np.int64)
    b = oracle.bounds(mesh)
    rows = [r for r in range(g["mesh"].size) if g["mesh"][r] == small]
    assert len(rows) == 4
    for r in rows:
        e = acts[picks[g["pick"][r]]]
        assert (e.from_, e.to) == (g["frm"][r], g["to"][r])
        views = (int(g["views"][r]), 0, 0xB1172026)
        gates = [settings(512.0, lim, views, 8, 8, 1.0) for lim in (2.0, 1.0, 2.0, 1.0)]
        v = oracle.audit_candidate(mesh, e, mesh, mesh, b, gates, preserve_uv=False)
        assert (v.accepted, v.failed_gate) == (g["accepted"][r], g["failed_gate"][r])
        for k in range(4):
            want = BoMeasurement.from_buffer_copy(g["gates"][r, k].tobytes())
            assert measurement_fields(v.gates[k]) == measurement_fields(want)
