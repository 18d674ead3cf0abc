"""Several sessions audited in one persistent launch: the verdicts equal each
session's own blitz_audit_candidates, with and without graph replay and after
autotuning, through the device and the host entry points, for meshes at LOD0,
after commits, and at rasters above 256 x 256 (large and huge tiers)."""
import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _gates(screen, views=(8, 0, 0xB1172026), ss=8):
    return [br.eval_settings(screen, 2.0, views, ss, ss, 1.0), br.eval_settings(screen, 1.0, views, ss, ss, 1.0),
            br.eval_settings(screen, 2.0, views, ss, ss, 0.5), br.eval_settings(screen, 1.0, views, ss, ss, 0.5)]


@pytest.mark.parametrize("screen", [24.0, 64.0])
def test_batch_equals_per_session(gpu_lib, screen):
    meshes = [syn.seamed_sphere(2000, 3), syn.seamed_torus(3000, 4, 8), syn.seamed_heightfield(5000, 5, 9),
              syn.noisy_icosphere(3, 6)]
    gates = _gates(screen)
    opts = br.neural_options(preserve_uv=0)
    sessions = [br.AuditSession(m, opts) for m in meshes]
    try:
        # one session after commits (state differs from its references)
        sessions[3].execute(meshes[3].face_count - 100, 200, gates, batch=8)
        picks = []
        for s in sessions:
            c = br.midpoint_collapses(s.actions())
            picks.append(c[:: max(1, c.size // 150)])
        want = [s.candidates(p, gates) for s, p in zip(sessions, picks)]
        import torch
        batch = br.AuditBatch(sessions)
        got = batch.candidates(picks, gates)
        for w, g in zip(want, got):
            assert np.array_equal(w, g)
        # fixed device buffers, so the captured graph is replayed
        counts = [int(p.size) for p in picks]
        cat = np.concatenate(picks)
        dev = torch.from_numpy(cat.view(np.uint8).copy()).cuda()
        out = torch.zeros(cat.size * br.VERDICT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        expect = np.concatenate(want)
        for flags in (br.BATCH_GRAPH, br.BATCH_GRAPH, br.BATCH_AUTOTUNE | br.BATCH_GRAPH, br.BATCH_GRAPH):
            out.zero_()
            batch.candidates_device(dev.data_ptr(), counts, gates, out.data_ptr(), flags)
            assert np.array_equal(out.cpu().numpy().view(br.VERDICT_DTYPE), expect), flags
        info = batch.info()
        assert info["tuned"] == 1 and info["graph_captured"] == 1 and info["graph_launches"] >= 2
        # host entry point: host collapses in, host verdicts out, graph replayed
        host_out = np.zeros(cat.size, br.VERDICT_DTYPE)
        for flags in (0, br.BATCH_GRAPH, br.BATCH_GRAPH):
            host_out[:] = 0
            batch.candidates_host(cat, counts, gates, host_out, flags)
            assert np.array_equal(host_out, expect), flags
        assert batch.info()["graph_launches"] > info["graph_launches"]
        batch.close()
    finally:
        for s in sessions:
            s.close()
