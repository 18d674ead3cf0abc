"""blitz_generate_neural on the GPU: a 4-level chain of a 1,280-face sphere
through the reference's public entry point (blitz.h:165) with a BLZNET policy
loaded by blitz_neural_model_load_v2. Every emitted level equals the oracle's
chain (schedule, four gates against the source and the previous level,
batched midpoint executor), level 0 is the source itself, and the lod info,
runtime levels, storage and proposals are consistent with the levels."""
import json

import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn

from test_generate import blznet
from test_gpu_executor import _oracle_chain

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("batch", [1, 8])
def test_generate_neural_matches_oracle_chain(gpu_lib, oracle, tmp_path, batch):
    mesh = syn.noisy_icosphere(3, 21)
    curve, search, audit = ((0.0, 1.0), (1.0, 3.0)), (6, 0, 5), (8, 0, 7)
    want = _oracle_chain(oracle, mesh, 4, 48.0, 12.0, curve, 2.0, search, audit, 4, batch, 120)
    policy = tmp_path / "policy.blzn"
    policy.write_bytes(blznet(2))
    model = br.NeuralModel(policy, br.neural_options(ranking=3, action_batch=batch, action_trials=120))
    config = br.settings(levels=4, profile=0, base_pixels=48.0, last_pixels=12.0, max_lod0_delta_px=2.0,
                         transition=curve, search_ortho=search[0], search_perspective=search[1],
                         search_seed=search[2], audit_ortho=audit[0], audit_perspective=audit[1], audit_seed=audit[2],
                         search_supersample=4, audit_supersample=4, max_supersample=4, max_changed_area=1.0)
    out = br.generate_neural(mesh, config, model, save_to=tmp_path / "chain")
    lods = out["lods"]
    assert len(lods) == 4
    assert np.array_equal(lods[0]["indices"], mesh.indices) and lods[0]["shared_vertices"] == 1
    for lv, w, prop in zip(lods[1:], want, out["proposals"]):
        assert np.array_equal(lv["indices"], w["indices"])
        used = np.unique(lv["indices"])
        assert np.array_equal(lv["positions"][used], w["positions"][used])
        assert lv["reference_triangles"] == lv["indices"].size // 3
        assert prop["trials"] == w["trials"] and prop["stop_reason"] == w["stop"]
        assert prop["final_triangles"] == lv["indices"].size // 3
        assert lv["passed"] == int(lv["source_error"] <= lv["source_limit"] and
                                   lv["transition_error"] <= lv["transition_limit"])
    p, t, b = oracle.schedule(48.0, 12.0, 4, [v for xy in curve for v in xy], 2.0)
    assert [lv["screen_pixels"] for lv in lods] == list(p)
    assert [lv["transition_limit"] for lv in lods[1:]] == list(t[1:])
    assert [lv["source_limit"] for lv in lods[1:]] == list(b[1:])
    assert out["runtime"][0] == 0 and out["runtime"] == sorted(set(out["runtime"]))
    st = out["storage"]
    assert st["index_bytes"] == sum(lods[i]["indices"].size * 4 for i in out["runtime"])
    assert st["source_vertex_bytes"] == mesh.vertex_count * 12
    assert out["info"]["legal_collapses"] == sum(len(w["commits"]) for w in want)
    # the exported chain: one node per level, one mesh per runtime level
    gltf = json.loads((tmp_path / "chain" / "chain.gltf").read_text())
    manifest = json.loads((tmp_path / "chain" / "lods.json").read_text())
    assert len(gltf["nodes"]) == 4 and len(gltf["meshes"]) == len(out["runtime"])
    assert gltf["buffers"][0]["byteLength"] == (tmp_path / "chain" / "chain.bin").stat().st_size
    assert [l["triangles"] for l in manifest["lods"]] == [lv["indices"].size // 3 for lv in lods]
    assert manifest["runtime_levels"] == out["runtime"]
    model.close()


def test_generate_neural_refuses_what_is_not_built(gpu_lib, tmp_path):
    policy = tmp_path / "policy.blzn"
    policy.write_bytes(blznet(2))
    mesh = syn.noisy_icosphere(2, 3)
    learned = br.NeuralModel(policy, br.neural_options(ranking=0))
    with pytest.raises(br.BlitzError) as e:
        br.generate_neural(mesh, br.settings(levels=2, profile=0, base_pixels=24.0, last_pixels=24.0), learned)
    assert e.value.status == br.BLITZ_UNAVAILABLE
    shortest = br.NeuralModel(policy, br.neural_options(ranking=3))
    with pytest.raises(br.BlitzError) as e:
        br.generate_neural(mesh, br.settings(levels=2, profile=1, base_pixels=24.0, last_pixels=24.0), shortest)
    assert e.value.status == br.BLITZ_UNAVAILABLE
