"""CPU checks of the C ABI: the library loads, exports every declared symbol,
keeps the reference's descriptor layouts, and refuses to run without a GPU."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import blitzremesher_b200 as br
from oracle.oracle import reference_root

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "blitz_audit.h"
_REF_ROOT = reference_root()
REFERENCE_HEADER = (_REF_ROOT / "include" / "blitz" / "blitz.h") if _REF_ROOT else None


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(blitz_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = br.load()
    names = declared_functions()
    assert "blitz_audit_candidates" in names and "blitz_audit_evaluate" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(br.library_path())], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (blitz_\w+)", out))
    assert set(names) <= exported


def _c_layout(source: str, include: Path, tmp_path: Path) -> dict:
    prog = tmp_path / "layout.c"
    prog.write_text(source)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", f"-I{include}", str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return dict(line.split("=") for line in out.split())


LAYOUT_SRC = r"""
#include <stdio.h>
#include <stddef.h>
#include "%s"
#define S(t) printf(#t "=%%zu\n", sizeof(t));
#define O(t, f) printf(#t "." #f "=%%zu\n", offsetof(t, f));
int main(void) {
  S(blitz_mesh) S(blitz_neural_options_v2) S(blitz_neural_info) S(blitz_stream)
  O(blitz_mesh, indices) O(blitz_mesh, double_sided_count)
  O(blitz_neural_options_v2, exact_position_bps) O(blitz_neural_options_v2, reserved)
  O(blitz_neural_info, fallback_levels)
  S(blitz_settings) S(blitz_lod_info) S(blitz_storage_info) S(blitz_runtime_lod_storage_info)
  S(blitz_neural_options) S(blitz_neural_action_proposal) S(blitz_curve_point) S(blitz_color_rgba8)
  O(blitz_settings, max_supersample) O(blitz_settings, search_seed) O(blitz_settings, max_changed_area)
  O(blitz_settings, attribute_importance_count) O(blitz_settings, user_data)
  O(blitz_lod_info, screen_pixels) O(blitz_lod_info, reference_triangles)
  O(blitz_lod_info, source_changed_area_worst_view)
  O(blitz_storage_info, max_added_vertex_bytes_bps) O(blitz_runtime_lod_storage_info, cumulative_added_vertex_bytes)
  O(blitz_neural_options, reserved) O(blitz_neural_action_proposal, screen_pixels)
  O(blitz_neural_action_proposal, reserved)
  %s
  return 0;
}
"""


def test_descriptor_layouts_match_python(tmp_path):
    extra = ("S(blitz_eval_settings) S(blitz_measurement) S(blitz_collapse) S(blitz_candidate_verdict) "
             "S(blitz_execute_options) S(blitz_audit_execution)")
    lay = _c_layout(LAYOUT_SRC % ("blitz_audit.h", extra), ROOT / "include", tmp_path)
    assert int(lay["blitz_mesh"]) == C.sizeof(br.BlitzMesh)
    assert int(lay["blitz_neural_options_v2"]) == C.sizeof(br.NeuralOptionsV2)
    assert int(lay["blitz_neural_info"]) == C.sizeof(br.NeuralInfo)
    assert int(lay["blitz_eval_settings"]) == C.sizeof(br.EvalSettings)
    assert int(lay["blitz_execute_options"]) == C.sizeof(br.ExecuteOptions)
    assert int(lay["blitz_audit_execution"]) == C.sizeof(br.Execution)
    assert int(lay["blitz_measurement"]) == C.sizeof(br.Measurement) == br.MEASUREMENT_DTYPE.itemsize
    assert int(lay["blitz_collapse"]) == C.sizeof(br.Collapse) == br.COLLAPSE_DTYPE.itemsize
    assert int(lay["blitz_candidate_verdict"]) == C.sizeof(br.Verdict) == br.VERDICT_DTYPE.itemsize


def test_batch_chain_profile_layouts_match_python(tmp_path):
    """The batch info, chain settings / level and profile records: sizes and
    the offsets of their last fields equal the ctypes mirrors'."""
    extra = ("S(blitz_audit_batch_info) S(blitz_chain_settings) S(blitz_chain_level) S(blitz_audit_profile) "
             "O(blitz_audit_batch_info, changed_samples) O(blitz_audit_batch_info, tier_cycles) "
             "O(blitz_audit_batch_info, flipped_samples) O(blitz_audit_batch_info, region_split) "
             "O(blitz_chain_settings, ranking) O(blitz_chain_level, transition_audit) "
             "O(blitz_audit_profile, record_bytes)")
    lay = _c_layout(LAYOUT_SRC % ("blitz_audit.h", extra), ROOT / "include", tmp_path)
    for c_name, py in [("blitz_audit_batch_info", br.BatchInfo), ("blitz_chain_settings", br.ChainSettings),
                       ("blitz_chain_level", br.ChainLevel), ("blitz_audit_profile", br.AuditProfile)]:
        assert int(lay[c_name]) == C.sizeof(py), c_name
    for c_name, py, field in [("blitz_audit_batch_info", br.BatchInfo, "changed_samples"),
                              ("blitz_audit_batch_info", br.BatchInfo, "tier_cycles"),
                              ("blitz_audit_batch_info", br.BatchInfo, "flipped_samples"),
                              ("blitz_audit_batch_info", br.BatchInfo, "region_split"),
                              ("blitz_chain_settings", br.ChainSettings, "ranking"),
                              ("blitz_chain_level", br.ChainLevel, "transition_audit"),
                              ("blitz_audit_profile", br.AuditProfile, "record_bytes")]:
        assert int(lay[f"{c_name}.{field}"]) == getattr(py, field).offset, (c_name, field)


@pytest.mark.skipif(REFERENCE_HEADER is None or not REFERENCE_HEADER.exists(),
                    reason="reference headers absent (set BLITZ_REFERENCE to the reference tree)")
def test_abi5_descriptors_identical_to_reference(tmp_path):
    ours = _c_layout(LAYOUT_SRC % ("blitz_audit.h", ""), ROOT / "include", tmp_path)
    (tmp_path / "ref").mkdir()
    theirs = _c_layout(LAYOUT_SRC % ("blitz/blitz.h", ""), REFERENCE_HEADER.parents[1], tmp_path / "ref")
    assert ours == theirs


def test_version_and_defaults():
    lib = br.load()
    assert lib.blitz_abi_version() == 5
    o = br.neural_options()
    assert o.struct_size == C.sizeof(br.NeuralOptionsV2) and o.version == 2 and o.memory_mib == 6144
    assert o.preserve_uv == 1 and o.action_batch == 32
    bad = br.NeuralOptionsV2()
    assert lib.blitz_neural_options_v2_init(C.byref(bad), 3) == br.BLITZ_INVALID_ARGUMENT
    s = br.eval_settings(24.0, 1.0)
    assert s.struct_size == C.sizeof(br.EvalSettings) and s.profile == 0


def test_session_rejects_invalid_descriptors():
    lib = br.load()
    mesh = br.synthetic.noisy_icosphere(1, 1)
    h = br._MeshHold(mesh)
    h.c.abi_version = 4
    handle = C.c_void_p()
    err = C.create_string_buffer(256)
    st = lib.blitz_audit_session_create(C.byref(h.c), None, C.byref(handle), err, 256)
    assert st in (br.BLITZ_INVALID_ARGUMENT, br.BLITZ_UNAVAILABLE)
    assert not handle.value


def test_no_gpu_means_unavailable():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(br.BlitzError) as exc:
        br.AuditSession(br.synthetic.noisy_icosphere(1, 1))
    assert exc.value.status == br.BLITZ_UNAVAILABLE


def test_synthetic_mesh_shapes():
    m = br.synthetic.config1_mesh()
    assert m.face_count == 20480 and m.vertex_count == 10242
    assert m.positions.dtype == np.float32 and m.indices.dtype == np.uint32
    r = np.linalg.norm(m.positions.astype(np.float64), axis=1)
    assert r.min() >= 0.98 - 1e-6 and r.max() <= 1.02 + 1e-6
    again = br.synthetic.config1_mesh()
    assert np.array_equal(m.positions, again.positions)
