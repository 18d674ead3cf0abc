"""The blitz.h generation surface (csrc/generate.cu) on the CPU: settings and
neural option defaults, BLZNET policy files (header, weight counts per
architecture, SHA-256 checksum; model_io.cpp:59-107), the classical
generator's refusal, and model option checks. The generation itself runs in
tests/test_gpu_generate.py."""
import ctypes as C
import hashlib
import struct

import numpy as np
import pytest

import blitzremesher_b200 as br
from oracle.oracle import reference_root


def policy_count(arch: int, width: int) -> int:
    if arch == 1:
        return sum(o * (i + 1) for i, o in zip((48, 128, 128, 72, 64), (64, 64, 64, 64, 4)))
    inputs, outputs = {2: (80, 3), 3: (128, 12), 4: (128, 12)}[arch]
    return width * (inputs + 1) + width * (width + 1) + outputs * (width + 1)


def blznet(arch: int, width: int = 64, use: int = 0, provenance: bytes = b"test", weights=None,
           count=None) -> bytes:
    """A BLZNET file in the layout of model_io.cpp:108-140 (save_weights)."""
    n = policy_count(arch, width) if count is None else count
    w = np.linspace(-1, 1, n, dtype=np.float32) if weights is None else np.asarray(weights, np.float32)
    version = b"3" if use else (b"2" if width != 64 else b"1")
    head = b"BLZNET0" + version + struct.pack("<III", arch, n, len(provenance))
    if version != b"1":
        head += struct.pack("<I", width)
    if use:
        head += struct.pack("<I", use)
    payload = head + provenance + w.astype("<f4").tobytes()
    return payload + hashlib.sha256(payload).hexdigest().encode()


def load(path, **opts):
    lib = br.load()
    o = br.neural_options(**opts)
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    st = lib.blitz_neural_model_load_v2(str(path).encode(), C.byref(o), C.byref(h), err, 256)
    sha = lib.blitz_neural_model_sha256(h).decode() if st == br.BLITZ_OK else None
    if h:
        lib.blitz_neural_model_destroy(h)
    return st, sha, err.value.decode()


@pytest.mark.parametrize("arch,width,use,prov", [(2, 64, 0, b""), (2, 128, 0, b"p" * 55), (3, 256, 0, b"q" * 56),
                                                 (4, 64, 1, b"r" * 119), (1, 64, 0, b"graph")])
def test_policy_files_load_with_their_sha256(tmp_path, arch, width, use, prov):
    data = blznet(arch, width, use, prov)
    f = tmp_path / "m.blzn"
    f.write_bytes(data)
    # the graph-encoder schema only allows the Learned ranking (generate.cpp:48-51)
    st, sha, msg = load(f, ranking=0 if arch == 1 else 3)
    assert st == br.BLITZ_OK, msg
    assert sha == hashlib.sha256(data).hexdigest()


def test_policy_files_are_checked(tmp_path):
    good = bytearray(blznet(2))
    bad = tmp_path / "bad.blzn"
    corrupt = bytearray(good)
    corrupt[40] ^= 1  # a weight byte: checksum mismatch
    bad.write_bytes(bytes(corrupt))
    assert load(bad)[0] == br.BLITZ_INVALID_ARGUMENT
    bad.write_bytes(blznet(2, count=policy_count(2, 64) - 1))  # wrong weight count
    assert load(bad)[0] == br.BLITZ_INVALID_ARGUMENT
    w = np.zeros(policy_count(2, 64), np.float32)
    w[7] = np.inf
    bad.write_bytes(blznet(2, weights=w))  # nonfinite weight, valid checksum
    assert load(bad)[0] == br.BLITZ_INVALID_ARGUMENT
    bad.write_bytes(bytes(good[:-1]))
    assert load(bad)[0] == br.BLITZ_INVALID_ARGUMENT
    bad.write_bytes(blznet(3, use=1))  # endpoint-reuse scope needs architecture 4
    assert load(bad)[0] == br.BLITZ_INVALID_ARGUMENT
    assert load(tmp_path / "missing.blzn")[0] == br.BLITZ_INVALID_ARGUMENT
    ok = tmp_path / "ok.blzn"
    ok.write_bytes(bytes(good))
    assert load(ok, preserve_uv=0)[0] == br.BLITZ_INVALID_ARGUMENT  # uv relaxation needs a v4 policy
    assert load(ok, action_batch=0)[0] == br.BLITZ_INVALID_ARGUMENT
    assert load(ok)[0] == br.BLITZ_OK


_ROOT = reference_root()
FIXTURE = None if _ROOT is None else _ROOT / "tests" / "fixtures" / "neural-cancellation" / "model.blzn"


@pytest.mark.skipif(FIXTURE is None or not FIXTURE.exists(), reason="reference model fixture absent")
def test_reference_policy_fixture_loads():
    """The reference's own BLZNET01 test model (tests/fixtures/neural-cancellation)."""
    st, sha, msg = load(FIXTURE, ranking=0)
    assert st == br.BLITZ_OK, msg
    assert sha == hashlib.sha256(FIXTURE.read_bytes()).hexdigest()


def test_settings_defaults_are_the_reference_defaults():
    """blitz_settings_init = blitz::Settings defaults (remesher.hpp:31-56,
    evaluate.hpp:8; c_api.cpp:82-122)."""
    s = br.settings()
    assert s.struct_size == C.sizeof(br.Settings) and s.abi_version == 5
    assert (s.levels, s.profile, s.objective, s.beam_width, s.candidate_budget) == (8, 1, 0, 8, 64)
    assert (s.triangle_overhead_bps, s.max_added_vertex_bytes_bps) == (0, 2000)
    assert (s.search_supersample, s.audit_supersample, s.max_supersample) == (4, 8, 32)
    assert (s.search_ortho, s.search_perspective, s.search_seed) == (42, 12, 0xB1172024)
    assert (s.audit_ortho, s.audit_perspective, s.audit_seed) == (642, 64, 0xB1172026)
    assert (s.pixels_per_meter, s.meters_per_unit, s.last_pixels, s.base_pixels, s.max_lod0_delta_px) == \
        (512.0, 1.0, 16.0, 0.0, 0.0)
    assert (s.max_changed_area, s.prune, s.force_scalar, s.coupled_wedges) == (1.0, 1, 0, 1)
    assert s.transition_count == 0 and not s.cancelled
    o = br.NeuralOptionsV1()
    assert br.load().blitz_neural_options_init(C.byref(o), C.sizeof(o)) == br.BLITZ_OK
    assert (o.struct_size, o.version, o.device, o.memory_mib, o.overdraw_tiebreak) == (C.sizeof(o), 1, 0, 6144, 1)


def test_classical_generation_is_unavailable():
    lib = br.load()
    out = C.c_void_p(1)
    err = C.create_string_buffer(256)
    assert lib.blitz_generate(None, None, C.byref(out), err, 256) == br.BLITZ_UNAVAILABLE
    assert not out.value and b"neural" in err.value
