"""The allocation-free coverage distance against the session entry point.

blitz_audit_coverage_distance_static serves callers that may not call
cudaMalloc (their device memory belongs to another allocator, or the loop must
not synchronise on allocation): its scratch is a static device array, its
inputs and output are caller-owned device buffers. This file is collected
last so a run that stops at the first failure has already run every other
test; it also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _blob_mask(rng, width, height, blobs):
    yy, xx = np.mgrid[0:height, 0:width]
    m = np.zeros((height, width), bool)
    for _ in range(blobs):
        cx, cy, r = rng.uniform(0, width), rng.uniform(0, height), rng.uniform(2, width / 6)
        m |= (xx - cx) ** 2 + (yy - cy) ** 2 < r * r
    bits = np.packbits(m.reshape(-1), bitorder="little")
    bits = np.concatenate([bits, np.zeros((-bits.size) % 8, np.uint8)])
    return bits.view(np.uint64)


def _static_distance(lib, a, b, width, height, ss):
    import torch

    da = torch.from_numpy(a.view(np.uint8).copy()).cuda()
    db = torch.from_numpy(b.view(np.uint8).copy()).cuda()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    err = C.create_string_buffer(256)
    st = lib.blitz_audit_coverage_distance_static(C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), width,
                                                  height, ss, C.c_void_p(out.data_ptr()), None, err, 256)
    torch.cuda.synchronize()
    return st, out.item(), err.value.decode()


def _bind(lib):
    fn = lib.blitz_audit_coverage_distance_static
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint8, C.c_void_p, C.c_void_p, C.c_char_p,
                   C.c_size_t]
    fn.restype = C.c_int


def test_static_scratch_matches_session_entry_point(gpu_lib, oracle):
    lib = br.load()
    _bind(lib)
    rng = np.random.default_rng(23)
    with br.AuditSession(syn.noisy_icosphere(1, 1)) as s:
        # Two calls in a row on different shapes: the second must not see the
        # first call's leftovers in the shared scratch. Each result is also
        # the oracle's (the reference's coverage distance restated on the CPU).
        for width, height, ss, blobs in ((257, 190, 1, 4), (512, 512, 8, 3), (13, 11, 2, 1)):
            a = _blob_mask(rng, width, height, blobs)
            b = _blob_mask(rng, width, height, blobs + 1)
            want = s.coverage_distance(a, b, width, height, ss)
            st, got, msg = _static_distance(lib, a, b, width, height, ss)
            assert st == br.BLITZ_OK, msg
            assert got == want, (width, height, ss, got, want)
            assert got == oracle.coverage_distance(a, b, width, height, ss)
        # Equal masks and one empty mask keep the session's semantics.
        a = _blob_mask(rng, 64, 64, 2)
        empty = np.zeros_like(a)
        assert _static_distance(lib, a, a, 64, 64, 1)[1] == s.coverage_distance(a, a, 64, 64, 1) == 0
        assert np.isinf(_static_distance(lib, a, empty, 64, 64, 1)[1])


def test_static_scratch_rejects_oversized_masks(gpu_lib):
    lib = br.load()
    _bind(lib)
    a = np.zeros((513 * 512 + 63) // 64, np.uint64)
    st, got, msg = _static_distance(lib, a, a, 513, 512, 1)
    assert st == br.BLITZ_INVALID_ARGUMENT and "512 x 512" in msg
    assert got == -1.0


def test_static_scratch_ignores_bits_past_the_last_sample(gpu_lib):
    """Bits set at or past width x height in the last word are not samples:
    the result equals that of the same masks with those bits cleared."""
    lib = br.load()
    _bind(lib)
    rng = np.random.default_rng(5)
    width, height, ss = 13, 11, 1  # 143 samples: the last u64 word holds 49 non-samples
    a = _blob_mask(rng, width, height, 2)
    b = _blob_mask(rng, width, height, 3)
    tail = ~np.uint64((1 << (width * height - 64 * (a.size - 1))) - 1)
    dirty_a, dirty_b = a.copy(), b.copy()
    dirty_a[-1] |= tail
    dirty_b[-1] |= tail & np.uint64(0x5555555555555555)
    st, clean, msg = _static_distance(lib, a, b, width, height, ss)
    assert st == br.BLITZ_OK, msg
    st, dirty, msg = _static_distance(lib, dirty_a, dirty_b, width, height, ss)
    assert st == br.BLITZ_OK, msg
    assert dirty == clean
    # Equal samples with different tails are still equal masks: distance 0.
    st, same, msg = _static_distance(lib, a, dirty_a, width, height, ss)
    assert st == br.BLITZ_OK and same == 0.0, msg
