"""The chain's schedule in the library (blitz_chain_schedule, the code that
blitz_audit_chain runs) against the oracle's restatement of blitz::schedule
(chain.cpp:101-118) and against the reference's own blitz::schedule
(oracle/_ref/schedule_ref, built from src/chain.cpp): per level the audited
screen size, the transition bound and the capped LOD0 bound, bit for bit.
CPU only."""
import subprocess

import numpy as np
import pytest

import blitzremesher_b200 as br
from oracle.oracle import HERE as ORACLE_DIR

SCHEDULE_REF = ORACLE_DIR / "_ref" / "schedule_ref"

CASES = [
    (6, 1024.0, 32.0, ((0.0, 1.0), (1.0, 3.0)), 2.0),
    (6, 240.0, 7.5, ((0.0, 1.0), (1.0, 3.0)), 2.0),
    (2, 24.0, 24.0, ((0.0, 1.0), (1.0, 1.0)), 2.0),
    (4, 48.0, 12.0, ((0.0, 1.0), (1.0, 3.0)), 2.0),
    (9, 2048.0, 16.0, ((0.0, 0.5), (0.3, 1.0), (0.8, 2.5), (1.0, 4.0)), 0.0),
    (32, 16384.0, 1.0, ((0.0, 2.0), (0.5, 1.0), (1.0, 0.25)), 5.0),
    (3, 100.0, 99.0, ((0.0, 1.5), (0.2, 1.5), (0.9, 0.5), (1.0, 0.5)), 1.0),
]


@pytest.mark.parametrize("levels,base,last,curve,lod0", CASES)
def test_schedule_matches_oracle(oracle, levels, base, last, curve, lod0):
    s = br.chain_settings(levels, base, last, curve, lod0)
    p, t, b = br.chain_schedule(s)
    # the settings keep the curve as float32: the oracle gets the same values
    want = oracle.schedule(base, last, levels, np.asarray(curve, np.float32), lod0)
    for got, exp in zip((p, t, b), want):
        assert np.array_equal(got, exp), (got, exp)


@pytest.mark.parametrize("levels,base,last,curve,lod0", [
    (6, 24.0, 48.0, ((0.0, 1.0), (1.0, 3.0)), 2.0),  # base below last
    (3, 100.0, 99.0, ((0.2, 1.5), (0.9, 0.5)), 1.0),  # curve not spanning [0, 1]
    (3, 100.0, 99.0, ((0.0, 1.0),), 1.0),
    (3, 100.0, 99.0, ((0.0, 1.0), (0.5, 2.0), (0.5, 3.0), (1.0, 1.0)), 1.0),  # x not increasing
    (3, 100.0, 99.0, ((0.0, -1.0), (1.0, 1.0)), 1.0),  # negative bound
    (1, 100.0, 99.0, ((0.0, 1.0), (1.0, 1.0)), 1.0),  # one level
])
def test_schedule_rejects_bad_settings(levels, base, last, curve, lod0):
    """Settings the reference's validation refuses (chain.cpp:37-94) are
    refused here too; the reference's own schedule is run on them where it is
    present and must refuse them as well."""
    s = br.chain_settings(levels, base, last, curve, lod0)
    with pytest.raises(br.BlitzError) as exc:
        br.chain_schedule(s)
    assert exc.value.status == br.BLITZ_INVALID_ARGUMENT
    if SCHEDULE_REF.exists():
        args = [str(SCHEDULE_REF), str(levels), repr(base), repr(last), repr(lod0)]
        for x, y in curve:
            args += [repr(x), repr(y)]
        if len(curve) == 1:
            return  # the runner's command line needs two points
        assert subprocess.run(args, capture_output=True, text=True).returncode == 1


@pytest.mark.skipif(not SCHEDULE_REF.exists(), reason="reference schedule runner (oracle/_ref) absent")
@pytest.mark.parametrize("levels,base,last,curve,lod0", CASES)
def test_schedule_matches_reference(oracle, levels, base, last, curve, lod0):
    args = [str(SCHEDULE_REF), str(levels), repr(base), repr(last), repr(lod0)]
    for x, y in curve:
        args += [repr(float(np.float32(x))), repr(float(np.float32(y)))]
    out = subprocess.run(args, capture_output=True, text=True, check=True).stdout.split()
    ref = np.array([float.fromhex(v) for v in out]).reshape(-1, 3)
    s = br.chain_settings(levels, base, last, curve, lod0)
    p, t, b = br.chain_schedule(s)
    assert np.array_equal(p, ref[:, 0]) and np.array_equal(t, ref[:, 1]) and np.array_equal(b, ref[:, 2])
    want = oracle.schedule(base, last, levels, np.asarray(curve, np.float32), lod0)
    assert all(np.array_equal(w, ref[:, k]) for k, w in enumerate(want))
