"""The chain's schedule in the library (blitz_chain_schedule, the code that
blitz_audit_chain runs) against the oracle's restatement of blitz::schedule
(chain.cpp:101-118): per level the audited screen size, the transition bound
and the capped LOD0 bound, bit for bit. CPU only."""
import numpy as np
import pytest

import blitzremesher_b200 as br

CASES = [
    (6, 1024.0, 32.0, ((0.0, 1.0), (1.0, 3.0)), 2.0),
    (6, 240.0, 7.5, ((0.0, 1.0), (1.0, 3.0)), 2.0),
    (2, 24.0, 24.0, ((0.0, 1.0),), 2.0),
    (4, 48.0, 12.0, ((0.0, 1.0), (1.0, 3.0)), 2.0),
    (9, 2048.0, 16.0, ((0.0, 0.5), (0.3, 1.0), (0.8, 2.5), (1.0, 4.0)), 0.0),
    (32, 16384.0, 1.0, ((0.0, 2.0), (0.5, 1.0), (1.0, 0.25)), 5.0),
    (3, 100.0, 99.0, ((0.2, 1.5), (0.9, 0.5)), 1.0),
]


@pytest.mark.parametrize("levels,base,last,curve,lod0", CASES)
def test_schedule_matches_oracle(oracle, levels, base, last, curve, lod0):
    s = br.chain_settings(levels, base, last, curve, lod0)
    p, t, b = br.chain_schedule(s)
    # the settings keep the curve as float32: the oracle gets the same values
    want = oracle.schedule(base, last, levels, np.asarray(curve, np.float32), lod0)
    for got, exp in zip((p, t, b), want):
        assert np.array_equal(got, exp), (got, exp)


def test_schedule_rejects_bad_settings():
    s = br.chain_settings(6, 24.0, 48.0)  # base below last
    with pytest.raises(br.BlitzError) as exc:
        br.chain_schedule(s)
    assert exc.value.status == br.BLITZ_INVALID_ARGUMENT
