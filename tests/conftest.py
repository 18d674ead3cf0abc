import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


FIELDS = ["error", "coverage", "coverage_upper", "changed_area", "normal_degrees", "worst_view",
          "changed_area_worst_view", "views_evaluated", "supersample", "complete", "passed", "resource_limited",
          "cancelled"]


def measurement_fields(m) -> tuple:
    """Every Measurement field, doubles as bit patterns (padding excluded)."""
    import struct

    if hasattr(m, "dtype"):  # numpy record
        get = lambda k: m[k].item()  # noqa: E731
    else:
        get = lambda k: getattr(m, k)  # noqa: E731
    out = []
    for k in FIELDS:
        v = get(k)
        out.append(struct.pack("<d", v) if k in FIELDS[:5] else int(v))
    return tuple(out)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference

    if not Reference.available():
        pytest.skip("reference CPU build (oracle/_ref) absent")
    return Reference()


@pytest.fixture(scope="session")
def gpu_lib():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blitzremesher_b200 as br

    return br.load()
