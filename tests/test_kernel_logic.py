"""CPU checks of the audit kernels' exact search logic (tests/kernel_logic.cpp):
the per-row coverage intervals equal face_covers sample by sample, and the
nearest-covered-sample search equals brute force. The C++ program is built
from the same headers as the CUDA library, with the library's FP64 flags."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_intervals_and_nearest_search(tmp_path):
    exe = tmp_path / "kernel_logic"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math",
                    str(HERE / "kernel_logic.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    lines = dict(l.split(" ", 1) for l in r.stdout.strip().splitlines())
    rows, bad_rows = map(int, lines["intervals"].split())
    queries, bad_queries = map(int, lines["nearest"].split())
    assert rows > 20_000 and queries == 12_000
    assert bad_rows == 0 and bad_queries == 0
    assert r.returncode == 0


CUDA_INCLUDE = Path("/usr/local/cuda/include")


@pytest.mark.skipif(shutil.which("g++") is None or not (CUDA_INCLUDE / "vector_types.h").exists(),
                    reason="needs g++ and the CUDA vector-type headers")
def test_uv_projection_matches_oracle_and_definition(tmp_path):
    """The uv transport's closest-point weights (csrc/placement.cuh) equal
    the oracle's bit for bit on 20,000 random cases (collinear and repeated
    corners included) and are the closest point of the triangle."""
    from oracle.oracle import HERE as ORACLE, build

    if not (ORACLE / "liboracle.so").exists():
        build(ref=False)
    exe = tmp_path / "placement_logic"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", f"-I{CUDA_INCLUDE}",
                    str(HERE / "placement_logic.cpp"), f"-L{ORACLE}", "-loracle", f"-Wl,-rpath,{ORACLE}",
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    cases, mismatch, not_closest = map(int, r.stdout.split()[1:4])
    assert cases == 20_000 and mismatch == 0 and not_closest == 0
    assert r.returncode == 0


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_view_measurement_matches_oracle(tmp_path):
    """finish_view and bounded_refinement (csrc/common.cuh, run by the verdict
    kernel) equal the oracle's restatements bit for bit on 200,000 random view
    records (clipped, empty-side, same-mask, conservative-screen cases) and
    11,628 refinement bounds."""
    from oracle.oracle import HERE as ORACLE, build

    if not (ORACLE / "liboracle.so").exists():
        build(ref=False)
    exe = tmp_path / "verdict_logic"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math",
                    str(HERE / "verdict_logic.cpp"), f"-L{ORACLE}", "-loracle", f"-Wl,-rpath,{ORACLE}",
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    lines = dict(l.split(" ", 1) for l in r.stdout.strip().splitlines())
    cases, bad = map(int, lines["finish_view"].split())
    rcases, rbad = map(int, lines["refinement"].split())
    assert cases == 200_000 and bad == 0 and rcases > 10_000 and rbad == 0
    assert r.returncode == 0


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_distance_field_values_match_oracle(tmp_path):
    """On a 4160 x 4160 raster: exact integer squared distances below 2^24,
    and cpu_field_value's float roundings from 2^24 up (csrc/common.cuh, the
    audit's full-raster path), equal the oracle's float distance field."""
    from oracle.oracle import HERE as ORACLE, build

    if not (ORACLE / "liboracle.so").exists():
        build(ref=False)
    exe = tmp_path / "field_logic"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math",
                    str(HERE / "field_logic.cpp"), f"-L{ORACLE}", "-loracle", f"-Wl,-rpath,{ORACLE}",
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    n, bad_exact, bad_round, rounded = map(int, r.stdout.split()[1:5])
    assert n == 3000 and rounded > 500 and bad_exact == 0 and bad_round == 0
    assert r.returncode == 0
