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
