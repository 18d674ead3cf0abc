"""CPU check of the library's collapse legality (csrc/legality.cuh, compiled
for the host by tests/legality_logic.cpp): on closed, open, seamed,
multi-material and broken meshes the legal edits, their wedge maps and
removed-face counts equal the oracle's legality with placement
(action_gpu.cu:487-624 restated), edit for edit in enumeration order."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from blitzremesher_b200 import synthetic as syn

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def legality(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    lib = tmp_path_factory.mktemp("legality") / "liblegality.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                    str(HERE / "legality_logic.cpp"), "-o", str(lib)], check=True)
    L = C.CDLL(str(lib))
    L.legality_actions.restype = C.c_int64
    L.legality_actions.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                   C.c_uint64]

    def run(mesh):
        pos = np.ascontiguousarray(mesh.positions, np.float32)
        idx = np.ascontiguousarray(mesh.indices, np.uint32)
        mat = None if mesh.materials is None else np.ascontiguousarray(mesh.materials, np.uint16)
        cap = 6 * mesh.face_count + 6
        out = np.zeros((cap, 7), np.uint32)
        n = L.legality_actions(pos.ctypes.data, pos.shape[0], idx.ctypes.data, idx.size // 3,
                               None if mat is None else mat.ctypes.data, out.ctypes.data, cap)
        assert 0 <= n <= cap
        return out[:n]

    return run


def _mesh(pos, faces, materials=None):
    return syn.Mesh(np.asarray(pos, np.float32), np.asarray(faces, np.uint32).reshape(-1),
                    materials=None if materials is None else np.asarray(materials, np.uint16))


def _special_meshes():
    tetra = _mesh([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], [[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])
    # Two fans meeting at vertex 0 only (bow-tie): vertex 0 is not one fan.
    bowtie = _mesh([[0, 0, 0], [1, 0, 0], [1, 1, 0], [-1, 0, 0], [-1, -1, 0], [2, 0.5, 0], [-2, -0.5, 0]],
                   [[0, 1, 2], [1, 5, 2], [0, 3, 4], [3, 6, 4]])
    # Three faces on one edge (non-manifold).
    fin = _mesh([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [1, 1, 1]],
                [[0, 1, 2], [1, 0, 3], [0, 1, 4], [1, 2, 5]])
    # A face with two corners at one position (degenerate in classes).
    degen = _mesh([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 0, 0], [1, 1, 0]], [[0, 1, 2], [1, 3, 4], [1, 4, 2]])
    # Materials by hemisphere and by face parity band on an icosphere.
    ico = syn.noisy_icosphere(2, 3)
    f = ico.indices.reshape(-1, 3)
    z = ico.positions[f].mean(axis=1)[:, 2]
    two_mat = ico.copy()
    two_mat.materials = (z > 0).astype(np.uint16)
    three_mat = ico.copy()
    three_mat.materials = np.digitize(z, [-0.3, 0.3]).astype(np.uint16)
    return {"tetra": tetra, "bowtie": bowtie, "fin": fin, "degenerate": degen, "two_materials": two_mat,
            "three_materials": three_mat}


CASES = {
    "icosphere3": lambda: syn.noisy_icosphere(3, 2),
    "grid6": lambda: syn.grid(6),
    "seamed_torus": lambda: syn.seamed_torus(3000, 4, 6),
    "seamed_heightfield": lambda: syn.seamed_heightfield(2500, 5, 4),
    "seamed_sphere": lambda: syn.seamed_sphere(2000, 3),
    "ribbons": lambda: syn.ribbons(40, seed=6),
}
CASES.update({k: (lambda m=m: m) for k, m in _special_meshes().items()})


@pytest.mark.parametrize("name", sorted(CASES))
def test_legal_edits_match_oracle(legality, oracle, name):
    mesh = CASES[name]()
    got = legality(mesh)
    want = oracle.actions(mesh, placement=True)
    assert got.shape[0] == len(want), (name, got.shape[0], len(want))
    for row, e in zip(got, want):
        w = int(e.wedges)
        assert (row[0], row[1]) == (e.from_, e.to)
        assert row[6] & 0xFF == w and row[6] >> 8 == e.removed, (name, e.from_, e.to)
        assert list(row[2:2 + w]) == list(e.source)[:w] and list(row[4:4 + w]) == list(e.target)[:w]


def test_broken_meshes_lose_their_edits(legality):
    """The rule is not vacuous on the broken meshes: the tetrahedron, the
    bow-tie centre and the non-manifold edge allow none of the collapses the
    fan and link rules forbid."""
    m = _special_meshes()
    assert legality(m["tetra"]).shape[0] == 0
    bow = legality(m["bowtie"])
    assert not np.any(bow[:, :2] == 0)
    fin = legality(m["fin"])
    assert not np.any((fin[:, 0] <= 1) & (fin[:, 1] <= 1))
