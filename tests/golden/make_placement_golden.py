"""Generates tests/golden/placement_ref.npz from the reference's own GPU
placement path (oracle/_ref/placement_ref: GpuActionState::trial with the
midpoint placement, src/neural/action_gpu.cu place_vertices 962-1067 and
validate_placement 1103-1156, built from the reference sources for sm_100a).

Needs a CUDA device. For seamed spheres, tori and heightfields, a rock with
8 uv charts and ribbon cards, each with and without preserve_uv, every k-th
legal action's trial is recorded: validity, face count, a SHA-256 of the
trial indices, and every vertex slot whose position or uv changed (slot,
position, uv).

    python tests/golden/make_placement_golden.py
"""
from __future__ import annotations

import hashlib
import struct
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "placement_ref.npz"
DRIVER = ROOT / "oracle" / "_ref" / "placement_ref"
TRIALS = 28


def cases():
    from blitzremesher_b200 import synthetic as syn

    meshes = {"torus": syn.seamed_torus(1200, 4, 6), "sphere": syn.seamed_sphere(800, 3),
              "heightfield": syn.seamed_heightfield(1000, 5, 4), "rock": syn.rock(2, 3),
              "ribbons": syn.ribbons(12, seed=6)}
    return [(name, mesh, preserve) for name, mesh in meshes.items() for preserve in (0, 1)]


def run_reference(mesh, preserve_uv: int, stride: int, tmp: Path):
    nv, nf = mesh.vertex_count, mesh.face_count
    has_uv = int(mesh.uv is not None)
    data = struct.pack("<5I", nv, nf, has_uv, preserve_uv, stride)
    data += np.ascontiguousarray(mesh.positions, np.float32).tobytes()
    if has_uv:
        data += np.ascontiguousarray(mesh.uv, np.float32).tobytes()
    data += np.ascontiguousarray(mesh.indices, np.uint32).tobytes()
    (tmp / "in.bin").write_bytes(data)
    subprocess.run([str(DRIVER), str(tmp / "in.bin"), str(tmp / "out.bin")], check=True)
    raw = (tmp / "out.bin").read_bytes()
    at, rows = 0, []
    while at < len(raw):
        frm, to, valid, faces = struct.unpack_from("<4I", raw, at)
        at += 16
        idx = pos = uv = None
        if valid:
            idx = np.frombuffer(raw, np.uint32, faces * 3, at)
            at += faces * 12
            pos = np.frombuffer(raw, np.float32, nv * 3, at).reshape(-1, 3)
            at += nv * 12
            if has_uv:
                uv = np.frombuffer(raw, np.float32, nv * 2, at).reshape(-1, 2)
                at += nv * 8
        rows.append((frm, to, valid, faces, idx, pos, uv))
    return rows


def changed_slots(mesh, pos, uv):
    moved = np.any(pos.view(np.uint32) != np.ascontiguousarray(mesh.positions, np.float32).view(np.uint32), axis=1)
    if uv is not None:
        moved |= np.any(uv.view(np.uint32) != np.ascontiguousarray(mesh.uv, np.float32).view(np.uint32), axis=1)
    return np.nonzero(moved)[0].astype(np.uint32)


def main() -> None:
    from oracle.oracle import Oracle

    O = Oracle()
    out = {}
    with tempfile.TemporaryDirectory() as d:
        tmp = Path(d)
        for name, mesh, preserve in cases():
            legal = len(O.actions(mesh, placement=True, preserve_uv=bool(preserve)))
            stride = max(1, legal // TRIALS)
            rows = run_reference(mesh, preserve, stride, tmp)
            key = f"{name}_uv{preserve}"
            ft, valid, faces, sha, slots, spos, suv, count = [], [], [], [], [], [], [], []
            for frm, to, ok, nfaces, idx, pos, uv in rows:
                ft.append((frm, to))
                valid.append(ok)
                faces.append(nfaces)
                if ok:
                    sha.append(hashlib.sha256(idx.tobytes()).hexdigest()[:32])
                    c = changed_slots(mesh, pos, uv)
                    slots.append(c)
                    spos.append(pos[c])
                    suv.append(uv[c] if uv is not None else np.zeros((c.size, 2), np.float32))
                    count.append(c.size)
                else:
                    sha.append("")
                    count.append(0)
            out[f"{key}_from_to"] = np.array(ft, np.uint32)
            out[f"{key}_valid"] = np.array(valid, np.uint8)
            out[f"{key}_faces"] = np.array(faces, np.uint32)
            out[f"{key}_sha"] = np.array(sha)
            out[f"{key}_count"] = np.array(count, np.uint32)
            out[f"{key}_slots"] = np.concatenate(slots) if slots else np.zeros(0, np.uint32)
            out[f"{key}_positions"] = np.concatenate(spos) if spos else np.zeros((0, 3), np.float32)
            out[f"{key}_uv"] = np.concatenate(suv) if suv else np.zeros((0, 2), np.float32)
            print(f"{key}: {len(rows)} trials, {sum(valid)} valid")
    np.savez_compressed(OUT, **out)


if __name__ == "__main__":
    main()
