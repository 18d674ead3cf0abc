"""Seeded synthetic meshes for the audit workloads.

The generators produce float32 positions, uint32 triangle indices (outward,
counter-clockwise) and optional float32 UVs. Every random draw comes from a
SplitMix64 stream keyed by the seed, so a mesh is identical across processes
and machines.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

MASK64 = (1 << 64) - 1


def splitmix64(seed: int, count: int) -> np.ndarray:
    """``count`` SplitMix64 outputs for ``seed`` (uint64)."""
    out = np.empty(count, dtype=np.uint64)
    x = seed & MASK64
    for i in range(count):
        x = (x + 0x9E3779B97F4A7C15) & MASK64
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        out[i] = z ^ (z >> 31)
    return out


def uniform(seed: int, count: int, lo: float, hi: float) -> np.ndarray:
    """Doubles uniform in [lo, hi) from the top 53 bits of SplitMix64."""
    u = (splitmix64(seed, count) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    return lo + (hi - lo) * u


@dataclass
class Mesh:
    """Host mesh in the layout the C ABI borrows (blitz_mesh streams)."""

    positions: np.ndarray  # (V,3) float32
    indices: np.ndarray  # (F*3,) uint32
    uv: Optional[np.ndarray] = None  # (V,2) float32
    materials: Optional[np.ndarray] = None  # (F,) uint16
    double_sided: Optional[np.ndarray] = None  # (M,) uint8
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def vertex_count(self) -> int:
        return int(self.positions.shape[0])

    @property
    def face_count(self) -> int:
        return int(self.indices.size // 3)

    def copy(self) -> "Mesh":
        return Mesh(
            self.positions.copy(),
            self.indices.copy(),
            None if self.uv is None else self.uv.copy(),
            None if self.materials is None else self.materials.copy(),
            None if self.double_sided is None else self.double_sided.copy(),
            self.name,
            dict(self.meta),
        )


def _orient_outward(pos: np.ndarray, faces: np.ndarray, center=(0.0, 0.0, 0.0)) -> np.ndarray:
    a, b, c = pos[faces[:, 0]], pos[faces[:, 1]], pos[faces[:, 2]]
    n = np.cross(b - a, c - a)
    centroid = (a + b + c) / 3.0 - np.asarray(center)
    flip = (n * centroid).sum(1) < 0
    faces = faces.copy()
    faces[flip, 1], faces[flip, 2] = faces[flip, 2].copy(), faces[flip, 1].copy()
    return faces


def icosphere(level: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20*4^level faces, 10*4^level+2 vertices (float64, int64)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
             (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    pos = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    f = np.array(faces, dtype=np.int64)
    for _ in range(level):
        cache: dict = {}

        def mid(i: int, j: int) -> int:
            key = (i, j) if i < j else (j, i)
            if key not in cache:
                p = pos[i] + pos[j]
                pos.append(p / np.linalg.norm(p))
                cache[key] = len(pos) - 1
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = np.array(nf, dtype=np.int64)
    p = np.stack(pos)
    return p, _orient_outward(p, f)


def noisy_icosphere(level: int = 5, seed: int = 1, amplitude: float = 0.02, radius: float = 1.0) -> Mesh:
    """Icosphere with per-vertex radial noise r*(1+u), u ~ U[-amplitude, amplitude]."""
    p, f = icosphere(level)
    u = uniform(seed, p.shape[0], -amplitude, amplitude)
    pos = (p * (radius * (1.0 + u))[:, None]).astype(np.float32)
    return Mesh(pos, f.astype(np.uint32).reshape(-1), name=f"icosphere{level}-seed{seed}",
                meta={"level": level, "seed": seed, "amplitude": amplitude})


def grid(n: int, scale: float = 1.0, bend: float = 0.0, two_sided: bool = True) -> Mesh:
    """Planar (n x n)-cell grid used by the reference precision fixtures."""
    pos, uv = [], []
    for y in range(n + 1):
        for x in range(n + 1):
            u, v = np.float32(x) / np.float32(n), np.float32(y) / np.float32(n)
            pos.append((np.float32(scale) * (u + np.float32(8)), np.float32(scale) * (v - np.float32(8)),
                        np.float32(scale) * np.float32(bend) * u * v))
            uv.append((u * np.float32(4) - np.float32(2), v * np.float32(3) - np.float32(1)))
    idx = []
    for y in range(n):
        for x in range(n):
            a = y * (n + 1) + x
            b, c = a + 1, a + n + 1
            d = c + 1
            idx += [a, b, d, a, d, c]
    return Mesh(np.array(pos, dtype=np.float32), np.array(idx, dtype=np.uint32),
                uv=np.array(uv, dtype=np.float32),
                double_sided=np.array([1 if two_sided else 0], dtype=np.uint8), name=f"grid{n}")


def config1_mesh(seed: int = 1) -> Mesh:
    """Plain-audit workload mesh: icosphere level 5 (20,480 faces), +-2% radial noise."""
    return noisy_icosphere(5, seed, 0.02)
