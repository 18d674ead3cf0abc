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


# ---------------------------------------------------------------------------
# Batched-audit mesh set: noise-displaced spheres, tori (R/r = 3) and open
# heightfield grids, each with FP32 UVs split into 4-16 charts. A chart seam
# duplicates its vertices (same position, different UV), so the position weld
# joins them into one geometric class with two wedges.

def _hash3(ix, iy, iz, seed: int) -> np.ndarray:
    """Vectorised 64-bit lattice hash -> doubles in [0, 1)."""
    with np.errstate(over="ignore"):
        h = (ix.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)) ^ \
            (iy.astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F)) ^ \
            (iz.astype(np.uint64) * np.uint64(0x165667B19E3779F9)) ^ np.uint64(seed * 0x27D4EB2F165667C5 & MASK64)
        h ^= h >> np.uint64(30)
        h *= np.uint64(0xBF58476D1CE4E5B9)
        h ^= h >> np.uint64(27)
        h *= np.uint64(0x94D049BB133111EB)
        h ^= h >> np.uint64(31)
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def value_noise(p: np.ndarray, seed: int, octaves: int = 4, frequency: float = 2.0) -> np.ndarray:
    """Sum of `octaves` octaves of trilinear value noise (smoothstep weights),
    amplitude halving and frequency doubling per octave, in about [-1, 1]."""
    p = np.asarray(p, np.float64)
    if p.shape[1] == 2:
        p = np.concatenate([p, np.zeros((p.shape[0], 1))], 1)
    total = np.zeros(p.shape[0])
    amp, norm = 1.0, 0.0
    for o in range(octaves):
        q = p * frequency * (2 ** o)
        i = np.floor(q).astype(np.int64)
        f = q - i
        w = f * f * (3 - 2 * f)
        acc = np.zeros(p.shape[0])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    h = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed + 7919 * o)
                    wx = w[:, 0] if dx else 1 - w[:, 0]
                    wy = w[:, 1] if dy else 1 - w[:, 1]
                    wz = w[:, 2] if dz else 1 - w[:, 2]
                    acc += (2 * h - 1) * wx * wy * wz
        total += amp * acc
        norm += amp
        amp *= 0.5
    return total / norm


def _cuts(n: int, parts: int) -> list:
    parts = max(1, min(parts, n))
    return [round(k * n / parts) for k in range(parts + 1)]


def _chart_grid(nu: int, nv: int, cuts_u: list, cuts_v: list, position, wrap_u: bool, wrap_v: bool):
    """Grid of nu x nv cells split into charts at the cut lines. `position(i, j)`
    maps integer lattice coordinates (already wrapped) to (k, 3) float32
    positions. Each chart owns its vertices; its UVs tile an atlas."""
    pos, uv, faces = [], [], []
    base = 0
    cu, cv = len(cuts_u) - 1, len(cuts_v) - 1
    for a in range(cu):
        for b in range(cv):
            u0, u1, v0, v1 = cuts_u[a], cuts_u[a + 1], cuts_v[b], cuts_v[b + 1]
            ii, jj = np.meshgrid(np.arange(u0, u1 + 1), np.arange(v0, v1 + 1), indexing="ij")
            ii, jj = ii.reshape(-1), jj.reshape(-1)
            wi = ii % nu if wrap_u else ii
            wj = jj % nv if wrap_v else jj
            pos.append(position(wi, wj))
            tile_u = (a + (ii - u0) / max(1, u1 - u0) * 0.9) / cu
            tile_v = (b + (jj - v0) / max(1, v1 - v0) * 0.9) / cv
            uv.append(np.stack([tile_u, tile_v], 1).astype(np.float32))
            w = v1 - v0 + 1
            ci, cj = np.meshgrid(np.arange(u1 - u0), np.arange(v1 - v0), indexing="ij")
            ci, cj = ci.reshape(-1), cj.reshape(-1)
            p00 = base + ci * w + cj
            p10, p01 = p00 + w, p00 + 1
            p11 = p10 + 1
            faces.append(np.stack([np.stack([p00, p10, p11], 1), np.stack([p00, p11, p01], 1)], 1).reshape(-1, 3))
            base += ii.size
    return np.concatenate(pos).astype(np.float32), np.concatenate(faces), np.concatenate(uv)


def _orient_by(pos: np.ndarray, faces: np.ndarray, outward: np.ndarray) -> np.ndarray:
    """Flips faces whose normal points against `outward` (per face)."""
    a, b, c = pos[faces[:, 0]].astype(np.float64), pos[faces[:, 1]].astype(np.float64), pos[faces[:, 2]].astype(
        np.float64)
    n = np.cross(b - a, c - a)
    flip = (n * outward).sum(1) < 0
    faces = faces.copy()
    faces[flip, 1], faces[flip, 2] = faces[flip, 2].copy(), faces[flip, 1].copy()
    return faces


def seamed_sphere(target_faces: int, seed: int, amplitude: float = 0.05) -> Mesh:
    """Cube-sphere (each cube face a chart, or two) with value-noise radial
    displacement; about target_faces faces (12 n^2)."""
    n = max(2, int(round((target_faces / 12) ** 0.5)))
    split = int(splitmix64(seed ^ 0x5EA, 1)[0] % np.uint64(2)) + 1  # 6 or 12 charts
    pos, faces, uv = [], [], []
    base = 0
    axes = [(0, 1, 2, 1.0), (0, 1, 2, -1.0), (1, 2, 0, 1.0), (1, 2, 0, -1.0), (2, 0, 1, 1.0), (2, 0, 1, -1.0)]
    for k, (ax, a1, a2, sign) in enumerate(axes):
        def position(i, j, ax=ax, a1=a1, a2=a2, sign=sign):
            c = np.zeros((i.size, 3))
            c[:, ax] = sign
            c[:, a1] = -1.0 + 2.0 * i / n
            c[:, a2] = -1.0 + 2.0 * j / n
            d = c / np.linalg.norm(c, axis=1, keepdims=True)
            r = 1.0 + amplitude * value_noise(d, seed)
            return (d * r[:, None]).astype(np.float32)
        p, f, t = _chart_grid(n, n, _cuts(n, split), [0, n], position, False, False)
        t = (t + np.array([k % 3, k // 3], np.float32)) / np.array([3, 2], np.float32)
        pos.append(p)
        faces.append(f + base)
        uv.append(t.astype(np.float32))
        base += p.shape[0]
    pos = np.concatenate(pos)
    faces = np.concatenate(faces)
    cent = pos[faces].astype(np.float64).mean(1)
    faces = _orient_by(pos, faces, cent)
    return Mesh(pos, faces.astype(np.uint32).reshape(-1), uv=np.concatenate(uv), name=f"sphere-{seed}",
                meta={"kind": "sphere", "charts": 6 * split, "seed": seed})


def seamed_torus(target_faces: int, seed: int, charts: int, amplitude: float = 0.02) -> Mesh:
    """Torus with R/r = 3 (R = 0.75, r = 0.25), nu = 3 nv cells, charts cut
    along both directions, light value-noise displacement."""
    nv = max(3, int(round((target_faces / 6) ** 0.5)))
    nu = 3 * nv
    cu = max(2, min(charts // 2, nu))
    cv = max(1, charts // cu)
    R, r = 0.75, 0.25

    def position(i, j):
        tu, tv = 2 * np.pi * i / nu, 2 * np.pi * j / nv
        base = np.stack([np.cos(tu), np.sin(tu), np.zeros_like(tu)], 1)
        p = base * (R + r * np.cos(tv))[:, None]
        p[:, 2] = r * np.sin(tv)
        return (p * (1.0 + amplitude * value_noise(p, seed))[:, None]).astype(np.float32)

    pos, faces, uv = _chart_grid(nu, nv, _cuts(nu, cu), _cuts(nv, cv), position, True, True)
    c = pos[faces].astype(np.float64).mean(1)
    ring = c.copy()
    ring[:, 2] = 0
    ring = ring / np.linalg.norm(ring, axis=1, keepdims=True) * R
    faces = _orient_by(pos, faces, c - ring)
    return Mesh(pos, faces.astype(np.uint32).reshape(-1), uv=uv, name=f"torus-{seed}",
                meta={"kind": "torus", "charts": cu * cv, "seed": seed})


def seamed_heightfield(target_faces: int, seed: int, charts: int, height: float = 0.15) -> Mesh:
    """Open n x n grid over [-1, 1]^2 with 4-octave value-noise heights."""
    n = max(2, int(round((target_faces / 2) ** 0.5)))
    cu = max(2, int(round(charts ** 0.5)))
    cv = max(2, charts // cu)

    def position(i, j):
        x, y = -1.0 + 2.0 * i / n, -1.0 + 2.0 * j / n
        z = height * value_noise(np.stack([x, y], 1), seed, octaves=4)
        return np.stack([x, y, z], 1).astype(np.float32)

    pos, faces, uv = _chart_grid(n, n, _cuts(n, cu), _cuts(n, cv), position, False, False)
    up = np.zeros((faces.shape[0], 3))
    up[:, 2] = 1
    faces = _orient_by(pos, faces, up)
    return Mesh(pos, faces.astype(np.uint32).reshape(-1), uv=uv, name=f"heightfield-{seed}",
                meta={"kind": "heightfield", "charts": cu * cv, "seed": seed})


def batched_set(count: int = 64, seed: int = 2, lo: int = 2000, hi: int = 200000) -> list:
    """The batched-audit mesh set: `count` meshes cycling sphere / torus /
    heightfield, face counts log-uniform in [lo, hi], 4-16 UV charts each."""
    u = uniform(seed, 2 * count, 0.0, 1.0)
    meshes = []
    for k in range(count):
        faces = int(round(np.exp(np.log(lo) + (np.log(hi) - np.log(lo)) * u[k])))
        charts = 4 + int(u[count + k] * 13)
        s = seed * 1000 + k
        if k % 3 == 0:
            meshes.append(seamed_sphere(faces, s))
        elif k % 3 == 1:
            meshes.append(seamed_torus(faces, s, charts))
        else:
            meshes.append(seamed_heightfield(faces, s, charts))
    return meshes


def ridged_noise(p: np.ndarray, seed: int, octaves: int = 6, frequency: float = 1.5) -> np.ndarray:
    """Ridged multifractal sum: per octave (1 - |n|)^2 of value noise, amplitude
    halving and frequency doubling, normalised to [0, 1]."""
    total = np.zeros(p.shape[0])
    amp, norm = 1.0, 0.0
    for o in range(octaves):
        n = value_noise(p * (2 ** o), seed + 104729 * o, octaves=1, frequency=frequency)
        total += amp * (1.0 - np.abs(n)) ** 2
        norm += amp
        amp *= 0.5
    return total / norm


def rock(level: int, seed: int = 3, relief: float = 0.25) -> Mesh:
    """A rock: icosphere (20 * 4^level faces) displaced radially by 6-octave
    ridged noise, with FP32 UVs on 8 charts (one per octant of the face
    centroid; vertices shared across charts are duplicated)."""
    p, f = icosphere(level)
    r = 1.0 + relief * (ridged_noise(p, seed) - 0.5)
    pos = (p * r[:, None]).astype(np.float32)
    cent = p[f].mean(1)
    chart = (cent[:, 0] > 0).astype(np.int64) | ((cent[:, 1] > 0) << 1) | ((cent[:, 2] > 0) << 2)
    key = f * 8 + chart[:, None]
    uniq, inv = np.unique(key.reshape(-1), return_inverse=True)
    slot_vertex, slot_chart = uniq // 8, uniq % 8
    d = p[slot_vertex]
    u = (np.arctan2(d[:, 1], d[:, 0]) / (2 * np.pi) + 0.5) * 0.24 + 0.25 * (slot_chart % 4)
    v = (np.arcsin(np.clip(d[:, 2], -1, 1)) / np.pi + 0.5) * 0.49 + 0.5 * (slot_chart // 4)
    faces = inv.reshape(-1, 3).astype(np.uint32)
    return Mesh(pos[slot_vertex], faces.reshape(-1), uv=np.stack([u, v], 1).astype(np.float32),
                name=f"rock{level}-seed{seed}", meta={"kind": "rock", "level": level, "charts": 8, "seed": seed})


def ribbons(count: int = 2000, seed: int = 5, height: float = 2.0, quads: int = 10) -> Mesh:
    """Ribbon cards (foliage / hair cards): `count` two-sided quad strips of
    quads x quads cells (2 * quads^2 triangles each), length 0.5-3% of the
    scene height (`height`, cards based in [-1, 1]^2 x [-height/2, height/2]),
    width a quarter of the length, random orientation, a seeded bend (arc of
    up to 90 degrees along the length) and twist (up to 90 degrees). Each card
    is its own uv chart, one cell of a square atlas."""
    n = quads + 1
    u = uniform(seed, 12 * count, 0.0, 1.0).reshape(12, count)
    base = np.stack([2 * u[0] - 1, height * (u[1] - 0.5), 2 * u[2] - 1], 1)
    length = height * (0.005 + 0.025 * u[3])
    width = 0.25 * length
    # orthonormal frame per card: strip axis a, bending normal b, binormal c
    z = 2 * u[4] - 1
    phi = 2 * np.pi * u[5]
    a = np.stack([np.sqrt(1 - z * z) * np.cos(phi), np.sqrt(1 - z * z) * np.sin(phi), z], 1)
    helper = np.where(np.abs(a[:, 0:1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    b = np.cross(a, helper)
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    rot = 2 * np.pi * u[6]
    c0 = np.cross(a, b)
    b, c = np.cos(rot)[:, None] * b + np.sin(rot)[:, None] * c0, -np.sin(rot)[:, None] * b + np.cos(rot)[:, None] * c0
    bend = (u[7] - 0.5) * np.pi  # total arc angle, -90..90 degrees
    twist = (u[8] - 0.5) * np.pi
    t = np.linspace(0.0, 1.0, n)                       # along the length
    s = np.linspace(-0.5, 0.5, n)                      # across the width
    theta = bend[:, None] * t[None, :]                 # (count, n)
    safe = np.where(np.abs(bend) < 1e-9, 1.0, bend)
    along = np.where(np.abs(bend)[:, None] < 1e-9, t[None, :], np.sin(theta) / safe[:, None])
    side = np.where(np.abs(bend)[:, None] < 1e-9, 0.0, (1 - np.cos(theta)) / safe[:, None])
    center = (base[:, None, :] + length[:, None, None] * (along[..., None] * a[:, None, :] +
                                                           side[..., None] * b[:, None, :]))
    tangent = np.cos(theta)[..., None] * a[:, None, :] + np.sin(theta)[..., None] * b[:, None, :]
    tw = twist[:, None] * t[None, :]
    cross_tc = np.cross(tangent, np.broadcast_to(c[:, None, :], tangent.shape))
    wdir = np.cos(tw)[..., None] * c[:, None, :] + np.sin(tw)[..., None] * cross_tc
    pos = center[:, :, None, :] + (width[:, None, None, None] * s[None, None, :, None]) * wdir[:, :, None, :]
    pos = pos.reshape(count * n * n, 3).astype(np.float32)
    # faces: cell (i, j) of card k -> two triangles, the same winding on every card
    i, j = np.meshgrid(np.arange(quads), np.arange(quads), indexing="ij")
    v00 = (i * n + j).reshape(-1)
    v01, v10, v11 = v00 + 1, v00 + n, v00 + n + 1
    cell = np.stack([np.stack([v00, v10, v11], 1), np.stack([v00, v11, v01], 1)], 1).reshape(-1, 3)
    faces = (cell[None, :, :] + (np.arange(count) * n * n)[:, None, None]).reshape(-1)
    # uv: card k in cell (k % side, k // side) of a side x side atlas, 10% margin
    side_cells = int(np.ceil(np.sqrt(count)))
    k = np.arange(count)
    cu, cv = (k % side_cells).astype(np.float64), (k // side_cells).astype(np.float64)
    uu = (cu[:, None, None] + 0.05 + 0.9 * (s[None, None, :] + 0.5)) / side_cells
    vv = (cv[:, None, None] + 0.05 + 0.9 * t[None, :, None]) / side_cells
    uv = np.stack(np.broadcast_arrays(uu, vv), -1).reshape(count * n * n, 2).astype(np.float32)
    return Mesh(pos, faces.astype(np.uint32), uv=uv, double_sided=np.array([1], np.uint8),
                name=f"ribbons{count}-seed{seed}",
                meta={"kind": "ribbons", "cards": count, "quads": quads, "seed": seed})
