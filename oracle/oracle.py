"""ctypes bindings to the CPU oracle — TEST INFRASTRUCTURE ONLY.

``Oracle`` wraps ``oracle/liboracle.so`` (this project's CPU restatement of the
reference audit path) and ``Reference`` wraps ``oracle/_ref/libblitz_ref.so``
(the reference's own CPU sources behind a C shim). Only tests, the smoke check
and the benchmark's CPU-baseline leg import this module, always as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


class BoMesh(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("vertex_count", C.c_uint32), ("indices", C.c_void_p),
                ("face_count", C.c_uint32), ("materials", C.c_void_p), ("double_sided", C.c_void_p),
                ("double_sided_count", C.c_uint32), ("uv", C.c_void_p)]


class BoBounds(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("radius", C.c_double)]


class BoCamera(C.Structure):
    _fields_ = [("right", C.c_float * 3), ("up", C.c_float * 3), ("forward", C.c_float * 3),
                ("distance", C.c_double), ("focal", C.c_double), ("scale", C.c_double),
                ("perspective", C.c_uint8), ("pad", C.c_uint8 * 7)]


class BoEvalSettings(C.Structure):
    _fields_ = [("screen_size", C.c_double), ("limit", C.c_double), ("max_changed_area", C.c_double),
                ("views_orthographic", C.c_uint16), ("views_perspective", C.c_uint16),
                ("views_seed", C.c_uint32), ("supersample", C.c_uint8), ("max_supersample", C.c_uint8),
                ("force_two_sided", C.c_uint8), ("conservative_screen", C.c_uint8),
                ("profile", C.c_uint8), ("pad", C.c_uint8 * 3)]


class BoMeasurement(C.Structure):
    _fields_ = [("error", C.c_double), ("coverage", C.c_double), ("coverage_upper", C.c_double),
                ("changed_area", C.c_double), ("normal_degrees", C.c_double),
                ("worst_view", C.c_uint32), ("changed_area_worst_view", C.c_uint32),
                ("views_evaluated", C.c_uint32), ("supersample", C.c_uint8), ("complete", C.c_uint8),
                ("passed", C.c_uint8), ("resource_limited", C.c_uint8), ("cancelled", C.c_uint8),
                ("pad", C.c_uint8 * 3)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class BoViewRecord(C.Structure):
    _fields_ = [("max_d2", C.c_double), ("changed", C.c_uint64), ("total", C.c_uint64),
                ("ca", C.c_uint8), ("cb", C.c_uint8), ("same", C.c_uint8), ("clipped_ref", C.c_uint8),
                ("clipped_cand", C.c_uint8), ("pad", C.c_uint8 * 3)]


class BoEdit(C.Structure):
    _fields_ = [("from_", C.c_uint32), ("to", C.c_uint32), ("source", C.c_uint32 * 2),
                ("target", C.c_uint32 * 2), ("wedges", C.c_uint8), ("removed", C.c_uint8),
                ("valid", C.c_uint8), ("pad", C.c_uint8)]


class BoVerdict(C.Structure):
    _fields_ = [("accepted", C.c_uint8), ("failed_gate", C.c_uint8), ("placement_valid", C.c_uint8),
                ("pad", C.c_uint8 * 5), ("gates", BoMeasurement * 4)]


def settings(screen: float, limit: float, views: tuple = (32, 0, 0xB1172026), supersample: int = 8,
             max_supersample: int = 8, max_changed_area: float = 1.0, force_two_sided: bool = False,
             conservative_screen: bool = False) -> BoEvalSettings:
    s = BoEvalSettings()
    s.screen_size, s.limit, s.max_changed_area = screen, limit, max_changed_area
    s.views_orthographic, s.views_perspective, s.views_seed = views
    s.supersample, s.max_supersample = supersample, max_supersample
    s.force_two_sided, s.conservative_screen, s.profile = int(force_two_sided), int(conservative_screen), 0
    return s


class _MeshHold:
    """Keeps numpy arrays alive while a BoMesh points at them."""

    def __init__(self, mesh):
        self.pos = np.ascontiguousarray(mesh.positions, dtype=np.float32)
        self.idx = np.ascontiguousarray(mesh.indices, dtype=np.uint32)
        self.mat = None if mesh.materials is None else np.ascontiguousarray(mesh.materials, dtype=np.uint16)
        self.ds = None if mesh.double_sided is None else np.ascontiguousarray(mesh.double_sided, dtype=np.uint8)
        self.uv = None if mesh.uv is None else np.ascontiguousarray(mesh.uv, dtype=np.float32)
        self.c = BoMesh(self.pos.ctypes.data, self.pos.shape[0], self.idx.ctypes.data, self.idx.size // 3,
                        None if self.mat is None else self.mat.ctypes.data,
                        None if self.ds is None else self.ds.ctypes.data,
                        0 if self.ds is None else self.ds.size,
                        None if self.uv is None else self.uv.ctypes.data)


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree exists, the reference shim)."""
    targets = ["liboracle.so"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE)] + targets, check=True)


class Oracle:
    def __init__(self, path: Path | None = None):
        path = path or HERE / "liboracle.so"
        if not path.exists():
            build(ref=False)
        self.lib = C.CDLL(str(path))
        L = self.lib
        P = C.POINTER
        L.bo_bounds_of.argtypes = [P(BoMesh), P(BoBounds)]
        L.bo_cameras.argtypes = [P(BoBounds), C.c_double, C.c_uint16, C.c_uint16, C.c_uint32, P(BoCamera)]
        L.bo_raster_size.argtypes = [C.c_double, C.c_uint8]
        L.bo_raster_size.restype = C.c_uint32
        L.bo_rasterize_coverage.argtypes = [P(BoMesh), P(BoBounds), P(BoCamera), C.c_double, C.c_uint8,
                                            C.c_int, C.c_void_p, P(C.c_uint8)]
        L.bo_coverage_distance.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint8,
                                           P(C.c_double)]
        L.bo_distance_field.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
        L.bo_view_record_of.argtypes = [P(BoMesh), P(BoMesh), P(BoBounds), P(BoCamera), C.c_double,
                                        C.c_uint8, C.c_int, P(BoViewRecord)]
        L.bo_finish_view.argtypes = [P(BoViewRecord), P(BoEvalSettings), C.c_uint8, P(BoMeasurement)]
        L.bo_evaluate.argtypes = [P(BoMesh), P(BoMesh), P(BoBounds), P(BoEvalSettings), P(BoMeasurement)]
        L.bo_bounded_refinement.argtypes = [C.c_double, C.c_uint8, C.c_uint8]
        L.bo_bounded_refinement.restype = C.c_uint8
        L.bo_schedule.argtypes = [C.c_double, C.c_double, C.c_uint32, C.c_void_p, C.c_uint32, C.c_double,
                                  C.c_void_p, C.c_void_p, C.c_void_p]
        L.bo_actions.argtypes = [P(BoMesh), C.c_int, C.c_int, P(BoEdit), C.c_uint64]
        L.bo_actions.restype = C.c_int64
        L.bo_topology_flags.argtypes = [P(BoMesh), C.c_void_p, C.c_void_p, C.c_void_p]
        L.bo_trial_midpoint.argtypes = [P(BoMesh), P(BoEdit), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                        P(C.c_uint8)]
        L.bo_trial_midpoint.restype = C.c_int64
        L.bo_audit_candidate.argtypes = [P(BoMesh), P(BoEdit), P(BoMesh), P(BoMesh), P(BoBounds),
                                         P(BoEvalSettings), C.c_int, P(BoVerdict)]

    def bounds(self, mesh) -> BoBounds:
        h = _MeshHold(mesh)
        b = BoBounds()
        assert self.lib.bo_bounds_of(C.byref(h.c), C.byref(b)) == 0
        return b

    def execute(self, source, target: int, budget: int, gates, previous=None, preserve_uv=True, batch=1,
                start=None, ranking=3) -> dict:
        """Greedy executor (ShortestEdge, midpoint placement), batches of up to
        `batch` independent collapses audited as one trial, from `start` (a
        later state of `source`; default the source)."""
        L = self.lib
        P = C.POINTER
        L.bo_execute_from.argtypes = [P(BoMesh), P(BoMesh), P(BoMesh), C.c_uint32, C.c_uint32, P(BoEvalSettings),
                                      C.c_int, C.c_uint32, C.c_int, C.c_void_p, C.c_uint32, P(C.c_uint32),
                                      P(C.c_uint32), C.c_void_p, P(C.c_uint32), C.c_void_p, P(C.c_uint8),
                                      C.c_void_p]
        hs = _MeshHold(source)
        hp = None if previous is None else _MeshHold(previous)
        hst = None if start is None else _MeshHold(start)
        cap = source.face_count
        ft = np.zeros(2 * cap, np.uint32)
        idx = np.zeros(source.face_count * 3, np.uint32)
        pos = np.zeros((source.vertex_count, 3), np.float32)
        uv = np.zeros((source.vertex_count, 2), np.float32)
        commits, trials, faces, stop = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint8()
        g = (BoEvalSettings * 4)(*gates)
        st = L.bo_execute_from(C.byref(hs.c), None if hp is None else C.byref(hp.c),
                               None if hst is None else C.byref(hst.c), target, budget, g, int(preserve_uv), batch,
                               ranking,
                               ft.ctypes.data, cap, C.byref(commits), C.byref(trials), idx.ctypes.data,
                               C.byref(faces), pos.ctypes.data, C.byref(stop), uv.ctypes.data)
        assert st == 0
        n = commits.value
        return {"commits": ft[: 2 * n].reshape(-1, 2), "trials": trials.value, "stop": stop.value,
                "indices": idx[: 3 * faces.value].copy(), "positions": pos,
                "uv": uv if source.uv is not None else None}

    def execute_endpoint(self, source, target: int, budget: int, gates, batch=1) -> dict:
        """The walk over endpoint collapses (the reference CPU executor's),
        ShortestEdge ranking, previous = source."""
        L = self.lib
        P = C.POINTER
        L.bo_execute_endpoint.argtypes = [P(BoMesh), C.c_uint32, C.c_uint32, P(BoEvalSettings), C.c_uint32,
                                          C.c_void_p, C.c_uint32, P(C.c_uint32), P(C.c_uint32), C.c_void_p,
                                          P(C.c_uint32), P(C.c_uint8)]
        hs = _MeshHold(source)
        cap = source.face_count
        ft = np.zeros(2 * cap, np.uint32)
        idx = np.zeros(source.face_count * 3, np.uint32)
        commits, trials, faces, stop = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint8()
        g = (BoEvalSettings * 4)(*gates)
        st = L.bo_execute_endpoint(C.byref(hs.c), target, budget, g, batch, ft.ctypes.data, cap, C.byref(commits),
                                   C.byref(trials), idx.ctypes.data, C.byref(faces), C.byref(stop))
        assert st == 0
        n = commits.value
        return {"commits": ft[: 2 * n].reshape(-1, 2), "trials": trials.value, "stop": stop.value,
                "indices": idx[: 3 * faces.value].copy()}

    def cameras(self, b: BoBounds, screen: float, views: tuple) -> list:
        n = views[0] + views[1]
        out = (BoCamera * n)()
        assert self.lib.bo_cameras(C.byref(b), screen, views[0], views[1], views[2], out) == 0
        return list(out)

    def raster_size(self, screen: float, ss: int) -> int:
        return int(self.lib.bo_raster_size(screen, ss))

    def rasterize(self, mesh, b, cam, screen, ss, two=False):
        size = self.raster_size(screen, ss)
        words = np.zeros((size * size + 63) // 64, dtype=np.uint64)
        clipped = C.c_uint8()
        h = _MeshHold(mesh)
        st = self.lib.bo_rasterize_coverage(C.byref(h.c), C.byref(b), C.byref(cam), screen, ss, int(two),
                                            words.ctypes.data, C.byref(clipped))
        if st:
            raise (MemoryError if st == 2 else ValueError)("rasterize failed")
        return words, bool(clipped.value), size

    def coverage_distance(self, a, b, width, height, ss) -> float:
        out = C.c_double()
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        assert self.lib.bo_coverage_distance(a.ctypes.data, b.ctypes.data, width, height, ss, C.byref(out)) == 0
        return out.value

    def distance_field(self, words, width, height) -> np.ndarray:
        out = np.zeros(width * height, dtype=np.float32)
        w = np.ascontiguousarray(words, dtype=np.uint64)
        assert self.lib.bo_distance_field(w.ctypes.data, width, height, out.ctypes.data) == 0
        return out

    def view_record(self, ref, cand, b, cam, screen, ss, two=False) -> BoViewRecord:
        hr, hc = _MeshHold(ref), _MeshHold(cand)
        r = BoViewRecord()
        st = self.lib.bo_view_record_of(C.byref(hr.c), C.byref(hc.c), C.byref(b), C.byref(cam), screen, ss,
                                        int(two), C.byref(r))
        assert st == 0
        return r

    def evaluate(self, ref, cand, b, s: BoEvalSettings) -> BoMeasurement:
        hr, hc = _MeshHold(ref), _MeshHold(cand)
        m = BoMeasurement()
        st = self.lib.bo_evaluate(C.byref(hr.c), C.byref(hc.c), C.byref(b), C.byref(s), C.byref(m))
        if st:
            raise ValueError("evaluate failed")
        return m

    def bounded_refinement(self, screen, ss, max_ss) -> int:
        return int(self.lib.bo_bounded_refinement(screen, ss, max_ss))

    def schedule(self, first, last, levels, curve, max_lod0=0.0):
        c = np.ascontiguousarray(np.asarray(curve, dtype=np.float32).reshape(-1))
        p, t, s = (np.zeros(levels) for _ in range(3))
        assert self.lib.bo_schedule(first, last, levels, c.ctypes.data, c.size // 2, max_lod0,
                                    p.ctypes.data, t.ctypes.data, s.ctypes.data) == 0
        return p, t, s

    def actions(self, mesh, placement=True, preserve_uv=True) -> list:
        h = _MeshHold(mesh)
        cap = 6 * mesh.face_count + 6
        out = (BoEdit * cap)()
        n = self.lib.bo_actions(C.byref(h.c), int(placement), int(preserve_uv), out, cap)
        assert n >= 0
        return list(out[:n])

    def topology_flags(self, mesh):
        h = _MeshHold(mesh)
        n = mesh.vertex_count
        g = np.zeros(n, np.uint32)
        bnd = np.zeros(n, np.uint8)
        inv = np.zeros(n, np.uint8)
        assert self.lib.bo_topology_flags(C.byref(h.c), g.ctypes.data, bnd.ctypes.data, inv.ctypes.data) == 0
        return g, bnd, inv

    def trial_midpoint(self, mesh, edit: BoEdit, preserve_uv=True):
        h = _MeshHold(mesh)
        idx = np.zeros(mesh.face_count * 3, np.uint32)
        pos = np.zeros((mesh.vertex_count, 3), np.float32)
        uv = np.zeros((mesh.vertex_count, 2), np.float32)
        valid = C.c_uint8()
        nf = self.lib.bo_trial_midpoint(C.byref(h.c), C.byref(edit), int(preserve_uv), idx.ctypes.data,
                                        pos.ctypes.data, uv.ctypes.data, C.byref(valid))
        assert nf >= 0
        return idx[: nf * 3].copy(), pos, (uv if mesh.uv is not None else None), bool(valid.value)

    def audit_candidate(self, parent, edit, source, previous, b, gates, preserve_uv=True) -> BoVerdict:
        hp, hs, hv = _MeshHold(parent), _MeshHold(source), _MeshHold(previous)
        g = (BoEvalSettings * 4)(*gates)
        v = BoVerdict()
        st = self.lib.bo_audit_candidate(C.byref(hp.c), C.byref(edit), C.byref(hs.c), C.byref(hv.c),
                                         C.byref(b), g, int(preserve_uv), C.byref(v))
        assert st == 0
        return v


def reference_root() -> Path | None:
    """The reference source tree: $BLITZ_REFERENCE, else the tree that
    oracle/Makefile compiled oracle/_ref from; None when neither exists."""
    env = os.environ.get("BLITZ_REFERENCE")
    if env:
        return Path(env) if Path(env).is_dir() else None
    rec = HERE / "_ref" / "source_root.txt"
    if rec.exists():
        p = Path(rec.read_text().strip())
        return p if p.is_dir() else None
    return None


class Reference:
    """The reference's own CPU sources (oracle/_ref/libblitz_ref.so)."""

    PATH = HERE / "_ref" / "libblitz_ref.so"

    @classmethod
    def available(cls) -> bool:
        return cls.PATH.exists()

    def __init__(self):
        self.lib = C.CDLL(str(self.PATH))
        L = self.lib
        P = C.POINTER
        L.br_bounds_of.argtypes = [P(BoMesh), P(BoBounds)]
        L.br_cameras.argtypes = [P(BoBounds), C.c_double, C.c_uint16, C.c_uint16, C.c_uint32, P(BoCamera)]
        L.br_rasterize_coverage.argtypes = [P(BoMesh), P(BoBounds), P(BoCamera), C.c_double, C.c_uint8,
                                            C.c_int, C.c_void_p, P(C.c_uint8)]
        L.br_coverage_distance.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint8, C.c_int,
                                           P(C.c_double)]
        L.br_evaluate.argtypes = [P(BoMesh), P(BoMesh), P(BoBounds), P(BoEvalSettings), P(BoMeasurement)]
        L.br_bounded_refinement.argtypes = [C.c_double, C.c_uint8, C.c_uint8]
        L.br_bounded_refinement.restype = C.c_uint8
        L.br_actions.argtypes = [P(BoMesh), C.c_void_p, C.c_uint64]
        L.br_actions.restype = C.c_int64
        L.br_precision_masks.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
        L.br_trial_endpoint.argtypes = [P(BoMesh), C.c_uint32, C.c_uint32, C.c_void_p]
        L.br_trial_endpoint.restype = C.c_int64

    def execute_actions(self, source, target: int, budget: int, gates, batch=1) -> dict:
        """neural::execute_actions itself (action.cpp:453-525): endpoint
        collapses, ShortestEdge ranking, the four gates over blitz::evaluate."""
        L = self.lib
        P = C.POINTER
        L.br_execute_actions.argtypes = [P(BoMesh), C.c_uint32, C.c_uint32, P(BoEvalSettings), C.c_uint32,
                                         C.c_void_p, P(C.c_uint32), P(C.c_uint64), P(C.c_uint64), P(C.c_uint64),
                                         P(C.c_uint8)]
        h = _MeshHold(source)
        idx = np.zeros(source.face_count * 3, np.uint32)
        faces, stop = C.c_uint32(), C.c_uint8()
        trials, accepted, rejected = C.c_uint64(), C.c_uint64(), C.c_uint64()
        g = (BoEvalSettings * 4)(*gates)
        st = L.br_execute_actions(C.byref(h.c), target, budget, g, batch, idx.ctypes.data, C.byref(faces),
                                  C.byref(trials), C.byref(accepted), C.byref(rejected), C.byref(stop))
        assert st == 0
        return {"trials": trials.value, "accepted": accepted.value, "rejected": rejected.value, "stop": stop.value,
                "indices": idx[: 3 * faces.value].copy()}

    def trial_endpoint(self, mesh, frm: int, to: int) -> np.ndarray:
        h = _MeshHold(mesh)
        out = np.zeros(mesh.face_count * 3, np.uint32)
        nf = self.lib.br_trial_endpoint(C.byref(h.c), frm, to, out.ctypes.data)
        assert nf >= 0
        return out[: 3 * nf].copy()

    def bounds(self, mesh) -> BoBounds:
        h = _MeshHold(mesh)
        b = BoBounds()
        assert self.lib.br_bounds_of(C.byref(h.c), C.byref(b)) == 0
        return b

    def cameras(self, b, screen, views) -> list:
        n = views[0] + views[1]
        out = (BoCamera * n)()
        assert self.lib.br_cameras(C.byref(b), screen, views[0], views[1], views[2], out) == 0
        return list(out)

    def rasterize(self, mesh, b, cam, screen, ss, two=False):
        size = int(np.ceil(screen + 8)) * ss
        words = np.zeros((size * size + 63) // 64, dtype=np.uint64)
        clipped = C.c_uint8()
        h = _MeshHold(mesh)
        st = self.lib.br_rasterize_coverage(C.byref(h.c), C.byref(b), C.byref(cam), screen, ss, int(two),
                                            words.ctypes.data, C.byref(clipped))
        if st:
            raise (MemoryError if st == 2 else ValueError)("rasterize failed")
        return words, bool(clipped.value), size

    def coverage_distance(self, a, b, width, height, ss, scalar=True) -> float:
        out = C.c_double()
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        assert self.lib.br_coverage_distance(a.ctypes.data, b.ctypes.data, width, height, ss, int(scalar),
                                             C.byref(out)) == 0
        return out.value

    def evaluate(self, ref, cand, b, s) -> BoMeasurement:
        hr, hc = _MeshHold(ref), _MeshHold(cand)
        m = BoMeasurement()
        st = self.lib.br_evaluate(C.byref(hr.c), C.byref(hc.c), C.byref(b), C.byref(s), C.byref(m))
        if st:
            raise ValueError("evaluate failed")
        return m

    def bounded_refinement(self, screen, ss, max_ss) -> int:
        return int(self.lib.br_bounded_refinement(screen, ss, max_ss))

    def actions(self, mesh) -> np.ndarray:
        h = _MeshHold(mesh)
        cap = 6 * mesh.face_count + 6
        out = np.zeros(2 * cap, np.uint32)
        n = self.lib.br_actions(C.byref(h.c), out.ctypes.data, cap)
        assert n >= 0
        return out[: 2 * n].reshape(-1, 2)

    def precision_masks(self, seed=2921, trials=40):
        a = np.zeros(3 * trials, np.uint64)
        b = np.zeros(3 * trials, np.uint64)
        self.lib.br_precision_masks(seed, trials, a.ctypes.data, b.ctypes.data)
        return a.reshape(trials, 3), b.reshape(trials, 3)
