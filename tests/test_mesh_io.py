"""Mesh files (csrc/mesh_io.cu) on the CPU: OBJ with shared corners, a
material library and polygons; PLY written by the library and read back
(ascii and both binary byte orders of the reader, vertex colours, per-face
materials); binary and ascii STL welded on exact positions; the reference's
refusals (non-opaque materials, non-triangle PLY faces, indices outside the
vertex stream, unknown formats)."""
import struct

import numpy as np
import pytest

import blitzremesher_b200 as br
from blitzremesher_b200 import synthetic as syn


def test_obj_corners_polygons_and_materials(tmp_path):
    (tmp_path / "m.mtl").write_text("newmtl red\nKd 1 0 0\nd 1\nnewmtl blue\nKd 0 0 1\n")
    (tmp_path / "m.obj").write_text(
        "mtllib m.mtl\n"
        "v 0 0 0 1 0 0\nv 1 0 0 0 1 0\nv 1 1 0 0 0 1\nv 0 1 0 1 1 1\nv 0.5 0.5 1\n"
        "vt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\nvn 0 0 1\n"
        "usemtl blue\nf 1/1/1 2/2/1 3/3/1 4/4/1\n"  # a quad: fanned into two triangles
        "usemtl red\nf 1/1/1 2/2/1 5/1/1\n"
        "f -5/1/1 -4/2/1 -3/3/1\n")  # negative (relative) indices: the same corners again
    m = br.load_mesh(tmp_path / "m.obj")
    assert m["indices"].tolist() == [0, 1, 2, 0, 2, 3, 0, 1, 4, 0, 1, 2]
    assert m["positions"].shape == (5, 3) and m["uv"].shape == (5, 2) and m["normals"].shape == (5, 3)
    assert np.array_equal(m["positions"][4], [0.5, 0.5, 1])
    assert m["materials"].tolist() == [2, 2, 1, 1]  # 1 + place in the library
    assert m["colors"][0].tolist() == [255, 0, 0, 255] and m["colors"][3].tolist() == [255, 255, 255, 255]


def test_obj_refusals(tmp_path):
    (tmp_path / "glass.mtl").write_text("newmtl glass\nd 0.5\n")
    (tmp_path / "a.obj").write_text("mtllib glass.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nusemtl glass\nf 1 2 3\n")
    with pytest.raises(br.BlitzError) as e:
        br.load_mesh(tmp_path / "a.obj")
    assert "nonopaque" in str(e.value)
    (tmp_path / "b.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n")
    with pytest.raises(br.BlitzError):
        br.load_mesh(tmp_path / "b.obj")
    (tmp_path / "c.xyz").write_text("1 2 3\n")
    with pytest.raises(br.BlitzError) as e:
        br.load_mesh(tmp_path / "c.xyz")
    assert e.value.status == br.BLITZ_INVALID_ARGUMENT
    (tmp_path / "d.glb").write_bytes(b"glTF")
    with pytest.raises(br.BlitzError) as e:
        br.load_mesh(tmp_path / "d.glb")
    assert e.value.status == br.BLITZ_UNAVAILABLE


def test_ply_round_trip(tmp_path):
    mesh = syn.seamed_torus(800, 3, 4)
    mesh.materials = (np.arange(mesh.face_count) % 3).astype(np.uint16)
    br.save_ply(mesh, tmp_path / "t.ply")
    m = br.load_mesh(tmp_path / "t.ply")
    assert np.array_equal(m["positions"], mesh.positions) and np.array_equal(m["indices"], mesh.indices)
    assert np.array_equal(m["uv"], mesh.uv) and np.array_equal(m["materials"], mesh.materials)
    assert m["normals"] is None and m["colors"] is None


@pytest.mark.parametrize("fmt", ["ascii", "binary_big_endian"])
def test_ply_formats_and_colors(tmp_path, fmt):
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    faces = [[0, 1, 2], [0, 2, 3]]
    cols = [[255, 0, 0], [0, 255, 0], [0, 0, 255], [10, 20, 30]]
    head = (f"ply\nformat {fmt} 1.0\nelement vertex 4\nproperty float x\nproperty float y\nproperty float z\n"
            "property uchar red\nproperty uchar green\nproperty uchar blue\nelement face 2\n"
            "property list uchar int vertex_indices\nproperty ushort material_index\nend_header\n").encode()
    if fmt == "ascii":
        body = "".join(f"{p[0]} {p[1]} {p[2]} {c[0]} {c[1]} {c[2]}\n" for p, c in zip(pos, cols))
        body += "".join(f"3 {f[0]} {f[1]} {f[2]} {k + 4}\n" for k, f in enumerate(faces))
        data = head + body.encode()
    else:
        data = head + b"".join(struct.pack(">fffBBB", *p, *c) for p, c in zip(pos, cols))
        data += b"".join(struct.pack(">BiiiH", 3, *f, k + 4) for k, f in enumerate(faces))
    (tmp_path / "c.ply").write_bytes(data)
    m = br.load_mesh(tmp_path / "c.ply")
    assert np.array_equal(m["positions"], pos) and m["indices"].tolist() == [0, 1, 2, 0, 2, 3]
    assert m["colors"][:, :3].tolist() == cols and m["colors"][:, 3].tolist() == [255] * 4
    assert m["materials"].tolist() == [4, 5]
    bad = data.replace(b"3 0 2 3", b"4 0 2 3 1") if fmt == "ascii" else None
    if bad is not None:
        (tmp_path / "q.ply").write_bytes(bad)
        with pytest.raises(br.BlitzError):
            br.load_mesh(tmp_path / "q.ply")


def test_stl_binary_and_ascii_weld(tmp_path):
    tris = [[(0, 0, 0), (1, 0, 0), (0, 1, 0)], [(1, 0, 0), (1, 1, 0), (0, 1, 0)], [(0, 0, 0), (0, 1, 0), (0, 0, 1)]]
    binary = b"\0" * 80 + struct.pack("<I", len(tris))
    for t in tris:
        binary += struct.pack("<3f", 0, 0, 1) + b"".join(struct.pack("<3f", *v) for v in t) + b"\0\0"
    (tmp_path / "b.stl").write_bytes(binary)
    text = "solid s\n" + "".join("facet normal 0 0 1\nouter loop\n" + "".join(f"vertex {x} {y} {z}\n" for x, y, z in t)
                                 + "endloop\nendfacet\n" for t in tris) + "endsolid s\n"
    (tmp_path / "a.stl").write_text(text)
    for name in ("b.stl", "a.stl"):
        m = br.load_mesh(tmp_path / name)
        assert m["positions"].shape == (5, 3)  # nine corners at five distinct positions
        assert m["indices"].tolist() == [0, 1, 2, 1, 3, 2, 0, 2, 4]
