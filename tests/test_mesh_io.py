"""PLY reading and writing (CPU) and the host-side checks of scene files.

The reader replaces smallgwn's test loader (tests/test_mesh_io.cpp:43-92, libigl): the fixtures of
smallgwn's tests/data are ASCII files with double positions and `uchar uint` index lists; the
writer here produces the same structure from the analytic meshes, and the reference project's own
files are read when they are present. Binary files of either byte order, mixed property types,
extra properties and elements, polygons (triangle fans) and the refusals (non-finite positions,
out-of-range indices, short faces, empty or truncated files) are covered.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from conftest import cube, open_cube
from oracle.build import REFERENCE_ROOT
from smallgwn_b200 import _lib, api, meshes

# smallgwn's own PLY fixtures, where the oracle's build recipe finds the reference project
REFERENCE_DATA = REFERENCE_ROOT / "tests" / "data"


def ply_text(mesh: dict, comment: str = "fixture") -> str:
    """ASCII PLY with double positions and `uchar uint` lists, the layout of smallgwn's fixtures."""
    lines = ["ply", "format ascii 1.0", f"comment {comment}", f"element vertex {mesh['x'].size}",
             "property double x", "property double y", "property double z", f"element face {mesh['i0'].size}",
             "property list uchar uint vertex_indices", "end_header"]
    lines += [f"{x:g} {y:g} {z:g}" for x, y, z in zip(mesh["x"], mesh["y"], mesh["z"])]
    lines += [f"3 {a} {b} {c}" for a, b, c in zip(mesh["i0"], mesh["i1"], mesh["i2"])]
    return "\n".join(lines) + "\n"


def same(a: dict, b: dict) -> bool:
    return all(np.array_equal(np.asarray(a[k]), np.asarray(b[k])) for k in ("x", "y", "z", "i0", "i1", "i2"))


@pytest.mark.parametrize("mesh_fn", [cube, open_cube])
def test_reads_fixture_layout(tmp_path, mesh_fn):
    m = mesh_fn()
    p = tmp_path / "m.ply"
    p.write_text(ply_text(m))
    assert same(api.read_ply(p), m)


@pytest.mark.skipif(not REFERENCE_DATA.exists(), reason="the reference project's fixtures are not here")
def test_reads_the_reference_fixtures():
    assert same(api.read_ply(REFERENCE_DATA / "closed_cube.ply"), cube())
    assert same(api.read_ply(REFERENCE_DATA / "open_cube.ply"), open_cube())
    m = api.read_ply(REFERENCE_DATA / "nonplanar_closed.ply")
    assert m["x"].size == 8 and m["i0"].size == 12
    np.testing.assert_array_equal(m["z"][4:], np.array([1, 1.25, 0.85, 1.1], np.float32))


@pytest.mark.parametrize("binary", [True, False])
def test_write_read_round_trip(tmp_path, binary):
    m = meshes.soup_mesh(40, seed=13)
    p = tmp_path / "soup.ply"
    api.write_ply(p, m, binary=binary)
    assert same(api.read_ply(p), m)


def test_big_endian_mixed_types_extra_data_and_polygons(tmp_path):
    """Big-endian body; x double, y float, z int16; per-vertex normals and colours; an `edge`
    element with its own list; a quad and a pentagon named `vertex_index` (fanned)."""
    header = "\n".join([
        "ply", "format binary_big_endian 1.0", "element vertex 5", "property double x", "property float y",
        "property short z", "property float nx", "property uchar red", "element edge 1",
        "property list uchar int vertex_pair", "element face 2", "property uchar flags",
        "property list uchar int vertex_index", "end_header"]) + "\n"
    body = b""
    pts = [(0.0, 0.0, 0), (1.0, 0.0, 0), (1.0, 1.0, 0), (0.0, 1.0, 0), (0.5, 2.0, 1)]
    for x, y, z in pts:
        body += np.array([x], ">f8").tobytes() + np.array([y], ">f4").tobytes() + np.array([z], ">i2").tobytes()
        body += np.array([0.5], ">f4").tobytes() + bytes([200])
    body += bytes([2]) + np.array([0, 1], ">i4").tobytes()
    body += bytes([7, 4]) + np.array([0, 1, 2, 3], ">i4").tobytes()
    body += bytes([0, 5]) + np.array([0, 1, 4, 2, 3], ">i4").tobytes()
    p = tmp_path / "be.ply"
    p.write_bytes(header.encode() + body)
    m = api.read_ply(p)
    np.testing.assert_array_equal(m["x"], [0, 1, 1, 0, 0.5])
    np.testing.assert_array_equal(m["z"], [0, 0, 0, 0, 1])
    # fans (0,1,2), (0,2,3) then (0,1,4), (0,4,2), (0,2,3)
    np.testing.assert_array_equal(m["i0"], [0, 0, 0, 0, 0])
    np.testing.assert_array_equal(m["i1"], [1, 2, 1, 4, 2])
    np.testing.assert_array_equal(m["i2"], [2, 3, 4, 2, 3])


@pytest.mark.parametrize("body, why", [
    ("0 0 0\n1 0 0\nnan 1 0\n3 0 1 2\n", "non-finite"),
    ("0 0 0\n1 0 0\n0 1 0\n3 0 1 3\n", "out of range"),
    ("0 0 0\n1 0 0\n0 1 0\n3 0 -1 2\n", "out of range"),
    ("0 0 0\n1 0 0\n0 1 0\n2 0 1\n", "fewer than three"),
    ("0 0 0\n1 0 0\n0 1 0\n3 0 1\n", "truncated"),
])
def test_refusals(tmp_path, body, why):
    head = ("ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
            "element face 1\nproperty list uchar int vertex_indices\nend_header\n")
    p = tmp_path / "bad.ply"
    p.write_text(head + body)
    with pytest.raises(ValueError, match=why):
        api.read_ply(p)


def test_refuses_missing_empty_and_foreign_files(tmp_path):
    with pytest.raises(ValueError, match="cannot open"):
        api.read_ply(tmp_path / "missing.ply")
    p = tmp_path / "empty.ply"
    p.write_text("ply\nformat ascii 1.0\nelement vertex 0\nproperty float x\nproperty float y\nproperty float z\n"
                 "element face 0\nproperty list uchar int vertex_indices\nend_header\n")
    with pytest.raises(ValueError, match="no vertices or no triangles"):
        api.read_ply(p)
    p.write_text("OFF\n3 1 0\n")
    with pytest.raises(ValueError, match="magic"):
        api.read_ply(p)


def test_scene_files_are_checked_on_the_host(tmp_path):
    """Saving invalid objects and loading missing, foreign or truncated files fail before any
    device work."""
    lib = _lib.load()
    g = _lib.geometry_f32()
    b = _lib.bvh4_f32()
    st = lib.gwnb_scene_save_f32(str(tmp_path / "s.gwnb").encode(), C.byref(g), C.byref(b), None, 0, None)
    assert st == _lib.GWNB_INVALID_ARGUMENT and "no queryable data" in _lib.last_error()
    ms = (_lib.moment4_f32 * 3)()
    mask = C.c_int()
    assert lib.gwnb_scene_load_f32(str(tmp_path / "missing").encode(), C.byref(g), C.byref(b), ms, C.byref(mask),
                                   None) == _lib.GWNB_INVALID_ARGUMENT
    p = tmp_path / "foreign.gwnb"
    p.write_bytes(b"NOTASCENE" * 20)
    assert lib.gwnb_scene_load_f32(str(p).encode(), C.byref(g), C.byref(b), ms, C.byref(mask),
                                   None) == _lib.GWNB_INVALID_ARGUMENT
    assert "magic" in _lib.last_error()
    p.write_bytes(b"GWNBSCN1" + bytes(100))
    assert lib.gwnb_scene_load_f32(str(p).encode(), C.byref(g), C.byref(b), ms, C.byref(mask),
                                   None) == _lib.GWNB_INVALID_ARGUMENT
    status, *_ = api.load_scene(tmp_path / "missing")
    assert status.error == api.gwn_error.invalid_argument


def test_matrix_upload_refusals():
    """gwn_upload_geometry_from_eigen refuses what smallgwn's Eigen bridge refuses, before any
    device work (include/gwn/gwn_eigen_bridge.cuh:32-113)."""
    geo = api.gwn_geometry_object()
    m = cube()
    V = np.stack([m["x"], m["y"], m["z"]], axis=1).astype(np.float64)
    F = np.stack([m["i0"], m["i1"], m["i2"]], axis=1).astype(np.int64)
    st = api.gwn_upload_geometry_from_eigen(geo, V[:, :2], F)
    assert st.error == api.gwn_error.invalid_argument and "Nx3" in st.message
    for bad in (-1, 8, 1.5, np.nan, np.inf):
        Fb = F.astype(np.float64)
        Fb[3, 1] = bad
        st = api.gwn_upload_geometry_from_eigen(geo, V, Fb)
        assert st.error == api.gwn_error.invalid_argument and "integer-valued" in st.message, bad
    Fi = F.copy()
    Fi[0, 0] = -2
    assert api.gwn_upload_geometry_from_eigen(geo, V, Fi).error == api.gwn_error.invalid_argument
    assert api.gwn_upload_geometry_from_eigen(geo, V, F.astype(bool)).error == api.gwn_error.invalid_argument
    assert not geo.has_data()


def _scene_checksum(body: bytes) -> int:
    """FNV-1a over little-endian 8-byte words, then the tail bytes (the scene file's checksum)."""
    h, prime, mask = 0xCBF29CE484222325, 0x100000001B3, (1 << 64) - 1
    n8 = len(body) // 8 * 8
    for (w,) in np.frombuffer(body[:n8], "<u8").reshape(-1, 1):
        h = ((h ^ int(w)) * prime) & mask
    for b in body[n8:]:
        h = ((h ^ b) * prime) & mask
    return h


def _crafted_scene(nodes_refs, prims, root_ref) -> bytes:
    """A scene of 4 vertices / 2 triangles with the given node references (one list of 4 per node),
    primitive order and root reference, and a correct checksum."""
    V, T, N, P = 4, 2, len(nodes_refs), len(prims)
    root = np.zeros(1, [("b", "<f4", 6), ("r", "<u8")])
    root["r"] = root_ref
    head = b"GWNBSCN1" + np.array([1, 0], "<u4").tobytes() + np.array([V, T, N, P], "<u8").tobytes()
    head += root.tobytes() + np.array([4, 8], "<u4").tobytes()
    assert len(head) == 88
    body = np.zeros(3 * V, "<f4").tobytes() + np.array([0, 1, 2, 3, 2, 1], "<u4").tobytes()
    node = np.zeros((N, 4), [("b", "<f4", 6), ("r", "<u8")])
    for n, refs in enumerate(nodes_refs):
        node["r"][n] = refs
    body += node.tobytes() + np.asarray(prims, "<u4").tobytes() + np.zeros(P * 9, "<f4").tobytes()
    blob = head + body
    return blob + _scene_checksum(blob).to_bytes(8, "little")


@pytest.mark.parametrize("nodes_refs, prims, root, why", [
    ([[(1 << 47) | 0, 0, 0, 0]], [0, 1], 1 << 47, "self loop"),                  # node 0 names itself
    ([[(1 << 47) | (1 << 48) | 1, (1 << 47) | (2 << 48) | 1, 0, 0]], [0, 1], 1 << 47, "leaf past the end"),
    ([[(1 << 47) | (1 << 48) | 0, (1 << 47) | (1 << 48) | 1, 0, 0]], [0, 5], 1 << 47, "bad primitive id"),
    ([[(1 << 47) | 1, (1 << 47) | (2 << 48) | 0, 0, 0], [0, 0, 0, 0]], [0, 1], (1 << 47) | 1, "root not node 0"),
    ([[(1 << 47) | 1, (1 << 47) | 1, 0, 0], [(1 << 47) | (2 << 48), 0, 0, 0]], [0, 1], 1 << 47, "two parents"),
    ([[], ], [0, 1], (1 << 47) | (2 << 48), "leaf root with nodes"),
])
def test_scene_load_refuses_malformed_trees_on_host(tmp_path, nodes_refs, prims, root, why):
    """Files with a correct checksum whose hierarchy is not a tree the kernels can walk are refused
    before any upload."""
    refs = [r + [0] * (4 - len(r)) for r in nodes_refs]
    p = tmp_path / "crafted.gwnb"
    p.write_bytes(_crafted_scene(refs, prims, root))
    lib = _lib.load()
    g, b = _lib.geometry_f32(), _lib.bvh4_f32()
    ms, mask = (_lib.moment4_f32 * 3)(), C.c_int()
    rc = lib.gwnb_scene_load_f32(str(p).encode(), C.byref(g), C.byref(b), ms, C.byref(mask), None)
    assert rc == _lib.GWNB_INVALID_ARGUMENT, why
    assert "not a valid BVH4 tree" in _lib.last_error(), (why, _lib.last_error())


@pytest.mark.parametrize("header_count, body", [
    ("element vertex 4000000000", "0 0 0\n"),                       # vertex count far beyond the body
    ("element vertex 3", "0 0 0\n1 0 0\n0 1 0\n4000000000 0 1 2\n"),  # list length far beyond the body
])
def test_refuses_counts_the_body_cannot_hold(tmp_path, header_count, body):
    """Counts in the header are checked against the bytes left before anything is allocated."""
    head = ("ply\nformat ascii 1.0\n" + header_count + "\nproperty float x\nproperty float y\nproperty float z\n"
            "element face 1\nproperty list uint int vertex_indices\nend_header\n")
    p = tmp_path / "huge.ply"
    p.write_text(head + body)
    with pytest.raises(ValueError, match="truncated"):
        api.read_ply(p)
    binary = tmp_path / "huge_bin.ply"
    binary.write_bytes(("ply\nformat binary_little_endian 1.0\nelement vertex 4000000000\nproperty float x\n"
                        "property float y\nproperty float z\nend_header\n").encode() + bytes(24))
    with pytest.raises(ValueError, match="truncated"):
        api.read_ply(binary)
