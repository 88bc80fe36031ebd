"""Command-line pipeline (cuacd_b200/cli.py) and its mesh files
(cuacd_b200/meshio.py), on the CPU: each reader on a cube written in its
format (quads, negative indices, both STL forms, three PLY encodings,
glTF node transforms and buffers), the GLB writer read back, and the
pipeline with stand-in GPU contexts (tests/cli_fakes.py) -- outputs and
their layout, one retry with a fresh context, and a decomposer that dies
by a signal reported with the mesh it was on."""
import base64
import json
import os
import struct

import numpy as np
import pytest

import cli_fakes
from conftest import box_mesh
from cuacd_b200 import cli, meshio

CUBE_V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], np.float32)
CUBE_Q = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (0, 4, 7, 3), (1, 2, 6, 5)]
CUBE_T = np.array([t for q in CUBE_Q for t in meshio.fan(list(q))], np.int32)


def same_surface(v, t, v0=CUBE_V, t0=CUBE_T):
    """Same triangles as point triples (vertex numbering may differ)."""
    a = sorted(tuple(map(tuple, v[tri])) for tri in np.asarray(t))
    b = sorted(tuple(map(tuple, v0[tri])) for tri in np.asarray(t0))
    return a == b


def test_clean_mesh_merges_and_drops():
    v = np.array([[9, 9, 9], [0, 0, 0], [1, 0, 0], [0, 1, 0], [-0.0, 0, 0], [1, 0, 0]], np.float32)
    t = np.array([[1, 2, 3], [4, 3, 5]])
    cv, ct = meshio.clean_mesh(v, t)
    assert cv.tolist() == [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    assert ct.tolist() == [[0, 1, 2], [0, 2, 1]]
    with pytest.raises(ValueError):
        meshio.clean_mesh(v, [[0, 1, 6]])
    with pytest.raises(ValueError):
        meshio.clean_mesh(np.array([[np.nan, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), [[0, 1, 2]])


def test_obj_quads_slashes_negative_indices(tmp_path):
    lines = ["# cube", "o cube", "g a"] + [f"v {x} {y} {z}" for x, y, z in CUBE_V] + ["vt 0 0", "vn 0 0 1"]
    for k, q in enumerate(CUBE_Q):
        if k % 3 == 0:
            lines.append("f " + " ".join(str(i + 1) for i in q))
        elif k % 3 == 1:
            lines.append("f " + " ".join(f"{i + 1}/1/1" for i in q))
        else:
            lines.append("f " + " ".join(f"{i - 8}//1" for i in q))
    p = tmp_path / "c.obj"
    p.write_text("\n".join(lines) + "\n")
    v, t = meshio.load_mesh(p)
    assert len(v) == 8 and len(t) == 12 and same_surface(v, t)


def test_stl_binary_and_ascii_weld_the_soup(tmp_path):
    tri_v = CUBE_V[CUBE_T]
    rec = np.zeros(len(CUBE_T), meshio._STL_REC)
    rec["v"] = tri_v
    (tmp_path / "b.stl").write_bytes(b"\0" * 80 + struct.pack("<I", len(CUBE_T)) + rec.tobytes())
    txt = ["solid cube"]
    for tri in tri_v:
        txt += ["facet normal 0 0 0", "outer loop"] + [f"vertex {x} {y} {z}" for x, y, z in tri] + ["endloop",
                                                                                                    "endfacet"]
    (tmp_path / "a.stl").write_text("\n".join(txt + ["endsolid cube"]))
    for name in ("a.stl", "b.stl"):
        v, t = meshio.load_mesh(tmp_path / name)
        assert len(v) == 8 and len(t) == 12 and same_surface(v, t)


@pytest.mark.parametrize("fmt", ["ascii", "binary_little_endian", "binary_big_endian"])
def test_ply_encodings(tmp_path, fmt):
    head = ["ply", f"format {fmt} 1.0", "comment cube", "element vertex 8", "property float x", "property float y",
            "property float z", "property uchar red", "element face 6", "property list uchar int vertex_indices",
            "element extra 1", "property short w", "end_header"]
    if fmt == "ascii":
        body = "\n".join([f"{x} {y} {z} 7" for x, y, z in CUBE_V] + ["4 " + " ".join(map(str, q)) for q in CUBE_Q]
                         + ["3"]) + "\n"
        data = ("\n".join(head) + "\n" + body).encode()
    else:
        bo = "<" if fmt.endswith("little_endian") else ">"
        vt = np.dtype([("x", bo + "f4"), ("y", bo + "f4"), ("z", bo + "f4"), ("r", "u1")])
        va = np.zeros(8, vt)
        va["x"], va["y"], va["z"] = CUBE_V.T
        faces = b"".join(struct.pack(bo + "B4i", 4, *q) for q in CUBE_Q)
        data = ("\n".join(head) + "\n").encode() + va.tobytes() + faces + struct.pack(bo + "h", 3)
    p = tmp_path / "c.ply"
    p.write_bytes(data)
    v, t = meshio.load_mesh(p)
    assert len(v) == 8 and len(t) == 12 and same_surface(v, t)


def test_ply_binary_triangles_bulk_path(tmp_path):
    head = ["ply", "format binary_little_endian 1.0", "element vertex 8", "property double x",
            "property double y", "property double z", "element face 12",
            "property list uchar uint vertex_indices", "end_header"]
    faces = b"".join(struct.pack("<B3I", 3, *tri) for tri in CUBE_T)
    p = tmp_path / "t.ply"
    p.write_bytes(("\n".join(head) + "\n").encode() + CUBE_V.astype("<f8").tobytes() + faces)
    v, t = meshio.load_mesh(p)
    assert v.tolist() == CUBE_V.tolist() and t.tolist() == CUBE_T.tolist()


def test_off(tmp_path):
    txt = ["OFF", "# cube", "8 6 12"] + [f"{x} {y} {z}" for x, y, z in CUBE_V] + \
          ["4 " + " ".join(map(str, q)) for q in CUBE_Q]
    p = tmp_path / "c.off"
    p.write_text("\n".join(txt) + "\n")
    v, t = meshio.load_mesh(p)
    assert v.tolist() == CUBE_V.tolist() and t.tolist() == CUBE_T.tolist()


def test_glb_writer_round_trip(tmp_path):
    parts = [(CUBE_V * 2 - 1, CUBE_T), (CUBE_V + 5, CUBE_T[:4]), (np.zeros((0, 3), np.float32), np.zeros((0, 3)))]
    data = meshio.glb_bytes(parts, ["m_0", "m_1", "m_2"])
    magic, version, length = struct.unpack_from("<III", data, 0)
    assert (magic, version, length) == (0x46546C67, 2, len(data)) and len(data) % 4 == 0
    js, binc = meshio.split_glb(data)
    assert js["asset"]["version"] == "2.0" and len(js["nodes"]) == 3 and "mesh" not in js["nodes"][2]
    for a in js["accessors"]:
        bv = js["bufferViews"][a["bufferView"]]
        assert bv["byteOffset"] % 4 == 0 and bv["byteOffset"] + bv["byteLength"] <= len(binc)
    got = meshio.read_glb_parts(data)
    cols = meshio.part_colors(3)
    assert [g[0] for g in got] == ["m_0", "m_1"]
    for (name, v, t, c), (v0, t0), c0 in zip(got, parts, cols):
        assert v.tolist() == np.asarray(v0, np.float32).tolist() and t.tolist() == np.asarray(t0).tolist()
        assert c.tolist() == c0.tolist() and c[3] == 255
    pos = js["accessors"][js["meshes"][0]["primitives"][0]["attributes"]["POSITION"]]
    assert pos["min"] == [-1.0, -1.0, -1.0] and pos["max"] == [1.0, 1.0, 1.0]
    (tmp_path / "s.glb").write_bytes(data)
    v, t = meshio.load_mesh(tmp_path / "s.glb")          # the scene flattened: 8 + 8 corners
    assert len(t) == 16 and len(v) == 16


def test_part_colors_follow_the_seeded_draws():
    rng = np.random.default_rng(0)
    want = [(rng.random(3) * 255).astype(np.uint8).tolist() for _ in range(4)]
    assert meshio.part_colors(4)[:, :3].tolist() == want


def _gltf_doc(v, t, nodes, uri=None):
    blob = np.ascontiguousarray(v, np.float32).tobytes() + np.ascontiguousarray(t, np.uint16).tobytes()
    pad = -len(blob) % 4
    buf = {"byteLength": len(blob) + pad}
    if uri is not None:
        buf["uri"] = uri
    js = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": [0]}], "nodes": nodes,
          "meshes": [{"primitives": [{"attributes": {"POSITION": 0}, "indices": 1}]}],
          "accessors": [{"bufferView": 0, "componentType": 5126, "count": len(v), "type": "VEC3"},
                        {"bufferView": 1, "componentType": 5123, "count": t.size, "type": "SCALAR"}],
          "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": 12 * len(v)},
                          {"buffer": 0, "byteOffset": 12 * len(v), "byteLength": 2 * t.size}],
          "buffers": [buf]}
    return js, blob + b"\0" * pad


def test_gltf_transforms_and_buffers(tmp_path):
    # root: translate (10, 0, 0); child: rotate 90 degrees about z, scale 2; grandchild holds the mesh
    s = np.sqrt(0.5)
    nodes = [{"translation": [10, 0, 0], "children": [1]},
             {"rotation": [0, 0, s, s], "scale": [2, 2, 2], "children": [2]},
             {"matrix": [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 3, 1], "mesh": 0}]
    js, blob = _gltf_doc(CUBE_V, CUBE_T, nodes)
    jb = json.dumps(js).encode()
    jb += b" " * (-len(jb) % 4)
    glb = struct.pack("<III", 0x46546C67, 2, 28 + len(jb) + len(blob)) + struct.pack("<II", len(jb), 0x4E4F534A) \
        + jb + struct.pack("<II", len(blob), 0x004E4942) + blob
    (tmp_path / "x.glb").write_bytes(glb)
    v, t = meshio.load_mesh(tmp_path / "x.glb")
    w = CUBE_V.astype(np.float64) + [0, 0, 3]                  # grandchild
    w = np.stack([-w[:, 1], w[:, 0], w[:, 2]], 1) * 2          # child: Rz(90) then scale
    w = (w + [10, 0, 0]).astype(np.float32)
    assert np.allclose(v, w, atol=1e-5) and t.tolist() == CUBE_T.tolist()
    # .gltf with a data URI, and with a side-by-side .bin file
    js2, blob2 = _gltf_doc(CUBE_V, CUBE_T, [{"mesh": 0}],
                           uri="data:application/octet-stream;base64," + base64.b64encode(_gltf_doc(
                               CUBE_V, CUBE_T, [{"mesh": 0}])[1]).decode())
    (tmp_path / "d.gltf").write_text(json.dumps(js2))
    js3, blob3 = _gltf_doc(CUBE_V, CUBE_T, [{"mesh": 0}], uri="c.bin")
    (tmp_path / "c.bin").write_bytes(blob3)
    (tmp_path / "e.gltf").write_text(json.dumps(js3))
    for name in ("d.gltf", "e.gltf"):
        v, t = meshio.load_mesh(tmp_path / name)
        assert v.tolist() == CUBE_V.tolist() and t.tolist() == CUBE_T.tolist()


def test_pool_size_parser():
    assert cli.parse_pool_bytes("0") == 0
    assert cli.parse_pool_bytes("512M") == 512 << 20
    assert cli.parse_pool_bytes("1.5g") == 3 << 29
    assert cli.parse_pool_bytes("64k") == 64 << 10
    with pytest.raises(Exception):
        cli.parse_pool_bytes("lots")


def _write_obj(path, v, t):
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text("\n".join([f"v {x!r} {y!r} {z!r}" for x, y, z in v.tolist()] +
                              [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in np.asarray(t).tolist()]) + "\n")


def _tree(tmp_path):
    src = tmp_path / "in"
    a = box_mesh([0, 0, 0], [2, 1, 1])
    b = box_mesh([-3, 1, 0.5], [-1, 4, 2])
    _write_obj(src / "a.obj", *a)
    _write_obj(src / "sub" / "b.obj", *b)
    pyr_v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0.5, 0.5, 1]], np.float32)
    pyr_t = np.array([[0, 2, 1], [0, 3, 2], [0, 1, 4], [1, 2, 4], [2, 3, 4], [3, 0, 4]])
    _write_obj(src / "sub" / "pyr.obj", pyr_v, pyr_t)
    (src / "notes.txt").write_text("not a mesh")
    return src, {"a": a, "b": b}


def test_pipeline_writes_parts_in_input_coordinates(tmp_path, capfd):
    src, meshes = _tree(tmp_path)
    out = tmp_path / "out"
    rc = cli.main([str(src), str(out), "-r"], context_factory=cli_fakes.ok_factory)
    so, se = capfd.readouterr()
    assert rc == 0, se
    assert sorted(p.relative_to(out).as_posix() for p in out.rglob("*.glb")) == ["a.glb", "sub/b.glb", "sub/pyr.glb"]
    for name, rel in (("a", "a.glb"), ("b", "sub/b.glb")):
        parts = meshio.read_glb_parts((out / rel).read_bytes())
        stem = rel.split("/")[-1][:-4]
        assert [p[0] for p in parts] == [f"{stem}_0", f"{stem}_1"]
        v0, t0 = meshes[name]
        assert np.allclose(parts[0][1], v0, atol=1e-6) and parts[0][2].tolist() == t0.tolist()
        assert np.allclose(parts[1][1].min(0), v0.min(0), atol=1e-6)
    assert "a.obj" in so and "2 parts" in so
    # not recursive: only the top-level mesh
    out2 = tmp_path / "out2"
    assert cli.main([str(src), str(out2)], context_factory=cli_fakes.ok_factory) == 0
    assert [p.name for p in out2.rglob("*.glb")] == ["a.glb"]


def test_pipeline_retries_with_a_fresh_context(tmp_path, capfd):
    src, _ = _tree(tmp_path)
    out = tmp_path / "out"
    rc = cli.main([str(src / "a.obj"), str(out)], context_factory=cli_fakes.flaky_factory)
    so, se = capfd.readouterr()
    assert rc == 0 and (out / "a.glb").exists()
    assert "reopening the context and retrying" in se


def test_pipeline_gives_up_after_one_retry(tmp_path, capfd):
    src, _ = _tree(tmp_path)
    out = tmp_path / "out"
    rc = cli.main([str(src), str(out), "-r"], context_factory=cli_fakes.failing_factory)
    so, se = capfd.readouterr()
    assert rc == 0 and not list(out.rglob("*.glb"))
    assert se.count("decompose error on retry") == 3


def test_pipeline_reports_a_dead_decomposer(tmp_path, capfd):
    src, _ = _tree(tmp_path)
    out = tmp_path / "out"
    rc = cli.main([str(src), str(out), "-r"], context_factory=cli_fakes.crash_factory)
    so, se = capfd.readouterr()
    assert rc == 1
    assert "decomposer exited with code -9 while decomposing 'sub/pyr.obj'" in se.replace(os.sep, "/")
    assert "native crash" in se


def test_preprocess_modes(tmp_path, capfd):
    """auto remeshes only what the audit flags (the fake flags an odd
    triangle count and remeshes to the bounding box); on always; off never."""
    src, meshes = _tree(tmp_path)
    _write_obj(src / "odd.obj", meshes["a"][0], meshes["a"][1][:11])
    for mode, remeshed in (("auto", {"odd"}), ("on", {"odd", "pyr"}), ("off", set())):
        out = tmp_path / mode
        assert cli.main([str(src), str(out), "-r", "--serial", "--preprocess", mode],
                        context_factory=cli_fakes.ok_factory) == 0
        for stem, rel in (("odd", "odd.glb"), ("pyr", "sub/pyr.glb")):       # 11 and 6 triangles as given
            part0 = meshio.read_glb_parts((out / rel).read_bytes())[0]
            assert (len(part0[2]) == 12) == (stem in remeshed), (mode, stem)
    capfd.readouterr()


def test_serial_and_bench_modes(tmp_path, capfd):
    src, _ = _tree(tmp_path)
    for flag, extra in (("--serial", ""), ("--bench", "MiB")):
        out = tmp_path / flag.strip("-")
        rc = cli.main([str(src), str(out), "-r", flag], context_factory=cli_fakes.ok_factory)
        so, se = capfd.readouterr()
        assert rc == 0, se
        assert len(list(out.rglob("*.glb"))) == 3
        assert all(extra in line for line in so.strip().splitlines())


def test_no_meshes(tmp_path, capfd):
    (tmp_path / "empty").mkdir()
    assert cli.main([str(tmp_path / "empty"), str(tmp_path / "o")], context_factory=cli_fakes.ok_factory) == 1


def test_supervisor_clean_and_failed_workers():
    assert cli.supervise([("loader", cli_fakes.FakeProc(0)), ("saver", cli_fakes.FakeProc(0))], poll=0) is None
    survivor = cli_fakes.FakeProc(0, ticks=10)
    assert cli.supervise([("decomposer", cli_fakes.FakeProc(-11)), ("loader", survivor)], poll=0) == \
        ("decomposer", -11)
    assert survivor.terminated


def test_supervisor_sees_a_failure_on_the_last_poll():
    # both end on the same poll; the non-zero one must not pass as a clean end
    assert cli.supervise([("loader", cli_fakes.FakeProc(0)), ("saver", cli_fakes.FakeProc(3))], poll=0) == \
        ("saver", 3)
    # the failing one is still alive on the first poll and ends with the other
    assert cli.supervise([("saver", cli_fakes.FakeProc(3, ticks=1)), ("loader", cli_fakes.FakeProc(0, ticks=1))],
                         poll=0) == ("saver", 3)


def test_supervisor_breaks_a_real_deadlock():
    """A consumer that dies after one item leaves its peer blocked on a queue
    forever; the supervisor ends the peer and reports the dead one."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q1, q2 = ctx.Queue(maxsize=2), ctx.Queue(maxsize=2)
    dead = ctx.Process(target=cli_fakes.exit_after_one_item, args=(q1,))
    blocked = ctx.Process(target=cli_fakes.wait_for_item, args=(q2,))
    dead.start()
    blocked.start()
    q1.put(("mesh.obj", None, None))
    try:
        assert cli.supervise([("decomposer", dead), ("saver", blocked)]) == ("decomposer", 3)
    finally:
        dead.join(10)
        blocked.join(10)
    assert not blocked.is_alive()


def test_current_mesh_buffer():
    import multiprocessing as mp
    buf = mp.get_context("spawn").Array("c", cli._CUR_BYTES)
    cli.set_current(buf, "dir/a.obj")
    assert cli.get_current(buf) == "dir/a.obj"
    cli.set_current(buf, "b.obj")                      # no tail of the longer name
    assert cli.get_current(buf) == "b.obj"
    cli.set_current(buf, "x" * (cli._CUR_BYTES + 64))  # truncated, not dropped
    assert cli.get_current(buf) == "x" * (cli._CUR_BYTES - 1)


def test_gltf_interleaved_accessor(tmp_path):
    """POSITION interleaved with a 4-byte attribute (byteStride 16)."""
    rows = np.zeros(8, np.dtype([("p", "<f4", (3,)), ("c", "u1", (4,))]))
    rows["p"] = CUBE_V
    idx = CUBE_T.astype("<u4").tobytes()
    blob = rows.tobytes() + idx
    js = {"asset": {"version": "2.0"}, "meshes": [{"primitives": [{"attributes": {"POSITION": 0}, "indices": 1}]}],
          "accessors": [{"bufferView": 0, "componentType": 5126, "count": 8, "type": "VEC3"},
                        {"bufferView": 1, "componentType": 5125, "count": CUBE_T.size, "type": "SCALAR"}],
          "bufferViews": [{"buffer": 0, "byteOffset": 0, "byteLength": 128, "byteStride": 16},
                          {"buffer": 0, "byteOffset": 128, "byteLength": len(idx)}],
          "buffers": [{"byteLength": len(blob), "uri": "data:application/octet-stream;base64,"
                       + base64.b64encode(blob).decode()}]}
    (tmp_path / "i.gltf").write_text(json.dumps(js))
    v, t = meshio.load_mesh(tmp_path / "i.gltf")             # no nodes: every mesh, untransformed
    assert v.tolist() == CUBE_V.tolist() and t.tolist() == CUBE_T.tolist()


def test_malformed_files_raise_value_error(tmp_path):
    good = meshio.glb_bytes([(CUBE_V, CUBE_T)], ["c_0"])
    cases = {"short.glb": good[:40], "bad.glb": b"glTF" + b"\0" * 16, "x.ply": b"ply\nformat ascii 1.0\n",
             "y.ply": b"ply\nformat binary_little_endian 1.0\nelement vertex 8\nproperty float x\n"
                      b"property float y\nproperty float z\nend_header\n" + b"\0" * 10,
             "z.off": b"OF\n", "w.obj": b"v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n", "q.stl": b"solid x\nvertex 0 0 0\n",
             "n.xyz": b"", "h.off": b"OFF\n", "s.stl": b"solid x\nvertex 0 0\n",
             "f.ply": b"ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
                      b"element face 1\nproperty list uchar int corners\nend_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n"}
    for name, data in cases.items():
        (tmp_path / name).write_bytes(data)
        with pytest.raises(ValueError):
            meshio.load_mesh(tmp_path / name)
