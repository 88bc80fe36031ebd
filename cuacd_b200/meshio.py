"""Mesh files for the command-line pipeline (cuacd_b200/cli.py).

Readers for OBJ, STL (binary and ASCII), PLY (ASCII and binary, either byte
order), OFF and glTF 2.0 (.glb, and .gltf with embedded or side-by-side
buffers), and a GLB writer for decomposition results.  They take the place
of the reference's `_load_mesh` / `_save_parts` (cuacd/cli.py:42-47,
87-102), which go through trimesh; trimesh is not part of this library's
dependencies.

Every reader returns (verts float32 (n, 3), tris int32 (m, 3)):
- polygons are split into fans from their first corner;
- vertices with exactly equal coordinates are merged and vertices no
  triangle uses are dropped, the rest keeping their file order, so that a
  mesh whose seams repeat vertices (an STL triangle soup, an OBJ split by
  texture coordinates) comes out closed;
- a glTF scene is flattened: every triangle primitive of every node of the
  default scene, moved by the node's world transform.
"""
import base64
import json
import os
import struct

import numpy as np

MESH_EXTS = (".obj", ".stl", ".ply", ".off", ".glb", ".gltf")


# --------------------------------------------------------------------------
# common
# --------------------------------------------------------------------------
def fan(poly):
    """Triangles (first, k, k+1) of one polygon's corner list."""
    return [(poly[0], poly[k], poly[k + 1]) for k in range(1, len(poly) - 1)]


def clean_mesh(verts, tris):
    """Merge exactly equal vertices (0.0 and -0.0 are equal), drop the ones
    no triangle references; the kept vertices stay in file order."""
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.int64).reshape(-1, 3)
    if len(t) and (t.min() < 0 or t.max() >= len(v)):
        raise ValueError(f"triangle index out of range (0..{len(v) - 1})")
    if len(t) == 0:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int32)
    used = np.zeros(len(v), bool)
    used[t.reshape(-1)] = True
    if not np.isfinite(v[used]).all():
        raise ValueError("non-finite vertex coordinates")
    key = np.ascontiguousarray(v + np.float32(0.0))            # -0.0 -> 0.0
    key = key.view(np.dtype((np.void, 12))).reshape(-1)
    keep = np.flatnonzero(used)
    _, first, inv = np.unique(key[keep], return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")                    # groups by first occurrence
    rank = np.empty(len(order), np.int64)
    rank[order] = np.arange(len(order))
    new_id = np.full(len(v), -1, np.int64)
    new_id[keep] = rank[inv.reshape(-1)]
    out_v = v[keep[first[order]]]
    return np.ascontiguousarray(out_v, np.float32), new_id[t].astype(np.int32)


def load_mesh(path):
    """(verts, tris) of a mesh file, by its extension.  A file that does not
    parse raises ValueError."""
    ext = os.path.splitext(str(path))[1].lower()
    with open(path, "rb") as f:
        data = f.read()
    try:
        return _load(data, ext, path)
    except (IndexError, KeyError, struct.error, UnicodeDecodeError) as e:
        raise ValueError(f"malformed {ext or 'mesh'} file: {type(e).__name__}: {e}") from None


def _load(data, ext, path):
    if ext == ".obj":
        v, t = read_obj(data)
    elif ext == ".stl":
        v, t = read_stl(data)
    elif ext == ".ply":
        v, t = read_ply(data)
    elif ext == ".off":
        v, t = read_off(data)
    elif ext == ".glb":
        v, t = read_glb(data)
    elif ext == ".gltf":
        v, t = read_gltf(data, os.path.dirname(os.path.abspath(str(path))))
    else:
        raise ValueError(f"unsupported mesh format: {ext or '(none)'}")
    return clean_mesh(v, t)


# --------------------------------------------------------------------------
# OBJ
# --------------------------------------------------------------------------
def read_obj(data):
    """`v x y z` and `f` records (indices 1-based or negative, `i`, `i/t`,
    `i//n`, `i/t/n`); everything else is ignored."""
    vs, tris = [], []
    for ln, line in enumerate(data.decode("utf-8", "replace").splitlines(), 1):
        rec = line.split("#", 1)[0].split()
        if not rec:
            continue
        if rec[0] == "v":
            if len(rec) < 4:
                raise ValueError(f"OBJ line {ln}: vertex with fewer than 3 coordinates")
            vs.append((float(rec[1]), float(rec[2]), float(rec[3])))
        elif rec[0] == "f":
            poly = []
            for c in rec[1:]:
                i = int(c.split("/", 1)[0])
                if i == 0:
                    raise ValueError(f"OBJ line {ln}: index 0")
                poly.append(i - 1 if i > 0 else len(vs) + i)
            tris += fan(poly)
    return np.asarray(vs, np.float32).reshape(-1, 3), np.asarray(tris, np.int64).reshape(-1, 3)


# --------------------------------------------------------------------------
# STL
# --------------------------------------------------------------------------
_STL_REC = np.dtype([("n", "<f4", (3,)), ("v", "<f4", (3, 3)), ("attr", "<u2")])


def read_stl(data):
    """Binary STL when the size matches its triangle count, else ASCII
    (`vertex x y z` records, three per facet)."""
    if len(data) >= 84:
        n = struct.unpack_from("<I", data, 80)[0]
        if 84 + 50 * n == len(data):
            rec = np.frombuffer(data, _STL_REC, count=n, offset=84)
            return rec["v"].reshape(-1, 3).astype(np.float32), np.arange(3 * n, dtype=np.int64).reshape(-1, 3)
    vs = []
    for line in data.decode("ascii", "replace").splitlines():
        rec = line.split()
        if rec and rec[0] == "vertex":
            vs.append((float(rec[1]), float(rec[2]), float(rec[3])))
    if len(vs) % 3:
        raise ValueError("ASCII STL: vertex count is not a multiple of 3")
    return np.asarray(vs, np.float32).reshape(-1, 3), np.arange(len(vs), dtype=np.int64).reshape(-1, 3)


# --------------------------------------------------------------------------
# PLY
# --------------------------------------------------------------------------
_PLY_TYPES = {"char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1", "short": "i2", "int16": "i2",
              "ushort": "u2", "uint16": "u2", "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4",
              "float": "f4", "float32": "f4", "double": "f8", "float64": "f8"}


def read_ply(data):
    """`vertex` element (x, y, z) and `face` element (`vertex_indices` or
    `vertex_index` list); other elements and properties are skipped."""
    end = data.find(b"end_header")
    if not data.startswith(b"ply") or end < 0:
        raise ValueError("PLY: missing header")
    body = data.index(b"\n", end) + 1
    fmt, elements = None, []
    for line in data[:end].decode("ascii", "replace").splitlines()[1:]:
        rec = line.split()
        if not rec or rec[0] in ("comment", "obj_info"):
            continue
        if rec[0] == "format":
            fmt = rec[1]
        elif rec[0] == "element":
            elements.append((rec[1], int(rec[2]), []))
        elif rec[0] == "property":
            if rec[1] == "list":
                elements[-1][2].append(("list", _PLY_TYPES[rec[2]], _PLY_TYPES[rec[3]], rec[4]))
            else:
                elements[-1][2].append(("scalar", _PLY_TYPES[rec[1]], rec[2]))
    if fmt not in ("ascii", "binary_little_endian", "binary_big_endian"):
        raise ValueError(f"PLY: unsupported format {fmt}")
    verts, tris, bulk = None, [], []
    if fmt == "ascii":
        tok = data[body:].split()
        pos = 0
        for name, count, props in elements:
            rows = []
            for _ in range(count):
                row = {}
                for p in props:
                    if p[0] == "scalar":
                        row[p[2]] = float(tok[pos]); pos += 1
                    else:
                        k = int(tok[pos]); pos += 1
                        row[p[3]] = [int(x) for x in tok[pos:pos + k]]; pos += k
                rows.append(row)
            if name == "vertex":
                verts = np.asarray([(r["x"], r["y"], r["z"]) for r in rows], np.float32).reshape(-1, 3)
            elif name == "face":
                key = "vertex_indices" if props and any(p[-1] == "vertex_indices" for p in props) else "vertex_index"
                for r in rows:
                    tris += fan(r[key])
    else:
        bo = "<" if fmt == "binary_little_endian" else ">"
        pos = body
        for name, count, props in elements:
            if all(p[0] == "scalar" for p in props):
                dt = np.dtype([(p[2], bo + p[1]) for p in props])
                arr = np.frombuffer(data, dt, count=count, offset=pos)
                pos += dt.itemsize * count
                if name == "vertex":
                    verts = np.stack([arr["x"], arr["y"], arr["z"]], 1).astype(np.float32)
                continue
            if name == "face" and len(props) == 1 and props[0][3] in ("vertex_indices", "vertex_index"):
                # every face a triangle: one bulk read
                dt = np.dtype([("k", bo + props[0][1]), ("i", bo + props[0][2], (3,))])
                if pos + dt.itemsize * count <= len(data):
                    arr = np.frombuffer(data, dt, count=count, offset=pos)
                    if (arr["k"] == 3).all():
                        bulk.append(arr["i"].astype(np.int64))
                        pos += dt.itemsize * count
                        continue
            for _ in range(count):
                for p in props:
                    if p[0] == "scalar":
                        pos += np.dtype(p[1]).itemsize
                        continue
                    ct, it = np.dtype(bo + p[1]), np.dtype(bo + p[2])
                    k = int(np.frombuffer(data, ct, 1, pos)[0]); pos += ct.itemsize
                    idx = np.frombuffer(data, it, k, pos).tolist(); pos += it.itemsize * k
                    if name == "face" and p[3] in ("vertex_indices", "vertex_index"):
                        tris += fan(idx)
    if verts is None:
        raise ValueError("PLY: no vertex element")
    return verts, np.concatenate(bulk + [np.asarray(tris, np.int64).reshape(-1, 3)])


# --------------------------------------------------------------------------
# OFF
# --------------------------------------------------------------------------
def read_off(data):
    """OFF / COFF / NOFF: counts, vertex rows (first three numbers), face
    rows `k i0 .. i(k-1)`."""
    lines = [l.split("#", 1)[0].split() for l in data.decode("ascii", "replace").splitlines()]
    lines = [l for l in lines if l]
    if not lines or not lines[0][0].endswith("OFF"):
        raise ValueError("OFF: missing header")
    head = lines[0][1:] if len(lines[0]) > 1 else lines[1]
    rest = lines[1:] if len(lines[0]) > 1 else lines[2:]
    nv, nf = int(head[0]), int(head[1])
    verts = np.asarray([[float(x) for x in r[:3]] for r in rest[:nv]], np.float32).reshape(-1, 3)
    tris = []
    for r in rest[nv:nv + nf]:
        k = int(r[0])
        tris += fan([int(x) for x in r[1:1 + k]])
    return verts, np.asarray(tris, np.int64).reshape(-1, 3)


# --------------------------------------------------------------------------
# glTF 2.0
# --------------------------------------------------------------------------
_GLB_MAGIC, _CHUNK_JSON, _CHUNK_BIN = 0x46546C67, 0x4E4F534A, 0x004E4942
_COMP = {5120: "i1", 5121: "u1", 5122: "i2", 5123: "u2", 5125: "u4", 5126: "f4"}
_NCOMP = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT2": 4, "MAT3": 9, "MAT4": 16}


def split_glb(data):
    """(json dict, BIN chunk bytes or None) of a GLB file."""
    if len(data) < 20:
        raise ValueError("GLB: too short")
    magic, version, length = struct.unpack_from("<III", data, 0)
    if magic != _GLB_MAGIC or version != 2:
        raise ValueError("GLB: not a glTF 2.0 binary")
    pos, js, binc = 12, None, None
    while pos + 8 <= min(length, len(data)):
        clen, ctype = struct.unpack_from("<II", data, pos)
        chunk = data[pos + 8:pos + 8 + clen]
        if ctype == _CHUNK_JSON:
            js = json.loads(chunk.decode("utf-8"))
        elif ctype == _CHUNK_BIN and binc is None:
            binc = bytes(chunk)
        pos += 8 + clen
    if js is None:
        raise ValueError("GLB: no JSON chunk")
    return js, binc


def read_glb(data):
    js, binc = split_glb(data)
    return _gltf_mesh(js, binc, None)


def read_gltf(data, base_dir):
    return _gltf_mesh(json.loads(data.decode("utf-8")), None, base_dir)


def _gltf_buffers(js, binc, base_dir):
    out = []
    for b in js.get("buffers", []):
        uri = b.get("uri")
        if uri is None:
            if binc is None:
                raise ValueError("glTF: buffer without data")
            out.append(binc)
        elif uri.startswith("data:"):
            out.append(base64.b64decode(uri.split(",", 1)[1]))
        else:
            if base_dir is None:
                raise ValueError("glTF: external buffer in a GLB")
            with open(os.path.join(base_dir, uri), "rb") as f:
                out.append(f.read())
    return out


def gltf_accessor(js, buffers, i):
    """Accessor i as a (count, components) array of its component type."""
    a = js["accessors"][i]
    if "sparse" in a:
        raise ValueError("glTF: sparse accessors are not supported")
    dt = np.dtype("<" + _COMP[a["componentType"]])
    nc, count = _NCOMP[a["type"]], a["count"]
    if "bufferView" not in a:
        return np.zeros((count, nc), dt)
    bv = js["bufferViews"][a["bufferView"]]
    buf = buffers[bv["buffer"]]
    off = bv.get("byteOffset", 0) + a.get("byteOffset", 0)
    stride = bv.get("byteStride", 0) or dt.itemsize * nc
    if stride == dt.itemsize * nc:
        return np.frombuffer(buf, dt, count * nc, off).reshape(count, nc)
    rows = np.frombuffer(buf, np.uint8, (count - 1) * stride + dt.itemsize * nc, off)
    return np.stack([rows[k * stride:k * stride + dt.itemsize * nc].view(dt) for k in range(count)])


def _node_matrix(node):
    if "matrix" in node:
        return np.asarray(node["matrix"], np.float64).reshape(4, 4).T        # column-major
    x, y, z, w = node.get("rotation", (0.0, 0.0, 0.0, 1.0))
    r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    m = np.eye(4)
    m[:3, :3] = r * np.asarray(node.get("scale", (1.0, 1.0, 1.0)), np.float64)[None, :]
    m[:3, 3] = node.get("translation", (0.0, 0.0, 0.0))
    return m


def _prim_tris(js, buffers, prim, nv):
    mode = prim.get("mode", 4)
    idx = (gltf_accessor(js, buffers, prim["indices"]).reshape(-1).astype(np.int64)
           if "indices" in prim else np.arange(nv, dtype=np.int64))
    if mode == 4:
        return idx[:len(idx) // 3 * 3].reshape(-1, 3)
    if mode == 5:                                    # strip: alternate winding
        t = [(idx[k], idx[k + 1], idx[k + 2]) if k % 2 == 0 else (idx[k + 1], idx[k], idx[k + 2])
             for k in range(len(idx) - 2)]
        return np.asarray(t, np.int64).reshape(-1, 3)
    if mode == 6:                                    # fan
        return np.asarray(fan(list(idx)), np.int64).reshape(-1, 3)
    return np.zeros((0, 3), np.int64)                # points and lines carry no surface


def _gltf_mesh(js, binc, base_dir):
    if js.get("extensionsRequired"):
        raise ValueError(f"glTF: required extensions {js['extensionsRequired']} are not supported")
    buffers = _gltf_buffers(js, binc, base_dir)
    nodes = js.get("nodes", [])
    if js.get("scenes"):
        roots = js["scenes"][js.get("scene", 0)].get("nodes", [])
    else:
        children = {c for n in nodes for c in n.get("children", [])}
        roots = [i for i in range(len(nodes)) if i not in children]
    vs, ts, base = [], [], 0
    stack = [(r, np.eye(4)) for r in reversed(roots)]
    placed = []
    while stack:
        i, parent = stack.pop()
        m = parent @ _node_matrix(nodes[i])
        if "mesh" in nodes[i]:
            placed.append((nodes[i]["mesh"], m))
        for c in reversed(nodes[i].get("children", [])):
            stack.append((c, m))
    if not nodes:
        placed = [(k, np.eye(4)) for k in range(len(js.get("meshes", [])))]
    for mi, m in placed:
        for prim in js["meshes"][mi]["primitives"]:
            p = gltf_accessor(js, buffers, prim["attributes"]["POSITION"]).astype(np.float64)
            t = _prim_tris(js, buffers, prim, len(p))
            if len(t) == 0:
                continue
            vs.append(p @ m[:3, :3].T + m[:3, 3])
            ts.append(t + base)
            base += len(p)
    if not vs:
        return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.int64)
    return np.concatenate(vs).astype(np.float32), np.concatenate(ts)


def part_colors(n, seed=0):
    """RGBA colour of each of n parts: three uniform bytes per part from a
    seeded generator (the reference draws `rng.random(3) * 255` per part
    from default_rng(0), cuacd/cli.py:89-96), alpha 255."""
    rng = np.random.default_rng(seed)
    out = np.full((n, 4), 255, np.uint8)
    for i in range(n):
        out[i, :3] = (rng.random(3) * 255).astype(np.uint8)
    return out


def glb_bytes(parts, names, colors=None):
    """A GLB scene with one node per part: node / mesh `names[i]`, float32
    positions (with their bounds), the part's colour on every vertex
    (COLOR_0, normalised bytes) and uint32 triangle indices."""
    if colors is None:
        colors = part_colors(len(parts))
    blob = bytearray()
    views, accessors, meshes, nodes = [], [], [], []

    def view(arr, target):
        while len(blob) % 4:
            blob.append(0)
        b = np.ascontiguousarray(arr).tobytes()
        views.append({"buffer": 0, "byteOffset": len(blob), "byteLength": len(b), "target": target})
        blob.extend(b)
        return len(views) - 1

    for i, (v, t) in enumerate(parts):
        v = np.ascontiguousarray(v, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(t, np.uint32).reshape(-1, 3)
        node = {"name": names[i]}
        if len(t) and len(v):
            col = np.broadcast_to(np.asarray(colors[i], np.uint8), (len(v), 4))
            accessors.append({"bufferView": view(v, 34962), "componentType": 5126, "count": len(v), "type": "VEC3",
                              "min": [float(x) for x in v.min(0)], "max": [float(x) for x in v.max(0)]})
            pa = len(accessors) - 1
            accessors.append({"bufferView": view(col, 34962), "componentType": 5121, "normalized": True,
                              "count": len(v), "type": "VEC4"})
            ca = len(accessors) - 1
            accessors.append({"bufferView": view(t, 34963), "componentType": 5125, "count": 3 * len(t),
                              "type": "SCALAR"})
            meshes.append({"name": names[i], "primitives": [{"attributes": {"POSITION": pa, "COLOR_0": ca},
                                                            "indices": len(accessors) - 1, "mode": 4}]})
            node["mesh"] = len(meshes) - 1
        nodes.append(node)
    while len(blob) % 4:
        blob.append(0)
    js = {"asset": {"version": "2.0", "generator": "cuacd_b200"}, "scene": 0,
          "scenes": [{"nodes": list(range(len(nodes)))}], "nodes": nodes}
    if meshes:
        js.update(meshes=meshes, accessors=accessors, bufferViews=views, buffers=[{"byteLength": len(blob)}])
    jb = json.dumps(js, separators=(",", ":")).encode("utf-8")
    jb += b" " * (-len(jb) % 4)
    out = struct.pack("<III", _GLB_MAGIC, 2, 12 + 8 + len(jb) + (8 + len(blob) if meshes else 0))
    out += struct.pack("<II", len(jb), _CHUNK_JSON) + jb
    if meshes:
        out += struct.pack("<II", len(blob), _CHUNK_BIN) + bytes(blob)
    return out


def read_glb_parts(data):
    """[(node name, verts, tris, RGBA colour or None)] of a GLB scene, one per
    node with a mesh (world transforms applied): the reader of glb_bytes'
    files, for checking them."""
    js, binc = split_glb(data)
    buffers = _gltf_buffers(js, binc, None)
    out = []
    for node in js.get("nodes", []):
        if "mesh" not in node:
            continue
        m = _node_matrix(node)
        vs, ts, col, base = [], [], None, 0
        for prim in js["meshes"][node["mesh"]]["primitives"]:
            p = gltf_accessor(js, buffers, prim["attributes"]["POSITION"]).astype(np.float64)
            vs.append(p @ m[:3, :3].T + m[:3, 3])
            ts.append(_prim_tris(js, buffers, prim, len(p)) + base)
            base += len(p)
            if "COLOR_0" in prim["attributes"] and col is None:
                col = gltf_accessor(js, buffers, prim["attributes"]["COLOR_0"])[0].copy()
        out.append((node.get("name"), np.concatenate(vs).astype(np.float32),
                    np.concatenate(ts).astype(np.int32), col))
    return out
