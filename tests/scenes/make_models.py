"""Writes the model files the XML test scenes load (run from any directory;
the outputs are committed next to this script, under models/):

* pyramid.obj + pyramid.mtl: a square pyramid, four triangular sides in one
  material and the quad base in another, no normals (the CLI's model loader
  generates smooth ones), texture coordinates on the sides, negative
  (relative) indices on the base;
* prism.gltf: a triangular prism (flat normals, texture coordinates, 16-bit
  indices) whose buffer is a base64 data URI, under a node with a matrix and
  a child node;
* prism.glb: the same prism in the binary container (JSON + BIN chunk).
"""
import base64
import json
import os
import struct

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "models")

PYRAMID_OBJ = """\
# Square pyramid: apex above a unit square base.
mtllib pyramid.mtl
o pyramid
v -0.5 0 -0.5
v 0.5 0 -0.5
v 0.5 0 0.5
v -0.5 0 0.5
v 0 0.8 0
vt 0 0
vt 1 0
vt 0.5 1
usemtl amber
s 1
f 4/1 3/2 5/3
f 3/1 2/2 5/3
f 2/1 1/2 5/3
f 1/1 4/2 5/3
usemtl slate
s off
f -5 -4 -3 -2
"""

PYRAMID_MTL = """\
# Materials of pyramid.obj
newmtl amber
Kd 0.9 0.55 0.15
Ks 0.04
Ns 50
illum 2

newmtl slate
Kd 0.2 0.3 0.6
illum 1
"""


def prism_geometry():
    """Flat-shaded triangular prism: 2 triangular caps and 3 quad sides."""
    import math
    tri = [(math.cos(a), math.sin(a)) for a in (math.pi / 2, math.pi / 2 + 2 * math.pi / 3,
                                                  math.pi / 2 + 4 * math.pi / 3)]
    pos, nrm, uv, idx = [], [], [], []

    def face(corners, n):
        base = len(pos)
        for k, p in enumerate(corners):
            pos.append(p)
            nrm.append(n)
            uv.append(((k & 1) * 1.0, (k >> 1) * 1.0))
        for k in range(1, len(corners) - 1):
            idx.extend([base, base + k, base + k + 1])

    h = 0.5
    face([(x * 0.5, y * 0.5, h) for x, y in tri], (0.0, 0.0, 1.0))
    face([(x * 0.5, y * 0.5, -h) for x, y in reversed(tri)], (0.0, 0.0, -1.0))
    for k in range(3):
        (x0, y0), (x1, y1) = tri[k], tri[(k + 1) % 3]
        nx, ny = (y1 - y0), -(x1 - x0)
        ln = math.hypot(nx, ny)
        face([(x0 * 0.5, y0 * 0.5, -h), (x1 * 0.5, y1 * 0.5, -h), (x1 * 0.5, y1 * 0.5, h),
              (x0 * 0.5, y0 * 0.5, h)], (nx / ln, ny / ln, 0.0))
    return pos, nrm, uv, idx


def prism_buffer_and_json(uri):
    pos, nrm, uv, idx = prism_geometry()
    b = bytearray()
    b += b"".join(struct.pack("<3f", *p) for p in pos)
    off_n = len(b)
    b += b"".join(struct.pack("<3f", *n) for n in nrm)
    off_uv = len(b)
    b += b"".join(struct.pack("<2f", *t) for t in uv)
    off_i = len(b)
    b += b"".join(struct.pack("<H", i) for i in idx)
    n = len(pos)
    lo = [min(p[k] for p in pos) for k in range(3)]
    hi = [max(p[k] for p in pos) for k in range(3)]
    doc = {
        "asset": {"version": "2.0", "generator": "make_models.py"},
        "scene": 0,
        "scenes": [{"nodes": [0]}],
        "nodes": [
            {"name": "root", "children": [1],
             "matrix": [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0.1, 0, 1]},
            {"name": "prism", "mesh": 0},
        ],
        "meshes": [{"primitives": [{"attributes": {"POSITION": 0, "NORMAL": 1, "TEXCOORD_0": 2},
                                    "indices": 3, "mode": 4}]}],
        "accessors": [
            {"bufferView": 0, "componentType": 5126, "count": n, "type": "VEC3", "min": lo, "max": hi},
            {"bufferView": 0, "byteOffset": off_n, "componentType": 5126, "count": n, "type": "VEC3"},
            {"bufferView": 0, "byteOffset": off_uv, "componentType": 5126, "count": n, "type": "VEC2"},
            {"bufferView": 1, "componentType": 5123, "count": len(idx), "type": "SCALAR"},
        ],
        "bufferViews": [
            {"buffer": 0, "byteOffset": 0, "byteLength": off_i},
            {"buffer": 0, "byteOffset": off_i, "byteLength": len(idx) * 2},
        ],
        "buffers": [{"byteLength": len(b)}],
    }
    if uri is not None:
        doc["buffers"][0]["uri"] = uri(bytes(b))
    return bytes(b), doc


def write_gltf(path):
    _, doc = prism_buffer_and_json(
        lambda data: "data:application/octet-stream;base64," + base64.b64encode(data).decode())
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")


def write_glb(path):
    data, doc = prism_buffer_and_json(None)
    js = json.dumps(doc, separators=(",", ":")).encode()
    js += b" " * (-len(js) % 4)
    data += b"\0" * (-len(data) % 4)
    total = 12 + 8 + len(js) + 8 + len(data)
    with open(path, "wb") as f:
        f.write(struct.pack("<III", 0x46546C67, 2, total))
        f.write(struct.pack("<II", len(js), 0x4E4F534A) + js)
        f.write(struct.pack("<II", len(data), 0x004E4942) + data)


def main():
    os.makedirs(OUT, exist_ok=True)
    with open(os.path.join(OUT, "pyramid.obj"), "w") as f:
        f.write(PYRAMID_OBJ)
    with open(os.path.join(OUT, "pyramid.mtl"), "w") as f:
        f.write(PYRAMID_MTL)
    write_gltf(os.path.join(OUT, "prism.gltf"))
    write_glb(os.path.join(OUT, "prism.glb"))


if __name__ == "__main__":
    main()
