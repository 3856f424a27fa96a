"""The reference's per-frame file writers, restated in Python — TEST INFRASTRUCTURE ONLY.

Only tests/ import this; the product's writers are in
2017multiphase_b200/csrc/host/export.cpp. Each function follows one writer of
gaoyangVR/2017Multiphase, Multiphase/Multiphase/spray.cu, line for line in
what it prints: outputPovRaywater (2250-2306), outputOBJwater (2308-2371),
outputBOBJwater (2373-2438), outputColoredParticle (2440-2466),
outputSoloBubblePovRay (2468-2496), outputAirParticlePovRay (2498-2526), with
verifyfloat3 (spray.cu:999-1008) and mapColorBlue2Red_h (spray.cpp:1299-1360).
C's "%f" and Python's "%f" both print the correctly rounded 6-decimal value of
the same double, so the texts agree byte for byte. The reference ships no
output files or tests for these writers; the writers themselves, compiled for
the host by oracle/make_refhost.py, pin the product's files in
tests/test_refhost_io.py, and this restatement stays as the checker that
travels without the reference tree.
"""
from __future__ import annotations

import struct

import numpy as np

TYPEAIR, TYPEAIRSOLO = 1, 4


def _verify3(v) -> bool:
    # verifyfloat3: !(x > 0 || x < 1) only for NaN
    return all((float(a) > 0 or float(a) < 1) for a in v)


def _checked(v):
    return [float(a) for a in v] if _verify3(v) else [0.0, 0.0, 0.0]


def pov_mesh(verts, normals, indices, name: str) -> bytes:
    """outputPovRaywater, spray.cu:2250-2306 (empty mesh: empty file)."""
    nv = len(verts)
    if nv == 0:
        return b""
    out = ["#declare watermesh=mesh2{\n", "vertex_vectors{\n", "%d,\n" % nv]
    for v in verts:
        out.append("< %f, %f, %f >,\n" % tuple(_checked(v)))
    out += ["}\n ", "normal_vectors{\n", "%d,\n" % nv]
    for v in normals:
        out.append("<%f, %f, %f>,\n" % tuple(_checked(v)))
    out += ["}\n ", "face_indices{\n", "%d,\n" % (len(indices) // 3)]
    for t in range(0, len(indices), 3):
        out.append("<%d, %d, %d>,\n" % (int(indices[t]), int(indices[t + 1]), int(indices[t + 2])))
    out += ["}\n ", "inside_vector <0,0,1> }\n ", "object{ watermesh material{%s_material} }\n " % name]
    return "".join(out).encode()


def obj_mesh(verts, normals, indices) -> bytes:
    """outputOBJwater, spray.cu:2308-2371 (1-based indices)."""
    if len(verts) == 0:
        return b""
    out = ["#obj model\n", "#vertex_vectors\n"]
    for v in verts:
        out.append("v  %f %f %f\n" % tuple(_checked(v)))
    out.append("#normal_vectors\n")
    for v in normals:
        out.append("vn  %f %f %f\n" % tuple(_checked(v)))
    out.append("#face_indices\n")
    for t in range(0, len(indices), 3):
        out.append("f  %d %d %d\n" % (int(indices[t]) + 1, int(indices[t + 1]) + 1, int(indices[t + 2]) + 1))
    return "".join(out).encode()


def bobj_payload(verts, normals, indices) -> bytes:
    """The uncompressed stream of outputBOBJwater, spray.cu:2373-2438: int
    count, float xyz per vertex; int count, float xyz per normal; int number
    of INDICES, int per index (little-endian, as the x86 writer)."""
    nv = len(verts)
    if nv == 0:
        return b""
    b = [struct.pack("<i", nv)]
    for v in verts:
        b.append(struct.pack("<3f", *_checked(v)))
    b.append(struct.pack("<i", nv))
    for v in normals:
        b.append(struct.pack("<3f", *_checked(v)))
    b.append(struct.pack("<i", len(indices)))
    for t in indices:
        b.append(struct.pack("<i", int(t)))
    return b"".join(b)


def blue2red(v: np.float32):
    """mapColorBlue2Red_h, spray.cpp:1299-1360, in float32 arithmetic."""
    f32 = np.float32
    v = f32(v)
    if v < 0:
        return (f32(0), f32(0), f32(1))
    ic = int(v)
    f = f32(v - f32(ic))
    h = f32(f / f32(2))
    table = {0: (f32(0), h, f32(1)),
             1: (f32(0), f32(h + f32(0.5)), f32(1)),
             2: (h, f32(1), f32(f32(1) - h)),
             3: (f32(h + f32(0.5)), f32(1), f32(f32(0.5) - h)),
             4: (f32(1), f32(f32(1.0) - h), f32(0)),
             5: (f32(1), f32(f32(0.5) - h), f32(0))}
    return table.get(ic, (f32(1), f32(0), f32(0)))


def particles(kind: int, pos, flag, temperature, t_min: float, t_max: float) -> bytes:
    """kind 0: outputColoredParticle (spray.cu:2440-2466); 1:
    outputSoloBubblePovRay (2468-2496, AIRSOLO); 2: outputAirParticlePovRay
    (2498-2526, AIR)."""
    f32 = np.float32
    out = []
    if kind == 0:
        r = float(f32(0.004))
        lo, hi = f32(t_min), f32(t_max)
        for p, T in zip(pos, temperature):
            c = blue2red(f32(f32(f32(T) - lo) / f32(hi - lo)) * f32(6.0))
            out.append("sphere{ <%f,%f,%f> %f texture{ finish{dropletFinish} pigment{ rgb<%f,%f,%f>}} }\n"
                       % (float(p[0]), float(p[1]), float(p[2]), r, float(c[0]), float(c[1]), float(c[2])))
    else:
        want = TYPEAIRSOLO if kind == 1 else TYPEAIR
        r = float(f32(0.005))
        for p, fl in zip(pos, flag):
            if int(fl) == want:
                out.append("sphere{ <%f,%f,%f> %f texture{bblTexture} }\n" % (float(p[0]), float(p[1]), float(p[2]), r))
    return "".join(out).encode()
