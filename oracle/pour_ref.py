"""Pouring emitters and pouringwater, restated in numpy — TEST INFRASTRUCTURE ONLY.

Only tests/ import this; the product's versions are mp_scene_pour
(2017multiphase_b200/csrc/host/scene.cpp) and k_pour_particles
(2017multiphase_b200/csrc/k_part.cu). Follows gaoyangVR/2017Multiphase:
CompPouringParam_Freezing / _Ineraction / _Ineraction2
(Multiphase/Multiphase/spray.cpp:1416-1545) for the emitter lattice, and
pouringwater (Multiphase/Multiphase/spray_k.cu:5575-5596) as called by
pouring / pouringgas (spray.cu:3012-3043, frame argument 0) for the particles
it appends. All arithmetic in float32, one rounding per operation, in the
reference's order. The reference ships no emitter data; its own
CompPouringParam_* and pouringwater, compiled for the host by
oracle/make_refhost.py, pin the product's emitters in tests/test_refhost_io.py
and tests/test_refhost_modes.py, and this restatement stays as the checker
that travels without the reference tree.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32
FREEZING, INTERACTION, INTERACTION2 = 0, 1, 2


def emitter(variant: int, samplespace: float, radius: float, center, vel, center2=None):
    ss = f32(samplespace) if variant == FREEZING else f32(f32(samplespace) * f32(2.0))
    num = int(f32(radius) / f32(samplespace)) * 3 if variant == FREEZING else int(f32(radius) / ss)
    pts = []
    centres = [center] + ([center2] if variant == INTERACTION2 else [])
    for c in centres:
        c = [f32(a) for a in c]
        for x in range(-num, num + 1):
            for y in range(-num, num + 1):
                p = [f32(c[0] + f32(f32(x) * ss)), f32(c[1] + f32(f32(y) * ss)), f32(c[2] + f32(0.0))]
                d = [f32(p[a] - c[a]) for a in range(3)]
                dd = f32(f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2]))
                if np.sqrt(dd, dtype=np.float32) > f32(radius):
                    continue
                pts.append(p)
    pos = np.array(pts, np.float32).reshape(-1, 3)
    vel3 = np.tile(np.array(vel, np.float32), (len(pos), 1))
    return pos, vel3


def pour(ppos, pvel, randfloat, posrand: float, velrand: float, samplespace: float):
    """Positions and velocities pouringwater gives the emitter's points."""
    rf = np.asarray(randfloat, np.float32)
    n, nr = len(ppos), len(rf)
    pos = np.zeros((n, 3), np.float32)
    vel = np.zeros((n, 3), np.float32)
    for idx in range(n):
        rb = (0 + idx) % (nr - 6)
        rv = [f32(f32(rf[rb + a] * f32(2.0)) - f32(1.0)) for a in range(3)]
        rb += 3
        rp = [f32(f32(rf[rb + a] * f32(2.0)) - f32(1.0)) for a in range(3)]
        for a in range(3):
            pos[idx, a] = f32(f32(ppos[idx][a]) + f32(f32(rp[a] * f32(posrand)) * f32(samplespace)))
            vel[idx, a] = f32(f32(pvel[idx][a]) + f32(rv[a] * f32(velrand)))
    return pos, vel
