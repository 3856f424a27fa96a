"""Scene inputs for the CPU oracle without the product library — TEST
INFRASTRUCTURE (the benchmark's reference arm and CPU baseline).

The oracle's library (oracle/_build/libmp_oracle.so) also compiles the host
sources that define the five benchmark configurations (parameters, seeded
particles, random table and nucleation cells, fixed-heat field) and the
marching-cubes case tables, so the reference arm builds the same inputs as
the GPU arm while loading nothing but the oracle. The field names and the
state record mirror include/mp.h (enum mp_field, mp_state); a CPU test checks
them against the product's ctypes mirror.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict

import numpy as np

from . import oracle as _oracle

# enum mp_field (include/mp.h)
FIELDS = [
    "press", "div", "lsfluid", "lsair", "lsmerge", "phifluid", "phiair", "phisolid",
    "phigrax", "phigray", "phigraz", "phigrax_air", "phigray_air", "phigraz_air",
    "surftension", "tp", "tp_save", "tp_old", "fixedheat", "mark",
    "waterux", "wateruy", "wateruz", "waterux_old", "wateruy_old", "wateruz_old",
    "airux", "airuy", "airuz", "airux_old", "airuy_old", "airuz_old",
    "solidux", "soliduy", "soliduz", "cellstart", "cellend",
    "pos", "vel", "flag", "mass", "temp", "lheat", "solubility", "gascontain",
]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}


class State(C.Structure):
    """mp_state (include/mp.h)."""
    _fields_ = [("frame", C.c_int32), ("par_num_now", C.c_int32), ("n_real_solpoint", C.c_int32),
                ("last_cg_iters", C.c_int32), ("last_cg_residual", C.c_double),
                ("last_heat_cg_iters", C.c_int32), ("last_heat_cg_residual", C.c_double),
                ("mc_verts", C.c_int32 * 3), ("mc_indices", C.c_int32 * 3), ("mc_active_voxels", C.c_int32 * 3),
                ("reserved", C.c_int32 * 6)]


_Params = None


def _lib():
    lib = _oracle.load()
    if not hasattr(lib, "_scene_bound"):
        vp = C.c_void_p
        lib.mp_params_describe.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.mp_params_size.restype = C.c_int
        lib.mp_scene_params.argtypes = [C.c_int, C.c_int, vp]
        lib.mp_scene_particles.argtypes = [vp, C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_int)] + [vp] * 8
        lib.mp_scene_tables.argtypes = [vp, C.c_int, C.c_uint64, vp, C.c_int, vp, C.c_int, C.POINTER(C.c_int)]
        lib.mp_scene_fixed_heat.argtypes = [vp, C.c_int, vp]
        lib.mp_internal_mc_tables.argtypes = [vp, vp, vp]
        lib.mp_internal_mc_tables.restype = None
        lib._scene_bound = True
    return lib


def Params():
    """A ctypes mp_params built from the oracle library's own field table."""
    global _Params
    lib = _lib()
    if _Params is None:
        members, last = [], 0
        i = 0
        while True:
            name = C.c_char_p(); off = C.c_int(); kind = C.c_int()
            if lib.mp_params_describe(i, C.byref(name), C.byref(off), C.byref(kind)) != 0:
                break
            members.append((name.value.decode(), C.c_float if kind.value == 1 else C.c_int32))
            last = off.value
            i += 1
        size = lib.mp_params_size()
        members.append(("reserved", C.c_int32 * ((size - (last + 4)) // 4)))

        class P(C.Structure):
            _fields_ = members

        if C.sizeof(P) != size:
            raise ImportError("mp_params size mismatch")
        _Params = P
    return _Params()


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def scene_params(config: int, n: int = 0):
    p = Params()
    _check(_lib().mp_scene_params(config, n, C.byref(p)), "mp_scene_params")
    return p


def scene_particles(p, config: int, seed: int) -> Dict[str, np.ndarray]:
    lib = _lib()
    n = C.c_int()
    _check(lib.mp_scene_particles(C.byref(p), config, seed, 0, C.byref(n), *([None] * 8)), "mp_scene_particles")
    cnt = n.value
    out = {"pos": np.zeros((cnt, 3), np.float32), "vel": np.zeros((cnt, 3), np.float32),
           "flag": np.zeros(cnt, np.int8), "mass": np.zeros(cnt, np.float32), "temp": np.zeros(cnt, np.float32),
           "lheat": np.zeros(cnt, np.float32), "solubility": np.zeros(cnt, np.float32),
           "gascontain": np.zeros(cnt, np.float32)}
    _check(lib.mp_scene_particles(C.byref(p), config, seed, cnt, C.byref(n), *[_ptr(out[k]) for k in
           ["pos", "vel", "flag", "mass", "temp", "lheat", "solubility", "gascontain"]]), "mp_scene_particles")
    return out


def scene_tables(p, config: int, seed: int, nrand: int = 10000):
    rf = np.zeros(nrand, np.float32)
    seeds = np.zeros(64, np.int32)
    ns = C.c_int()
    _check(_lib().mp_scene_tables(C.byref(p), config, seed, _ptr(rf), nrand, _ptr(seeds), 64, C.byref(ns)),
           "mp_scene_tables")
    return rf, seeds[:ns.value].copy()


def scene_fixed_heat(p, config: int) -> np.ndarray:
    fh = np.zeros(p.nx * p.ny * p.nz, np.float32)
    _check(_lib().mp_scene_fixed_heat(C.byref(p), config, _ptr(fh)), "mp_scene_fixed_heat")
    return fh


def mc_tables():
    nv = np.zeros(256, np.int32); tri = np.zeros(256 * 16, np.int32); edge = np.zeros(256, np.int32)
    _lib().mp_internal_mc_tables(_ptr(nv), _ptr(tri), _ptr(edge))
    return nv, tri, edge


def make_oracle(config: int, n: int, seed: int, threads: int = 0):
    """An oracle holding configuration `config` at n^3 from `seed`: the
    inputs the GPU arm's Sim.from_config builds (returns (oracle, params,
    particle count))."""
    p = scene_params(config, n)
    orc = _oracle.Oracle(p, FIELD_ID, State, mc_tables=mc_tables(), threads=threads)
    parts = scene_particles(p, config, seed)
    orc.upload_particles(**parts)
    rf, seeds = scene_tables(p, config, seed)
    orc.set_tables(rf, seeds)
    orc.set_field("fixedheat", scene_fixed_heat(p, config))
    st = orc.state()
    st.n_real_solpoint = int((parts["flag"] == 5).sum())
    orc.set_state(st)
    return orc, p, len(parts["flag"])
