"""B200 multiphase FLIP step — Python host mirror of the reference's `cspray`.

The simulation runs in ``libmp.so`` (hand-written sm_100a CUDA behind the C ABI
declared in ``include/mp.h``). This module binds that ABI with ctypes and mirrors
the reference's stage methods (Multiphase/Multiphase/spray.h:21-337) under
their reference names, so a caller of ``cspray`` finds the same operations:

    sim = Sim.from_config(1)            # scene set-up (cspray::initparam + init)
    sim.bubblesim()                     # one time step (spray.cpp:979-1233)
    sim.hashAndSortParticles()          # or one stage at a time
    p = sim.get_field("press")

There is no CPU fallback: if the library or a GPU is missing, construction
raises.
"""
from __future__ import annotations

import ctypes as C
import os
import warnings
from typing import Dict, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmp.so")
INCLUDE_H = os.path.join(os.path.dirname(_HERE), "include", "mp.h")

# status codes (mp.h)
MP_OK, MP_ERR_CUDA, MP_ERR_CAPACITY, MP_ERR_NOCONVERGE, MP_ERR_TIMEOUT, MP_ERR_ARG, MP_ERR_STATE, MP_ERR_IO = range(8)
_ERR_NAMES = {1: "MP_ERR_CUDA", 2: "MP_ERR_CAPACITY", 3: "MP_ERR_NOCONVERGE", 4: "MP_ERR_TIMEOUT",
              5: "MP_ERR_ARG", 6: "MP_ERR_STATE", 7: "MP_ERR_IO"}
# per-frame file formats and particle kinds (mp.h, cspray::output*)
OUT_POV_MESH, OUT_OBJ_MESH, OUT_BOBJ_GZ = range(3)
OUT_PARTICLES_COLORED, OUT_PARTICLES_SOLO, OUT_PARTICLES_AIR = range(3)
# pouring emitter layouts (mp_scene_pour)
POUR_FREEZING, POUR_INTERACTION, POUR_INTERACTION2 = range(3)

# particle and cell types (utility.h:13-19)
TYPEFLUID, TYPEAIR, TYPEBOUNDARY, TYPEVACUUM, TYPEAIRSOLO, TYPESOLID = range(6)
# scenes (utility.h:114-131)
(SCENE_FLUIDSPHERE, SCENE_SMOKE, SCENE_BOILING, SCENE_BOILING_HIGHRES, SCENE_MULTIBUBBLE, SCENE_DAMBREAK,
 SCENE_MELTING, SCENE_MELTINGPOUR, SCENE_FREEZING, SCENE_INTERACTION, SCENE_INTERACTION_HIGHRES, SCENE_MELTANDBOIL,
 SCENE_MELTANDBOIL_HIGHRES, SCENE_HEATTRANSFER) = range(14)
SCENE_ALL = 15
MC_SOLID, MC_FLUID, MC_GAS = 0, 1, 2
PREC_MIXED, PREC_FP64 = 0, 1
TOL_REF_ABS, TOL_REL = 0, 1
KT_CG_STENCIL, KT_CG_UPDATE, KT_P2G, KT_G2P, KT_SORT, KT_LEVELSET, KT_MC_DENS, KT_CORRECT = range(8)

# field ids in the order of enum mp_field (mp.h)
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
_DTYPE = {"mark": np.int8, "flag": np.int8, "cellstart": np.uint32, "cellend": np.uint32}


class MPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class MPState(C.Structure):
    _fields_ = [("frame", C.c_int32), ("par_num_now", C.c_int32), ("n_real_solpoint", C.c_int32),
                ("last_cg_iters", C.c_int32), ("last_cg_residual", C.c_double),
                ("last_heat_cg_iters", C.c_int32), ("last_heat_cg_residual", C.c_double),
                ("mc_verts", C.c_int32 * 3), ("mc_indices", C.c_int32 * 3), ("mc_active_voxels", C.c_int32 * 3),
                ("reserved", C.c_int32 * 6)]


class MPSceneInfo(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("sim_mode", C.c_int32),
                ("init_fluid_particles", C.c_int32), ("split_num", C.c_int32), ("par_num_extra", C.c_int32),
                ("seed_num", C.c_int32), ("pour_variant", C.c_int32), ("pour_radius", C.c_float),
                ("pour_pos", C.c_float * 3), ("pour_pos2", C.c_float * 3), ("pour_vel", C.c_float * 3),
                ("solid_init_pos", C.c_float * 3), ("t_render_min", C.c_float), ("t_render_max", C.c_float),
                ("frame_max", C.c_int32), ("output_colored_particles", C.c_int32), ("reserved", C.c_int32 * 8)]


class MPGrad(C.Structure):
    """mp_grad: device arrays of doubles, xyz (or one temperature) per particle
    (NULL members allowed)."""
    _fields_ = [("pos", C.c_void_p), ("vel", C.c_void_p), ("temp", C.c_void_p)]


class MPOutput(C.Structure):
    _fields_ = [("dir", C.c_char_p), ("pov", C.c_int32), ("obj", C.c_int32), ("colored_particles", C.c_int32),
                ("t_render_min", C.c_float), ("t_render_max", C.c_float)]


_lib = None
_Params = None


def load_library() -> C.CDLL:
    """Loads libmp.so; raises if it has not been built."""
    global _lib, _Params
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() (make -C csrc)")
    lib = C.CDLL(LIB_PATH)
    lib.mp_params_describe.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.mp_params_size.restype = C.c_int
    fields = []
    i = 0
    while True:
        name = C.c_char_p(); off = C.c_int(); kind = C.c_int()
        if lib.mp_params_describe(i, C.byref(name), C.byref(off), C.byref(kind)) != 0:
            break
        fields.append((name.value.decode(), off.value, kind.value))
        i += 1
    # rebuild the struct from the library's own table (offsets checked below)
    members = []
    for nm, off, kind in fields:
        members.append((nm, C.c_float if kind == 1 else C.c_int32))
    size = lib.mp_params_size()
    pad = (size - (fields[-1][1] + 4)) // 4
    members.append(("reserved", C.c_int32 * pad))

    class Params(C.Structure):
        _fields_ = members

    for nm, off, _ in fields:
        if getattr(Params, nm).offset != off:
            raise ImportError(f"mp_params layout mismatch at {nm}")
    if C.sizeof(Params) != size:
        raise ImportError("mp_params size mismatch")
    _Params = Params
    vp = C.c_void_p
    P = C.POINTER(Params)
    sig = {
        "mp_params_default": ([P, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
        "mp_params_derive": ([P], C.c_int),
        "mp_create": ([P, C.POINTER(vp)], C.c_int),
        "mp_destroy": ([vp], C.c_int),
        "mp_set_params": ([vp, P], C.c_int),
        "mp_get_params": ([vp, P], C.c_int),
        "mp_get_state": ([vp, C.POINTER(MPState)], C.c_int),
        "mp_set_state": ([vp, C.POINTER(MPState)], C.c_int),
        "mp_last_error": ([vp, C.c_char_p, C.c_size_t], C.c_int),
        "mp_set_stream": ([vp, vp], C.c_int),
        "mp_get_stream": ([vp, C.POINTER(vp)], C.c_int),
        "mp_synchronize": ([vp], C.c_int),
        "mp_upload_particles": ([vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "mp_download_particles": ([vp, C.POINTER(C.c_int), vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "mp_field_info": ([vp, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)], C.c_int),
        "mp_get_field": ([vp, C.c_int, vp, C.c_size_t], C.c_int),
        "mp_set_field": ([vp, C.c_int, vp, C.c_size_t], C.c_int),
        "mp_set_tables": ([vp, vp, C.c_int, vp, C.c_int], C.c_int),
        "mp_mc_tables": ([vp, vp, vp], C.c_int),
        "mp_set_mc_tables": ([vp, vp, vp], C.c_int),
        "mp_init_particle_heat": ([vp], C.c_int),
        "mp_levelset": ([vp, C.c_float], C.c_int),
        "mp_sweep_phi": ([vp, C.c_int], C.c_int),
        "mp_sweep_u": ([vp, C.c_int], C.c_int),
        "mp_set_boundary_u": ([vp, C.c_int], C.c_int),
        "mp_project": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_double)], C.c_int),
        "mp_adj_record": ([vp, C.c_int, C.c_int], C.c_int),
        "mp_adj_set_targets": ([vp, vp, C.c_int], C.c_int),
        "mp_adj_info": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
        "mp_adj_order": ([vp, vp], C.c_int),
        "mp_adj_loss": ([vp, C.c_int, vp, C.POINTER(C.c_double)], C.c_int),
        "mp_adj_gradient": ([vp, C.c_int, vp, vp, C.POINTER(C.c_double)], C.c_int),
        "mp_adj_release": ([vp], C.c_int),
        "mp_adj_forward": ([vp, C.c_int, C.POINTER(MPGrad), C.POINTER(MPGrad)], C.c_int),
        "mp_step_adjoint": ([vp, C.c_int, C.POINTER(MPGrad), C.POINTER(MPGrad), C.POINTER(MPGrad)], C.c_int),
        "mp_adj_level_set_loss": ([vp, C.c_int, vp, C.POINTER(C.c_double), vp], C.c_int),
        "mp_checkpoint_size": ([vp, C.POINTER(C.c_size_t)], C.c_int),
        "mp_checkpoint_save": ([vp, vp, C.c_size_t], C.c_int),
        "mp_checkpoint_load": ([vp, vp, C.c_size_t], C.c_int),
        "mp_pressure_cg_static": ([C.c_int, C.c_int, C.c_int, C.c_float, vp, vp, vp, C.c_int, C.c_int, C.c_float, vp,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double)], C.c_int),
        "mp_mc": ([vp, C.c_int], C.c_int),
        "mp_mc_download": ([vp, C.c_int, vp, vp, vp, C.c_int, C.c_int], C.c_int),
        "mp_mc_download_field": ([vp, vp, vp], C.c_int),
        "mp_kernel_timing": ([vp, C.c_int, C.c_int], C.c_int),
        "mp_kernel_timing_read": ([vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64)], C.c_int),
        "mp_kernel_timing_reset": ([vp], C.c_int),
        "mp_launch_count": ([vp], C.c_int64),
        "mp_work_counts": ([vp, C.POINTER(C.c_int64), C.c_int], C.c_int),
        "mp_scene_params": ([C.c_int, C.c_int, P], C.c_int),
        "mp_scene_particles": ([P, C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_int), vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "mp_scene_tables": ([P, C.c_int, C.c_uint64, vp, C.c_int, vp, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "mp_scene_fixed_heat": ([P, C.c_int, vp], C.c_int),
        "mp_write_mesh": ([C.c_int, C.c_char_p, C.c_char_p, vp, vp, C.c_int, vp, C.c_int], C.c_int),
        "mp_write_particles": ([C.c_int, C.c_char_p, vp, vp, vp, C.c_int, C.c_float, C.c_float], C.c_int),
        "mp_export_mesh": ([vp, C.c_int, C.c_int, C.c_char_p], C.c_int),
        "mp_export_particles": ([vp, C.c_int, C.c_char_p, C.c_float, C.c_float], C.c_int),
        "mp_set_output": ([vp, C.POINTER(MPOutput)], C.c_int),
        "mp_scene_pour": ([C.c_int, C.c_float, C.c_float, vp, vp, vp, C.c_int, vp, vp, C.POINTER(C.c_int)], C.c_int),
        "mp_set_pour": ([vp, vp, vp, C.c_int], C.c_int),
        "mp_reference_scene": ([C.c_int, P, C.POINTER(MPSceneInfo)], C.c_int),
        "mp_project_water": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_double)], C.c_int),
    }
    for nm, (args, res) in sig.items():
        f = getattr(lib, nm)
        f.argtypes = args
        f.restype = res
    for nm in ["mp_hash_sort", "mp_external_force", "mp_sweep_ls_mark", "mp_mark_solo_air", "mp_surface_tension",
               "mp_markgrid_bubble", "mp_p2g", "mp_drag", "mp_g2p", "mp_solid_motion", "mp_solo_air_update",
               "mp_collide_advect", "mp_correct_pos", "mp_correct_pos_bubble", "mp_heat", "mp_gen_gas", "mp_delete",
               "mp_melt", "mp_freeze", "mp_mc_presort", "mp_step", "mp_pour", "mp_heatsim",
               "mp_init_heat_grid", "mp_flip_mark", "mp_water_p2g", "mp_water_g2p", "mp_water_advect",
               "mp_watersim"]:
        f = getattr(lib, nm)
        f.argtypes = [vp]
        f.restype = C.c_int
    _lib = lib
    return lib


def Params():
    """The ctypes mirror of mp_params, built from the library's field table."""
    load_library()
    return _Params()


def params_to_dict(p) -> Dict[str, float]:
    return {nm: getattr(p, nm) for nm, _ in p._fields_ if nm != "reserved"}


def scene_params(config: int, n: int = 0):
    """Parameters of benchmark configuration 1..5 (mp_scene_params)."""
    lib = load_library()
    p = Params()
    _check(lib.mp_scene_params(config, n, C.byref(p)), None)
    return p


def default_params(nx: int, ny: int, nz: int, par_num_max: int):
    lib = load_library()
    p = Params()
    _check(lib.mp_params_default(C.byref(p), nx, ny, nz, par_num_max), None)
    return p


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc: int, ctx, allow_noconverge=False) -> int:
    if rc == MP_OK:
        return rc
    if rc == MP_ERR_NOCONVERGE and allow_noconverge:
        warnings.warn("CG stopped at its iteration limit", RuntimeWarning)
        return rc
    buf = C.create_string_buffer(512)
    load_library().mp_last_error(ctx, buf, 512)
    raise MPError(rc, buf.value.decode(errors="replace"))


def scene_particles(p, config: int, seed: int) -> Dict[str, np.ndarray]:
    """Initial particles of a configuration (mp_scene_particles), as numpy arrays."""
    lib = load_library()
    n = C.c_int()
    _check(lib.mp_scene_particles(C.byref(p), config, seed, 0, C.byref(n), None, None, None, None, None, None, None,
                                  None), None)
    cnt = n.value
    out = {"pos": np.zeros((cnt, 3), np.float32), "vel": np.zeros((cnt, 3), np.float32),
           "flag": np.zeros(cnt, np.int8), "mass": np.zeros(cnt, np.float32), "temp": np.zeros(cnt, np.float32),
           "lheat": np.zeros(cnt, np.float32), "solubility": np.zeros(cnt, np.float32),
           "gascontain": np.zeros(cnt, np.float32)}
    _check(lib.mp_scene_particles(C.byref(p), config, seed, cnt, C.byref(n), *[_ptr(out[k]) for k in
                                  ["pos", "vel", "flag", "mass", "temp", "lheat", "solubility", "gascontain"]]), None)
    return out


def scene_tables(p, config: int, seed: int, nrand: int = 10000):
    lib = load_library()
    rf = np.zeros(nrand, np.float32)
    seeds = np.zeros(64, np.int32)
    ns = C.c_int()
    _check(lib.mp_scene_tables(C.byref(p), config, seed, _ptr(rf), nrand, _ptr(seeds), 64, C.byref(ns)), None)
    return rf, seeds[:ns.value].copy()


def scene_fixed_heat(p, config: int) -> np.ndarray:
    lib = load_library()
    fh = np.zeros(p.nx * p.ny * p.nz, np.float32)
    _check(lib.mp_scene_fixed_heat(C.byref(p), config, _ptr(fh)), None)
    return fh


def write_mesh(fmt: int, path: str, verts: np.ndarray, normals: np.ndarray, indices: np.ndarray,
               object_name: str = "water"):
    """One mesh from host arrays in the reference's POV-Ray / OBJ / BOBJ.gz
    format (mp_write_mesh)."""
    lib = load_library()
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    nr = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
    ix = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    _check(lib.mp_write_mesh(fmt, os.fsencode(path), object_name.encode(), _ptr(v), _ptr(nr), len(v), _ptr(ix),
                             len(ix)), None)


def write_particles(kind: int, path: str, pos: np.ndarray, flag: Optional[np.ndarray] = None,
                    temperature: Optional[np.ndarray] = None, t_min: float = 273.0, t_max: float = 373.0):
    """POV-Ray particle spheres from host arrays (mp_write_particles)."""
    lib = load_library()
    p3 = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    fl = None if flag is None else np.ascontiguousarray(flag, np.int8)
    T = None if temperature is None else np.ascontiguousarray(temperature, np.float32)
    _check(lib.mp_write_particles(kind, os.fsencode(path), _ptr(p3), _ptr(fl), _ptr(T), len(p3), t_min, t_max),
           None)


SIM_WATER, SIM_SOLIDCOUPLING, SIM_SMOKE, SIM_BUBBLE, SIM_HEATONLY = range(5)


def reference_scene(scene: int):
    """cspray::initparam's parameters for the reference's named scene (mp_reference_scene):
    (params, info) with info a dict of the branch's other settings."""
    lib = load_library()
    p = Params()
    info = MPSceneInfo()
    _check(lib.mp_reference_scene(scene, C.byref(p), C.byref(info)), None)
    d = {}
    for nm, typ in MPSceneInfo._fields_:
        if nm == "reserved":
            continue
        v = getattr(info, nm)
        d[nm] = list(v) if hasattr(v, "__len__") else v
    return p, d


def scene_pour(variant: int, samplespace: float, radius: float, center, vel, center2=None):
    """The emitter points of CompPouringParam_* (mp_scene_pour): (pos, vel) float32 (n, 3)."""
    lib = load_library()
    c1 = np.ascontiguousarray(center, np.float32)
    c2 = None if center2 is None else np.ascontiguousarray(center2, np.float32)
    v = np.ascontiguousarray(vel, np.float32)
    n = C.c_int()
    _check(lib.mp_scene_pour(variant, samplespace, radius, _ptr(c1), _ptr(c2), _ptr(v), 0, None, None, C.byref(n)),
           None)
    pos = np.zeros((n.value, 3), np.float32); vel3 = np.zeros((n.value, 3), np.float32)
    _check(lib.mp_scene_pour(variant, samplespace, radius, _ptr(c1), _ptr(c2), _ptr(v), n.value, _ptr(pos),
                             _ptr(vel3), C.byref(n)), None)
    return pos, vel3


def mc_tables():
    lib = load_library()
    nv = np.zeros(256, np.int32); tri = np.zeros(256 * 16, np.int32); edge = np.zeros(256, np.int32)
    lib.mp_mc_tables(_ptr(nv), _ptr(tri), _ptr(edge))
    return nv, tri, edge


class Sim:
    """One simulation context on the current CUDA device (the reference's cspray)."""

    def __init__(self, params):
        self.lib = load_library()
        self.params = params
        self.ctx = C.c_void_p()
        _check(self.lib.mp_create(C.byref(params), C.byref(self.ctx)), None)

    @classmethod
    def from_config(cls, config: int, n: int = 0, seed: int = 2017000, params=None, **overrides):
        """cspray::initparam + init for benchmark configuration `config`."""
        p = params if params is not None else scene_params(config, n)
        for k, v in overrides.items():
            setattr(p, k, v)
        parts = scene_particles(p, config, seed)
        sim = cls(p)
        sim.upload_particles(**parts)
        rf, seeds = scene_tables(p, config, seed)
        sim.set_tables(rf, seeds)
        sim.set_field("fixedheat", scene_fixed_heat(p, config))
        st = sim.state()
        st.n_real_solpoint = int((parts["flag"] == TYPESOLID).sum())
        sim.set_state(st)
        sim.config, sim.seed = config, seed
        return sim

    def close(self):
        if self.ctx:
            self.lib.mp_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- data -------------------------------------------------------------
    def upload_particles(self, pos, flag, mass, vel=None, temp=None, lheat=None, solubility=None, gascontain=None):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        n = pos.shape[0]
        arrs = [pos, None if vel is None else np.ascontiguousarray(vel, np.float32).reshape(-1, 3),
                np.ascontiguousarray(flag, np.int8), np.ascontiguousarray(mass, np.float32)]
        arrs += [None if a is None else np.ascontiguousarray(a, np.float32) for a in (temp, lheat, solubility, gascontain)]
        _check(self.lib.mp_upload_particles(self.ctx, n, *[_ptr(a) for a in arrs]), self.ctx)

    def download_particles(self) -> Dict[str, np.ndarray]:
        n = self.state().par_num_now
        out = {"pos": np.zeros((n, 3), np.float32), "vel": np.zeros((n, 3), np.float32), "flag": np.zeros(n, np.int8),
               "mass": np.zeros(n, np.float32), "temp": np.zeros(n, np.float32), "lheat": np.zeros(n, np.float32),
               "solubility": np.zeros(n, np.float32), "gascontain": np.zeros(n, np.float32)}
        cnt = C.c_int()
        _check(self.lib.mp_download_particles(self.ctx, C.byref(cnt), *[_ptr(out[k]) for k in
               ["pos", "vel", "flag", "mass", "temp", "lheat", "solubility", "gascontain"]]), self.ctx)
        return out

    def field_info(self, name: str):
        cnt = C.c_size_t(); eb = C.c_size_t()
        _check(self.lib.mp_field_info(self.ctx, FIELD_ID[name], C.byref(cnt), C.byref(eb)), self.ctx)
        return cnt.value, eb.value

    def get_field(self, name: str) -> np.ndarray:
        cnt, eb = self.field_info(name)
        a = np.zeros(cnt, _DTYPE.get(name, np.float32))
        _check(self.lib.mp_get_field(self.ctx, FIELD_ID[name], _ptr(a), a.nbytes), self.ctx)
        return a

    def set_field(self, name: str, a: np.ndarray):
        a = np.ascontiguousarray(a, _DTYPE.get(name, np.float32)).ravel()
        _check(self.lib.mp_set_field(self.ctx, FIELD_ID[name], _ptr(a), a.nbytes), self.ctx)

    def set_tables(self, randfloat: np.ndarray, seeds: np.ndarray):
        rf = np.ascontiguousarray(randfloat, np.float32)
        sd = np.ascontiguousarray(seeds, np.int32)
        _check(self.lib.mp_set_tables(self.ctx, _ptr(rf), rf.size, _ptr(sd), sd.size), self.ctx)

    def checkpoint(self) -> bytes:
        """mp_checkpoint_save: the state the next step starts from."""
        nb = C.c_size_t()
        _check(self.lib.mp_checkpoint_size(self.ctx, C.byref(nb)), self.ctx)
        buf = C.create_string_buffer(nb.value)
        _check(self.lib.mp_checkpoint_save(self.ctx, buf, nb.value), self.ctx)
        return buf.raw

    def restore(self, blob: bytes):
        """mp_checkpoint_load of a checkpoint taken with the same parameters."""
        _check(self.lib.mp_checkpoint_load(self.ctx, C.c_char_p(blob), len(blob)), self.ctx)

    def state(self) -> MPState:
        s = MPState()
        _check(self.lib.mp_get_state(self.ctx, C.byref(s)), self.ctx)
        return s

    def set_state(self, s: MPState):
        _check(self.lib.mp_set_state(self.ctx, C.byref(s)), self.ctx)

    def get_params(self):
        p = Params()
        _check(self.lib.mp_get_params(self.ctx, C.byref(p)), self.ctx)
        return p

    def set_params(self, p):
        _check(self.lib.mp_set_params(self.ctx, C.byref(p)), self.ctx)
        self.params = p

    def synchronize(self):
        _check(self.lib.mp_synchronize(self.ctx), self.ctx)

    # ---- stages, under the reference's method names (spray.h) ------------
    def _stage(self, name, *args, allow_noconverge=False):
        return _check(getattr(self.lib, name)(self.ctx, *args), self.ctx, allow_noconverge)

    def initHeatAndSolubility(self): return self._stage("mp_init_particle_heat")
    def hashAndSortParticles(self): return self._stage("mp_hash_sort")
    def addexternalforce(self): return self._stage("mp_external_force")
    def computeLevelset(self, offset=0.0): return self._stage("mp_levelset", C.c_float(offset))
    def sweepLSAndMardGrid(self): return self._stage("mp_sweep_ls_mark")
    def markSoloAirParticle(self): return self._stage("mp_mark_solo_air")
    def computesurfacetension(self): return self._stage("mp_surface_tension")
    def markgrid_bubble(self): return self._stage("mp_markgrid_bubble")
    def mapvelp2g_bubble(self): return self._stage("mp_p2g")
    def enforceDragForce(self): return self._stage("mp_drag")
    def sweepPhi(self, phase): return self._stage("mp_sweep_phi", phase)
    def sweepU(self, phase): return self._stage("mp_sweep_u", phase)
    def setWaterBoundaryU(self, phase): return self._stage("mp_set_boundary_u", phase)

    def project_CG_bubble(self):
        it = C.c_int(); res = C.c_double()
        rc = _check(self.lib.mp_project(self.ctx, C.byref(it), C.byref(res)), self.ctx, allow_noconverge=True)
        return it.value, res.value, rc

    def mapvelg2p_bubble(self): return self._stage("mp_g2p")
    def solidmotion(self): return self._stage("mp_solid_motion")
    def updateSoloAirParticle(self): return self._stage("mp_solo_air_update")
    def CollisionSolid(self): return self._stage("mp_collide_advect")
    def correctpos(self): return self._stage("mp_correct_pos")
    def correctpos_bubble(self): return self._stage("mp_correct_pos_bubble")
    def updateTemperature(self): return self._stage("mp_heat", allow_noconverge=True)
    def GenerateGasParticle(self): return self._stage("mp_gen_gas")
    def deleteAirFluidParticle(self): return self._stage("mp_delete")
    def MeltSolid(self): return self._stage("mp_melt")
    def Freezing(self): return self._stage("mp_freeze")
    def preMC(self): return self._stage("mp_mc_presort")
    def runMC(self, surface): return self._stage("mp_mc", surface)
    def bubblesim(self):
        rc = self._stage("mp_step", allow_noconverge=True)
        # the frame-scripted switches of some scenes change the parameters
        self.params = self.get_params()
        return rc
    simstep = bubblesim

    def mc_mesh(self, surface: int):
        s = self.state()
        nv, ni = s.mc_verts[surface], s.mc_indices[surface]
        v = np.zeros((nv, 3), np.float32); nr = np.zeros((nv, 3), np.float32); ix = np.zeros(ni, np.uint32)
        _check(self.lib.mp_mc_download(self.ctx, surface, _ptr(v), _ptr(nr), _ptr(ix), nv, ni), self.ctx)
        return v, nr, ix

    # ---- pouring (cspray::pouring / pouringgas) ------------------------------
    def set_mc_tables(self, num_verts: np.ndarray, tri: np.ndarray):
        """Replaces the marching-cubes case tables of this context (mp_set_mc_tables)."""
        nv = np.ascontiguousarray(num_verts, np.int32).reshape(256)
        tr = np.ascontiguousarray(tri, np.int32).reshape(256 * 16)
        _check(self.lib.mp_set_mc_tables(self.ctx, _ptr(nv), _ptr(tr)), self.ctx)

    def set_pour(self, pos: np.ndarray, vel: np.ndarray):
        """The emitter (dpourpos / dpourvel) the step pours from (mp_set_pour)."""
        p3 = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        v3 = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        _check(self.lib.mp_set_pour(self.ctx, _ptr(p3), _ptr(v3), len(p3)), self.ctx)

    def pouring(self): return self._stage("mp_pour")

    # ---- water-only mode (SIMULATION_WATER) ----------------------------------
    def flipMark_sphere(self): return self._stage("mp_flip_mark")
    def mapvelp2g(self): return self._stage("mp_water_p2g")
    def mapvelg2p(self): return self._stage("mp_water_g2p")
    def wateradvect(self): return self._stage("mp_water_advect")

    def project_CG(self):
        it = C.c_int(); res = C.c_double()
        rc = _check(self.lib.mp_project_water(self.ctx, C.byref(it), C.byref(res)), self.ctx, allow_noconverge=True)
        return it.value, res.value, rc

    def watersim(self): return self._stage("mp_watersim", allow_noconverge=True)

    # ---- heat-only mode (SIMULATION_HEATONLY) --------------------------------
    def initheat_grid(self): return self._stage("mp_init_heat_grid")
    def heatsim(self): return self._stage("mp_heatsim", allow_noconverge=True)

    # ---- per-frame files (cspray::output*) ----------------------------------
    def export_mesh(self, surface: int, fmt: int, path: str):
        """The last extraction of `surface` as a file (mp_export_mesh)."""
        _check(self.lib.mp_export_mesh(self.ctx, surface, fmt, os.fsencode(path)), self.ctx)

    def export_particles(self, kind: int, path: str, t_min: float = 273.0, t_max: float = 373.0):
        _check(self.lib.mp_export_particles(self.ctx, kind, os.fsencode(path), t_min, t_max), self.ctx)

    def set_output(self, out_dir: Optional[str], pov: bool = False, obj: bool = True, colored_particles: bool = True,
                   t_render_min: float = 273.0, t_render_max: float = 373.0):
        """Per-frame files written by each step that extracts meshes (mp_set_output);
        defaults are cspray::initparam's (spray.cpp:30-33, 61). None turns it off.
        `out_dir` is a prefix used as written, so it ends with a separator."""
        if out_dir is None:
            self._out = None
            _check(self.lib.mp_set_output(self.ctx, None), self.ctx)
            return
        self._out = MPOutput(os.fsencode(out_dir), int(pov), int(obj), int(colored_particles), t_render_min,
                             t_render_max)
        _check(self.lib.mp_set_output(self.ctx, C.byref(self._out)), self.ctx)

    def mc_field(self):
        p = self.params
        dens = np.zeros((2 * p.nx + 1) * (2 * p.ny + 1) * (2 * p.nz + 1), np.float32)
        cube = np.zeros(8 * p.nx * p.ny * p.nz, np.uint8)
        _check(self.lib.mp_mc_download_field(self.ctx, _ptr(dens), _ptr(cube)), self.ctx)
        return dens, cube

    # ---- adjoint of the FLUID-only step (mp_adj_*) -------------------------
    def adj_record(self, nsteps: int, checkpoint_every: int):
        """Runs `nsteps` steps from the current particles, recording the discrete
        state the derivative holds fixed (mp_adj_record)."""
        _check(self.lib.mp_adj_record(self.ctx, nsteps, checkpoint_every), self.ctx)
        self._adj_heat = bool(self.params.b_heat_trans)

    def adj_set_targets(self, samples: np.ndarray):
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, 3)
        _check(self.lib.mp_adj_set_targets(self.ctx, _ptr(s), len(s)), self.ctx)

    def adj_num_particles(self) -> int:
        n = C.c_int(); k = C.c_int()
        _check(self.lib.mp_adj_info(self.ctx, C.byref(n), C.byref(k)), self.ctx)
        return n.value

    def adj_order(self):
        """Recording index of the particle in each slot of the context now
        (mp_adj_order), as a CUDA int64 tensor: the engine's particles after
        the recording, reordered by it, line up with the replay's final state."""
        import torch
        n = self.adj_num_particles()
        ids = torch.empty(n, dtype=torch.int32, device=f"cuda:{torch.cuda.current_device()}")
        torch.cuda.synchronize()
        _check(self.lib.mp_adj_order(self.ctx, C.c_void_p(ids.data_ptr())), self.ctx)
        return ids.to(torch.int64)

    def adj_loss(self, v0=None, precision: int = PREC_MIXED) -> float:
        """Loss of the recorded program from initial velocities v0 (a CUDA
        float64 tensor (np, 3) in recording order, or None for the recorded ones)."""
        loss = C.c_double()
        vp = None if v0 is None else C.c_void_p(v0.data_ptr())
        _check(self.lib.mp_adj_loss(self.ctx, precision, vp, C.byref(loss)), self.ctx)
        return loss.value

    def adj_gradient(self, v0=None, precision: int = PREC_MIXED):
        """(loss, dL/dv0) as a CUDA float64 tensor (np, 3)."""
        import torch
        n = self.adj_num_particles()
        g = torch.empty((n, 3), dtype=torch.float64, device=f"cuda:{torch.cuda.current_device()}")
        loss = C.c_double()
        vp = None if v0 is None else C.c_void_p(v0.data_ptr())
        torch.cuda.synchronize()
        _check(self.lib.mp_adj_gradient(self.ctx, precision, vp, C.c_void_p(g.data_ptr()), C.byref(loss)), self.ctx)
        return loss.value, g

    @staticmethod
    def _grad(pos=None, vel=None, temp=None):
        return MPGrad(None if pos is None else pos.data_ptr(), None if vel is None else vel.data_ptr(),
                      None if temp is None else temp.data_ptr())

    def _empty3(self, cols=3):
        import torch
        shape = (self.adj_num_particles(), cols) if cols > 1 else (self.adj_num_particles(),)
        return torch.empty(shape, dtype=torch.float64, device=f"cuda:{torch.cuda.current_device()}")

    def adj_forward(self, x0=None, v0=None, precision: int = PREC_MIXED, T0=None):
        """The recorded program from initial positions/velocities (CUDA float64
        (np, 3) tensors in recording order, None: the recorded ones) and, when
        the recording ran the heat stage, initial temperatures (np,), to the
        final (xT, vT) or (xT, vT, TT) (mp_adj_forward)."""
        import torch
        heat = getattr(self, "_adj_heat", False)
        xT, vT = self._empty3(), self._empty3()
        TT = self._empty3(1) if heat else None
        inp, out = self._grad(x0, v0, T0 if heat else None), self._grad(xT, vT, TT)
        torch.cuda.synchronize()
        _check(self.lib.mp_adj_forward(self.ctx, precision, C.byref(inp), C.byref(out)), self.ctx)
        return (xT, vT, TT) if heat else (xT, vT)

    def step_adjoint(self, x0=None, v0=None, xT_bar=None, vT_bar=None, precision: int = PREC_MIXED, T0=None,
                     TT_bar=None):
        """The vector-Jacobian product of the recorded program at (x0, v0[, T0]):
        (x0_bar, v0_bar[, T0_bar]) = J^T (xT_bar, vT_bar[, TT_bar]) (mp_step_adjoint)."""
        import torch
        heat = getattr(self, "_adj_heat", False)
        x0b, v0b = self._empty3(), self._empty3()
        T0b = self._empty3(1) if heat else None
        inp = self._grad(x0, v0, T0 if heat else None)
        dout = self._grad(xT_bar, vT_bar, TT_bar if heat else None)
        din = self._grad(x0b, v0b, T0b)
        torch.cuda.synchronize()
        _check(self.lib.mp_step_adjoint(self.ctx, precision, C.byref(inp), C.byref(dout), C.byref(din)), self.ctx)
        return (x0b, v0b, T0b) if heat else (x0b, v0b)

    def adj_level_set_loss(self, xT, precision: int = PREC_MIXED, grad: bool = True):
        """(L, dL/dxT) of the target-point loss at final positions xT."""
        import torch
        loss = C.c_double()
        g = self._empty3() if grad else None
        torch.cuda.synchronize()
        _check(self.lib.mp_adj_level_set_loss(self.ctx, precision, C.c_void_p(xT.data_ptr()), C.byref(loss),
                                              None if g is None else C.c_void_p(g.data_ptr())), self.ctx)
        return loss.value, g

    # ---- measurement ------------------------------------------------------
    def kernel_timing(self, cls: int, enable: bool = True):
        _check(self.lib.mp_kernel_timing(self.ctx, cls, int(enable)), self.ctx)

    def kernel_timing_read(self, cls: int):
        ms = C.c_double(); n = C.c_int64()
        _check(self.lib.mp_kernel_timing_read(self.ctx, cls, C.byref(ms), C.byref(n)), self.ctx)
        return ms.value, n.value

    def kernel_timing_reset(self):
        _check(self.lib.mp_kernel_timing_reset(self.ctx), self.ctx)

    def launch_count(self) -> int:
        return int(self.lib.mp_launch_count(self.ctx))

    def work_counts(self) -> Dict[str, int]:
        """mp_work_counts: sorts that reordered / found the order, CG iterations,
        reverse sweeps from the engine's states / after a full replay."""
        a = (C.c_int64 * 5)()
        _check(self.lib.mp_work_counts(self.ctx, a, 5), self.ctx)
        return {"sort_full": int(a[0]), "sort_fast": int(a[1]), "cg_iters": int(a[2]),
                "adj_engine": int(a[3]), "adj_replay": int(a[4])}

    def stream_handle(self) -> int:
        s = C.c_void_p()
        _check(self.lib.mp_get_stream(self.ctx, C.byref(s)), self.ctx)
        return s.value or 0


def dam_break_targets(nsamples: int, seed: int, height: float = 0.3, margin: float = 0.1) -> np.ndarray:
    """Target points of configuration 4's loss: (x, y) uniform in the box
    interior from `seed`, on the surface z = height."""
    rng = np.random.default_rng(seed)
    xy = rng.uniform(margin, 1.0 - margin, size=(nsamples, 2))
    return np.concatenate([xy, np.full((nsamples, 1), height)], axis=1).astype(np.float32)


def _functions():
    import torch

    class MPStep(torch.autograd.Function):
        """The recorded steps (Sim.adj_record) as a function of the particles'
        initial positions and velocities, and of their temperatures when the
        recording ran the heat stage: (x0, v0[, T0]) -> (xT, vT[, TT]), CUDA
        float64 tensors in recording order. backward is the hand-written
        adjoint (mp_step_adjoint), run only when a gradient is asked for. The
        discrete state (splat order, cell marks, extrapolation choices) is the
        recorded one, so the inputs should stay near the recorded state."""

        @staticmethod
        def forward(ctx, x0, v0, T0, sim, precision):
            x0 = x0.detach().to(torch.float64).contiguous()
            v0 = v0.detach().to(torch.float64).contiguous()
            T0 = None if T0 is None else T0.detach().to(torch.float64).contiguous()
            ctx.heat = T0 is not None
            ctx.save_for_backward(x0, v0, T0)
            ctx.sim, ctx.precision = sim, precision
            return sim.adj_forward(x0, v0, precision, T0=T0)

        @staticmethod
        def backward(ctx, *grads):
            if not any(ctx.needs_input_grad[:3]):
                return None, None, None, None, None
            x0, v0, T0 = ctx.saved_tensors
            g = [None if q is None else q.to(torch.float64).contiguous() for q in grads]
            out = ctx.sim.step_adjoint(x0, v0, g[0], g[1], ctx.precision, T0=T0,
                                       TT_bar=g[2] if ctx.heat else None)
            x0b, v0b = out[0], out[1]
            T0b = out[2] if ctx.heat else None
            need = ctx.needs_input_grad
            return (x0b if need[0] else None), (v0b if need[1] else None), (T0b if need[2] else None), None, None

    class LevelSetLoss(torch.autograd.Function):
        """sum_s phi(y_s)^2 of the final fluid distance field at the target
        points (mp_adj_set_targets) as a function of the final positions."""

        @staticmethod
        def forward(ctx, xT, sim, precision):
            xT = xT.detach().to(torch.float64).contiguous()
            ctx.save_for_backward(xT)
            ctx.sim, ctx.precision = sim, precision
            loss, _ = sim.adj_level_set_loss(xT, precision, grad=False)
            return torch.tensor(loss, dtype=torch.float64, device=xT.device)

        @staticmethod
        def backward(ctx, gout):
            if not ctx.needs_input_grad[0]:
                return None, None, None
            (xT,) = ctx.saved_tensors
            _, g = ctx.sim.adj_level_set_loss(xT, ctx.precision, grad=True)
            return gout * g, None, None

    class DamBreakLoss(torch.autograd.Function):
        """Loss of the recorded FLUID-only program as a function of the initial
        particle velocities; forward evaluates the loss only, backward runs the
        adjoint (mp_adj_gradient)."""

        @staticmethod
        def forward(ctx, v0, sim, precision):
            v0 = v0.detach().to(torch.float64).contiguous()
            ctx.save_for_backward(v0)
            ctx.sim, ctx.precision = sim, precision
            return torch.tensor(sim.adj_loss(v0, precision), dtype=torch.float64, device=v0.device)

        @staticmethod
        def backward(ctx, gout):
            if not ctx.needs_input_grad[0]:
                return None, None, None
            (v0,) = ctx.saved_tensors
            _, grad = ctx.sim.adj_gradient(v0, ctx.precision)
            return gout * grad, None, None

    return MPStep, LevelSetLoss, DamBreakLoss


_FUNCS = None


def _fn(i):
    global _FUNCS
    if _FUNCS is None:
        _FUNCS = _functions()
    return _FUNCS[i]


def mp_step(x0, v0, sim, precision: int = PREC_MIXED, T0=None):
    """torch.autograd entry: (xT, vT) of the recorded steps from (x0, v0), or
    (xT, vT, TT) from (x0, v0, T0) when the recording ran the heat stage."""
    return _fn(0).apply(x0, v0, T0, sim, precision)


def level_set_loss(xT, sim, precision: int = PREC_MIXED):
    """torch.autograd entry: the target-point level-set loss of final positions."""
    return _fn(1).apply(xT, sim, precision)


def dam_break_loss(v0, sim, precision: int = PREC_MIXED):
    """torch.autograd entry: loss(v0) with d loss / d v0 from the adjoint."""
    return _fn(2).apply(v0, sim, precision)
