"""ctypes binding of oracle/_ref/librefhost.so — TEST INFRASTRUCTURE ONLY.

The library is the reference's own kernels (Multiphase/Multiphase/spray_k.cu),
compiled for the host by oracle/make_refhost.py and launched stage by stage
the way the reference's host code launches them (oracle/refhost/stages.inc).
RefHost holds one cspray state in numpy arrays under the library's field names
and runs bubblesim's stages under the reference's method names, so that the
oracle's stages can be compared with the reference's arithmetic on the same
inputs.  Only tests/ use it; it needs the reference source tree to build.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "librefhost.so")
_lib = None

PARTICLES = ["pos", "vel", "flag", "mass", "temp", "lheat", "solubility", "gascontain"]
_DT = {"mark": np.int8, "flag": np.int8, "cellstart": np.uint32, "cellend": np.uint32}


class RHState(C.Structure):
    _fields_ = [("f", C.c_void_p * 45), ("np", C.c_int32), ("cap", C.c_int32), ("frame", C.c_int32),
                ("n_real_solid", C.c_int32), ("randfloat", C.c_void_p), ("nrand", C.c_int32),
                ("seeds", C.c_void_p), ("nseed", C.c_int32), ("iters", C.c_int32), ("residual", C.c_double),
                ("capped", C.c_int32), ("pour_pos", C.c_void_p), ("pour_vel", C.c_void_p), ("npour", C.c_int32),
                ("solid_verts", C.c_void_p), ("nsolid_verts", C.c_int32), ("run_mc_solid", C.c_int32)]


class RHMesh(C.Structure):
    _fields_ = [("dens", C.c_void_p), ("voxel_verts", C.c_void_p), ("verts", C.c_void_p), ("normals", C.c_void_p),
                ("indices", C.c_void_p), ("maxv", C.c_int32), ("maxi", C.c_int32), ("nverts", C.c_int32),
                ("nindices", C.c_int32), ("active", C.c_int32)]


def load(src_dir=None):
    """Loads the library, building it from the reference source first when it
    is missing (raises FileNotFoundError without the reference tree)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        from oracle import make_refhost
        make_refhost.build(src_dir or make_refhost.DEFAULT_SRC, quiet=True)
    lib = C.CDLL(LIB)
    lib.rh_stage.argtypes = [C.c_char_p, C.POINTER(RHState), C.c_void_p, C.c_float]
    lib.rh_stage.restype = C.c_int
    lib.rh_last_error.restype = C.c_char_p
    lib.rh_verify_own_writes.argtypes = [C.c_int]
    lib.rh_mc.argtypes = [C.POINTER(RHState), C.c_void_p, C.c_int, C.POINTER(RHMesh)]
    lib.rh_mc.restype = C.c_int
    lib.rh_smooth_normals.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int]
    lib.rh_smooth_normals.restype = None
    _lib = lib
    return lib


class RefHost:
    """One cspray state run by the reference's kernels on the CPU."""

    def __init__(self, params, fields, state_cls):
        self.lib = load()
        self.params = params
        self.FIELD_ID = fields
        self.State = state_cls
        nx, ny, nz = params.nx, params.ny, params.nz
        n = nx * ny * nz
        cap = params.par_num_max
        faces = {"ux": (nx + 1) * ny * nz, "uy": nx * (ny + 1) * nz, "uz": nx * ny * (nz + 1)}
        self.a = {}
        for name in fields:
            if name in PARTICLES:
                cnt = cap * 3 if name in ("pos", "vel") else cap
            else:
                axis = [k for k in faces if name.startswith(("water" + k, "air" + k, "solid" + k))]
                cnt = faces[axis[0]] if axis else n
            self.a[name] = np.zeros(cnt, _DT.get(name, np.float32))
        self.np = 0
        self.frame = 0
        self.n_real_solid = 0
        self.iters, self.residual, self.capped = 0, 0.0, 0
        self.rf = np.zeros(1, np.float32)
        self.seeds = np.zeros(1, np.int32)
        self.mesh = {}
        self.pour_pos = np.zeros((0, 3), np.float32)
        self.pour_vel = np.zeros((0, 3), np.float32)
        self.solid_verts = np.zeros((0, 3), np.float32)   # the kept solid surface solidmotion moves
        self.dens = np.zeros((2 * nx + 1) * (2 * ny + 1) * (2 * nz + 1), np.float32)
        self.voxel_verts = np.zeros(8 * n, np.uint32)

    # ---- state, in the Oracle's interface --------------------------------------
    def get_field(self, name):
        a = self.a[name]
        if name in PARTICLES:
            return a[: self.np * (3 if name in ("pos", "vel") else 1)].copy()
        return a.copy()

    def set_field(self, name, v):
        v = np.ascontiguousarray(v, self.a[name].dtype).ravel()
        self.a[name][: v.size] = v

    def upload_particles(self, pos, flag, mass, vel=None, temp=None, lheat=None, solubility=None, gascontain=None):
        pos = np.asarray(pos, np.float32).reshape(-1, 3)
        self.np = pos.shape[0]
        for k in PARTICLES:     # unused slots read as a fresh, zeroed buffer
            self.a[k][:] = 0
        vals = dict(pos=pos, vel=vel, flag=flag, mass=mass, temp=temp, lheat=lheat, solubility=solubility,
                    gascontain=gascontain)
        for k, v in vals.items():
            if v is not None:
                self.set_field(k, v)

    def download_particles(self):
        out = {k: self.get_field(k) for k in PARTICLES}
        out["pos"] = out["pos"].reshape(-1, 3)
        out["vel"] = out["vel"].reshape(-1, 3)
        return out

    def set_tables(self, randfloat, seeds):
        self.rf = np.ascontiguousarray(randfloat, np.float32)
        self.seeds = np.ascontiguousarray(seeds, np.int32)

    def set_pour(self, pos, vel):
        self.pour_pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        self.pour_vel = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)

    def set_state(self, s):
        self.frame = s.frame
        self.n_real_solid = s.n_real_solpoint

    def state(self):
        s = self.State()
        s.frame, s.par_num_now, s.n_real_solpoint = self.frame, self.np, self.n_real_solid
        s.last_cg_iters, s.last_cg_residual = self.iters, self.residual
        return s

    # ---- stages ------------------------------------------------------------------
    def _state(self):
        st = RHState()
        for fname, fid in self.FIELD_ID.items():
            st.f[fid] = self.a[fname].ctypes.data
        st.np, st.cap, st.frame, st.n_real_solid = self.np, self.params.par_num_max, self.frame, self.n_real_solid
        st.randfloat, st.nrand = self.rf.ctypes.data, self.rf.size
        st.seeds, st.nseed = self.seeds.ctypes.data, self.seeds.size
        st.pour_pos, st.pour_vel, st.npour = self.pour_pos.ctypes.data, self.pour_vel.ctypes.data, len(self.pour_pos)
        st.solid_verts, st.nsolid_verts = self.solid_verts.ctypes.data, len(self.solid_verts)
        st.run_mc_solid = self.params.b_run_mc_solid
        return st

    def run(self, name, arg=0.0):
        st = self._state()
        rc = self.lib.rh_stage(name.encode(), C.byref(st), C.addressof(self.params), C.c_float(arg))
        if rc:
            raise RuntimeError(f"reference stage {name}: {self.lib.rh_last_error().decode()}")
        self.np, self.n_real_solid = st.np, st.n_real_solid
        self.iters, self.residual, self.capped = st.iters, st.residual, st.capped
        return rc

    def runMC(self, surface, maxv=2_000_000, maxi=6_000_000):
        """runMC_smooth for one surface (MP_MC_*); preMC must have run."""
        st = self._state()
        v = np.zeros((maxv, 3), np.float32)
        nr = np.zeros((maxv, 3), np.float32)
        ix = np.zeros(maxi, np.uint32)
        m = RHMesh(self.dens.ctypes.data, self.voxel_verts.ctypes.data, v.ctypes.data, nr.ctypes.data,
                   ix.ctypes.data, maxv, maxi, 0, 0, 0)
        rc = self.lib.rh_mc(C.byref(st), C.addressof(self.params), surface, C.byref(m))
        if rc:
            raise RuntimeError(f"reference runMC: {self.lib.rh_last_error().decode()}")
        self.mesh[surface] = (v[: m.nverts].copy(), nr[: m.nverts].copy(), ix[: m.nindices].copy(), m.active)
        return rc

    def smooth_and_normals(self, verts, indices, smooth, iters):
        """smoothMesh (when smooth) and calNormals on a given mesh; returns
        the smoothed vertices and the normals."""
        v = np.ascontiguousarray(verts, np.float32).copy()
        ix = np.ascontiguousarray(indices, np.uint32)
        nr = np.zeros_like(v)
        self.lib.rh_smooth_normals(v.ctypes.data, nr.ctypes.data, len(v), ix.ctypes.data, ix.size, int(smooth),
                                   int(iters))
        return v, nr

    def mc_mesh(self, surface):
        v, nr, ix, _ = self.mesh[surface]
        return v, nr, ix

    def mc_field(self):
        """The last density field and classifyVoxel's per-voxel vertex counts."""
        return self.dens.copy(), self.voxel_verts.copy()

    def __getattr__(self, name):
        if name.startswith("_") or name in ("a", "lib"):
            raise AttributeError(name)
        return lambda *args: self.run(name, float(args[0]) if args else 0.0)
