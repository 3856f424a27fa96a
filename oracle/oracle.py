"""ctypes binding of the CPU oracle (oracle/oracle.cpp) — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this;
the product never does. The oracle restates the reference's multiphase FLIP
step (gaoyangVR/2017Multiphase, Multiphase/Multiphase/spray.cpp:979-1233 and the
spray_k.cu kernels it launches) on the CPU. Parity status: pinned to the
reference's own kernels compiled for the host (oracle/make_refhost.py,
tests/test_refhost_*.py; see oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "libmp_oracle.so")
_lib = None


def build(quiet: bool = True) -> str:
    """Compiles the oracle with its Makefile (g++, no GPU needed)."""
    r = subprocess.run(["make", "-C", _HERE], capture_output=quiet, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + (r.stdout or "") + (r.stderr or ""))
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    vp = C.c_void_p
    for nm in ["or_hash_sort", "or_external_force", "or_sweep_ls_mark", "or_mark_solo_air", "or_surface_tension",
               "or_markgrid_bubble", "or_p2g", "or_drag", "or_g2p", "or_solid_motion", "or_solo_air_update",
               "or_collide_advect", "or_correct_pos", "or_correct_pos_bubble", "or_heat", "or_gen_gas", "or_delete",
               "or_melt", "or_freeze", "or_mc_presort", "or_step", "or_init_particle_heat", "or_heatsim",
               "or_init_heat_grid", "or_flip_mark", "or_water_p2g", "or_water_g2p", "or_water_advect", "or_watersim",
               "or_pour"]:
        f = getattr(lib, nm)
        f.argtypes = [vp]
        f.restype = C.c_int
    lib.or_create.argtypes = [vp, C.POINTER(vp)]
    lib.or_destroy.argtypes = [vp]
    lib.or_destroy.restype = None
    lib.or_set_params.argtypes = [vp, vp]
    lib.or_get_state.argtypes = [vp, vp]
    lib.or_set_state.argtypes = [vp, vp]
    lib.or_upload_particles.argtypes = [vp, C.c_int] + [vp] * 8
    lib.or_field_info.argtypes = [vp, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    lib.or_get_field.argtypes = [vp, C.c_int, vp, C.c_size_t]
    lib.or_set_field.argtypes = [vp, C.c_int, vp, C.c_size_t]
    lib.or_set_tables.argtypes = [vp, vp, C.c_int, vp, C.c_int]
    lib.or_set_mc_tables.argtypes = [vp, vp, vp]
    lib.or_levelset.argtypes = [vp, C.c_float]
    lib.or_sweep_phi.argtypes = [vp, C.c_int]
    lib.or_sweep_u.argtypes = [vp, C.c_int]
    lib.or_set_boundary_u.argtypes = [vp, C.c_int]
    lib.or_project.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.or_project_water.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.or_set_pour.argtypes = [vp, vp, vp, C.c_int]
    lib.or_get_params.argtypes = [vp, vp]
    lib.or_mc_sphere.argtypes = [vp, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float]
    lib.or_mc.argtypes = [vp, C.c_int]
    lib.or_mc_get.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, C.c_int]
    lib.or_mc_get_field.argtypes = [vp, vp, vp]
    lib.or_set_threads.argtypes = [C.c_int]
    lib.or_set_threads.restype = None
    _lib = lib
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """CPU restatement of one cspray context; same field names as the product's Sim."""

    def __init__(self, params, fields, state_cls, mc_tables=None, threads: int = 0):
        self.lib = load()
        if threads:
            self.lib.or_set_threads(threads)
        self.params = params
        self.FIELD_ID = fields
        self.State = state_cls
        self.h = C.c_void_p()
        rc = self.lib.or_create(C.byref(params), C.byref(self.h))
        if rc:
            raise RuntimeError(f"or_create failed: {rc}")
        if mc_tables is not None:
            nv, tri = mc_tables[0], mc_tables[1]
            self.lib.or_set_mc_tables(self.h, _ptr(np.ascontiguousarray(nv, np.int32)),
                                      _ptr(np.ascontiguousarray(tri, np.int32)))

    def __del__(self):
        try:
            if self.h:
                self.lib.or_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def _rc(self, rc, ok=(0,)):
        if rc not in ok:
            raise RuntimeError(f"oracle stage failed with status {rc}")
        return rc

    def upload_particles(self, pos, flag, mass, vel=None, temp=None, lheat=None, solubility=None, gascontain=None):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        arrs = [pos, None if vel is None else np.ascontiguousarray(vel, np.float32).reshape(-1, 3),
                np.ascontiguousarray(flag, np.int8), np.ascontiguousarray(mass, np.float32)]
        arrs += [None if a is None else np.ascontiguousarray(a, np.float32) for a in (temp, lheat, solubility, gascontain)]
        self._rc(self.lib.or_upload_particles(self.h, pos.shape[0], *[_ptr(a) for a in arrs]))

    def get_field(self, name: str) -> np.ndarray:
        cnt = C.c_size_t(); eb = C.c_size_t()
        self._rc(self.lib.or_field_info(self.h, self.FIELD_ID[name], C.byref(cnt), C.byref(eb)))
        dt = {"mark": np.int8, "flag": np.int8, "cellstart": np.uint32, "cellend": np.uint32}.get(name, np.float32)
        a = np.zeros(cnt.value, dt)
        self._rc(self.lib.or_get_field(self.h, self.FIELD_ID[name], _ptr(a), a.nbytes))
        return a

    def set_field(self, name: str, a: np.ndarray):
        dt = {"mark": np.int8, "flag": np.int8, "cellstart": np.uint32, "cellend": np.uint32}.get(name, np.float32)
        a = np.ascontiguousarray(a, dt).ravel()
        self._rc(self.lib.or_set_field(self.h, self.FIELD_ID[name], _ptr(a), a.nbytes))

    def set_tables(self, randfloat, seeds):
        rf = np.ascontiguousarray(randfloat, np.float32)
        sd = np.ascontiguousarray(seeds, np.int32)
        self._rc(self.lib.or_set_tables(self.h, _ptr(rf), rf.size, _ptr(sd), sd.size))

    def state(self):
        s = self.State()
        self.lib.or_get_state(self.h, C.byref(s))
        return s

    def set_state(self, s):
        self._rc(self.lib.or_set_state(self.h, C.byref(s)))

    def set_params(self, p):
        self._rc(self.lib.or_set_params(self.h, C.byref(p)))
        self.params = p

    def download_particles(self) -> Dict[str, np.ndarray]:
        out = {k: self.get_field(k) for k in ["pos", "vel", "flag", "mass", "temp", "lheat", "solubility",
                                              "gascontain"]}
        out["pos"] = out["pos"].reshape(-1, 3)
        out["vel"] = out["vel"].reshape(-1, 3)
        return out

    # stages under the reference's names
    def initHeatAndSolubility(self): return self._rc(self.lib.or_init_particle_heat(self.h))
    def hashAndSortParticles(self): return self._rc(self.lib.or_hash_sort(self.h))
    def addexternalforce(self): return self._rc(self.lib.or_external_force(self.h))
    def computeLevelset(self, offset=0.0): return self._rc(self.lib.or_levelset(self.h, C.c_float(offset)))
    def sweepLSAndMardGrid(self): return self._rc(self.lib.or_sweep_ls_mark(self.h))
    def markSoloAirParticle(self): return self._rc(self.lib.or_mark_solo_air(self.h))
    def computesurfacetension(self): return self._rc(self.lib.or_surface_tension(self.h))
    def markgrid_bubble(self): return self._rc(self.lib.or_markgrid_bubble(self.h))
    def mapvelp2g_bubble(self): return self._rc(self.lib.or_p2g(self.h))
    def enforceDragForce(self): return self._rc(self.lib.or_drag(self.h))
    def sweepPhi(self, ph): return self._rc(self.lib.or_sweep_phi(self.h, ph))
    def sweepU(self, ph): return self._rc(self.lib.or_sweep_u(self.h, ph))
    def setWaterBoundaryU(self, ph): return self._rc(self.lib.or_set_boundary_u(self.h, ph))

    def project_CG_bubble(self):
        it = C.c_int(); res = C.c_double()
        rc = self._rc(self.lib.or_project(self.h, C.byref(it), C.byref(res)), ok=(0, 3))
        return it.value, res.value, rc

    def mapvelg2p_bubble(self): return self._rc(self.lib.or_g2p(self.h))
    def solidmotion(self): return self._rc(self.lib.or_solid_motion(self.h))
    def updateSoloAirParticle(self): return self._rc(self.lib.or_solo_air_update(self.h))
    def CollisionSolid(self): return self._rc(self.lib.or_collide_advect(self.h))
    def correctpos(self): return self._rc(self.lib.or_correct_pos(self.h))
    def correctpos_bubble(self): return self._rc(self.lib.or_correct_pos_bubble(self.h))
    def updateTemperature(self): return self._rc(self.lib.or_heat(self.h), ok=(0, 3))
    def heatsim(self): return self._rc(self.lib.or_heatsim(self.h), ok=(0, 3))
    def set_pour(self, pos, vel):
        p3 = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        v3 = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        return self._rc(self.lib.or_set_pour(self.h, _ptr(p3), _ptr(v3), len(p3)))

    def get_params(self, p):
        """Fills the ctypes mp_params `p` with the oracle's current parameters."""
        return self._rc(self.lib.or_get_params(self.h, C.byref(p)))

    def pouring(self): return self._rc(self.lib.or_pour(self.h))
    def runMC_sphere(self, s, center, radius):
        return self._rc(self.lib.or_mc_sphere(self.h, s, *[float(c) for c in center], float(radius)))
    def flipMark_sphere(self): return self._rc(self.lib.or_flip_mark(self.h))
    def mapvelp2g(self): return self._rc(self.lib.or_water_p2g(self.h))
    def mapvelg2p(self): return self._rc(self.lib.or_water_g2p(self.h))
    def wateradvect(self): return self._rc(self.lib.or_water_advect(self.h))
    def watersim(self): return self._rc(self.lib.or_watersim(self.h), ok=(0, 3))

    def project_CG(self):
        it = C.c_int(); res = C.c_double()
        rc = self._rc(self.lib.or_project_water(self.h, C.byref(it), C.byref(res)), ok=(0, 3))
        return it.value, res.value, rc
    def initheat_grid(self): return self._rc(self.lib.or_init_heat_grid(self.h))
    def GenerateGasParticle(self): return self._rc(self.lib.or_gen_gas(self.h))
    def deleteAirFluidParticle(self): return self._rc(self.lib.or_delete(self.h))
    def MeltSolid(self): return self._rc(self.lib.or_melt(self.h))
    def Freezing(self): return self._rc(self.lib.or_freeze(self.h))
    def preMC(self): return self._rc(self.lib.or_mc_presort(self.h))
    def runMC(self, s): return self._rc(self.lib.or_mc(self.h, s))
    def bubblesim(self): return self._rc(self.lib.or_step(self.h), ok=(0, 3))

    def mc_mesh(self, surface):
        s = self.state()
        nv, ni = s.mc_verts[surface], s.mc_indices[surface]
        v = np.zeros((nv, 3), np.float32); nr = np.zeros((nv, 3), np.float32); ix = np.zeros(ni, np.uint32)
        self._rc(self.lib.or_mc_get(self.h, surface, _ptr(v), _ptr(nr), _ptr(ix), nv, ni))
        return v, nr, ix

    def mc_field(self):
        p = self.params
        dens = np.zeros((2 * p.nx + 1) * (2 * p.ny + 1) * (2 * p.nz + 1), np.float32)
        cube = np.zeros(8 * p.nx * p.ny * p.nz, np.uint8)
        self._rc(self.lib.or_mc_get_field(self.h, _ptr(dens), _ptr(cube)))
        return dens, cube
