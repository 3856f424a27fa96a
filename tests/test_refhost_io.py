"""The product's per-frame file writers (mp_write_mesh / mp_write_particles,
csrc/host/export.cpp) against the reference's own writers compiled for the
host (outputPovRaywater, outputOBJwater, outputBOBJwater,
outputColoredParticle, outputSoloBubblePovRay, outputAirParticlePovRay in
spray.cu, mapColorBlue2Red_h in spray.cpp; oracle/make_refhost.py).  The
same mesh and particles go through both and the files must be equal byte for
byte, the BOBJ.gz files included (both write through zlib's gzopen "wb1").
The reference names its files with Windows separators; on this host those
are part of the file name.  Skipped without the reference source tree."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from test_refhost_stages import SRC

pytestmark = pytest.mark.skipif(not os.path.exists(SRC + "/spray_k.cu"), reason="reference source tree not present")


def _mesh(rng, nv=257, nt=401, bad=True):
    v = rng.uniform(-1, 2, (nv, 3)).astype(np.float32)
    n = rng.normal(size=(nv, 3)).astype(np.float32)
    if bad:                                   # verifyfloat3 writes NaN vertices as 0
        v[3, 1] = np.nan
        n[5, 2] = np.nan
        v[7] = [1e-30, -1e-30, 123456.789]
    ix = rng.integers(0, nv, 3 * nt).astype(np.uint32)
    return v, n, ix


def _read(p):
    with open(p, "rb") as f:
        return f.read()


@pytest.fixture
def shortdir():
    """cspray::outputdir holds 29 characters: a short directory prefix."""
    d = tempfile.mkdtemp(prefix="rh", dir="/tmp")
    yield d + "/"
    for f in os.listdir(d):
        os.remove(os.path.join(d, f))
    os.rmdir(d)


def _lib(refhost):
    lib = refhost.load()
    vp = C.c_void_p
    lib.rh_write_mesh.argtypes = [C.c_int, C.c_char_p, C.c_int, vp, vp, C.c_int, vp, C.c_int, C.c_char_p]
    lib.rh_write_mesh.restype = C.c_int
    lib.rh_write_particles.argtypes = [C.c_int, C.c_char_p, C.c_int, vp, vp, vp, C.c_int, C.c_float, C.c_float]
    lib.rh_write_particles.restype = None
    return lib


@pytest.mark.parametrize("name", ["water", "gas", "solid"])
@pytest.mark.parametrize("empty", [False, True])
def test_mesh_files_equal_the_reference_writers(mp, refhost, shortdir, name, empty):
    lib = _lib(refhost)
    v, n, ix = _mesh(np.random.default_rng(11 + len(name)))
    if empty:
        v, n, ix = v[:0], n[:0], ix[:0]
    frame = 7
    refs = {mp.OUT_POV_MESH: f"waterdata\\{name}{frame:05d}.pov", mp.OUT_OBJ_MESH: f"waterOBJdata\\{name}{frame:05d}.obj",
            mp.OUT_BOBJ_GZ: f"{name}BOBJdata\\fluidsurface_final_{frame - 1:04d}.bobj.gz"}
    for fmt, fn in refs.items():
        code = {mp.OUT_POV_MESH: 0, mp.OUT_OBJ_MESH: 1, mp.OUT_BOBJ_GZ: 2}[fmt]
        assert lib.rh_write_mesh(code, shortdir.encode(), frame, v.ctypes.data, n.ctypes.data, len(v), ix.ctypes.data,
                                 len(ix), name.encode()) == 0
        ours = os.path.join(shortdir, f"ours{fmt}")
        mp.write_mesh(fmt, ours, v, n, ix, name)
        assert _read(ours) == _read(os.path.join(shortdir, fn)), (fmt, fn)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_particle_files_equal_the_reference_writers(mp, refhost, shortdir, kind):
    lib = _lib(refhost)
    rng = np.random.default_rng(21 + kind)
    npart = 999
    pos = rng.uniform(0, 1, (npart, 3)).astype(np.float32)
    flag = rng.integers(0, 6, npart).astype(np.int8)
    temp = rng.uniform(250, 400, npart).astype(np.float32)
    frame = 12
    lib.rh_write_particles(kind, shortdir.encode(), frame, pos.ctypes.data, flag.ctypes.data, temp.ctypes.data, npart,
                           263.0, 383.0)
    fn = {0: f"waterdata\\allparticles{frame:05d}.pov", 1: f"waterdata\\solobubble{frame:05d}.pov",
          2: f"waterdata\\solobubble{frame:05d}.pov"}[kind]
    ours = os.path.join(shortdir, "ours.pov")
    kinds = {0: mp.OUT_PARTICLES_COLORED, 1: mp.OUT_PARTICLES_SOLO, 2: mp.OUT_PARTICLES_AIR}
    mp.write_particles(kinds[kind], ours, pos, flag, temp, 263.0, 383.0)
    ref = _read(os.path.join(shortdir, fn))
    assert len(ref) > 0 and _read(ours) == ref


@pytest.mark.parametrize("variant, radius, c2", [(0, 0.035, None), (1, 0.05, None), (2, 0.04, (0.3, 0.7, 0.8)),
                                                 (0, 0.0, None)])
def test_pouring_emitters_equal_the_reference(mp, refhost, variant, radius, c2):
    """mp_scene_pour against CompPouringParam_Freezing / _Ineraction /
    _Ineraction2 (spray.cpp:1416-1545), points and velocities bit for bit."""
    lib = refhost.load()
    vp = C.c_void_p
    lib.rh_pour_lattice.argtypes = [C.c_int, C.c_float, C.c_float, vp, vp, vp, vp, vp, C.c_int]
    lib.rh_pour_lattice.restype = C.c_int
    ss = np.float32(1.0 / 64 * 0.5)
    c1 = np.array([0.5, 0.45, 0.9], np.float32)
    vel = np.array([0.0, 0.1, -0.5], np.float32)
    cc2 = None if c2 is None else np.array(c2, np.float32)
    cap = 100000
    rp = np.zeros((cap, 3), np.float32)
    rv = np.zeros((cap, 3), np.float32)
    n = lib.rh_pour_lattice(variant, ss, radius, c1.ctypes.data, None if cc2 is None else cc2.ctypes.data,
                            vel.ctypes.data, rp.ctypes.data, rv.ctypes.data, cap)
    pos, pvel = mp.scene_pour(variant, float(ss), radius, c1, vel, center2=cc2)
    assert len(pos) == n
    assert np.array_equal(pos.view(np.uint32), rp[:n].view(np.uint32))
    assert np.array_equal(pvel.view(np.uint32), rv[:n].view(np.uint32))
