"""The C ABI: libmp.so loads without a GPU and exports every function include/mp.h
declares; the Python mirrors of mp_params, mp_state and enum mp_field agree with
the header."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT

HDR = os.path.join(ROOT, "include", "mp.h")


def _header():
    with open(HDR) as f:
        return f.read()


def _decls():
    txt = re.sub(r"/\*.*?\*/", "", _header(), flags=re.S)
    return sorted(set(re.findall(r"\b(?:int|int64_t)\s+(mp_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(mp):
    lib = mp.load_library()
    names = _decls()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_params_struct_matches_header(mp):
    txt = re.sub(r"/\*.*?\*/", "", _header(), flags=re.S)
    body = re.search(r"typedef struct mp_params \{(.*?)\} mp_params;", txt, re.S).group(1)
    names = []
    for line in body.split(";"):
        line = line.strip()
        if not line:
            continue
        m = re.match(r"(int32_t|float)\s+(.*)", line)
        assert m, line
        for part in m.group(2).split(","):
            nm = part.strip().split("[")[0].strip()
            names.append(nm)
    p = mp.Params()
    py = [f for f, _ in p._fields_]
    assert py == names, (py, names)
    assert C.sizeof(p) == mp.load_library().mp_params_size()


def test_field_enum_matches_header(mp):
    txt = _header()
    body = re.search(r"enum mp_field \{(.*?)\};", txt, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    ids = [x.strip().split("=")[0].strip() for x in body.split(",") if x.strip()]
    ids = [i for i in ids if i != "MP_FIELD_COUNT"]
    py = [("MP_P_" if n in ("pos", "vel", "flag", "mass", "temp", "lheat", "solubility", "gascontain") else "MP_F_") + n.upper()
          for n in mp.FIELDS]
    py = [s.replace("MP_F_SURFTENSION", "MP_F_SURFTENSION") for s in py]
    assert py == ids


def test_state_struct_size(mp):
    # mp_state: 4 ints, double, int (+pad), double, 3x3 ints, 6 reserved -> 104 bytes
    assert C.sizeof(mp.MPState) == 104


def test_params_default_and_derive(mp):
    p = mp.default_params(64, 64, 64, 1000)
    assert p.version == 4 and p.nx == 64 and abs(p.cellsize - 1 / 64) < 1e-9
    # spray.cpp:573-588: m0 = waterrho / (1/samplespace)^3, airm0 = m0
    assert abs(p.m0 - 1000.0 * (0.5 / 64) ** 3) < 1e-9 and p.airm0 == p.m0
    assert p.cg_max_iter == 800 and p.heat_cg_max_iter == 3800 and p.heat_clamp == 378.0


def test_bad_arguments_are_rejected_without_a_gpu(mp):
    lib = mp.load_library()
    ctx = C.c_void_p()
    p = mp.default_params(64, 64, 64, 10)
    p.version = 99
    assert lib.mp_create(C.byref(p), C.byref(ctx)) == mp.MP_ERR_ARG
    buf = C.create_string_buffer(256)
    lib.mp_last_error(None, buf, 256)
    assert b"version" in buf.value
    assert lib.mp_hash_sort(None) == mp.MP_ERR_ARG


def test_scene_presets(mp):
    for cfg, n in [(1, 32), (2, 64), (3, 128), (4, 64), (5, 256)]:
        p = mp.scene_params(cfg, 0)
        # configuration 5 shrinks the step with h^2 below 64^3 cells per side
        dt = 1 / 240 if cfg < 5 else (1 / 240) * (64 / n) ** 2
        assert p.nx == n and abs(p.cellsize - 1.0 / n) < 1e-9 and abs(p.dt - dt) < 1e-9
    p = mp.scene_params(2, 0)
    assert p.b_gen_gas and p.b_heat_trans and p.b_fixed_heat and p.boiling_point == 1.0
    p = mp.scene_params(3, 0)
    assert p.b_melt and p.b_freeze and p.melting_point == 1.0
    with pytest.raises(mp.MPError):
        mp.scene_params(9, 0)


def test_unsupported_seed_redraw_is_rejected(mp):
    """updateSeedCell's host-rand() re-draw is not part of the step, so asking
    for it fails at mp_create with a message instead of being ignored."""
    import ctypes as C
    lib = mp.load_library()
    p = mp.default_params(16, 16, 16, 100)
    p.seed_redraw = 1
    ctx = C.c_void_p()
    assert lib.mp_create(C.byref(p), C.byref(ctx)) == mp.MP_ERR_ARG
    buf = C.create_string_buffer(256)
    lib.mp_last_error(None, buf, 256)
    assert b"seed_redraw" in buf.value
