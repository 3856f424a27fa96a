"""mp_reference_scene against cspray::initparam (Multiphase/Multiphase/spray.cpp:23-626)
read as text: the common defaults, each scene's branch and the settings after the
branches are parsed from the reference source (where the reference tree is
present), replayed in order, and every mapped member is compared with the
library's parameters and scene info. A layout check of mp_scene_info from C
runs everywhere."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

# the reference's source directory: the one the oracle's recipe compiles from
from oracle.make_refhost import DEFAULT_SRC  # noqa: E402
SPRAY_CPP = os.path.join(DEFAULT_SRC, "spray.cpp")

# reference member -> mp_params field (p) or mp_scene_info field (i)
PARAM = {
    "surfacetensionsigma": "surfacetension_sigma", "heatalphafluid": "heatalpha_fluid",
    "heatalphaair": "heatalpha_air", "heatalphasolid": "heatalpha_solid", "heatalphavacuum": "heatalpha_vacuum",
    "defaulttemperature": "default_temperature", "Temperature0": "temperature0", "meltingpoint": "melting_point",
    "boilingpoint": "boiling_point", "dragParamSolo": "drag_param_solo", "dragParamGrid": "drag_param_grid",
    "viscosiySPH": "viscosity_sph", "m_bSolid": "b_solid", "m_bMelt": "b_melt", "m_bFreeze": "b_freeze",
    "m_bFixSolid": "b_fix_solid", "m_bGenGas": "b_gen_gas", "m_bHeatTrans": "b_heat_trans",
    "m_bAddHeatBottom": "b_add_heat_bottom", "m_bExtendHeatToBoundary": "b_extend_heat_to_boundary",
    "m_bCorrectPosition": "b_correct_position", "SolidbounceParam": "solid_bounce_param",
    "defaultSolidT": "default_solid_T", "defaultLiquidT": "default_liquid_T", "LiquidHeatTh": "liquid_heat_th",
    "posrandparam": "pos_rand_param", "velrandparam": "vel_rand_param", "alphaTempTrans": "alpha_temp_trans",
    "bounceVelParam": "bounce_vel_param", "bouncePosParam": "bounce_pos_param",
    "initdissolvegasrate": "init_dissolve_gas_rate", "initgasrate": "init_gas_rate",
    "vaporGenRate": "vapor_gen_rate", "m_bSmoothMC": "b_smooth_mc", "bRunMCSolid": "b_run_mc_solid",
    "bubbleMaxVel": "bubble_max_vel", "updateSeedFrameDelta": "update_seed_frame_delta",
    "buoyanceRateAir": "buoyance_rate_air", "buoyanceRateSolo": "buoyance_rate_solo", "m_beginFrame": "begin_frame",
    "heatIncreaseBottom": "heat_increase_bottom", "outputframeDelta": "mc_every", "fMCDensity": "mc_density",
    "smoothIterTimes": "smooth_iters", "correctionspring": "correction_spring",
    "correctionradius": "correction_radius", "hparam.dt": "dt", "hparam.waterrho": "waterrho",
    "hparam.solidrho": "solidrho",
}
INFO = {
    "seednum": "seed_num", "initfluidparticle": "init_fluid_particles", "splitnum": "split_num",
    "pourRadius": "pour_radius", "pourpos": "pour_pos", "pourpos2": "pour_pos2", "pourvel": "pour_vel",
    "solidInitPos": "solid_init_pos", "temperatureMax_render": "t_render_max",
    "temperatureMin_render": "t_render_min", "frameMax": "frame_max",
    "bOutputColoredParticle": "output_colored_particles",
}
SIM = {"SIMULATION_WATER": 0, "SIMULATION_SOLIDCOUPLING": 1, "SIMULATION_SMOKE": 2, "SIMULATION_BUBBLE": 3,
       "SIMULATION_HEATONLY": 4}
POUR = {"CompPouringParam_Freezing": 0, "CompPouringParam_Ineraction": 1, "CompPouringParam_Ineraction2": 2}


def _value(expr):
    expr = expr.strip()
    m = re.fullmatch(r"make_float3\((.*)\)", expr)
    if m:
        parts = [x.strip() for x in m.group(1).split(",")]
        return [_value(x) for x in parts] if len(parts) == 3 else None
    if expr in ("true", "false"):
        return 1 if expr == "true" else 0
    m = re.fullmatch(r"-?\d+(\.\d*)?f?", expr)
    if m:
        return float(expr.rstrip("f"))
    return None


def _statements(block):
    block = re.sub(r"//[^\n]*", "", block)
    block = re.sub(r"/\*.*?\*/", "", block, flags=re.S)
    block = block.replace("{", ";").replace("}", ";")
    for st in block.split(";"):
        # split top-level commas: a = x, b = y
        depth, cur, parts = 0, "", []
        for ch in st:
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
            if ch == "," and depth == 0:
                parts.append(cur); cur = ""
            else:
                cur += ch
        parts.append(cur)
        for part in parts:
            m = re.fullmatch(r"\s*([A-Za-z_][\w.]*)\s*=\s*(.+?)\s*", part, flags=re.S)
            if m and "==" not in part and "!=" not in part:
                yield m.group(1), m.group(2)


def _branches(txt):
    body = txt[txt.index("void cspray::initparam()"):]
    body = body[:body.index("\n}\n")]
    first = body.index("if (mscene == SCENE_DAMBREAK)")
    base = body[:first]
    out = {}
    pos = first
    tail = ""
    for m in re.finditer(r"(?:else )?if \(mscene == (SCENE_\w+)\)", body[first:]):
        start = first + m.end()
        if start < pos:
            continue
        b0 = body.index("{", start)
        depth, i = 0, b0
        while True:
            if body[i] == "{":
                depth += 1
            elif body[i] == "}":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        out[m.group(1)] = body[b0 + 1:i]
        pos = i
        tail = body[i + 1:]
    return base, out, tail


def _replay(mp, base, branch, tail):
    p, info = {}, {"pour_variant": -1, "split_num": 1}
    for blk in (base, branch, tail):
        for name, expr in _statements(blk):
            v = _value(expr)
            if name in PARAM and v is not None:
                p[PARAM[name]] = v
            elif name in INFO and v is not None:
                info[INFO[name]] = v
            elif name == "simmode":
                info["sim_mode"] = SIM[expr.strip()]
    for fn, v in POUR.items():
        if re.search(fn + r"\(\)\s*;", re.sub(r"//[^\n]*", "", branch)):
            info["pour_variant"] = v
    g = re.search(r"NX\s*!=\s*(\d+)\s*\|\|\s*NY\s*!=\s*(\d+)\s*\|\|\s*NZ\s*!=\s*(\d+)", branch)
    info["grid"] = tuple(int(x) for x in g.groups())
    m = re.search(r"parNumMax\s*=\s*(?:(\d+)\s*\+\s*)?parNumNow(\s*\*\s*splitnum)?\s*;", re.sub(r"//[^\n]*", "", branch))
    if m:
        info["par_num_extra"] = int(m.group(1) or 0)
        if not m.group(2):
            info["split_num"] = 1
    else:
        m = re.search(r"parNumMax\s*=\s*(\d+)\s*;", branch)
        info["par_num_extra"] = int(m.group(1)); info["split_num"] = 0
    return p, info


@pytest.mark.skipif(not os.path.exists(SPRAY_CPP), reason="reference tree not present")
def test_every_scene_matches_initparam(mp):
    with open(SPRAY_CPP, encoding="latin-1") as f:
        txt = f.read()
    base, branches, tail = _branches(txt)
    assert len(branches) == 14, sorted(branches)
    for name, branch in branches.items():
        exp_p, exp_i = _replay(mp, base, branch, tail)
        p, info = mp.reference_scene(getattr(mp, name))
        assert (p.nx, p.ny, p.nz) == exp_i["grid"] == (info["nx"], info["ny"], info["nz"]), name
        for k, v in exp_p.items():
            assert np.float32(getattr(p, k)) == np.float32(v), (name, k, getattr(p, k), v)
        for k, v in exp_i.items():
            if k == "grid":
                continue
            got = info[k]
            if isinstance(v, list):
                assert np.array_equal(np.float32(got), np.float32(v)), (name, k, got, v)
            else:
                assert np.float32(got) == np.float32(v), (name, k, got, v)
        assert p.par_num_max == info["par_num_extra"] + info["init_fluid_particles"] * info["split_num"]


def test_reference_scene_basics(mp):
    p, info = mp.reference_scene(mp.SCENE_BOILING)
    assert info["sim_mode"] == mp.SIM_BUBBLE and p.b_gen_gas == 1 and p.heat_increase_bottom == np.float32(1.5)
    assert p.dt == np.float32(0.003) and p.m0 > 0 and p.mc_every == 2
    p, info = mp.reference_scene(mp.SCENE_HEATTRANSFER)
    assert info["sim_mode"] == mp.SIM_HEATONLY and p.par_num_max == 1
    with pytest.raises(mp.MPError):
        mp.reference_scene(mp.SCENE_SMOKE)             # initparam has no branch for it


def test_scene_info_layout_from_c(mp, tmp_path):
    """A C program reads mp_scene_info through the header; the Python mirror
    sees the same values."""
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    src = tmp_path / "s.c"
    src.write_text(r"""
#include <stdio.h>
#include "mp.h"
int main(void) {
    mp_params p; mp_scene_info s;
    if (mp_reference_scene(MP_SCENE_INTERACTION, &p, &s) != MP_OK) return 1;
    printf("%d %d %d %d %d %d %.9g %.9g %.9g %d %d\n", s.nx, s.ny, s.nz, s.par_num_extra, s.seed_num, s.pour_variant,
           s.pour_pos2[0], s.solid_init_pos[2], s.t_render_max, s.frame_max, (int)sizeof(mp_scene_info));
    return 0;
}
""")
    pkg = os.path.join(ROOT, "2017multiphase_b200")
    exe = tmp_path / "s"
    r = subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe), "-L", pkg,
                        "-lmp", "-Wl,-rpath," + pkg], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()
    _, info = mp.reference_scene(mp.SCENE_INTERACTION)
    assert [int(x) for x in out[:6]] == [info["nx"], info["ny"], info["nz"], info["par_num_extra"],
                                         info["seed_num"], info["pour_variant"]]
    f32 = np.float32
    assert f32(float(out[6])) == f32(info["pour_pos2"][0]) and f32(float(out[7])) == f32(info["solid_init_pos"][2])
    assert f32(float(out[8])) == f32(info["t_render_max"]) and int(out[9]) == info["frame_max"]
    import ctypes
    assert int(out[10]) == ctypes.sizeof(mp.MPSceneInfo)
