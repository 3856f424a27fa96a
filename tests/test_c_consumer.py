"""The drop-in boundary from C: include/mp.h compiles as C99 (gcc -std=c99
-Wall -Werror -pedantic) and as C++17, and a C program linked against libmp.so
calls the host-only entry points (parameter set-up, the pouring emitter, the
file writers) with the results the Python binding sees. No GPU needed."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HDR_DIR = os.path.join(ROOT, "include")
PKG = os.path.join(ROOT, "2017multiphase_b200")

C_SRC = r"""
#include <stdio.h>
#include <string.h>
#include "mp.h"

int main(int argc, char** argv) {
    mp_params p;
    if (mp_params_default(&p, 32, 32, 32, 1000) != MP_OK) return 1;
    if (p.version != MP_PARAMS_VERSION || p.nx != 32) return 2;
    if (mp_params_size() != (int)sizeof(mp_params)) return 3;
    float c[3] = {0.5f, 0.5f, 0.75f}, v[3] = {0.f, 0.f, -0.5f};
    int n = 0;
    if (mp_scene_pour(MP_POUR_FREEZING, p.samplespace, 0.035f, c, NULL, v, 0, NULL, NULL, &n) != MP_OK) return 4;
    float pos[3 * 4096], vel[3 * 4096];
    if (n > 4096 || mp_scene_pour(MP_POUR_FREEZING, p.samplespace, 0.035f, c, NULL, v, n, pos, vel, &n) != MP_OK)
        return 5;
    float verts[9] = {0, 0, 0, 1, 0, 0, 0, 1, 0}, nrm[9] = {0, 0, 1, 0, 0, 1, 0, 0, 1};
    uint32_t idx[3] = {0, 1, 2};
    if (mp_write_mesh(MP_OUT_OBJ_MESH, argv[1], "water", verts, nrm, 3, idx, 3) != MP_OK) return 6;
    if (mp_write_mesh(MP_OUT_OBJ_MESH, "/nonexistent-dir/x.obj", "water", verts, nrm, 3, idx, 3) != MP_ERR_IO) return 7;
    int32_t nvt[256], tri[256 * 16], edge[256];
    if (mp_mc_tables(nvt, tri, edge) != MP_OK || nvt[1] != 3) return 8;
    if (mp_set_mc_tables(NULL, nvt, tri) != MP_ERR_ARG) return 9;      /* no context: refused, no GPU needed */
    printf("%d %.9g %.9g %.9g\n", n, pos[0], pos[1], pos[2]);
    return 0;
}
"""


def _cc():
    for c in ("gcc", "cc"):
        if shutil.which(c):
            return c
    pytest.skip("no C compiler")


def test_header_compiles_as_c99_and_cxx17(tmp_path):
    src = tmp_path / "h.c"
    src.write_text('#include "mp.h"\nint main(void) { mp_params p; (void)p; return 0; }\n')
    r = subprocess.run([_cc(), "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", HDR_DIR, "-c", str(src), "-o",
                        str(tmp_path / "h.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    if shutil.which("g++"):
        cpp = tmp_path / "h.cpp"
        cpp.write_text('#include "mp.h"\nint main() { mp_output o{}; (void)o; return 0; }\n')
        r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", HDR_DIR, "-c", str(cpp), "-o",
                            str(tmp_path / "hc.o")], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_c_program_calls_host_entry_points(mp, tmp_path):
    src = tmp_path / "consumer.c"
    src.write_text(C_SRC)
    exe = tmp_path / "consumer"
    r = subprocess.run([_cc(), "-std=c99", "-Wall", "-I", HDR_DIR, str(src), "-o", str(exe), "-L", PKG, "-lmp",
                        "-Wl,-rpath," + PKG], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    obj = tmp_path / "m.obj"
    r = subprocess.run([str(exe), str(obj)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    n, x, y, z = r.stdout.split()
    p = mp.default_params(32, 32, 32, 1000)
    pos, _ = mp.scene_pour(mp.POUR_FREEZING, p.samplespace, 0.035, (0.5, 0.5, 0.75), (0.0, 0.0, -0.5))
    assert int(n) == len(pos)
    assert np.allclose([float(x), float(y), float(z)], pos[0], rtol=0, atol=0)
    assert obj.read_text().endswith("f  1 2 3\n")
