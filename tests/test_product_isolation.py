"""The product never reaches the oracle: no module of the package imports it,
libmp.so declares no dependency on the oracle's library (its only shared
dependencies are the C/C++ runtime and zlib; the CUDA runtime is linked
statically), and the package's library loader maps libmp.so and no oracle
library."""
import ast
import glob
import json
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "2017multiphase_b200")
LIB = os.path.join(PKG, "libmp.so")


def test_package_modules_do_not_import_the_oracle():
    for path in glob.glob(os.path.join(PKG, "**", "*.py"), recursive=True):
        tree = ast.parse(open(path).read(), path)
        for node in ast.walk(tree):
            names = []
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                names = [node.module or ""]
            assert not [n for n in names if n.split(".")[0] == "oracle"], (path, names)


@pytest.mark.skipif(not os.path.exists(LIB) or shutil.which("readelf") is None, reason="libmp.so or readelf missing")
def test_library_dependencies():
    out = subprocess.run(["readelf", "-d", LIB], capture_output=True, text=True, check=True).stdout
    needed = sorted(l.split("[", 1)[1].rstrip("]") for l in out.splitlines() if "(NEEDED)" in l)
    assert not [n for n in needed if "oracle" in n], needed
    allowed = ("libz.", "libstdc++.", "libm.", "libgcc_s.", "libc.", "ld-linux", "libdl.", "libpthread.", "librt.")
    assert all(n.startswith(allowed) for n in needed), needed


PROBE = r"""
import importlib, json
mp = importlib.import_module("2017multiphase_b200")
mp.load_library()
libs = sorted({l.split()[-1] for l in open("/proc/self/maps") if l.rstrip().endswith(".so")})
print(json.dumps(libs))
"""


@pytest.mark.skipif(not os.path.exists(LIB), reason="libmp.so not built")
def test_loader_maps_the_library_and_no_oracle():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    libs = json.loads(r.stdout.strip().splitlines()[-1])
    assert [l for l in libs if os.path.basename(l) == "libmp.so"], libs
    assert not [l for l in libs if "oracle" in l], libs
