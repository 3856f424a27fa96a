"""Builds oracle/_ref/librefhost.so: the reference's own CUDA kernels, compiled
for the host CPU, used by tests/test_refhost_*.py to pin the oracle against the
reference's arithmetic.  TEST INFRASTRUCTURE ONLY.

The reference's spray_k.cu does not compile as a whole anywhere but on its
original Windows/CUDA 7.5 setup: it includes the CUDA samples' helper_cuda.h
and helper_math.h (not present), declares texture references (removed in
CUDA 12) and mixes its kernels with host launch code.  Most of its kernels,
though, are plain per-thread functions.  This recipe reads spray_k.cu where it
lies, takes the text of every `__device__` helper and of the kernels named in
KERNELS (unchanged, in file order), and compiles them with g++ under
oracle/refhost/shim.h (and the per-frame file writers of class cspray under
oracle/refhost/cspray_io.h), which gives the CUDA execution model (threadIdx,
blockIdx, ...), helper_math's float3 arithmetic and the few intrinsics the
kernels use a host meaning.  oracle/refhost/stages.inc then launches them the
way spray.cu does, one emulated thread after another.  The extracted source
goes to oracle/_ref/ only (and is deleted once compiled, unless kept for
debugging), which git ignores: nothing of the reference is committed.

Usage: python oracle/make_refhost.py [reference-source-dir] [--keep-source]
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's source directory; MP_REFERENCE_SRC points at another checkout
DEFAULT_SRC = os.environ.get("MP_REFERENCE_SRC", "/root/reference/Multiphase/Multiphase")
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "librefhost.so")

# Kernels launched by refhost/stages.inc (spray_k.cu names).  Thrust's sort
# and scan (spray_thrust.cu) and the float reductions (product(),
# accumulate_GPU_f3) are not the reference's kernels: the sort and the scan are
# restated by their definitions (stable ascending sort, exclusive sum).
KERNELS = [
    "addgravityforce_k", "addbuoyancyforce_vel", "genlevelset", "markLS_bigpositive",
    "setLSback_bigpositive", "preparels", "setLSback", "mergeLSAndMarkGrid", "computePhigra",
    "initphi", "sweepphibytype", "sweepphi", "initSolidPhi",
    "verifySoloAirParticle", "compsurfacetension_k", "enforcesurfacetension_p", "markfluid_dense",
    "mapvelp2g_k_fluidSolid", "mapvelp2g_k_air", "mapvelp2g_k_solid", "calDragForce",
    "sweepu_k_bubble", "setWaterBoundaryU_k", "cptdivergence_bubble2", "computeAx_bubble",
    "pcg_op_bubble", "subGradPress", "computeDeltaU", "mapvelg2p_flip_bubble",
    "calcDensPress_Air", "enforceForceSoloAirP", "CollisionWithSolid_k", "CollisionWithSolid_Freezing",
    "correctparticlepos", "correctbubblepos", "correctbubblepos_air",
    "mapHeatp2g_hash", "addHeatAtBottom", "compb_heat", "computeAx_heat", "pcg_op_heat",
    "setBoundaryHeat", "compTpChange", "mapHeatg2p", "mapHeatg2p_MeltAndBoil", "updateLatentHeat_k",
    "updatesolubility", "GenerateGasParticle_k", "sweepVacuum", "markDeleteAirParticle",
    "deleteparticles", "MeltingSolidByHeat", "FreezingSolidByHeat", "calcHashD", "calcHashD_MC",
    "genWaterDensfield_liquidAndGas", "genWaterDensfield_Gas", "genWaterDensfield_GY",
    "genSphereDensfield", "classifyVoxel", "initheat_grid_k", "markBoundaryCell",
    "pouringwater", "computeSolidVertex_k", "computePosSolid_k", "computeVelSolid_k",
    "set_nonsolid_2_zero", "setVelZeroSolid_k", "solidCollisionWithBound", "compute_cI_k",
    "cptdivergence", "computeAx", "pcg_op", "mapvelg2p_flip",
    "advectparticle_RK2", "flipAirVacuum", "markfluid", "markair", "initHeatParticle", "initsolubility_k",
    "reorderDataAndFindCellStartD", "compactVoxels", "markActiveEdge_MC", "generateTriangles_indices",
    "smooth_computedisplacement", "smooth_addDisplacement", "calnormal_k", "normalizeTriangleNor_k",
    "arrayproduct_k", "accumulate_GPU_k",
]
# __device__ helpers that need what the shim does not give (triangle hashing,
# rendering); nothing in KERNELS calls them.
SKIP_DEVICE = {"collideCell", "IntersectTriangle_q", "calcGridHash_q"}


def _definitions(text):
    """Yields (name, kind, start, end) of every top-level function definition
    whose header carries __device__ or __global__."""
    depth = 0
    i = 0
    n = len(text)
    head_start = 0
    while i < n:
        c = text[i]
        if text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
            continue
        if text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
            continue
        if c == '"' or c == "'":
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            i = j + 1
            continue
        if depth == 0 and c == ";":
            head_start = i + 1
        elif c == "{":
            if depth == 0:
                header = text[head_start:i]
                body_start = i
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                hdr = re.sub(r"//[^\n]*|/\*.*?\*/", "", header, flags=re.S)
                kind = "global" if "__global__" in hdr else ("device" if "__device__" in hdr else None)
                m = re.search(r"([A-Za-z_]\w*)\s*\([^()]*(?:\([^()]*\)[^()]*)*\)\s*$", hdr.strip())
                if kind and m and "(" in hdr:
                    # the header starts after the previous definition/statement
                    start = head_start
                    while start < body_start and text[start] in " \t\r\n":
                        start += 1
                    # drop comment lines directly above the definition
                    yield m.group(1), kind, start, i + 1
                head_start = i + 1
        i += 1


def extract(src_dir):
    path = os.path.join(src_dir, "spray_k.cu")
    with open(path, encoding="latin-1") as f:
        text = f.read()
    parts = []
    found = set()
    for name, kind, s, e in _definitions(text):
        if kind == "global" and name not in KERNELS:
            continue
        if kind == "device" and name in SKIP_DEVICE:
            continue
        chunk = text[s:e]
        # strip comment lines that preceded the header inside the chunk
        line = text.count("\n", 0, s) + 1
        parts.append(f'#line {line} "spray_k.cu"\n{chunk}\n')
        if kind == "global":
            found.add(name)
    missing = [k for k in KERNELS if k not in found]
    if missing:
        raise SystemExit(f"kernels not found in {path}: {missing}")
    return "".join(parts)


# The per-frame file writers and the pouring emitters (host code of class
# cspray) and the helpers they call, compiled under refhost/cspray_io.h.
HOST_FUNCTIONS = [
    ("spray.cu", "verifyfloat3"), ("spray.cpp", "cspray::mapColorBlue2Red_h"),
    ("spray.cu", "cspray::outputPovRaywater"), ("spray.cu", "cspray::outputOBJwater"),
    ("spray.cu", "cspray::outputBOBJwater"), ("spray.cu", "cspray::outputColoredParticle"),
    ("spray.cu", "cspray::outputSoloBubblePovRay"), ("spray.cu", "cspray::outputAirParticlePovRay"),
    ("spray.cpp", "cspray::CompPouringParam_Freezing"), ("spray.cpp", "cspray::CompPouringParam_Ineraction"),
    ("spray.cpp", "cspray::CompPouringParam_Ineraction2"),
]


def _host_function(text, name, fname):
    """The text of one top-level host function definition, found by name."""
    m = re.search(r"^[A-Za-z_][\w \t\*&]*\b" + re.escape(name) + r"\s*\([^)]*\)\s*\{", text, re.M)
    if not m:
        raise SystemExit(f"{name} not found in {fname}")
    depth, i = 0, m.end() - 1
    while True:
        c = text[i]
        if c in "\"'":                       # skip string and character literals
            j = i + 1
            while text[j] != c:
                j += 2 if text[j] == "\\" else 1
            i = j
        elif text.startswith("//", i):
            i = text.index("\n", i)
        elif text.startswith("/*", i):
            i = text.index("*/", i) + 1
        elif c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                break
        i += 1
    line = text.count("\n", 0, m.start()) + 1
    return f'#line {line} "{fname}"\n' + text[m.start():i + 1] + "\n"


def extract_io(src_dir):
    parts = []
    for fname, name in HOST_FUNCTIONS:
        with open(os.path.join(src_dir, fname), encoding="latin-1") as f:
            parts.append(_host_function(f.read(), name, fname))
    return "".join(parts)


def build(src_dir=DEFAULT_SRC, quiet=False, keep_source=False):
    if not os.path.exists(os.path.join(src_dir, "spray_k.cu")):
        raise FileNotFoundError(f"reference source not found under {src_dir}")
    os.makedirs(OUT_DIR, exist_ok=True)
    body = extract(src_dir)
    cpp = os.path.join(OUT_DIR, "spray_k_host.cpp")
    with open(cpp, "w") as f:
        f.write('// generated by oracle/make_refhost.py from the reference spray_k.cu; not committed\n')
        f.write('#include "shim.h"\n#include "utility.h"\n#include "globals.inc"\n')
        f.write('#include "tables.h"\n' if os.path.exists(os.path.join(src_dir, "tables.h")) else "")
        f.write(body)
        f.write('#include "stages.inc"\n')
    io = os.path.join(OUT_DIR, "spray_io_host.cpp")
    with open(io, "w") as f:
        f.write('// generated by oracle/make_refhost.py from the reference spray.cu / spray.cpp; not committed\n')
        f.write('#include "cspray_io.h"\n')
        f.write(extract_io(src_dir))
        f.write('#include "io.inc"\n')
    inc = os.path.join(HERE, "refhost")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-w",
           "-I", inc, "-I", src_dir, "-I", os.path.join(HERE, "..", "include"), "-I", "/usr/local/cuda/include",
           cpp, io, "-o", LIB, "-lz"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("refhost build failed:\n" + r.stderr[-6000:])
    if not keep_source:
        os.remove(cpp)
        os.remove(io)
    if not quiet:
        print(LIB)
    return LIB


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    build(args[0] if args else DEFAULT_SRC, keep_source="--keep-source" in sys.argv)
