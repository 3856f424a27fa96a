"""Helpers for GPU-vs-oracle parity: the same scene on both sides, state transplant
(GPU state copied into the oracle so one stage can be checked in isolation), and
field comparison."""
import numpy as np

CELL_FIELDS = ["press", "div", "lsfluid", "lsair", "lsmerge", "phifluid", "phiair", "phisolid",
               "phigrax", "phigray", "phigraz", "phigrax_air", "phigray_air", "phigraz_air",
               "surftension", "tp", "tp_save", "tp_old", "fixedheat", "mark"]
FACE_FIELDS = ["waterux", "wateruy", "wateruz", "waterux_old", "wateruy_old", "wateruz_old",
               "airux", "airuy", "airuz", "airux_old", "airuy_old", "airuz_old",
               "solidux", "soliduy", "soliduz"]
PART_FIELDS = ["pos", "vel", "flag", "mass", "temp", "lheat", "solubility", "gascontain"]


def bubblesim_stages(p, frame):
    """The stage sequence of one bubblesim step (spray.cpp:979-1233) for params p."""
    s = [("hashAndSortParticles",), ("addexternalforce",), ("computeLevelset", 0.0), ("sweepLSAndMardGrid",),
         ("markSoloAirParticle",), ("computesurfacetension",)]
    if p.scene in (6, 8):   # MELTING, FREEZING
        s.append(("markgrid_bubble",))
    s += [("mapvelp2g_bubble",), ("enforceDragForce",), ("sweepPhi", 1), ("sweepU", 1), ("sweepPhi", 0), ("sweepU", 0),
          ("setWaterBoundaryU", 1), ("setWaterBoundaryU", 0), ("project_CG_bubble",), ("sweepU", 1), ("sweepU", 0),
          ("setWaterBoundaryU", 1), ("setWaterBoundaryU", 0), ("mapvelg2p_bubble",), ("solidmotion",),
          ("updateSoloAirParticle",), ("hashAndSortParticles",), ("CollisionSolid",)]
    if p.b_correct_position:
        s += [("hashAndSortParticles",), ("correctpos",), ("hashAndSortParticles",), ("computeLevelset", 0.15),
              ("sweepLSAndMardGrid",), ("correctpos_bubble",)]
    else:
        s += [("hashAndSortParticles",), ("computeLevelset", 0.15), ("sweepLSAndMardGrid",)]
    s.append(("hashAndSortParticles",))
    if p.b_heat_trans:
        s.append(("updateTemperature",))
    if p.b_gen_gas and frame % 2 == 0:
        s.append(("GenerateGasParticle",))
    s += [("hashAndSortParticles",), ("deleteAirFluidParticle",), ("hashAndSortParticles",)]
    if p.b_melt:
        s.append(("MeltSolid",))
    if p.b_freeze:
        s.append(("Freezing",))
    return s


def grid_params(mp, config, nx, ny=None, nz=None):
    """The parameters of configuration `config` at cell size 1/nx on an
    nx x ny x nz grid (the configuration's shapes clipped to that box); a
    non-cubic grid keeps the cubic grid's cell size and particle capacity."""
    p = mp.scene_params(config, nx)
    p.ny = ny or nx
    p.nz = nz or nx
    return p


def make_pair(mp, oracle_mod, config, n, seed, params=None, **overrides):
    """A GPU Sim and an oracle with identical parameters, particles and tables."""
    p = params if params is not None else mp.scene_params(config, n)
    for k, v in overrides.items():
        setattr(p, k, v)
    sim = mp.Sim.from_config(config, n, seed, params=p)
    orc = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    parts = mp.scene_particles(p, config, seed)
    orc.upload_particles(**parts)
    rf, seeds = mp.scene_tables(p, config, seed)
    orc.set_tables(rf, seeds)
    orc.set_field("fixedheat", mp.scene_fixed_heat(p, config))
    orc.set_state(sim.state())
    return sim, orc


def transplant(sim, orc, with_cells=True):
    """Copies the complete GPU state into the oracle."""
    for f in CELL_FIELDS + FACE_FIELDS:
        orc.set_field(f, sim.get_field(f))
    parts = sim.download_particles()
    st = sim.state()
    orc.set_state(st)
    orc.upload_particles(**parts)
    if with_cells:
        orc.set_field("cellstart", sim.get_field("cellstart"))
        orc.set_field("cellend", sim.get_field("cellend"))


def snapshot(obj):
    out = {f: obj.get_field(f) for f in CELL_FIELDS + FACE_FIELDS}
    out.update(obj.download_particles())
    return out


def rel_err(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    if a.shape != b.shape:
        return np.inf
    if a.size == 0:
        return 0.0
    fin = np.isfinite(b) & np.isfinite(a)
    if not np.array_equal(np.isfinite(a), np.isfinite(b)):
        return np.inf
    scale = max(np.abs(b[fin]).max() if fin.any() else 0.0, 1e-30)
    return float(np.abs(a[fin] - b[fin]).max() / scale) if fin.any() else 0.0


def rel_l2(a, b):
    """||a - b||_2 / ||b||_2 over the entries finite on both sides (0 when b is 0)."""
    a = np.asarray(a, np.float64).ravel(); b = np.asarray(b, np.float64).ravel()
    if a.shape != b.shape:
        return np.inf
    fin = np.isfinite(a) & np.isfinite(b)
    den = np.linalg.norm(b[fin])
    return float(np.linalg.norm(a[fin] - b[fin]) / den) if den > 0 else float(np.linalg.norm(a[fin]))


DRIFT_GRID = ["press", "lsmerge", "tp", "waterux", "wateruy", "wateruz", "airux", "airuy", "airuz"]


def drift(gpu, ref):
    """Drift of the GPU run from the oracle's after many steps: relative L2 error
    of the grid fields, the fraction of cells whose mark differs, the relative
    difference of the particle counts, and, while the counts agree, the relative
    L2 error of the particle positions, velocities and temperatures."""
    out = {f: rel_l2(gpu[f], ref[f]) for f in DRIFT_GRID}
    out["mark"] = float((gpu["mark"] != ref["mark"]).mean())
    ng, nr = len(gpu["flag"]), len(ref["flag"])
    out["count"] = abs(ng - nr) / max(nr, 1)
    for f in ("pos", "vel", "temp"):
        out[f] = rel_l2(gpu[f], ref[f]) if ng == nr else np.inf
    ag, ar = aggregates(gpu), aggregates(ref)
    for k in ar:
        out["agg_" + k] = abs(ag[k] - ar[k]) / max(abs(ar[k]), 1e-30)
    return out


def aggregates(snap):
    """Whole-domain quantities of a state: particle kinetic energy, the mean
    particle temperature, the centroid height of the gas particles (AIR and
    AIRSOLO) and of the liquid, and the cell counts of liquid and gas."""
    f = snap["flag"]
    v = snap["vel"].astype(np.float64); m = snap["mass"].astype(np.float64)
    z = snap["pos"][:, 2].astype(np.float64)
    gas = (f == 1) | (f == 4)
    liq = f == 0
    return {"kinetic": float((m * (v * v).sum(1)).sum()) + 1e-30,
            "temp": float(snap["temp"].astype(np.float64).mean()) if len(f) else 0.0,
            "gas_z": float(z[gas].mean()) if gas.any() else 0.0,
            "liquid_z": float(z[liq].mean()) if liq.any() else 0.0,
            "fluid_cells": float((snap["mark"] == 0).sum()),
            "gas_cells": float((snap["mark"] == 1).sum())}


def check_one_step(sim, orc, config, rtol=1e-5):
    """One whole bubblesim step on both sides from identical inputs: frame and
    particle count equal, marks and flags equal except for a handful of
    threshold flips, float fields within rtol (max-norm relative, per field)."""
    sim.bubblesim()
    orc.bubblesim()
    gs, rs = sim.state(), orc.state()
    assert gs.frame == rs.frame == 1
    assert gs.par_num_now == rs.par_num_now
    g, r = snapshot(sim), snapshot(orc)
    mism = (g["mark"] != r["mark"]).mean()
    assert mism <= 1e-3, f"marks differ in {mism:.2e} of cells"
    assert (g["flag"] != r["flag"]).mean() <= 1e-3
    for f in ["press", "lsmerge", "lsfluid", "lsair", "tp", "waterux", "wateruy", "wateruz", "airux", "airuy", "airuz",
              "pos", "vel", "temp"]:
        e = rel_err(g[f], r[f])
        assert e <= rtol, f"config {config} {f}: rel err {e:.3e}"
    return gs, rs


def compare(gpu, ref, exact=True, rtol=1e-5, skip=()):
    """Returns a list of (field, problem) for fields that differ."""
    bad = []
    for k, v in ref.items():
        if k in skip:
            continue
        g = gpu[k]
        if np.asarray(g).shape != np.asarray(v).shape:
            bad.append((k, f"shape {np.asarray(g).shape} vs {np.asarray(v).shape}"))
            continue
        if exact or v.dtype.kind in "iu":
            same = np.array_equal(g, v, equal_nan=v.dtype.kind == "f")
            if not same:
                if v.dtype.kind == "f":
                    d = np.abs(g.astype(np.float64) - v.astype(np.float64))
                    bad.append((k, f"not bit-exact: {int((g != v).sum())} differ, max |d| {np.nanmax(d):.3e}, "
                                   f"rel {rel_err(g, v):.3e}"))
                else:
                    bad.append((k, f"not equal: {int((g != v).sum())} of {v.size} differ"))
        else:
            e = rel_err(g, v)
            if e > rtol:
                bad.append((k, f"rel err {e:.3e} > {rtol}"))
    return bad


def state_digest(obj):
    """SHA-256 over the whole state: every field and particle attribute, the
    cell starts, and the cell ends of the occupied cells (the reference leaves
    the others stale)."""
    import hashlib
    h = hashlib.sha256()
    snap = snapshot(obj)
    for k in sorted(snap):
        h.update(k.encode())
        h.update(np.ascontiguousarray(snap[k]).tobytes())
    cs, ce = obj.get_field("cellstart"), obj.get_field("cellend")
    h.update(cs.tobytes())
    h.update(np.where(cs != 0xFFFFFFFF, ce, 0).astype(np.uint32).tobytes())
    return h.hexdigest()


def staged_digests(obj, p, frames, mc=True):
    """Runs `frames` bubblesim frames stage by stage on obj (the oracle or the
    reference's kernels), and the three surfaces' extraction after the last;
    returns [(frame, stage, digest)] after every stage, then the surfaces'
    density digests and counts."""
    import hashlib
    out = []
    for frame in range(frames):
        st = obj.state()
        st.frame = frame
        obj.set_state(st)
        for stage in bubblesim_stages(p, frame):
            getattr(obj, stage[0])(*stage[1:])
            out.append([frame, " ".join(str(x) for x in stage), state_digest(obj)])
    if mc:
        obj.preMC()
        out.append([frames, "preMC", state_digest(obj)])
        for surf in (0, 1, 2):
            obj.runMC(surf)
            dens = obj.mc_field()[0]
            verts, _, idx = obj.mc_mesh(surf)
            out.append([frames, f"runMC {surf}", hashlib.sha256(dens.tobytes()).hexdigest(),
                        int(len(verts)), int(len(idx))])
    return out
