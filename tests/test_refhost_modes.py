"""The oracle against the reference's own kernels (oracle/make_refhost.py,
oracle/refhost/stages.inc), beyond bubblesim's stage list: the rigid solid
motion, the water-only mode (cspray::watersim, spray.cpp:741-797), the
heat-only mode (initheat_grid, heatsim: spray.cu:1949-1987) and the pouring
emitters (pouring / pouringgas, spray.cu:3012-3043).  Every field and particle
attribute must agree bit for bit.  Skipped without the reference source tree."""
import numpy as np
import pytest

from parity_util import bubblesim_stages, compare, snapshot
from test_refhost_stages import SRC, copy_state, reference_mode

pytestmark = pytest.mark.skipif(not __import__("os").path.exists(SRC + "/spray_k.cu"),
                                reason="reference source tree not present")
N = 16
TF = 0


def _pair(mp, oracle_mod, refhost, config, seed, keep=None, **overrides):
    p, parts, rf, seeds = reference_mode(mp, config, N, seed)
    if keep is not None:        # a subset of the configuration's particles
        idx = keep(parts)
        parts = {k: (None if v is None else np.asarray(v)[idx]) for k, v in parts.items()}
    for k, v in overrides.items():
        setattr(p, k, v)
    orc = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    orc.upload_particles(**parts)
    orc.set_tables(rf, seeds)
    st = orc.state()
    st.n_real_solpoint = int((np.asarray(parts["flag"]) == mp.TYPESOLID).sum())
    orc.set_state(st)
    ref = refhost.RefHost(p, mp.FIELD_ID, mp.MPState)
    ref.set_tables(rf, seeds)
    return p, orc, ref, rf


def _stage(orc, ref, st):
    copy_state(orc, ref)
    ref.run(st[0], float(st[1]) if len(st) > 1 else 0.0)
    getattr(orc, st[0])(*st[1:])
    return compare(snapshot(ref), snapshot(orc), exact=True)


def test_rigid_solid_motion(mp, oracle_mod, refhost):
    """solidmotion with a free solid (the melting configuration), and
    solidmotion_fixed: the reference's kernels with the FP64 sums the oracle
    defines for accumulate_GPU_f3."""
    for fix in (0, 1):
        p, orc, ref, _ = _pair(mp, oracle_mod, refhost, 3, 2017_730 + fix, b_fix_solid=fix)
        assert orc.state().n_real_solpoint > 0
        for st in bubblesim_stages(p, 0):
            if st[0] == "solidmotion":
                before = orc.download_particles()["pos"]
                assert not _stage(orc, ref, st)
                moved = np.abs(orc.download_particles()["pos"] - before).max()
                assert (moved > 0) == (not fix)
                break
            getattr(orc, st[0])(*st[1:])


WATER = [("hashAndSortParticles",), ("sweepPhi", TF), ("computeLevelset", 0.0), ("sweepLSAndMardGrid",),
         ("flipMark_sphere",), ("computesurfacetension",), ("mapvelp2g",), ("sweepU", TF), ("setWaterBoundaryU", TF),
         ("project_CG",), ("sweepU", TF), ("setWaterBoundaryU", TF), ("mapvelg2p",), ("wateradvect",),
         ("hashAndSortParticles",), ("correctpos",)]


def test_water_mode_stages(mp, oracle_mod, refhost):
    """watersim's stages (spray.cpp:741-797) on the dam break, two frames."""
    p, orc, ref, _ = _pair(mp, oracle_mod, refhost, 4, 2017_740, b_correct_position=1)
    for frame in range(2):
        for st in WATER:
            bad = _stage(orc, ref, st)
            assert not bad, (frame, st, bad)
            if st[0] == "project_CG":
                assert ref.iters > 0 and ref.iters == orc.state().last_cg_iters
        s = orc.state()
        s.frame += 1
        orc.set_state(s)


@pytest.mark.parametrize("case", ["empty", "one", "sparse"])
def test_water_mode_stages_on_edge_inputs(mp, oracle_mod, refhost, case):
    """watersim's stages on the dam break with no particles, one particle
    (the block's first) and one particle in forty: bit for bit."""
    keep = {"empty": lambda q: np.zeros(0, np.int64), "one": lambda q: [0],
            "sparse": lambda q: np.arange(len(q["flag"]))[::40]}[case]
    p, orc, ref, _ = _pair(mp, oracle_mod, refhost, 4, 2017_740, keep=keep, b_correct_position=1)
    for frame in range(2):
        for st in WATER:
            bad = _stage(orc, ref, st)
            assert not bad, (frame, st, bad)
        s = orc.state()
        s.frame += 1
        orc.set_state(s)
    assert orc.state().par_num_now == {"empty": 0, "one": 1}.get(case, orc.state().par_num_now)


@pytest.mark.parametrize("extend", [1, 0])
def test_heat_only_mode(mp, oracle_mod, refhost, extend):
    """initheat_grid's two-disc scene (spray_k.cu:5603-5621) and heatsim steps,
    with the boundary cells' temperature extended from the interior or not."""
    p, orc, ref, _ = _pair(mp, oracle_mod, refhost, 1, 2017_750, b_extend_heat_to_boundary=extend)
    assert not _stage(orc, ref, ("initheat_grid",))
    for _ in range(3):
        assert not _stage(orc, ref, ("heatsim",))
        assert ref.iters > 0 and ref.iters == orc.state().last_heat_cg_iters


@pytest.mark.parametrize("scene, frames", [("MELTINGPOUR", (0, 1, 4)), ("INTERACTION", (0, 3, 6))])
def test_pouring(mp, oracle_mod, refhost, scene, frames):
    """pouring's liquid every fourth frame, and pouringgas's AIRSOLO every sixth
    frame from m_beginFrame in the interaction scenes."""
    p, orc, ref, _ = _pair(mp, oracle_mod, refhost, 1, 2017_760, scene=getattr(mp, "SCENE_" + scene), begin_frame=2)
    ppos, pvel = mp.scene_pour(mp.POUR_FREEZING, p.samplespace, 0.035, (0.5, 0.5, 0.6), (0.0, 0.0, -0.5))
    orc.set_pour(ppos, pvel)
    ref.set_pour(ppos, pvel)
    for f in frames:
        s = orc.state()
        s.frame = f
        orc.set_state(s)
        n0 = orc.state().par_num_now
        assert not _stage(orc, ref, ("pouring",))
        poured = orc.state().par_num_now - n0
        every = 6 if (scene == "INTERACTION" and f >= 2) else 4
        assert poured == (len(ppos) if f % every == 0 else 0)


@pytest.mark.parametrize("config", [2, 3])
def test_particle_heat_initialisation(mp, oracle_mod, refhost, config):
    """initTemperature + initSolubility (spray.cu:1989-1999): initHeatParticle
    and initsolubility_k, and the SOLID count the step starts from."""
    p, orc, ref, _ = _pair(mp, oracle_mod, refhost, config, 2017_790 + config)
    assert not _stage(orc, ref, ("initHeatAndSolubility",))
    assert ref.n_real_solid == orc.state().n_real_solpoint
    assert (orc.download_particles()["solubility"] > 0).any()


def test_kept_solid_surface_moves_with_the_solid(mp, oracle_mod, refhost):
    """runMC_interaction keeps the solid surface extracted at frame 0 when
    bRunMCSolid is off, and solidmotion moves it with computeSolidVertex_k
    (spray.cu:2770-2772, spray_k.cu:5254-5263): the moved vertices equal the
    reference's, bit for bit, with the particles."""
    p, orc, ref, _ = _pair(mp, oracle_mod, refhost, 3, 2017_795, scene=mp.SCENE_MELTANDBOIL, b_fix_solid=0,
                           b_run_mc_solid=0, b_run_mc=1)
    for st in bubblesim_stages(p, 0):
        getattr(orc, st[0])(*st[1:])
    orc.preMC()
    orc.runMC(mp.MC_SOLID)                         # the surface kept from frame 0
    kept = orc.mc_mesh(mp.MC_SOLID)[0]
    assert len(kept) > 0
    s = orc.state()
    s.frame = 1
    orc.set_state(s)
    for st in bubblesim_stages(p, 1):
        if st[0] == "solidmotion":
            ref.solid_verts = kept.copy()
            assert not _stage(orc, ref, st)
            moved = orc.mc_mesh(mp.MC_SOLID)[0]
            assert np.array_equal(ref.solid_verts, moved)
            assert np.abs(moved - kept).max() > 0
            break
        getattr(orc, st[0])(*st[1:])


def test_fp64_solid_sums_against_the_reference_float_reductions(mp, oracle_mod, refhost):
    """solidmotion's sums in FP64 (the oracle's definition) against the
    reference's accumulate_GPU_f3 (float3 tree sums per block,
    accumulate_GPU_k spray_k.cu:5167-5186, then a float sum on the host): the
    moved particles within 1e-6 relative (measured: positions equal,
    velocities within 1.4e-7)."""
    from parity_util import rel_err
    p, orc, ref, _ = _pair(mp, oracle_mod, refhost, 3, 2017_796, b_fix_solid=0)
    for st in bubblesim_stages(p, 0):
        if st[0] == "solidmotion":
            copy_state(orc, ref)
            ref.run("solidmotion_float")
            orc.solidmotion()
            a, b = snapshot(ref), snapshot(orc)
            assert rel_err(a["pos"], b["pos"]) <= 1e-6 and rel_err(a["vel"], b["vel"]) <= 1e-5
            return
        getattr(orc, st[0])(*st[1:])
    pytest.fail("no solid motion in the step")
