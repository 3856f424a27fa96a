"""The water-only mode (cspray::watersim, spray.cpp:741-797) on the GPU
against the oracle: every stage from a transplanted state (bit for bit except
the CG, compared at 1e-5 relative as the bubble projection is), and whole steps
with the bounds of the bubblesim step test."""
import numpy as np
import pytest

from parity_util import compare, make_pair, rel_err, snapshot, transplant

pytestmark = pytest.mark.gpu

TF = 0
STAGES = [("hashAndSortParticles",), ("sweepPhi", TF), ("computeLevelset", 0.0), ("sweepLSAndMardGrid",),
          ("flipMark_sphere",), ("computesurfacetension",), ("mapvelp2g",), ("sweepU", TF), ("setWaterBoundaryU", TF),
          ("project_CG",), ("sweepU", TF), ("setWaterBoundaryU", TF), ("mapvelg2p",), ("wateradvect",),
          ("hashAndSortParticles",), ("correctpos",)]
CONFIG, N, SEED = 4, 32, 2017_400   # the dam break: FLUID particles only


def _run(obj, st):
    return getattr(obj, st[0])(*st[1:])


@pytest.mark.parametrize("k", range(len(STAGES)))
def test_water_stage(mp, oracle_mod, k):
    sim, orc = make_pair(mp, oracle_mod, CONFIG, N, SEED, b_correct_position=1)
    for st in STAGES[:k]:
        _run(sim, st)
    transplant(sim, orc)
    st = STAGES[k]
    _run(sim, st); _run(orc, st)
    g, r = snapshot(sim), snapshot(orc)
    bad = compare(g, r, exact=st[0] != "project_CG", rtol=1e-5)
    assert not bad, f"stage {k} {st}: {bad}"
    if st[0] == "flipMark_sphere":
        assert not (sim.get_field("mark") == mp.TYPEVACUUM).any()
    if st[0] == "project_CG":
        assert sim.state().last_cg_iters > 0
    sim.close()


def test_water_steps(mp, oracle_mod):
    sim, orc = make_pair(mp, oracle_mod, CONFIG, N, SEED + 1, b_correct_position=1, b_run_mc=1)
    for step in range(2):
        sim.watersim(); orc.watersim()
        gs, rs = sim.state(), orc.state()
        assert gs.frame == rs.frame == step + 1 and gs.par_num_now == rs.par_num_now
        g, r = snapshot(sim), snapshot(orc)
        assert (g["mark"] != r["mark"]).mean() <= 1e-3
        for f in ["press", "lsfluid", "waterux", "wateruy", "wateruz", "pos", "vel"]:
            e = rel_err(g[f], r[f])
            assert e <= 1e-5 * (step + 1), f"step {step} {f}: rel err {e:.3e}"
    # the fluid surface is extracted every step (counts within the threshold
    # flips of a 1e-5 field difference)
    gv, rv = sim.state().mc_verts[mp.MC_FLUID], orc.state().mc_verts[mp.MC_FLUID]
    assert gv > 0 and abs(gv - rv) <= max(10, rv // 1000)
    sim.close()
