"""The heat-only mode (SIMULATION_HEATONLY, SCENE_HEATTRANSFER): the two-disc
initial grid bit for bit, and implicit heat steps against the oracle's
restatement of heatsim (spray.cu:1959-1987) within the CG parity tolerance."""
import numpy as np
import pytest

from parity_util import compare

pytestmark = pytest.mark.gpu


def _heat_params(mp, n):
    p = mp.default_params(n, n, n, 1)
    p.scene = mp.SCENE_HEATTRANSFER
    p.b_extend_heat_to_boundary = 1
    # spray.cpp:531-546
    p.heatalpha_fluid, p.heatalpha_air, p.heatalpha_solid, p.heatalpha_vacuum = 0.0001, 0.005, 0.015, 0.05
    return p


@pytest.mark.parametrize("n", [32, 64])
def test_heat_only_matches_oracle(mp, oracle_mod, n):
    p = _heat_params(mp, n)
    sim = mp.Sim(p)
    orc = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    sim.initheat_grid(); orc.initheat_grid()
    for f in ("tp", "mark"):
        assert np.array_equal(sim.get_field(f), orc.get_field(f)), f
    mark = sim.get_field("mark")
    assert set(np.unique(mark)) == {mp.TYPEFLUID, mp.TYPEAIR, mp.TYPEBOUNDARY, mp.TYPEVACUUM, mp.TYPESOLID}
    for step in range(3):
        sim.heatsim(); orc.heatsim()
        bad = compare({"tp": sim.get_field("tp")}, {"tp": orc.get_field("tp")}, exact=False, rtol=1e-5)
        assert not bad, (step, bad)
        assert sim.state().last_heat_cg_iters > 0
    assert sim.state().frame == 3
    # diffusion stays within the initial range (up to the CG tolerance) and
    # moves heat out of the hot disc
    tp = sim.get_field("tp")
    assert tp.min() > -0.01 and tp.max() < 100.0
    assert np.ptp(tp) > 0
    sim.close()
