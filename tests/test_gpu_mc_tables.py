"""mp_set_mc_tables: a context extracts its surfaces with the case tables it
is given.  A variant of the generated tables (each triangle's vertices
rotated, the triangles of each case in reverse order) on the GPU against the
oracle with the same tables, bit for bit; malformed tables are refused.  With
the reference's own tables.h the oracle reproduces the reference kernels'
index lists (tests/test_refhost_stages.py)."""
import numpy as np
import pytest

from parity_util import bubblesim_stages, make_pair, transplant

pytestmark = pytest.mark.gpu


def _variant(mp):
    nv, tri, _ = mp.mc_tables()
    tri = tri.reshape(256, 16).copy()
    for c in range(256):
        k = nv[c] // 3
        if k:
            ts = tri[c, :nv[c]].reshape(k, 3)
            tri[c, :nv[c]] = np.roll(ts, 1, axis=1)[::-1].reshape(-1)
    return nv.astype(np.int32), tri.reshape(-1).astype(np.int32)


def test_extraction_follows_the_given_tables(mp, oracle_mod):
    nv, tri = _variant(mp)
    sim, orc_default = make_pair(mp, oracle_mod, 1, 32, 2017_880)
    for st in bubblesim_stages(sim.params, 0):
        getattr(sim, st[0])(*st[1:])
    orc = oracle_mod.Oracle(sim.params, mp.FIELD_ID, mp.MPState, mc_tables=(nv, tri))
    transplant(sim, orc)
    transplant(sim, orc_default)
    sim.set_mc_tables(nv, tri)
    for o in (sim, orc, orc_default):
        o.preMC()
    differs = False
    for surf in (mp.MC_FLUID, mp.MC_GAS):
        for o in (sim, orc, orc_default):
            o.runMC(surf)
        gv, gn, gi = sim.mc_mesh(surf)
        rv, rn, ri = orc.mc_mesh(surf)
        assert np.array_equal(gi, ri) and np.array_equal(gv, rv) and np.array_equal(gn, rn), surf
        di = orc_default.mc_mesh(surf)[2]
        assert len(di) == len(gi)
        differs |= len(gi) > 0 and not np.array_equal(di, gi)
    assert differs
    sim.close()


def test_malformed_tables_are_refused(mp):
    sim = mp.Sim.from_config(1, 16, 2017_881)
    nv, tri = _variant(mp)
    bad = nv.copy(); bad[1] = 4
    with pytest.raises(mp.MPError) as e:
        sim.set_mc_tables(bad, tri)
    assert e.value.code == mp.MP_ERR_ARG
    bad_tri = tri.copy().reshape(256, 16); bad_tri[1, 0] = 5       # case 1 crosses edges 0, 3, 8 only
    with pytest.raises(mp.MPError) as e:
        sim.set_mc_tables(nv, bad_tri)
    assert e.value.code == mp.MP_ERR_ARG
    sim.set_mc_tables(nv, tri)
    sim.close()
