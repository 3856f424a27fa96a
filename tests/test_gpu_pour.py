"""Pouring (mp_pour / mp_step), the frame-scripted parameter switches of
bubblesim, and the interaction scenes' solid surface that moves with the
rigid solid motion (runMC_interaction, computeSolidVertex_k)."""
import numpy as np
import pytest

from oracle import pour_ref

pytestmark = pytest.mark.gpu


def _append_ok(mp, sim, ppos, pvel, rf, np0, flag):
    p = sim.params
    parts = sim.download_particles()
    n = len(ppos)
    assert len(parts["pos"]) == np0 + n
    rpos, rvel = pour_ref.pour(ppos, pvel, rf, p.pos_rand_param, p.vel_rand_param, p.samplespace)
    t = slice(np0, np0 + n)
    assert np.array_equal(parts["pos"][t].view(np.uint32), rpos.view(np.uint32))
    assert np.array_equal(parts["vel"][t].view(np.uint32), rvel.view(np.uint32))
    assert np.all(parts["flag"][t] == flag)
    assert np.all(parts["mass"][t] == np.float32(p.m0))
    assert np.all(parts["temp"][t] == np.float32(p.default_liquid_T))
    assert np.all(parts["lheat"][t] == np.float32(p.liquid_heat_th))
    assert np.all(parts["gascontain"][t] == 0) and np.all(parts["solubility"][t] == 0)
    return parts


def _at_frame(sim, f):
    st = sim.state(); st.frame = f; sim.set_state(st)


def test_pouring_appends_the_emitter_every_fourth_frame(mp):
    seed = 7401
    sim = mp.Sim.from_config(1, 32, seed)
    p = sim.params
    rf, _ = mp.scene_tables(p, 1, seed)
    ppos, pvel = mp.scene_pour(mp.POUR_FREEZING, p.samplespace, 0.035, (0.5, 0.5, 0.5), (0.0, 0.0, -0.5))
    sim.set_pour(ppos, pvel)
    before = sim.download_particles()
    np0 = len(before["pos"])
    sim.pouring()                                   # frame 0
    parts = _append_ok(mp, sim, ppos, pvel, rf, np0, mp.TYPEFLUID)
    for k in before:
        assert np.array_equal(parts[k][:np0].view(np.uint8), before[k].view(np.uint8)), k
    for f in (1, 2, 3):
        _at_frame(sim, f)
        sim.pouring()
        assert sim.state().par_num_now == np0 + len(ppos)
    _at_frame(sim, 4)
    sim.pouring()
    assert sim.state().par_num_now == np0 + 2 * len(ppos)
    # an emitter that no longer fits under par_num_max pours nothing
    room = p.par_num_max - sim.state().par_num_now
    big = np.tile(ppos, (room // len(ppos) + 1, 1))
    sim.set_pour(big, np.zeros_like(big))
    _at_frame(sim, 8)
    npb = sim.state().par_num_now
    sim.pouring()
    assert sim.state().par_num_now == npb
    sim.close()


def test_interaction_scene_pours_gas_from_begin_frame(mp):
    seed = 7402
    sim = mp.Sim.from_config(1, 32, seed, scene=mp.SCENE_INTERACTION, begin_frame=2)
    p = sim.params
    rf, _ = mp.scene_tables(p, 1, seed)
    ppos, pvel = mp.scene_pour(mp.POUR_INTERACTION2, p.samplespace, 0.05, (0.27, 0.25, 0.05), (0.0, 0.0, 1.1),
                               center2=(0.45, 0.25, 0.05))
    sim.set_pour(ppos, pvel)
    np0 = sim.state().par_num_now
    sim.pouring()                                   # frame 0 < begin_frame: water, 0 % 4 == 0
    _append_ok(mp, sim, ppos, pvel, rf, np0, mp.TYPEFLUID)
    np1 = sim.state().par_num_now
    _at_frame(sim, 4)                               # gas from frame 2 on, every 6th frame
    sim.pouring()
    assert sim.state().par_num_now == np1
    _at_frame(sim, 6)
    sim.pouring()
    _append_ok(mp, sim, ppos, pvel, rf, np1, mp.TYPEAIRSOLO)
    sim.close()


def test_step_pours_first(mp):
    a = mp.Sim.from_config(1, 32, 7403)
    b = mp.Sim.from_config(1, 32, 7403)
    p = a.params
    ppos, pvel = mp.scene_pour(mp.POUR_FREEZING, p.samplespace, 0.035, (0.5, 0.5, 0.7), (0.0, 0.0, -0.5))
    a.set_pour(ppos, pvel)
    a.bubblesim(); b.bubblesim()
    # the twin without an emitter: the poured water (above the liquid, far from
    # the bubble) is the only difference in the particle count
    assert a.state().par_num_now == b.state().par_num_now + len(ppos)
    assert (a.download_particles()["pos"][:, 2] > 0.65).sum() >= len(ppos)
    a.close(); b.close()


@pytest.mark.parametrize("scene,frame,changes", [
    ("SCENE_MELTANDBOIL", 300, {"b_fix_solid": 0}),
    ("SCENE_MELTANDBOIL", 400, {"b_gen_gas": 1}),
    ("SCENE_MELTANDBOIL", 700, {"b_gen_gas": 1, "drag_param_grid": 0.03, "vapor_gen_rate": 0.005}),
    ("SCENE_MELTANDBOIL_HIGHRES", 400, {"b_add_heat_bottom": 0}),
    ("SCENE_ALL", 0, {"b_fix_solid": 0, "b_add_heat_bottom": 0, "b_gen_gas": 0, "b_melt": 0, "b_freeze": 1}),
    ("SCENE_ALL", 520, {"b_add_heat_bottom": 1, "b_melt": 1}),
    ("SCENE_INTERACTION", 5, {"b_fix_solid": 0}),
])
def test_frame_scripted_switches(mp, scene, frame, changes):
    start = {"b_fix_solid": 1, "b_gen_gas": 0, "b_add_heat_bottom": 1, "b_melt": 0, "b_freeze": 0}
    if scene == "SCENE_ALL" and frame == 520:
        start.update(b_add_heat_bottom=0, b_melt=0)
    sim = mp.Sim.from_config(3, 32, 7404, scene=getattr(mp, scene), begin_frame=5, **start)
    if frame > 0:
        _at_frame(sim, frame - 1)
        sim.bubblesim()                             # frame - 1: nothing switches
        for k, v in start.items():
            assert getattr(sim.params, k) == v, (k, "switched a frame early")
    sim.bubblesim()                                 # frame: the switches
    for k, v in changes.items():
        assert getattr(sim.params, k) == pytest.approx(v), k
    sim.close()


def _rigid_fit(a, b):
    ca, cb = a.mean(0), b.mean(0)
    u, _, vt = np.linalg.svd((a - ca).T @ (b - cb))
    d = np.sign(np.linalg.det(vt.T @ u.T))
    r = vt.T @ np.diag([1, 1, d]) @ u.T
    return lambda x: (x - ca) @ r.T + cb


def _normals(v, ix):
    n = np.zeros_like(v)
    tri = ix.reshape(-1, 3)
    for t in tri:
        p1, p2, p3 = v[t[0]], v[t[1]], v[t[2]]
        c = np.cross(p2 - p1, p3 - p1)
        for k in t:
            n[k] += c
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    return np.where(ln > 0, n / np.where(ln > 0, ln, 1), 0)


@pytest.mark.parametrize("run_mc_solid", [0, 1])
def test_interaction_solid_surface_follows_the_solid(mp, run_mc_solid):
    sim = mp.Sim.from_config(3, 32, 7405, scene=mp.SCENE_MELTANDBOIL, b_run_mc_solid=run_mc_solid, b_fix_solid=0,
                             b_melt=0, b_freeze=0, mc_every=2)
    sim.bubblesim()                                 # frame 0 extracts the solid surface
    v0, n0, i0 = sim.mc_mesh(mp.MC_SOLID)
    assert len(v0) > 0
    parts0 = sim.download_particles()
    sim.solidmotion()                               # frame 1
    parts1 = sim.download_particles()
    v1 = sim.mc_mesh(mp.MC_SOLID)[0]
    if run_mc_solid:
        assert np.array_equal(v1, v0)               # re-extracted at MC frames instead
    else:
        s = parts0["flag"] == mp.TYPESOLID
        a, b = parts0["pos"][s].astype(np.float64), parts1["pos"][s].astype(np.float64)
        assert np.abs(b - a).max() > 1e-7           # the solid did move
        fit = _rigid_fit(a, b)
        assert np.abs(fit(v0.astype(np.float64)) - v1).max() < 2e-5
    _at_frame(sim, 1)
    sim.bubblesim()                                 # frame 1: no extraction
    sim.bubblesim()                                 # frame 2: extraction frame
    v2, n2, i2 = sim.mc_mesh(mp.MC_SOLID)
    if not run_mc_solid:
        assert np.array_equal(i2, i0) and len(v2) == len(v0)
        assert not np.array_equal(v2, v0)
        err = np.abs(n2 - _normals(v2.astype(np.float64), i2)).max(axis=1)
        assert (err > 1e-4).mean() < 1e-3, err.max()
    sim.close()


def test_step_with_pouring_switches_and_kept_solid_surface_matches_oracle(mp, oracle_mod):
    """Whole steps of a melt-and-boil scene with an emitter and bRunMCSolid off,
    GPU against the oracle: the same particles poured, the same switches, the
    solid surface of frame 0 moved and re-normalled, fields within the bounds
    of the bubblesim step test."""
    from parity_util import make_pair, rel_err, snapshot
    sim, orc = make_pair(mp, oracle_mod, 3, 32, 7406, scene=mp.SCENE_MELTANDBOIL, b_run_mc_solid=0, b_fix_solid=0,
                         b_melt=0, b_freeze=0, mc_every=2)
    p = sim.params
    ppos, pvel = mp.scene_pour(mp.POUR_FREEZING, p.samplespace, 0.035, (0.6, 0.45, 0.75), (0.0, 0.0, -0.5))
    sim.set_pour(ppos, pvel); orc.set_pour(ppos, pvel)
    i0 = None
    for step in range(3):
        sim.bubblesim(); orc.bubblesim()
        gs, rs = sim.state(), orc.state()
        assert gs.frame == rs.frame == step + 1 and gs.par_num_now == rs.par_num_now
        g, r = snapshot(sim), snapshot(orc)
        for f in ["press", "lsmerge", "waterux", "wateruy", "wateruz", "pos", "vel"]:
            e = rel_err(g[f], r[f])
            assert e <= 1e-5 * (step + 1), f"step {step} {f}: rel err {e:.3e}"
        gv, gn, gi = sim.mc_mesh(mp.MC_SOLID)
        rv, rn, ri = orc.mc_mesh(mp.MC_SOLID)
        assert len(gv) > 0 and len(rv) > 0
        # the frame-0 extraction sees fields 1e-5 apart, so its case indices can
        # flip at a threshold; where the surfaces agree, so do their motions
        if np.array_equal(gi, ri):
            assert rel_err(gv, rv) <= 1e-5 * (step + 1)
        if i0 is None:
            i0, r0 = gi, ri
        assert np.array_equal(gi, i0) and np.array_equal(ri, r0)   # the frame-0 surfaces, never re-extracted
    # the emitter poured at frame 0
    assert sim.state().par_num_now >= len(ppos)
    sim.close()
