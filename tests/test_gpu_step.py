"""Whole-step parity (bubblesim, spray.cpp:979-1233) and precision checks on the GPU.

After one full step from identical inputs the GPU and the oracle differ only by
the order of FP64 additions inside the CG dot products and by libm's expf/powf,
so float fields agree to 1e-5 relative (max-norm, per field) and discrete state
(particle count, flags, cell marks) agrees except for a handful of threshold
flips, bounded below. The mixed FP32/FP64 projection is compared with the
all-FP64 one at the 1e-5 relative pressure error the benchmark states.
"""
import numpy as np
import pytest

from parity_util import FACE_FIELDS, check_one_step, make_pair, rel_err, transplant

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("config", [1, 2, 3, 5])
def test_one_step(mp, oracle_mod, config):
    sim, orc = make_pair(mp, oracle_mod, config, 32, 4242 + config)
    gs, rs = check_one_step(sim, orc, config)
    # marching cubes ran on frame 0: counts from the same density field
    assert list(gs.mc_active_voxels) == list(rs.mc_active_voxels) or config in (2, 3)
    sim.close()


@pytest.mark.parametrize("config", [1, 5])
def test_mixed_vs_fp64_pressure(mp, oracle_mod, config):
    """Mixed FP32-vector / FP64-dot CG reaches <= 1e-5 relative pressure error
    against the all-FP64 projection on the same GPU state."""
    sim, _ = make_pair(mp, oracle_mod, config, 64, 99 + config)
    for st in ["hashAndSortParticles", "addexternalforce"]:
        getattr(sim, st)()
    sim.computeLevelset(0.0); sim.sweepLSAndMardGrid()
    sim.mapvelp2g_bubble()
    for ph in (1, 0):
        sim.sweepPhi(ph); sim.sweepU(ph)
    sim.setWaterBoundaryU(1); sim.setWaterBoundaryU(0)
    faces = {f: sim.get_field(f) for f in FACE_FIELDS}
    p = sim.params
    p.precision = mp.PREC_FP64; p.cg_tol = 1e-10; p.cg_max_iter = 5000
    sim.set_params(p)
    it64, _, rc = sim.project_CG_bubble()
    assert rc == 0
    ref = sim.get_field("press").astype(np.float64)
    for f, a in faces.items():
        sim.set_field(f, a)
    p.precision = mp.PREC_MIXED; p.cg_tol = 1e-6; p.cg_max_iter = 3000
    sim.set_params(p)
    it, _, rc = sim.project_CG_bubble()
    assert rc == 0
    x = sim.get_field("press").astype(np.float64)
    err = np.linalg.norm(x - ref) / np.linalg.norm(ref)
    assert err <= 1e-5, f"mixed vs fp64 relative pressure error {err:.3e} ({it} vs {it64} iterations)"
    sim.close()


def test_cg_matches_oracle_iterations(mp, oracle_mod):
    """Same system, same stopping rule: iteration counts agree within one."""
    sim, orc = make_pair(mp, oracle_mod, 1, 32, 7)
    for st in ["hashAndSortParticles", "addexternalforce"]:
        getattr(sim, st)()
    sim.computeLevelset(0.0); sim.sweepLSAndMardGrid(); sim.mapvelp2g_bubble()
    for ph in (1, 0):
        sim.sweepPhi(ph); sim.sweepU(ph)
    sim.setWaterBoundaryU(1); sim.setWaterBoundaryU(0)
    transplant(sim, orc)
    ig, rg, _ = sim.project_CG_bubble()
    io, ro, _ = orc.project_CG_bubble()
    assert abs(ig - io) <= 1, (ig, io)
    assert rel_err(sim.get_field("press"), orc.get_field("press")) <= 1e-5
    sim.close()


@pytest.mark.parametrize("config,shape", [(5, (64, 64, 64)), (1, (40, 24, 48))], ids=["64^3", "40x24x48"])
def test_cg_tma_matches_float4_passes(mp, oracle_mod, monkeypatch, config, shape):
    """The TMA plane-marching CG passes write the same vectors as the float4
    passes (their FP64 dot products add in another order): same iteration
    count within one, pressure within 1e-5, on a cube and on a grid whose
    tiles are partial in j and k."""
    from parity_util import grid_params
    out = {}
    for kernel in ("v4", "tma"):
        monkeypatch.setenv("MP_CG_KERNEL", kernel)
        p = grid_params(mp, config, *shape)
        sim = mp.Sim.from_config(config, shape[0], 77 + config, params=p)
        for st in ["hashAndSortParticles", "addexternalforce"]:
            getattr(sim, st)()
        sim.computeLevelset(0.0); sim.sweepLSAndMardGrid(); sim.mapvelp2g_bubble()
        for ph in (1, 0):
            sim.sweepPhi(ph); sim.sweepU(ph)
        sim.setWaterBoundaryU(1); sim.setWaterBoundaryU(0)
        it, res, rc = sim.project_CG_bubble()
        assert rc == 0
        out[kernel] = (it, sim.get_field("press"), sim.get_field("waterux"))
        sim.close()
    assert abs(out["v4"][0] - out["tma"][0]) <= 1, (out["v4"][0], out["tma"][0])
    assert rel_err(out["tma"][1], out["v4"][1]) <= 1e-5
    assert rel_err(out["tma"][2], out["v4"][2]) <= 1e-5


@pytest.mark.parametrize("config,n", [(2, 64), (3, 64)])
def test_mixed_form_fields_against_fp64_form(mp, oracle_mod, config, n):
    """One whole step from the same state in the mixed FP32/FP64 form (one CG
    pass, the reference's recurrence), in the mixed form with the periodic
    FP64 true-residual recompute (cg_refine_tol), in the all-FP64 form
    (projection and heat solve in FP64) at the same stop rule, and in FP64
    with the pressure solved to 1e-12 (the reference for all). Pressure,
    temperature and level set of both mixed forms are within 1e-5 (relative
    L2) of the reference. A velocity face's error is the CG's own error (a
    relative residual of 1e-6 leaves a smooth pressure error whose gradient
    is ~1e-5 of the splatted velocity); with FP32 storage of x the single
    pass adds ~eps*cond on top (1e-5..1e-3 of the splatted velocity in these
    liquids near rest), which the FP64 true residual removes: the refined
    mixed form's faces are as close to the reference as the FP64 form's
    (within 3x, plus 2e-6 of the splatted velocity), the single pass's
    within 2e-3."""
    from parity_util import rel_l2
    sim = mp.Sim.from_config(config, n, 9300 + config)
    blob = sim.checkpoint()
    p0 = sim.get_params()
    out = {}
    for name, prec, tol, refine in (("ref", mp.PREC_FP64, 1e-12, 0.0), ("fp64", mp.PREC_FP64, p0.cg_tol, 0.0),
                                    ("mixed", mp.PREC_MIXED, p0.cg_tol, 0.0),
                                    ("refined", mp.PREC_MIXED, p0.cg_tol, 1e-3)):
        sim.set_params(p0)
        sim.restore(blob)
        p = sim.get_params(); p.precision = prec; p.cg_tol = tol; p.cg_max_iter = 20000; p.cg_refine_tol = refine
        sim.set_params(p)
        sim.bubblesim()
        out[name] = {f: sim.get_field(f) for f in ["press", "waterux", "wateruy", "wateruz", "airux", "airuy",
                                                   "airuz", "tp", "lsmerge", "waterux_old", "wateruy_old",
                                                   "wateruz_old", "airux_old", "airuy_old", "airuz_old"]}
    for form in ("mixed", "refined"):
        for f in ["press", "tp", "lsmerge"]:
            e = rel_l2(out[form][f], out["ref"][f])
            assert e <= 1e-5, f"config {config} {f}: {form} form rel L2 {e:.3e}"
    for f in ["waterux", "wateruy", "wateruz", "airux", "airuy", "airuz"]:
        scale = max(np.linalg.norm(out["ref"][f + "_old"].astype(np.float64)), 1e-30)
        err = {form: float(np.linalg.norm(out[form][f].astype(np.float64) - out["ref"][f]) / scale)
               for form in ("fp64", "mixed", "refined")}
        assert err["refined"] <= 3 * err["fp64"] + 2e-6, f"config {config} {f}: {err}"
        assert err["mixed"] <= 2e-3, f"config {config} {f}: {err}"
    sim.close()


@pytest.mark.parametrize("config", [1, 5])
def test_refined_mixed_pressure_against_fp64(mp, oracle_mod, config):
    """Mixed-precision iterative refinement (cg_refine_tol): FP32-vector CG
    corrections with the solution and the true residual in FP64 reach the
    FP64 solve's pressure to 1e-6 relative at the configuration's 1e-6 stop,
    and the stop test holds on the FP64 true residual."""
    sim, _ = make_pair(mp, oracle_mod, config, 64, 199 + config)
    for st in ["hashAndSortParticles", "addexternalforce"]:
        getattr(sim, st)()
    sim.computeLevelset(0.0); sim.sweepLSAndMardGrid()
    sim.mapvelp2g_bubble()
    for ph in (1, 0):
        sim.sweepPhi(ph); sim.sweepU(ph)
    sim.setWaterBoundaryU(1); sim.setWaterBoundaryU(0)
    faces = {f: sim.get_field(f) for f in FACE_FIELDS}
    p0 = sim.get_params()
    p = sim.get_params()
    p.precision = mp.PREC_FP64; p.cg_tol = 1e-12; p.cg_max_iter = 8000
    sim.set_params(p)
    _, _, rc = sim.project_CG_bubble()
    assert rc == 0
    ref = sim.get_field("press").astype(np.float64)
    for f, a in faces.items():
        sim.set_field(f, a)
    p = p0
    p.cg_refine_tol = 1e-3
    sim.set_params(p)
    it, res, rc = sim.project_CG_bubble()
    assert rc == 0
    x = sim.get_field("press").astype(np.float64)
    err = np.linalg.norm(x - ref) / np.linalg.norm(ref)
    assert err <= 1e-6, f"refined mixed vs fp64 relative pressure error {err:.3e} ({it} iterations)"
    sim.close()
