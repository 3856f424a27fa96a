"""The adjoint of the two-phase step: FLUID and AIR particles (a rising air
bubble, configuration 1's scene, and the bubble column of configuration 5 at
a reduced grid), with position correction off.

The program differentiated is bubblesim's without the solo-air stages: the
buoyancy of AIR, both splats, both extrapolations, the two-phase projection
(the level-set blend at liquid-air faces), each phase's FLIP/PIC gather and
advection. The engine's own run of it (mp_adj_record) is checked against the
replay; the FP64 adjoint against central differences of the FP64 replay, on
seeded directions of the initial velocities and positions; the FP32 adjoint
against the FP64 one.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(mp, config, n, steps, every, seed, height, nsamples=1024):
    import torch
    p = mp.scene_params(config, n)
    p.b_correct_position = 0
    sim = mp.Sim.from_config(config, n, seed, params=p)
    parts = sim.download_particles()
    assert (parts["flag"] == mp.TYPEAIR).any() and (parts["flag"] == mp.TYPEFLUID).any()
    x0 = torch.from_numpy(parts["pos"].astype(np.float64)).cuda()
    v0 = torch.from_numpy(parts["vel"].astype(np.float64)).cuda()
    sim.adj_record(steps, every)
    sim.adj_set_targets(mp.dam_break_targets(nsamples, seed, height=height))
    sim._flag0 = parts["flag"]
    return sim, x0, v0


def _directions(shape, k, seed):
    import torch
    gen = torch.Generator(device="cpu").manual_seed(seed)
    return [torch.randn(shape, generator=gen, dtype=torch.float64).cuda() for _ in range(k)]


def test_replay_reproduces_the_engine_run(mp):
    """The FP32 replay of the recorded two-phase program runs the engine's
    arithmetic in the engine's order (the splats, the extrapolation weights,
    the projection with the same CG kernels from x = 0, the gather and the
    advection), so it ends exactly where the engine's own steps ended."""
    import torch
    sim, x0, v0 = _setup(mp, 1, 32, 4, 2, 2017001, 0.45)
    parts = sim.download_particles()
    ids = sim.adj_order().cpu().numpy()
    xe = np.empty_like(parts["pos"]); ve = np.empty_like(parts["vel"])
    xe[ids] = parts["pos"]; ve[ids] = parts["vel"]
    xT, vT = sim.adj_forward(x0, v0, mp.PREC_MIXED)
    xT, vT = xT.cpu().numpy(), vT.cpu().numpy()
    air = np.zeros(len(ids), bool)
    air[ids] = parts["flag"] == mp.TYPEAIR
    assert air.any()
    xT, vT = xT.astype(np.float32), vT.astype(np.float32)   # FP32 values carried in doubles
    dx = np.abs(xT - xe).max()
    dv = np.abs(vT - ve).max()
    assert dx == 0 and dv == 0, f"positions differ by {dx:.3e}, velocities by {dv:.3e}"
    sim.close()


@pytest.mark.parametrize("config,n,steps,every,seed,height", [(1, 32, 4, 2, 2017001, 0.45),
                                                               (5, 32, 3, 3, 2017005, 0.7)])
def test_fp64_adjoint_matches_central_differences(mp, config, n, steps, every, seed, height):
    sim, x0, v0 = _setup(mp, config, n, steps, every, seed, height)
    L, g = sim.adj_gradient(v0, mp.PREC_FP64)
    assert np.isfinite(L) and L > 0
    # 1e-6: small enough that no particle crosses a kink of the program (wall
    # clamp, kernel cut-off, the buoyancy's speed limit), large enough for
    # FP64 round-off
    eps = 1e-6
    for d in _directions(v0.shape, 4, 31):
        lp = sim.adj_loss(v0 + eps * d, mp.PREC_FP64)
        lm = sim.adj_loss(v0 - eps * d, mp.PREC_FP64)
        fd = (lp - lm) / (2 * eps)
        ad = float((g * d).sum())
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad), 1e-12 * L), f"fd {fd:.9e} adjoint {ad:.9e}"
    sim.close()


def test_vector_jacobian_product_matches_central_differences(mp):
    """mp_step_adjoint with arbitrary cotangents on the final positions and
    velocities of FLUID and AIR particles, along seeded directions of the
    initial velocities and positions, over two steps (checkpoints every step).

    The splat is discontinuous where a face's last particle leaves its window
    (u = s/W for W > 0, else 0), and around a bubble more faces hang on one
    particle: with cotangents on every particle, central differences over
    four steps cross such a jump at any step size (errors of 1e-3 to 1e-1
    that do not shrink with it), while over one step they agree to 1e-9 and
    over two to 1e-8 at a step of 1e-7."""
    import torch
    sim, x0, v0 = _setup(mp, 1, 32, 2, 1, 2017001, 0.45)
    xT, vT = sim.adj_forward(x0, v0, mp.PREC_FP64)
    gen = torch.Generator(device="cpu").manual_seed(41)
    wx = torch.randn(xT.shape, generator=gen, dtype=torch.float64).cuda()
    wv = torch.randn(vT.shape, generator=gen, dtype=torch.float64).cuda()
    x0b, v0b = sim.step_adjoint(x0, v0, wx, wv, mp.PREC_FP64)
    assert torch.isfinite(x0b).all() and torch.isfinite(v0b).all()

    def f(x, v):
        a, b = sim.adj_forward(x, v, mp.PREC_FP64)
        return float((a * wx).sum() + (b * wv).sum())

    for i, d in enumerate(_directions(v0.shape, 3, 43)):
        eps = 1e-7
        fd = (f(x0, v0 + eps * d) - f(x0, v0 - eps * d)) / (2 * eps)
        ad = float((v0b * d).sum())
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)), f"v direction {i}: fd {fd:.9e} adjoint {ad:.9e}"
    for i, d in enumerate(_directions(x0.shape, 3, 47)):
        eps = 1e-8
        fd = (f(x0 + eps * d, v0) - f(x0 - eps * d, v0)) / (2 * eps)
        ad = float((x0b * d).sum())
        assert abs(fd - ad) <= 1e-4 * max(abs(fd), abs(ad)), f"x direction {i}: fd {fd:.9e} adjoint {ad:.9e}"
    sim.close()


def test_fp32_adjoint_against_fp64(mp):
    sim, x0, v0 = _setup(mp, 1, 32, 4, 2, 2017001, 0.45)
    L64, g64 = sim.adj_gradient(v0, mp.PREC_FP64)
    L32, g32 = sim.adj_gradient(v0, mp.PREC_MIXED)
    assert abs(L32 - L64) <= 1e-4 * abs(L64)
    rel = float((g32 - g64).norm() / g64.norm())
    assert rel <= 1e-2, f"FP32 gradient rel err {rel:.3e}"
    sim.close()


def test_air_particles_receive_gradient(mp):
    """The loss reads the FLUID distance field only, yet the bubble's initial
    velocities change it through the two-phase projection: the AIR particles'
    rows of dL/dv0 are not all zero."""
    import torch
    sim, x0, v0 = _setup(mp, 1, 32, 4, 2, 2017001, 0.45)
    L, g = sim.adj_gradient(v0, mp.PREC_FP64)
    air = torch.from_numpy(sim._flag0 == mp.TYPEAIR).cuda()
    assert float(g[air].abs().max()) > 0
    sim.close()


def test_non_cubic_grid(mp):
    """The two-phase program on a 32 x 24 x 30 grid (extents that differ and
    do not fill the node tiles of the warp-staged splat and G2P transpose):
    the FP64 adjoint against central differences along velocity and position
    directions, over two steps."""
    import torch
    from parity_util import grid_params
    p = grid_params(mp, 1, 32, 24, 30)
    p.b_correct_position = 0
    sim = mp.Sim.from_config(1, 32, 2017011, params=p)
    parts = sim.download_particles()
    assert (parts["flag"] == mp.TYPEAIR).any()
    x0 = torch.from_numpy(parts["pos"].astype(np.float64)).cuda()
    v0 = torch.from_numpy(parts["vel"].astype(np.float64)).cuda()
    sim.adj_record(2, 1)
    xT, vT = sim.adj_forward(x0, v0, mp.PREC_FP64)
    gen = torch.Generator(device="cpu").manual_seed(51)
    wx = torch.randn(xT.shape, generator=gen, dtype=torch.float64).cuda()
    wv = torch.randn(vT.shape, generator=gen, dtype=torch.float64).cuda()
    x0b, v0b = sim.step_adjoint(x0, v0, wx, wv, mp.PREC_FP64)

    def f(x, v):
        a, b = sim.adj_forward(x, v, mp.PREC_FP64)
        return float((a * wx).sum() + (b * wv).sum())

    for i, d in enumerate(_directions(v0.shape, 2, 53)):
        eps = 1e-7
        fd = (f(x0, v0 + eps * d) - f(x0, v0 - eps * d)) / (2 * eps)
        ad = float((v0b * d).sum())
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)), f"v direction {i}: fd {fd:.9e} adjoint {ad:.9e}"
    for i, d in enumerate(_directions(x0.shape, 2, 59)):
        eps = 1e-8
        fd = (f(x0 + eps * d, v0) - f(x0 - eps * d, v0)) / (2 * eps)
        ad = float((x0b * d).sum())
        assert abs(fd - ad) <= 1e-4 * max(abs(fd), abs(ad)), f"x direction {i}: fd {fd:.9e} adjoint {ad:.9e}"
    sim.close()


def test_gradient_at_the_recorded_inputs_from_the_engine_states(mp):
    """The two-phase program: the gradient at the recorded inputs, from the
    engine's recorded states, equals the one from the full replay bit for
    bit."""
    import torch
    sim, x0, v0 = _setup(mp, 1, 32, 4, 2, 2017001, 0.45)
    w0 = sim.work_counts()
    L1, g1 = sim.adj_gradient(None, mp.PREC_MIXED)
    w1 = sim.work_counts()
    L2, g2 = sim.adj_gradient(v0, mp.PREC_MIXED)
    assert w1["adj_engine"] == w0["adj_engine"] + 1 and w1["adj_replay"] == w0["adj_replay"]
    assert L1 == L2 and torch.equal(g1, g2)
    sim.close()
