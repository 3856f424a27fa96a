"""The adjoint of the FLUID-only step (configuration 4, the dam break).

The derivative is that of the recorded program with its discrete state held
fixed, so it is checked against central differences of the same program
replayed in FP64 (mp_adj_loss), on seeded directions; the FP32 adjoint is
checked against the FP64 one; the torch.autograd entry returns the same
gradient.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(mp, n, steps, every, seed=2017004, nsamples=1024):
    import torch
    sim = mp.Sim.from_config(4, n, seed)
    parts = sim.download_particles()
    v0 = torch.from_numpy(parts["vel"].astype(np.float64)).cuda()
    sim._x0_recorded = torch.from_numpy(parts["pos"].astype(np.float64)).cuda()
    sim.adj_record(steps, every)
    sim.adj_set_targets(mp.dam_break_targets(nsamples, seed, height=0.3))
    return sim, v0


def _directions(v0, k, seed):
    import torch
    gen = torch.Generator(device="cpu").manual_seed(seed)
    return [torch.randn(v0.shape, generator=gen, dtype=torch.float64).cuda() for _ in range(k)]


@pytest.mark.parametrize("n,steps,every", [(32, 6, 3), (32, 8, 8)])
def test_fp64_adjoint_matches_central_differences(mp, n, steps, every):
    sim, v0 = _setup(mp, n, steps, every)
    L, g = sim.adj_gradient(v0, mp.PREC_FP64)
    assert np.isfinite(L) and L > 0
    # 1e-6: small enough that no particle crosses a kink of the program
    # (wall clamp, kernel cut-off), large enough for FP64 round-off
    eps = 1e-6
    for d in _directions(v0, 4, 11):
        lp = sim.adj_loss(v0 + eps * d, mp.PREC_FP64)
        lm = sim.adj_loss(v0 - eps * d, mp.PREC_FP64)
        fd = (lp - lm) / (2 * eps)
        ad = float((g * d).sum())
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad), 1e-12 * L), f"fd {fd:.9e} adjoint {ad:.9e}"
    sim.close()


def test_configuration4_gradient(mp):
    """The dam break as configured: 64^3, 32 steps, checkpoints every 8, 16
    seeded directions. Over 32 steps of ~0.46M particles a perturbation of
    1e-7 or more already moves some particle-face pair across a kink of the
    program (the kernel cut-off, the wall clamp), and the central difference
    then differs by up to 1e-1; at 1e-8 it agrees to a few 1e-6 (FP64
    round-off takes over below)."""
    sim, v0 = _setup(mp, 64, 32, 8)
    L, g = sim.adj_gradient(v0, mp.PREC_FP64)
    eps = 1e-8
    bad = 0
    for d in _directions(v0, 16, 13):
        lp = sim.adj_loss(v0 + eps * d, mp.PREC_FP64)
        lm = sim.adj_loss(v0 - eps * d, mp.PREC_FP64)
        fd = (lp - lm) / (2 * eps)
        ad = float((g * d).sum())
        bad += abs(fd - ad) > 1e-4 * max(abs(fd), abs(ad))
    assert bad == 0, f"{bad} of 16 directions off by more than 1e-4"
    sim.close()


def test_gradient_does_not_depend_on_the_checkpoint_interval(mp):
    """Recomputing from checkpoints replays the same arithmetic: the gradient
    is the same bit for bit whatever the interval."""
    out = []
    for every in (1, 3, 8):
        sim, v0 = _setup(mp, 32, 8, every)
        out.append(sim.adj_gradient(v0, mp.PREC_MIXED)[1])
        sim.close()
    import torch
    assert torch.equal(out[0], out[1]) and torch.equal(out[0], out[2])


def test_fp32_adjoint_against_fp64(mp):
    sim, v0 = _setup(mp, 32, 6, 3)
    L64, g64 = sim.adj_gradient(v0, mp.PREC_FP64)
    L32, g32 = sim.adj_gradient(v0, mp.PREC_MIXED)
    assert abs(L32 - L64) <= 1e-4 * abs(L64)
    rel = float((g32 - g64).norm() / g64.norm())
    assert rel <= 1e-2, f"FP32 gradient rel err {rel:.3e}"
    for d in _directions(v0, 4, 12):
        a32, a64 = float((g32 * d).sum()), float((g64 * d).sum())
        assert abs(a32 - a64) <= 1e-2 * abs(a64) + 1e-6 * float(g64.norm() * d.norm())
    sim.close()


def test_autograd_entry_returns_the_adjoint(mp):
    import torch
    sim, v0 = _setup(mp, 32, 4, 2)
    L64, g64 = sim.adj_gradient(v0, mp.PREC_FP64)
    v = v0.clone().requires_grad_(True)
    loss = mp.dam_break_loss(v, sim, mp.PREC_FP64)
    loss.backward()
    assert abs(float(loss.detach()) - L64) <= 1e-12 * abs(L64)
    assert torch.equal(v.grad, g64)
    sim.close()


def test_record_rejects_programs_outside_the_adjoint(mp):
    sim = mp.Sim.from_config(1, 32, 2017001)   # air bubble: not FLUID-only
    with pytest.raises(mp.MPError):
        sim.adj_record(2, 1)
    sim.close()


def test_vector_jacobian_product_matches_central_differences(mp):
    """mp_step_adjoint with arbitrary cotangents w on the final positions and
    velocities: <J^T w, d> equals the central difference of <w, f(x0, v0)>
    along seeded directions d of the initial velocities and of the initial
    positions (FP64 replays of the recorded program)."""
    import torch
    sim, v0 = _setup(mp, 32, 6, 3)
    x0 = sim._x0_recorded
    xT, vT = sim.adj_forward(x0, v0, mp.PREC_FP64)
    gen = torch.Generator(device="cpu").manual_seed(21)
    wx = torch.randn(xT.shape, generator=gen, dtype=torch.float64).cuda()
    wv = torch.randn(vT.shape, generator=gen, dtype=torch.float64).cuda()
    x0b, v0b = sim.step_adjoint(x0, v0, wx, wv, mp.PREC_FP64)
    assert torch.isfinite(x0b).all() and torch.isfinite(v0b).all()

    def f(x, v):
        a, b = sim.adj_forward(x, v, mp.PREC_FP64)
        return float((a * wx).sum() + (b * wv).sum())

    for i, d in enumerate(_directions(v0, 3, 23)):
        eps = 1e-6
        fd = (f(x0, v0 + eps * d) - f(x0, v0 - eps * d)) / (2 * eps)
        ad = float((v0b * d).sum())
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)), f"v direction {i}: fd {fd:.9e} adjoint {ad:.9e}"
    for i, d in enumerate(_directions(v0, 3, 29)):
        eps = 1e-8
        fd = (f(x0 + eps * d, v0) - f(x0 - eps * d, v0)) / (2 * eps)
        ad = float((x0b * d).sum())
        assert abs(fd - ad) <= 1e-4 * max(abs(fd), abs(ad)), f"x direction {i}: fd {fd:.9e} adjoint {ad:.9e}"
    sim.close()


def test_autograd_composition_equals_the_loss_gradient(mp):
    """The loss composed through autograd, level_set_loss(mp_step(x0, v0)[0]),
    gives the gradient mp_adj_gradient computes for the same program; backward
    runs only for the inputs that ask for it."""
    import torch
    sim, v0 = _setup(mp, 32, 4, 2)
    L64, g64 = sim.adj_gradient(v0, mp.PREC_FP64)
    x = sim._x0_recorded.clone()
    v = v0.clone().requires_grad_(True)
    xT, vT = mp.mp_step(x, v, sim, mp.PREC_FP64)
    loss = mp.level_set_loss(xT, sim, mp.PREC_FP64)
    loss.backward()
    assert abs(float(loss.detach()) - L64) <= 1e-12 * abs(L64)
    assert x.grad is None
    rel = float((v.grad - g64).norm() / g64.norm())
    assert rel <= 1e-10, f"composed gradient differs by {rel:.3e}"
    sim.close()


def _setup_heat(mp, n, steps, every, seed=2017006):
    """The dam break with the heat stage on: a hot bottom plate held at 1.25,
    initial temperatures 0.95 + 0.05 N(0, 1), FLIP/PIC temperature transfer
    0.3, melting and boiling points outside the range reached (no clamp)."""
    import torch
    p = mp.scene_params(4, n)
    p.b_heat_trans = 1; p.b_fixed_heat = 1; p.b_extend_heat_to_boundary = 1
    p.heatalpha_fluid = 0.05; p.heatalpha_vacuum = 0.0001
    p.default_temperature = 1.0; p.melting_point = 0.2; p.boiling_point = 5.0
    p.alpha_temp_trans = 0.3
    sim = mp.Sim.from_config(4, n, seed, params=p)
    parts = sim.download_particles()
    rng = np.random.default_rng(seed)
    parts["temp"] = (0.95 + 0.05 * rng.standard_normal(len(parts["temp"]))).astype(np.float32)
    sim.upload_particles(**parts)
    fh = np.full(n ** 3, -10000.0, np.float32).reshape(n, n, n)   # MP_UNDEF_TEMPERATURE: not held
    fh[1:-1, 1:-1, :4] = 1.25
    sim.set_field("fixedheat", fh.ravel())
    x0 = torch.from_numpy(parts["pos"].astype(np.float64)).cuda()
    v0 = torch.from_numpy(parts["vel"].astype(np.float64)).cuda()
    T0 = torch.from_numpy(parts["temp"].astype(np.float64)).cuda()
    sim.adj_record(steps, every)
    return sim, x0, v0, T0


def test_heat_adjoint_matches_central_differences(mp):
    """The heat stage's transpose (the splat of particle temperatures, the
    implicit diffusion as a second solve on the symmetric heat matrix, the
    boundary copy, the FLIP/PIC transfer back): <J^T w, d> against central
    differences of the FP64 replay. With a cotangent on the final
    temperatures only, the directions of the initial temperatures test the
    temperature path alone, and those of the initial velocities and positions
    the heat stage's dependence on where the particles are (splat weights,
    interpolation); a cotangent on the whole final state checks the sum."""
    import torch
    sim, x0, v0, T0 = _setup_heat(mp, 32, 4, 2)
    xT, vT, TT = sim.adj_forward(x0, v0, mp.PREC_FP64, T0=T0)
    assert torch.isfinite(TT).all() and float((TT - T0).abs().max()) > 1e-4   # the heat stage did something
    gen = torch.Generator(device="cpu").manual_seed(31)
    wx = torch.randn(xT.shape, generator=gen, dtype=torch.float64).cuda()
    wv = torch.randn(vT.shape, generator=gen, dtype=torch.float64).cuda()
    wT = torch.randn(TT.shape, generator=gen, dtype=torch.float64).cuda()

    def check(cx, cv, cT, dirs_T, dirs_v, dirs_x, tol_vx):
        x0b, v0b, T0b = sim.step_adjoint(x0, v0, cx, cv, mp.PREC_FP64, T0=T0, TT_bar=cT)

        def f(x, v, T):
            a, b, c = sim.adj_forward(x, v, mp.PREC_FP64, T0=T)
            out = (c * cT).sum()
            if cx is not None:
                out = out + (a * cx).sum() + (b * cv).sum()
            return float(out)

        # positions: the splat weights and the trilinear temperature transfer
        # are piecewise smooth, and at eps = 1e-8 about one particle per
        # direction crosses a cell face of the interpolation in 4 steps,
        # which moves the central difference by ~1e-4
        for name, base, grad, dirs, eps, tol in (("T", T0, T0b, dirs_T, 1e-6, 1e-5),
                                                  ("v", v0, v0b, dirs_v, 1e-6, tol_vx),
                                                  ("x", x0, x0b, dirs_x, 1e-8, 3e-4)):
            for i, d in enumerate(dirs):
                args = {"T": (x0, v0, T0), "v": (x0, v0, T0), "x": (x0, v0, T0)}[name]
                plus = [a + eps * d if a is base else a for a in args]
                minus = [a - eps * d if a is base else a for a in args]
                fd = (f(*plus) - f(*minus)) / (2 * eps)
                ad = float((grad * d).sum())
                assert abs(fd - ad) <= tol * max(abs(fd), abs(ad)), \
                    f"{name} direction {i}: fd {fd:.9e} adjoint {ad:.9e}"

    gd = torch.Generator(device="cpu").manual_seed(37)
    dT = [torch.randn(T0.shape, generator=gd, dtype=torch.float64).cuda() for _ in range(2)]
    # the temperature cotangent alone
    check(None, None, wT, dT, _directions(v0, 2, 41), _directions(v0, 2, 43), 1e-4)
    # the whole final state
    check(wx, wv, wT, dT[:1], _directions(v0, 1, 47), _directions(v0, 1, 53), 1e-4)
    sim.close()


def test_heat_autograd_and_fp32_against_fp64(mp):
    """torch.autograd through the heat-recorded program: the gradient of
    sum(TT^2) with respect to T0 from mp_step equals the FP64 VJP. The FP32
    replay keeps the engine's own stop rule for the heat solve (the
    reference's absolute |r|^2 < 0.01 n, a relative residual of about 2e-2
    here), so its temperatures, and its gradient, differ from the FP64
    replay's (solved to 1e-13) at that level: within 5e-2."""
    import torch
    sim, x0, v0, T0 = _setup_heat(mp, 32, 4, 2)
    T = T0.clone().requires_grad_(True)
    xT, vT, TT = mp.mp_step(x0, v0, sim, mp.PREC_FP64, T0=T)
    (TT * TT).sum().backward()
    _, _, TT64 = sim.adj_forward(x0, v0, mp.PREC_FP64, T0=T0)
    _, _, g64 = sim.step_adjoint(x0, v0, None, None, mp.PREC_FP64, T0=T0, TT_bar=2 * TT64)
    assert float((T.grad - g64).norm() / g64.norm()) <= 1e-12
    _, _, TT32 = sim.adj_forward(x0, v0, mp.PREC_MIXED, T0=T0)
    _, _, g32 = sim.step_adjoint(x0, v0, None, None, mp.PREC_MIXED, T0=T0, TT_bar=2 * TT32)
    rel = float((g32 - g64).norm() / g64.norm())
    assert rel <= 5e-2, f"FP32 heat gradient rel err {rel:.3e}"
    sim.close()


def test_replay_reproduces_the_engine_run(mp):
    """The FP32 replay of the recorded FLUID program runs the engine's
    arithmetic in the engine's order, so after four steps its final state is
    the engine's own, bit for bit (mp_adj_order maps the engine's slots)."""
    import torch
    sim, v0 = _setup(mp, 32, 4, 2)
    x0 = sim._x0_recorded
    parts = sim.download_particles()
    ids = sim.adj_order().cpu().numpy()
    xe = np.empty_like(parts["pos"]); ve = np.empty_like(parts["vel"])
    xe[ids] = parts["pos"]; ve[ids] = parts["vel"]
    xT, vT = sim.adj_forward(x0, v0, mp.PREC_MIXED)
    xT = xT.cpu().numpy().astype(np.float32); vT = vT.cpu().numpy().astype(np.float32)
    assert np.array_equal(xT, xe) and np.array_equal(vT, ve)
    sim.close()


def test_gradient_at_the_recorded_inputs_from_the_engine_states(mp):
    """A gradient at the recorded inputs (NULL initial state) takes its
    segment starts, final state and pressures from the engine's recorded run
    instead of a first replay; it equals the gradient from explicit inputs
    (the full replay) bit for bit, for several checkpoint intervals."""
    import torch
    for every in (8, 3):
        sim, v0 = _setup(mp, 32, 8, every)
        w0 = sim.work_counts()
        L1, g1 = sim.adj_gradient(None, mp.PREC_MIXED)
        w1 = sim.work_counts()
        L2, g2 = sim.adj_gradient(v0, mp.PREC_MIXED)
        w2 = sim.work_counts()
        assert w1["adj_engine"] == w0["adj_engine"] + 1 and w1["adj_replay"] == w0["adj_replay"]
        assert w2["adj_replay"] == w1["adj_replay"] + 1
        assert L1 == L2 and torch.equal(g1, g2)
        sim.close()
