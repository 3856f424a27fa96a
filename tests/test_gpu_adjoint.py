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
