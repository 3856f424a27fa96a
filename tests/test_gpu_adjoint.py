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
    v0 = torch.from_numpy(sim.download_particles()["vel"].astype(np.float64)).cuda()
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
