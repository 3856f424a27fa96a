"""The exact exits of the level-set sweep (k_sweep, sweepphibytype /
sweepphi spray_k.cu:755-788), checked on the CPU in float32 arithmetic.

An octant (a, b, c) of a cell with value res is skipped without its
solvedistance when m = min(a, b, c) >= res and either m + 1 <= max(a, b, c)
or m is "settled" (3m - 2m == m, or m > 1e-30 with m two ulps down >= res).
The claim is that solvedistance would then leave res unchanged. The cell
exit takes the same conclusion for all octants at once when the six
neighbours' minimum is >= res and all six are settled. Both are checked here
against solvedistance itself on seeded random values, the far-field values
the sweeps see (5, 3 N) and values a few ulps from res.
"""
import numpy as np

f32 = np.float32


def solvedistance(a, b, c, x):
    a, b, c, x = f32(a), f32(b), f32(c), f32(x)
    d = f32(min(a, min(b, c)) + f32(1))
    if d > max(a, max(b, c)):
        s = f32(3) - (a - b) * (a - b) - (a - c) * (a - c) - (b - c) * (b - c)
        with np.errstate(invalid="ignore"):
            d = f32((a + b + c + np.sqrt(f32(s))) / f32(3))
    return d if d < x else x


def settled(m, res):
    m, res = f32(m), f32(res)
    t = f32(f32(3) * m)
    if f32(t - f32(2) * m) == m:
        return True
    if m > f32(1e-30):
        down = np.frombuffer(np.array([m], dtype=f32).tobytes(), dtype=np.int32)[0] - 2
        return np.frombuffer(np.array([down], dtype=np.int32).tobytes(), dtype=f32)[0] >= res
    return False


def skipped(a, b, c, res):
    m = f32(min(a, min(b, c)))
    if not (m >= res):
        return False
    mx = f32(max(a, max(b, c)))
    if not (f32(m + f32(1)) > mx):
        return True
    return settled(m, res)


def samples(rng, n):
    base = rng.choice(np.array([0.0, 0.5, 1.0, 1.5, 2.0, 5.0, 96.0, 768.0, 1e-3, 3.7], dtype=f32), size=(n, 4))
    jitter = rng.integers(-3, 4, size=(n, 4)).astype(np.int32)
    bits = base.view(np.int32) + jitter * (base != 0)
    vals = bits.view(f32)
    rnd = rng.uniform(-0.5, 6.0, size=(n, 4)).astype(f32)
    pick = rng.random((n, 4)) < 0.5
    return np.where(pick, vals, rnd)


def test_octant_skip_leaves_the_cell_unchanged():
    rng = np.random.default_rng(2017)
    v = samples(rng, 40000)
    n = 0
    for a, b, c, res in v:
        if skipped(a, b, c, res):
            n += 1
            assert solvedistance(a, b, c, res) == f32(res), (a, b, c, res)
    assert n > 1000   # the skip is exercised


def test_cell_exit_leaves_the_cell_unchanged():
    rng = np.random.default_rng(2018)
    v = samples(rng, 12000)
    nb = samples(rng, 12000)
    n = 0
    for (n0, n1, n2, res), (n3, n4, n5, _) in zip(v, nb):
        six = [n0, n1, n2, n3, n4, n5]
        if not (f32(min(six)) >= res and all(settled(x, res) for x in six)):
            continue
        n += 1
        x = f32(res)
        for a in (n0, n3):
            for b in (n1, n4):
                for c in (n2, n5):
                    x = solvedistance(a, b, c, x)
        assert x == f32(res), (six, res)
    assert n > 100   # the exit is exercised
