"""The adjoint's nearest-FLUID-particle search (k_ad_nearest) with its bound
from the 27 nearest cells, checked on the CPU in float32: for every cell it
picks the same particle as the plain scan of the +-2 cell box in its fixed
order (first minimum kept, nothing beyond 2.5 cells), on seeded particle
clouds with coincident and boundary-hugging particles."""
import numpy as np

f32 = np.float32


def cells_of(pos, n, h):
    idx = np.floor(pos / h).astype(np.int64)
    idx = np.where((pos >= 0) & (pos < n * h), idx, 0)
    return idx


def nearest_plain(pos, cell, n, h, i, j, k):
    gp = (np.array([i, j, k], dtype=f32) + f32(0.5)) * f32(h)
    best, who = f32(6.25) * f32(h) * f32(h), -1
    for di in range(-2, 3):
        for dj in range(-2, 3):
            for dk in range(-2, 3):
                a, b, c = i + di, j + dj, k + dk
                if not (0 <= a < n and 0 <= b < n and 0 <= c < n):
                    continue
                for q in np.nonzero((cell[:, 0] == a) & (cell[:, 1] == b) & (cell[:, 2] == c))[0]:
                    d = (pos[q] - gp).astype(f32)
                    d2 = f32(f32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
                    if d2 < best:
                        best, who = d2, q
    return who


def nearest_bounded(pos, cell, n, h, i, j, k):
    gp = (np.array([i, j, k], dtype=f32) + f32(0.5)) * f32(h)
    h = f32(h)
    cap = f32(6.25) * h * h

    def members(a, b, c):
        return np.nonzero((cell[:, 0] == a) & (cell[:, 1] == b) & (cell[:, 2] == c))[0]

    def d2_of(q):
        d = (pos[q] - gp).astype(f32)
        return f32(f32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])

    bound = cap
    for di in range(-1, 2):
        for dj in range(-1, 2):
            for dk in range(-1, 2):
                a, b, c = i + di, j + dj, k + dk
                if 0 <= a < n and 0 <= b < n and 0 <= c < n:
                    for q in members(a, b, c):
                        bound = min(bound, d2_of(q))
    best, who = cap, -1
    for di in range(-2, 3):
        for dj in range(-2, 3):
            for dk in range(-2, 3):
                a, b, c = i + di, j + dj, k + dk
                if not (0 <= a < n and 0 <= b < n and 0 <= c < n):
                    continue
                bx = f32(0) if di == 0 else f32(abs(di)) - f32(0.5)
                by = f32(0) if dj == 0 else f32(abs(dj)) - f32(0.5)
                bz = f32(0) if dk == 0 else f32(abs(dk)) - f32(0.5)
                if f32(f32(f32(bx * bx + by * by) + bz * bz) * h * h * f32(0.9999)) > bound:
                    continue
                for q in members(a, b, c):
                    d2 = d2_of(q)
                    if d2 < best:
                        best, who = d2, q
    return who


def test_bounded_search_picks_the_same_particle():
    rng = np.random.default_rng(2017)
    n, h = 6, f32(1.0 / 6)
    pos = rng.uniform(0, 1, size=(700, 3)).astype(f32)
    pos[:40] = pos[40:80]                          # coincident pairs (ties: first kept)
    pos[80:120, 0] = f32(0.5) * h                   # on a cell's mid-plane
    pos[120:160] = np.floor(pos[120:160] / h) * h   # on cell corners
    cell = cells_of(pos, n, h)
    for i in range(n):
        for j in range(n):
            for k in range(n):
                assert nearest_bounded(pos, cell, n, h, i, j, k) == nearest_plain(pos, cell, n, h, i, j, k)
