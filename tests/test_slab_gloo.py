"""The x-slab decomposition (2017multiphase_b200/slab.py) on CPU ranks.

The plan's partition, particle routing and block reduction are checked
directly, and the decomposition of the projection's CG (solver_cg_bubble,
spray.cu:1613-1687, with computeAx_bubble spray_k.cu:3423-3447) runs on 2 and
4 gloo ranks: each rank holds its slab of the pressure system with one ghost
plane per side, exchanges the search direction's edge planes before every
matrix application and combines the dot products' block partials with one
all-reduce.  A numpy model of the oracle's CG arithmetic (float32 vectors in
the oracle's operation order, FP64 block sums) stands in for the GPU kernels,
which this 1-GPU setting cannot run on several GPUs.  The gathered pressure
and the iteration count equal the single-domain oracle's bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from conftest import ROOT

TF, TA, TB = 0, 1, 2


def _slab():
    import importlib
    return importlib.import_module("2017multiphase_b200.slab")


def test_partition_covers_the_grid_on_block_boundaries():
    sl = _slab()
    for nx, ny, nz in [(32, 32, 32), (64, 64, 64), (16, 16, 16), (37, 32, 32), (256, 256, 256)]:
        unit = sl.plane_unit(ny, nz)
        assert (unit * ny * nz) % sl.BLOCK == 0
        for world in (1, 2, 3, 4, 8):
            if -(-nx // unit) < world:
                with pytest.raises(ValueError):
                    sl.partition(nx, ny, nz, world)
                continue
            b = sl.partition(nx, ny, nz, world)
            assert b[0][0] == 0 and b[-1][1] == nx
            assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
            assert all(x0 * ny * nz % sl.BLOCK == 0 for x0, _ in b)
            sizes = [x1 - x0 for x0, x1 in b]
            assert min(sizes) > 0 and max(sizes) - min(sizes) <= unit


def test_particle_routing_follows_the_hash_cell(mp):
    sl = _slab()
    p = mp.scene_params(1, 32)
    parts = mp.scene_particles(p, 1, 5)
    pos = np.asarray(parts["pos"], np.float32).reshape(-1, 3)
    pos[:3, 0] = [-0.5, 99.0, np.float32(p.cellsize) * 16]        # outside the grid -> cell 0; a slab boundary
    b = sl.partition(p.nx, p.ny, p.nz, 4)
    owner = sl.route_particles(pos, p.cellsize, p.gmin_x, p.nx, b)
    assert owner[0] == 0 and owner[1] == 0 and owner[2] == sl.owner_of_planes(16, b)
    i = np.floor((pos[3:, 0] - np.float32(p.gmin_x)) / np.float32(p.cellsize)).astype(int)
    assert np.array_equal(owner[3:], sl.owner_of_planes(i, b))
    assert set(owner.tolist()) == {0, 1, 2, 3}


def test_block_reduction_is_independent_of_the_rank_count():
    sl = _slab()
    rng = np.random.default_rng(3)
    nx, ny, nz = 32, 32, 32
    a = rng.normal(size=(nx, ny, nz)).astype(np.float32)
    b = rng.normal(size=(nx, ny, nz)).astype(np.float32)
    nblk = -(-a.size // sl.BLOCK)
    whole = sl.combine_blocks(nblk, 0, sl.block_partials(a, b))
    for world in (2, 4, 8):
        v_sum = np.zeros(nblk)
        for x0, x1 in sl.partition(nx, ny, nz, world):
            b0, _ = sl.block_range(x0, x1, ny, nz)
            part = sl.block_partials(a[x0:x1], b[x0:x1])
            v_sum[b0:b0 + len(part)] += part
        assert sl.combine_blocks(nblk, 0, v_sum) == whole


# ---- the CG on gloo ranks -------------------------------------------------------

def _apply_A(x_ext, m_ext, h2):
    """computeAx_bubble on the owned planes of a slab with one ghost plane per
    side, in the oracle's operation order: -6c, then +x, +y, +z, -x, -y, -z
    neighbours (a BOUNDARY neighbour contributes c); rows other than FLUID/AIR
    are 0."""
    c, m = x_ext[1:-1], m_ext[1:-1]

    def nb(xq, mq):
        return np.where(mq == TB, c, xq)

    s = np.float32(-6.0) * c
    s = s + nb(x_ext[2:], m_ext[2:])
    s = s + nb(np.roll(c, -1, 1), np.roll(m, -1, 1))
    s = s + nb(np.roll(c, -1, 2), np.roll(m, -1, 2))
    s = s + nb(x_ext[:-2], m_ext[:-2])
    s = s + nb(np.roll(c, 1, 1), np.roll(m, 1, 1))
    s = s + nb(np.roll(c, 1, 2), np.roll(m, 1, 2))
    out = s / h2
    return np.where((m == TF) | (m == TA), out, np.float32(0)).astype(np.float32)


def _worker(rank, world, port, inp, outdir, pipelined=False):
    import sys
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import importlib
    sl = importlib.import_module("2017multiphase_b200.slab")
    d = np.load(inp)
    mark, div = d["mark"], d["div"]
    nx, ny, nz = mark.shape
    h2 = np.float32(d["h"]) * np.float32(d["h"])
    x0, x1 = sl.partition(nx, ny, nz, world)[rank]
    b0, _ = sl.block_range(x0, x1, ny, nz)
    nblk = -(-mark.size // sl.BLOCK)
    nl = x1 - x0
    m_ext = np.full((nl + 2, ny, nz), TB, np.int8)
    m_ext[1:-1] = mark[x0:x1]
    m_t = torch.from_numpy(m_ext)
    sl.exchange_ghosts(m_t, rank, world)            # the marks' ghost planes, once
    mask = (mark[x0:x1] == TF) | (mark[x0:x1] == TA)
    b = div[x0:x1].astype(np.float32)
    ext = torch.zeros((nl + 2, ny, nz), dtype=torch.float32)
    e = ext.numpy()

    def A(v):                                        # halo exchange, then the local rows
        e[1:-1] = v
        sl.exchange_ghosts(ext, rank, world)
        return _apply_A(e, m_ext, h2)

    n_reduce = [0]

    def count(v):
        n_reduce[0] += 1
        sl.torch_all_reduce(v)

    def dot(u, v):
        return sl.combine_blocks(nblk, b0, sl.block_partials(u, v), count)

    x = np.zeros((nl, ny, nz), np.float32)
    z = A(x)
    r = np.where(mask, b + np.float32(-1.0) * z, np.float32(0)).astype(np.float32)
    rr = dot(r, r)
    eps = float(np.float32(d["tol"]) * np.float32(mark.size))
    k = 0
    if pipelined and not rr < eps:
        # Chronopoulos-Gear: one all-reduce per iteration for both dot products
        def dots2(u, v, w, t):
            return sl.combine_blocks_many(nblk, b0, [sl.block_partials(u, v), sl.block_partials(w, t)], count)
        u = r.copy()
        w = A(u)
        gamma, delta = dots2(r, u, w, u)
        p, s = u.copy(), w.copy()
        alpha = gamma / delta
        while True:
            af = np.float32(alpha)
            x = np.where(mask, x + af * p, np.float32(0)).astype(np.float32)
            r = np.where(mask, r + (-af) * s, np.float32(0)).astype(np.float32)
            k += 1
            u = r
            w = A(u)
            gamma_new, delta = dots2(r, u, w, u)
            if gamma_new < eps or k >= int(d["maxiter"]):
                rr = gamma_new
                break
            beta = gamma_new / gamma
            alpha = gamma_new / (delta - beta * gamma_new / alpha)
            gamma = gamma_new
            bf = np.float32(beta)
            p = np.where(mask, u + bf * p, np.float32(0)).astype(np.float32)
            s = np.where(mask, w + bf * s, np.float32(0)).astype(np.float32)
    elif not rr < eps:
        p = r.copy()
        a = rr
        while True:
            if k >= int(d["maxiter"]):
                break
            z = A(p)
            zp = dot(z, p)
            if zp == 0:
                break
            af = np.float32(a / zp)
            x = np.where(mask, x + af * p, np.float32(0)).astype(np.float32)
            r = np.where(mask, r + (-af) * z, np.float32(0)).astype(np.float32)
            rr = dot(r, r)
            if rr < eps:
                k += 1
                break
            bf = np.float32(rr / a)
            p = np.where(mask, r + bf * p, np.float32(0)).astype(np.float32)
            a = rr
            k += 1
    np.savez(os.path.join(outdir, f"x{rank}.npz"), x=x, x0=x0, x1=x1, iters=k, rr=rr, reductions=n_reduce[0])
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _projection_system(mp, oracle_mod, tmp_path):
    """The pressure system of configuration 1 at 32^3 before its projection, and
    the oracle's single-domain solve of it."""
    from parity_util import bubblesim_stages
    p = mp.scene_params(1, 32)
    p.cg_tol_mode, p.cg_tol, p.cg_max_iter = mp.TOL_REF_ABS, 0.01, 800
    o = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    o.upload_particles(**mp.scene_particles(p, 1, 2017_910))
    rf, seeds = mp.scene_tables(p, 1, 2017_910)
    o.set_tables(rf, seeds)
    for st in bubblesim_stages(p, 0):
        if st[0] == "project_CG_bubble":
            break
        getattr(o, st[0])(*st[1:])
    it, res, rc = o.project_CG_bubble()
    shape = (p.nx, p.ny, p.nz)
    inp = tmp_path / "in.npz"
    np.savez(inp, mark=o.get_field("mark").reshape(shape), div=o.get_field("div").reshape(shape), h=p.cellsize,
             tol=p.cg_tol, maxiter=p.cg_max_iter)
    return inp, shape, it, o.get_field("press").reshape(shape)


def _gather(tmp_path, world, shape):
    press = np.zeros(shape, np.float32)
    iters, reductions = set(), set()
    for r in range(world):
        d = np.load(tmp_path / f"x{r}.npz")
        press[int(d["x0"]):int(d["x1"])] = d["x"]
        iters.add(int(d["iters"]))
        reductions.add(int(d["reductions"]))
    assert len(iters) == 1 and len(reductions) == 1
    return press, iters.pop(), reductions.pop()


@pytest.mark.parametrize("world", [2, 4])
def test_slab_cg_equals_the_single_domain_solve(mp, oracle_mod, tmp_path, world):
    inp, shape, it, ref = _projection_system(mp, oracle_mod, tmp_path)
    tmp.spawn(_worker, args=(world, _free_port(), str(inp), str(tmp_path)), nprocs=world, join=True)
    press, iters, reductions = _gather(tmp_path, world, shape)
    assert iters == it and it > 0
    assert reductions == 2 * it + 1                  # r.r at the start, z.p and r.r per iteration
    assert np.array_equal(press, ref), f"max |d| {np.abs(press - ref).max()}"


def test_single_reduction_cg_on_slabs(mp, oracle_mod, tmp_path):
    """The Chronopoulos-Gear form of the CG, which computes both dot products
    of an iteration in one all-reduce: half the reductions (the latency that
    bounds a decomposed solve), the same iteration count within two, and the
    pressure within 1e-5 of the single-domain solve."""
    inp, shape, it, ref = _projection_system(mp, oracle_mod, tmp_path)
    tmp.spawn(_worker, args=(2, _free_port(), str(inp), str(tmp_path), True), nprocs=2, join=True)
    press, iters, reductions = _gather(tmp_path, 2, shape)
    assert abs(iters - it) <= 2
    assert reductions == iters + 2                   # r.r and the first pair at the start, one per iteration
    scale = np.abs(ref).max()
    assert np.abs(press.astype(np.float64) - ref).max() <= 1e-5 * scale


# ---- particle migration -----------------------------------------------------------

PARTS = ["pos", "vel", "flag", "mass", "temp", "lheat", "solubility", "gascontain"]


def _migrate_worker(rank, world, port, inp, outdir):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import importlib
    sl = importlib.import_module("2017multiphase_b200.slab")
    d = np.load(inp)
    dims = tuple(int(x) for x in d["dims"])
    nx, ny, nz = dims
    x0, x1 = sl.partition(nx, ny, nz, world)[rank]
    g0, g1 = x0 * ny * nz, x1 * ny * nz
    mine = (d["old_cell"] >= g0) & (d["old_cell"] < g1)          # this rank's particles before the move
    arrays = {k: d[k][mine] for k in PARTS}
    owner = sl.route_particles(arrays["pos"], float(d["h"]), float(d["gmin"][0]), nx, sl.partition(nx, ny, nz, world))
    got = sl.migrate(arrays, owner, world)
    cell = sl.hash_cells(got["pos"], float(d["h"]), d["gmin"], dims)
    assert ((cell >= g0) & (cell < g1)).all()
    order = np.argsort(cell, kind="stable")                       # sortParticles, on the slab
    out = {k: v[order] for k, v in got.items()}
    cs = cell[order]
    start = np.full(g1 - g0, 0xFFFFFFFF, np.uint32)
    end = np.zeros(g1 - g0, np.uint32)
    for q in range(len(cs)):                                      # reorderDataAndFindCellStartD, by definition
        if q == 0 or cs[q] != cs[q - 1]:
            start[cs[q] - g0] = q
            if q > 0:
                end[cs[q - 1] - g0] = q
        if q == len(cs) - 1:
            end[cs[q] - g0] = q + 1
    np.savez(os.path.join(outdir, f"m{rank}.npz"), start=start, end=end, g0=g0, g1=g1, n=len(cs), **out)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_migration_and_local_sort_equal_the_global_sort(mp, oracle_mod, tmp_path, world):
    """After collision and advection moved the particles, each rank sends its
    particles to the slab of their new cell and sorts what it holds: the
    result is, slab by slab, the single-domain hashAndSortParticles (particle
    order, every attribute, cell ranges)."""
    from parity_util import bubblesim_stages
    p = mp.scene_params(1, 32)
    o = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    o.upload_particles(**mp.scene_particles(p, 1, 2017_920))
    rf, seeds = mp.scene_tables(p, 1, 2017_920)
    o.set_tables(rf, seeds)
    for st in bubblesim_stages(p, 0):
        getattr(o, st[0])(*st[1:])
        if st[0] == "CollisionSolid":
            break
    before = o.download_particles()
    cs, ce = o.get_field("cellstart"), o.get_field("cellend")     # the sort before the move
    old_cell = np.zeros(len(before["pos"]), np.int64)
    for c in np.nonzero(cs != 0xFFFFFFFF)[0]:
        old_cell[cs[c]:ce[c]] = c
    inp = tmp_path / "in.npz"
    np.savez(inp, dims=np.array([p.nx, p.ny, p.nz]), h=p.cellsize, gmin=np.array([p.gmin_x, p.gmin_y, p.gmin_z]),
             old_cell=old_cell, **before)
    tmp.spawn(_migrate_worker, args=(world, _free_port(), str(inp), str(tmp_path)), nprocs=world, join=True)
    o.hashAndSortParticles()
    after = o.download_particles()
    gcs, gce = o.get_field("cellstart"), o.get_field("cellend")
    off = 0
    for r in range(world):
        d = np.load(tmp_path / f"m{r}.npz")
        n, g0, g1 = int(d["n"]), int(d["g0"]), int(d["g1"])
        for k in PARTS:
            assert np.array_equal(d[k], after[k][off:off + n]), (r, k)
        occ = gcs[g0:g1] != 0xFFFFFFFF
        assert np.array_equal(d["start"] != 0xFFFFFFFF, occ)
        assert np.array_equal(d["start"][occ].astype(np.int64) + off, gcs[g0:g1][occ])
        assert np.array_equal(d["end"][occ].astype(np.int64) + off, gce[g0:g1][occ])
        off += n
    assert off == len(after["pos"])
    sl = _slab()
    bounds = sl.partition(p.nx, p.ny, p.nz, world)
    old_rank = sl.owner_of_planes(old_cell // (p.ny * p.nz), bounds)
    new_rank = sl.route_particles(before["pos"], p.cellsize, p.gmin_x, p.nx, bounds)
    assert (old_rank != new_rank).sum() > 0            # particles did cross slab boundaries
