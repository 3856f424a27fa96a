"""x-slab decomposition of the grid across ranks: the host-side plan.

The reference is a single-GPU program; this is the plan by which the step's
grid is split over N GPUs, one rank per GPU.  The grid is row-major with x
slowest (farray, utility.h:49-63; getidx, spray_k.cu:66-69), so the x-planes
[x0, x1) of a rank, with g ghost planes on each side, are one contiguous range
of every cell array (and of every face array, whose x extent is one plane
longer for ux).

Ghost planes each stage needs, from its stencil (in simulation-grid planes):

* 1: the projection (computeAx_bubble spray_k.cu:3423-3447,
  cptdivergence_bubble2 :3138-3263, subGradPress :198-224), one pass of the
  level-set and velocity sweeps (sweepphibytype :771-788, sweepu_k_bubble
  :3779-3880), the water P2G (mapvelp2g_k_fluidSolid, cells -1..0 / -1..1 per
  axis, :2829-2871), G2P and collision (trilinear reads of one cell and its
  upper neighbour, :111-122);
* 2: genlevelset's 5-cell window (:2774-2806) and the air P2G's -2..+1 cells
  (mapvelp2g_k_air, :2894-2937);
* 1 (= 2 planes of the 2x grid): the marching-cubes density window
  (genWaterDensfield_*, :1595-1772).

Reductions (the CG's dot products, spray.cu:1101-1116): each rank sums its
cells in FP64 in fixed blocks of BLOCK consecutive global cells, the blocks'
partial sums are combined with one all-reduce of a vector in which each block
has exactly one non-zero contributor (so the all-reduce adds only zeros to
it), and every rank then adds the blocks in global order.  The result does not
depend on the number of ranks, and equals a single-domain sum over the same
blocks bit for bit.  partition() therefore puts every slab boundary on a block
boundary.

Particles belong to the rank whose slab holds their cell, the cell of
calcHashD's getijkfrompos (spray_k.cu:51-57): a coordinate outside the grid
maps to cell 0.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

BLOCK = 4096

# ghost planes per stage (simulation-grid planes), from the stencils above
HALO = {
    "project": 1, "sweep_pass": 1, "p2g_water": 1, "g2p": 1, "collide": 1,
    "levelset": 2, "p2g_air": 2, "mc_density": 1,
}


def plane_unit(ny: int, nz: int, block: int = BLOCK) -> int:
    """The fewest x-planes whose cell count is a multiple of `block`."""
    return block // math.gcd(block, ny * nz)


def partition(nx: int, ny: int, nz: int, world: int, block: int = BLOCK) -> List[Tuple[int, int]]:
    """[(x0, x1)] per rank: contiguous x-slabs covering the grid, every
    boundary on a reduction block boundary, sizes within one plane unit of
    each other.  Raises ValueError when a rank would get no planes."""
    if world < 1:
        raise ValueError("world must be >= 1")
    unit = plane_unit(ny, nz, block)
    units = -(-nx // unit)                       # the last unit may be short
    if units < world:
        raise ValueError(f"{nx} planes in units of {unit} do not give {world} ranks a slab each")
    out = []
    for r in range(world):
        u0, u1 = r * units // world, (r + 1) * units // world
        out.append((min(u0 * unit, nx), min(u1 * unit, nx)))
    return out


def owner_of_planes(i: np.ndarray, bounds: Sequence[Tuple[int, int]]) -> np.ndarray:
    """The rank owning each x-plane index."""
    starts = np.array([b[0] for b in bounds])
    return np.searchsorted(starts, np.asarray(i), side="right") - 1


def hash_cells(pos: np.ndarray, cellsize: float, gmin: Sequence[float], dims: Sequence[int]) -> np.ndarray:
    """calcHashD's cell index of each particle (getijkfrompos, spray_k.cu:51-57,
    and getidx): (pos - gmin) / cellsize per axis in float32, truncated, an
    axis outside the grid giving 0."""
    p = np.asarray(pos, np.float32).reshape(-1, 3)
    ijk = []
    for a in range(3):
        u = (p[:, a] - np.float32(gmin[a])) / np.float32(cellsize)
        ijk.append(np.where((u >= 0) & (u < dims[a]), u.astype(np.int64), 0))
    return (ijk[0] * dims[1] + ijk[1]) * dims[2] + ijk[2]


def route_particles(pos: np.ndarray, cellsize: float, gmin_x: float, nx: int,
                    bounds: Sequence[Tuple[int, int]]) -> np.ndarray:
    """The owning rank of each particle (float32 positions, (n, 3))."""
    x = (np.asarray(pos, np.float32)[:, 0] - np.float32(gmin_x)) / np.float32(cellsize)
    i = np.where((x >= 0) & (x < nx), x.astype(np.int64), 0)
    return owner_of_planes(i, bounds)


def migrate(arrays: dict, owner: np.ndarray, world: int) -> dict:
    """Moves particles to the ranks `owner` names, over torch.distributed
    all-to-all.  Every rank receives the particles sent to it in source-rank
    order, each source's in its own order.  A rank's slice of the previous
    (cell-sorted) particle array is in global order, and slabs follow in rank
    order, so the received particles are in the global previous order.  A
    local stable sort by cell then gives the slab exactly its part of the
    single-domain stable sort."""
    import torch
    import torch.distributed as dist
    owner = np.asarray(owner, np.int64)
    order = np.argsort(owner, kind="stable")
    send_counts = torch.from_numpy(np.bincount(owner, minlength=world).astype(np.int64))
    recv_counts = torch.empty(world, dtype=torch.int64)
    dist.all_to_all_single(recv_counts, send_counts)
    sc, rc = send_counts.tolist(), recv_counts.tolist()
    out = {}
    for name, a in arrays.items():
        a = np.ascontiguousarray(np.asarray(a)[order])
        w = a.dtype.itemsize * int(np.prod(a.shape[1:], dtype=np.int64))     # bytes per particle
        b = a.view(np.uint8).reshape(len(a), w)
        pad = (-w) % 4                                                      # sent as int32 words
        if pad:
            b = np.concatenate([b, np.zeros((len(b), pad), np.uint8)], axis=1)
        send = torch.from_numpy(np.ascontiguousarray(b).view(np.int32))
        recv = torch.empty((sum(rc), send.shape[1]), dtype=torch.int32)
        dist.all_to_all_single(recv, send, rc, sc)
        rb = np.ascontiguousarray(recv.numpy().view(np.uint8)[:, :w])
        out[name] = rb.view(a.dtype).reshape((sum(rc),) + a.shape[1:])
    return out


def block_range(x0: int, x1: int, ny: int, nz: int, block: int = BLOCK) -> Tuple[int, int]:
    """The global reduction blocks [b0, b1) a slab owns."""
    g0, g1 = x0 * ny * nz, x1 * ny * nz
    return g0 // block, -(-g1 // block)


def block_partials(a: np.ndarray, b: np.ndarray, block: int = BLOCK) -> np.ndarray:
    """FP64 sums of a*b over consecutive blocks of a slab's owned cells (its
    first cell on a block boundary), each summed in cell order."""
    prod = np.asarray(a, np.float64).ravel() * np.asarray(b, np.float64).ravel()
    nb = -(-prod.size // block)
    out = np.empty(nb)
    for q in range(nb):
        out[q] = np.cumsum(prod[q * block:(q + 1) * block])[-1]
    return out


def combine_blocks(total_blocks: int, b0: int, partials: np.ndarray, all_reduce=None) -> float:
    """The global dot product from this rank's block partials: placed in a
    vector of all blocks (zero elsewhere), summed across ranks by `all_reduce`
    (a callable reducing a float64 numpy vector in place, e.g. over
    torch.distributed), then added in block order."""
    v = np.zeros(total_blocks)
    v[b0:b0 + len(partials)] = partials
    if all_reduce is not None:
        all_reduce(v)
    s = 0.0
    for x in v:
        s += x
    return s


def combine_blocks_many(total_blocks: int, b0: int, partials: Sequence[np.ndarray], all_reduce=None) -> List[float]:
    """Several dot products from one all-reduce: the block vectors of each are
    stacked, reduced together and each added in block order (a CG that needs
    two dot products per iteration pays one reduction's latency for both)."""
    v = np.zeros((len(partials), total_blocks))
    for q, part in enumerate(partials):
        v[q, b0:b0 + len(part)] = part
    flat = v.reshape(-1)
    if all_reduce is not None:
        all_reduce(flat)
    out = []
    for q in range(len(partials)):
        s = 0.0
        for x in flat[q * total_blocks:(q + 1) * total_blocks]:
            s += x
        out.append(s)
    return out


def exchange_ghosts(ext, rank: int, world: int, width: int = 1) -> None:
    """Fills the `width` ghost planes on each side of `ext` (a tensor of shape
    (owned planes + 2*width, ny, nz)) with the neighbouring ranks' edge planes,
    over torch.distributed point-to-point; the ghost planes beyond the grid's
    ends are left as they are.  Every rank calls it at the same point."""
    import torch.distributed as dist
    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, ext[width:2 * width].contiguous(), rank - 1))
        ops.append(dist.P2POp(dist.irecv, ext[:width], rank - 1))
    if rank < world - 1:
        ops.append(dist.P2POp(dist.isend, ext[-2 * width:-width].contiguous(), rank + 1))
        ops.append(dist.P2POp(dist.irecv, ext[-width:], rank + 1))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def torch_all_reduce(v: np.ndarray) -> None:
    """combine_blocks' all-reduce over torch.distributed (SUM, in place)."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(v)
    dist.all_reduce(t)
