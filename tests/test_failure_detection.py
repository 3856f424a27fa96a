"""Failure detection without a GPU fault: the failures are made on the host.

* A rank that leaves between steps (before the next collective) makes the
  other rank's collective end with an error within the process group's short
  timeout instead of waiting for ever: the pattern bench.py's barrier and
  max-over-ranks reduction rely on.
* A CG that reaches its iteration cap reports MP_ERR_NOCONVERGE (the
  reference paused, spray.cu:1642-1649) and the step carries on.
"""
import datetime
import os
import socket
import time

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as tmp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, outdir):
    import sys
    import torch
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    # one step's worth of collectives together
    t = torch.tensor([float(rank)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 1:
        # the failing rank leaves between steps, with no collective in flight
        np.save(os.path.join(outdir, "r1.npy"), np.array([t.item()]))
        os._exit(0)
    t0 = time.monotonic()
    err = ""
    try:
        dist.barrier()
        t = torch.tensor([0.0], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    except Exception as e:   # the expected outcome: an error, not a hang
        err = type(e).__name__ + ": " + str(e)[:200]
    np.savez(os.path.join(outdir, "r0.npz"), waited=time.monotonic() - t0, err=err)
    os._exit(0)


def test_a_dead_rank_ends_the_next_collective_with_an_error(tmp_path):
    port = _free_port()
    ctx = tmp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=False)
    deadline = time.monotonic() + 120
    while not ctx.join(timeout=5):
        assert time.monotonic() < deadline, "a rank is still waiting"
    r0 = np.load(tmp_path / "r0.npz")
    assert float(np.load(tmp_path / "r1.npy")[0]) == 1.0          # the first step's reduction completed
    assert str(r0["err"]) != ""                                     # the survivor saw the failure
    assert float(r0["waited"]) < 60.0


def test_forced_iteration_cap_reports_noconverge(mp, oracle_mod):
    p = mp.scene_params(1, 16)
    p.cg_max_iter = 2
    p.cg_tol_mode = mp.TOL_REL
    p.cg_tol = 1e-12
    o = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    o.upload_particles(**mp.scene_particles(p, 1, 31))
    rf, seeds = mp.scene_tables(p, 1, 31)
    o.set_tables(rf, seeds)
    o.hashAndSortParticles(); o.addexternalforce(); o.computeLevelset(0.0); o.sweepLSAndMardGrid()
    o.mapvelp2g_bubble()
    for ph in (1, 0):
        o.sweepPhi(ph); o.sweepU(ph)
    o.setWaterBoundaryU(1); o.setWaterBoundaryU(0)
    it, res, rc = o.project_CG_bubble()
    assert rc == mp.MP_ERR_NOCONVERGE and it == 2 and res > 0
    # the whole step carries on past the cap and reports it
    o2 = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    o2.upload_particles(**mp.scene_particles(p, 1, 31))
    o2.set_tables(rf, seeds)
    rc = o2.bubblesim()
    assert rc == mp.MP_ERR_NOCONVERGE and o2.state().frame == 1
