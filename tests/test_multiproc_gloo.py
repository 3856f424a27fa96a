"""The N>1 host path of bench.py on CPU: two gloo ranks each step an independent
replica (its own seed) of a small configuration with the oracle, reduce their
times with MAX and compute the whole-job throughput. The step does not shard
(replicas only), so no collective touches the data path."""
import os
import socket

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
    import importlib
    import sys
    import time
    import torch
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    mp = importlib.import_module("2017multiphase_b200")
    from oracle import oracle as oracle_mod
    seed = bench.replica_seed(900, rank)
    p = mp.scene_params(1, 12)
    o = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables(), threads=1)
    o.upload_particles(**mp.scene_particles(p, 1, seed))
    rf, seeds = mp.scene_tables(p, 1, seed)
    o.set_tables(rf, seeds)
    dist.barrier()
    t0 = time.perf_counter()
    o.bubblesim()
    ms = (time.perf_counter() - t0) * 1e3
    t = torch.tensor([ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    value = bench.aggregate_steps_per_s(world, 1, float(t.item()))
    np.savez(os.path.join(outdir, f"r{rank}.npz"), press=o.get_field("press"), ms=ms, max_ms=float(t.item()),
             value=value, seed=seed)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas(tmp_path):
    port = _free_port()
    tmp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r0 = np.load(tmp_path / "r0.npz"); r1 = np.load(tmp_path / "r1.npz")
    assert int(r0["seed"]) != int(r1["seed"])
    assert float(r0["max_ms"]) == float(r1["max_ms"]) == max(float(r0["ms"]), float(r1["ms"]))
    assert abs(float(r0["value"]) - 2 / (float(r0["max_ms"]) / 1e3)) < 1e-9
    assert not np.array_equal(r0["press"], r1["press"])      # independent replicas
