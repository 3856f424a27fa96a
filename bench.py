"""Benchmark: bubblesim steps/s of the bubble-column configuration (256^3).

One step = one full multiphase FLIP time step (cspray::bubblesim,
spray.cpp:979-1233) with marching cubes every step, on ~105M particles.
The path does not shard across GPUs (it is one coupled grid solve), so with
N GPUs every rank runs an independent replica with its own seed ("replicas
only"); value = N*K / max-over-ranks time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FLIP steps/s at 256³ (fwd, fwd+adjoint) at ≤1e-5 rel err; PCG HBM GB/s"
FALLBACK_HBM_GBS = 6650.0
# Algorithmic bytes per cell per launch of the two CG kernels (FP32 vectors,
# int8 marks): k_cg_dir reads r, p_old, mark and writes p_new; k_cg_upd reads
# p, x, r, mark and writes x, r.
CG_DIR_BYTES_PER_CELL = 13
CG_UPD_BYTES_PER_CELL = 21


def names_kt(mp):
    return {mp.KT_CG_STENCIL: "k_cg_dir", mp.KT_CG_UPDATE: "k_cg_upd", mp.KT_P2G: "k_p2g",
            mp.KT_G2P: "k_g2p", mp.KT_SORT: "sort", mp.KT_LEVELSET: "k_genlevelset", mp.KT_MC_DENS: "k_mc_density",
            mp.KT_CORRECT: "k_correct_pos"}


# DRAM bytes per launch from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum),
# as functions of (cells, particles): the capture's bytes scaled by the units a
# launch processes
TRAFFIC_PER_LAUNCH = {
    # the TMA CG passes captured at 256^3: 189.4 MB and 294.5 MB per launch
    "k_cg_dir": lambda n, np_: 189.36e6 * n / 256 ** 3,
    "k_cg_upd": lambda n, np_: 294.46e6 * n / 256 ** 3,
    # the MC density pass captured at 128^3 (12.9M particles): 711.9 MB per
    # launch; nodes and particles both grow with the cells
    "k_mc_density": lambda n, np_: 711.91e6 * n / 128 ** 3,
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=5)
    ap.add_argument("--n", type=int, default=0, help="grid size (0: the configuration's own, 256)")
    ap.add_argument("--seed", type=int, default=2017005)
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="steps of the end-to-end measurement (0: as many as --steps, on the same frames)")
    ap.add_argument("--ref-steps", type=int, default=2, help="reference arm: at most this many timed oracle steps")
    ap.add_argument("--ref-warmup", type=int, default=0, help="reference arm: at most this many warm-up steps")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adj-steps", type=int, default=16, help="steps of the forward+adjoint measurement (0: skip)")
    ap.add_argument("--adj-every", type=int, default=16, help="checkpoint interval of the adjoint")
    ap.add_argument("--class-steps", type=int, default=5,
                    help="steps of the per-kernel-class timing pass after the timed region")
    ap.add_argument("--precision-steps", type=int, default=3,
                    help="steps of the all-FP64 form timed after the main region (0: skip the precision report)")
    ap.add_argument("--profile-case", default="", choices=["", "cg", "step"],
                    help="small-footprint cases for ncu captures instead of the bench line: "
                         "cg = one pressure solve on an n^3 liquid slab (z < 0.8) with a seeded divergence; "
                         "step = one warm-up and one bubblesim step of the configuration at n^3")
    return ap.parse_args()


def replica_seed(base: int, rank: int) -> int:
    """Each rank simulates its own replica of the workload."""
    return base + rank


def aggregate_steps_per_s(world: int, steps: int, max_ms: float) -> float:
    """Whole-job throughput: all ranks' steps over the slowest rank's time."""
    return world * steps / (max_ms / 1e3)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush(); self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1])); mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def workload_config(p, npart0, seed, world):
    """The `config` object of both arms' JSON lines (the same workload)."""
    return {"workload": f"bubble column {p.nx}^3: liquid z<0.8, 200 air bubbles r~U[0.01,0.04], "
                        f"8 jittered particles/cell, dt=1/{1.0 / p.dt:.0f} (1/240 x (64/n)^2), FLIP 0.95, "
                        f"constant-coefficient projection (the reference's; coef_mode ref), "
                        f"CG rel 1e-6, marching cubes every step",
            "grid": p.nx, "particles": int(npart0), "seed": seed,
            "l2": (f"inputs larger than L2 (the three particle streams alone are {48 * npart0 / 1e9:.1f} GB)"
                   if 48 * npart0 > 126e6 else
                   f"inputs smaller than L2 ({48 * npart0 / 1e6:.0f} MB of particle streams): a reduced grid"),
            "parallelism": f"replicas x{world}"}


def oracle_steps(config, n, seed, steps, warm, threads=None):
    """The CPU oracle (the reference step restated in C++, OpenMP over the
    host cores) on configuration `config` at n^3, built from the oracle's own
    scene inputs (oracle/scene.py: nothing of the product is loaded). Returns
    (per-step seconds, threads, initial particles, params)."""
    from oracle import scene
    threads = threads or os.cpu_count() or 1
    orc, p, npart = scene.make_oracle(config, n, seed, threads=threads)
    for _ in range(warm):
        orc.bubblesim()
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        orc.bubblesim()
        times.append(time.perf_counter() - t)
    return times, threads, npart, p


def cpu_baseline(config, n, seed, single_n=64):
    """The GPU arm's `cpu_baseline`: one whole oracle step of the same
    configuration at n^3 on all host threads (no warm-up), and beside it one
    whole step on a single host thread at min(single_n, n)^3, a grid that one
    thread finishes in seconds (reported as measured, not scaled to n^3)."""
    t0 = time.perf_counter()
    times, threads, npart, _ = oracle_steps(config, n, seed, 1, 0)
    out = {"value": 1.0 / times[0], "unit": "steps/s", "cores": threads, "kind": "port",
           "sample": f"one whole oracle step of the same configuration at {n}^3 ({npart} particles, "
                     f"{times[0]:.1f} s; {time.perf_counter() - t0:.0f} s with set-up), no warm-up"}
    n1 = min(single_n, n)
    try:
        times1, _, npart1, _ = oracle_steps(config, n1, seed, 1, 0, threads=1)
    finally:   # the oracle's thread count is process-wide: put it back
        from oracle import oracle as orc_lib
        orc_lib.load().or_set_threads(threads)
    out["single_thread"] = {"value": 1.0 / times1[0], "unit": "steps/s", "cores": 1, "kind": "port",
                            "sample": f"one whole oracle step of the same configuration at {n1}^3 on one host "
                                      f"thread ({npart1} particles, {times1[0]:.1f} s), no warm-up; a smaller "
                                      f"grid, not scaled"}
    return out


def run_reference(args, rank):
    """The reference arm: whole oracle steps of the same configuration at the
    same grid on the host cores. A step at 256^3 takes minutes on the CPU, so
    it times min(steps, --ref-steps) steps after min(warmup, --ref-warmup)."""
    if rank != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    n = args.n or 256
    steps = max(1, min(args.steps, args.ref_steps))
    warm = min(args.warmup, args.ref_warmup)
    t0 = time.perf_counter()
    times, threads, npart, p = oracle_steps(args.config, n, replica_seed(args.seed, rank), steps, warm)
    per_step = sum(times) / len(times)
    value = 1.0 / per_step
    sample = (f"{steps} whole oracle step(s) of the same configuration at {n}^3 ({npart} particles) after "
              f"{warm} warm-up step(s), {threads} host threads; {time.perf_counter() - t0:.0f} s including set-up")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
           "steps": steps, "steps_requested": args.steps, "warmup": warm, "ms_per_step": per_step * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (CG dots in f64)",
           "data": "synthetic", "config": workload_config(p, npart, args.seed, world),
           "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def profile_case(args):
    """Cases sized for ncu: the device holds a few GB at most. Prints the
    kernel-class timings of the measured part (CUDA events)."""
    import importlib
    import numpy as np
    import torch
    mp = importlib.import_module("2017multiphase_b200")
    n = args.n or 256
    if args.profile_case == "cg":
        p = mp.scene_params(args.config, n)
        p.par_num_max = 16
        p.b_run_mc = 0
        sim = mp.Sim(p)
        mark = np.zeros((n, n, n), np.int8)
        mark[:, :, int(0.8 * n):] = mp.TYPEVACUUM
        mark[0], mark[-1] = mp.TYPEBOUNDARY, mp.TYPEBOUNDARY
        mark[:, 0], mark[:, -1] = mp.TYPEBOUNDARY, mp.TYPEBOUNDARY
        mark[:, :, 0], mark[:, :, -1] = mp.TYPEBOUNDARY, mp.TYPEBOUNDARY
        sim.set_field("mark", mark.ravel())
        sim.set_field("lsmerge", np.full(n ** 3, -0.5 / n, np.float32))
        rng = np.random.default_rng(args.seed)
        for f, cnt in [("waterux", (n + 1) * n * n), ("wateruy", n * (n + 1) * n), ("wateruz", n * n * (n + 1))]:
            sim.set_field(f, (0.01 * rng.standard_normal(cnt)).astype(np.float32))
        classes = {mp.KT_CG_STENCIL: ("k_cg_dir", CG_DIR_BYTES_PER_CELL), mp.KT_CG_UPDATE: ("k_cg_upd", CG_UPD_BYTES_PER_CELL)}
        for k in classes:
            sim.kernel_timing(k, True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, res, rc = sim.project_CG_bubble()
        torch.cuda.synchronize()
        out = {"case": "cg", "n": n, "iterations": it, "rc": rc, "solve_ms": (time.perf_counter() - t0) * 1e3}
        for k, (nm, bpc) in classes.items():
            ms, nl = sim.kernel_timing_read(k)
            per = ms / max(nl, 1)
            out[nm] = {"launches": nl, "us_per_launch": per * 1e3, "algorithmic_GBps": bpc * n ** 3 / (per / 1e3) / 1e9}
    else:
        sim = mp.Sim.from_config(args.config, n, args.seed)
        sim.bubblesim()
        classes = names_kt(mp)
        for k in classes:
            sim.kernel_timing(k, True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.bubblesim()
        torch.cuda.synchronize()
        out = {"case": "step", "n": n, "config": args.config, "step_ms": (time.perf_counter() - t0) * 1e3,
               "particles": int(sim.state().par_num_now)}
        for k, nm in classes.items():
            ms, nl = sim.kernel_timing_read(k)
            out[nm] = {"launches": nl, "ms": ms}
    print(json.dumps(out), flush=True)
    sim.close()


# the stages of bubblesim before the projection (spray.cpp:979-1233), bubble scenes
PRE_PROJECTION = [("hashAndSortParticles",), ("addexternalforce",), ("computeLevelset", 0.0),
                  ("sweepLSAndMardGrid",), ("markSoloAirParticle",), ("computesurfacetension",),
                  ("mapvelp2g_bubble",), ("enforceDragForce",), ("sweepPhi", 1), ("sweepU", 1), ("sweepPhi", 0),
                  ("sweepU", 0), ("setWaterBoundaryU", 1), ("setWaterBoundaryU", 0)]
STEP_FIELDS = ["press", "waterux", "wateruy", "wateruz", "airux", "airuy", "airuz", "lsmerge"]


def rel_l2(a, b):
    import numpy as np
    a = np.asarray(a, np.float64).ravel(); b = np.asarray(b, np.float64).ravel()
    den = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a))


def precision_report(sim, mp, stream, fp64_steps):
    """The mixed FP32/FP64 form against the all-FP64 form on the bench's own
    state: (1) one projection from the same faces solved three ways -- FP64 to
    a relative residual of 1e-12 (the exact pressure to FP64 precision), the
    FP64 form and the mixed form at the configuration's stop rule -- with each
    form's relative L2 pressure error against the first and its solve time;
    (2) one whole step from the same checkpoint in each form, with the
    relative L2 difference of every output field; (3) the FP64 form's
    steps/s over `fp64_steps` steps (CUDA events on the context stream)."""
    import numpy as np
    import torch
    p0 = sim.get_params()
    for st in PRE_PROJECTION:
        getattr(sim, st[0])(*st[1:])
    faces = {f: sim.get_field(f) for f in ["waterux", "wateruy", "wateruz", "airux", "airuy", "airuz"]}

    def solve(prec, tol, maxit, refine=0.0):
        p = sim.get_params()
        p.precision, p.cg_tol, p.cg_max_iter, p.cg_refine_tol = prec, tol, maxit, refine
        sim.set_params(p)
        for f, a in faces.items():
            sim.set_field(f, a)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        it, _, rc = sim.project_CG_bubble()
        e1.record(stream)
        torch.cuda.synchronize()
        return sim.get_field("press"), it, rc, e0.elapsed_time(e1)

    pref, it_ref, rc_ref, _ = solve(mp.PREC_FP64, 1e-12, 20000)
    p64, it64, rc64, ms64 = solve(mp.PREC_FP64, p0.cg_tol, p0.cg_max_iter)
    p32, it32, rc32, ms32 = solve(mp.PREC_MIXED, p0.cg_tol, p0.cg_max_iter)
    pr, itr, rcr, msr = solve(mp.PREC_MIXED, p0.cg_tol, p0.cg_max_iter, refine=1e-3)
    out = {"projection": {
        "reference": f"FP64 CG to relative residual 1e-12 ({it_ref} iterations, rc {rc_ref})",
        "mixed": {"pressure_rel_err": rel_l2(p32, pref), "iterations": it32, "solve_ms": ms32, "rc": rc32},
        "mixed_refined": {"pressure_rel_err": rel_l2(pr, pref), "iterations": itr, "solve_ms": msr, "rc": rcr,
                          "what": "FP32-vector CG corrections to 1e-3, solution and true residual in FP64, "
                                  "stop on the FP64 true residual"},
        "fp64": {"pressure_rel_err": rel_l2(p64, pref), "iterations": it64, "solve_ms": ms64, "rc": rc64}}}
    sim.set_params(p0)
    # one whole step from the same state in each form
    blob = sim.checkpoint()
    snaps = {}
    for name, prec in (("fp64", mp.PREC_FP64), ("mixed", mp.PREC_MIXED)):
        sim.set_params(p0)
        sim.restore(blob)
        p = sim.get_params(); p.precision = prec; sim.set_params(p)
        sim.bubblesim()
        snaps[name] = {f: sim.get_field(f) for f in STEP_FIELDS}
        parts = sim.download_particles()
        v = parts["vel"].astype(np.float64)
        gas = (parts["flag"] == mp.TYPEAIR) | (parts["flag"] == mp.TYPEAIRSOLO)
        snaps[name]["particle_kinetic_energy"] = float((parts["mass"] * (v * v).sum(1)).sum())
        snaps[name]["gas_particle_mean_z"] = float(parts["pos"][gas, 2].astype(np.float64).mean())
        snaps[name]["particles"] = len(parts["flag"])
    # per cell / face: relative L2 difference; particles (whose order after the
    # step's re-sorts is not comparable index by index): whole-domain sums
    out["step_fields_rel_l2"] = {f: rel_l2(snaps["mixed"][f], snaps["fp64"][f]) for f in STEP_FIELDS
                                 if snaps["mixed"][f].shape == snaps["fp64"][f].shape}
    out["step_particles_rel"] = {q: abs(snaps["mixed"][q] - snaps["fp64"][q]) / max(abs(snaps["fp64"][q]), 1e-30)
                                 for q in ("particle_kinetic_energy", "gas_particle_mean_z", "particles")}
    # the FP64 form's throughput
    sim.set_params(p0)
    sim.restore(blob)
    p = sim.get_params(); p.precision = mp.PREC_FP64; sim.set_params(p)
    sim.bubblesim()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(fp64_steps):
        sim.bubblesim()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out["fp64_form"] = {"value": fp64_steps / (ms / 1e3), "unit": "steps/s", "steps": fp64_steps,
                        "ms_per_step": ms / fp64_steps,
                        "what": "the same step with the projection (divergence, CG vectors and scalars, "
                                "gradient) and the heat solve in FP64"}
    sim.set_params(p0)
    return out


def fwd_adjoint(args, n, local, dist):
    """Forward + adjoint throughput of the two-phase program the adjoint covers
    on the bubble column (configuration 5's scene and step at the bench's
    grid, FLUID and AIR particles, position correction off, without the
    solo-air stages): the recorded engine steps plus the gradient of the loss
    with respect to the initial particle velocities (FP32 replay and
    transpose, checkpoints every --adj-every steps), timed with CUDA events on
    the context's stream, max over ranks."""
    import importlib
    import torch
    mp = importlib.import_module("2017multiphase_b200")
    p = mp.scene_params(5, n)
    p.b_correct_position = 0
    p.b_run_mc = 0   # the recorded program extracts no surface
    sim = mp.Sim.from_config(5, n, replica_seed(2017005, int(os.environ.get("RANK", "0"))), params=p)
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    targets = mp.dam_break_targets(4096, 2017005, height=0.7)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    sim.adj_record(args.adj_steps, args.adj_every)
    e1.record(stream)
    sim.adj_set_targets(targets)
    loss, grad = sim.adj_gradient(None, mp.PREC_MIXED)
    e2.record(stream)
    torch.cuda.synchronize()
    fwd_ms, adj_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    tot = fwd_ms + adj_ms
    if dist:
        t = torch.tensor([tot], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot = float(t.item())
    world = int(os.environ.get("WORLD_SIZE", "1"))
    res = {"value": world * args.adj_steps / (tot / 1e3), "unit": "steps/s", "steps": args.adj_steps,
           "checkpoint_every": args.adj_every, "fwd_ms_per_step": fwd_ms / args.adj_steps,
           "adjoint_ms_per_step": adj_ms / args.adj_steps, "particles": sim.adj_num_particles(),
           "loss": loss, "grad_norm": float(grad.norm()),
           "workload": f"bubble column {n}^3 (liquid z<0.8 with AIR bubbles; FLUID and AIR, the two-phase "
                       f"projection; position correction and the solo-air stages off), "
                       f"loss = sum phi^2 of the fluid level set on 4096 target points at z=0.7, dL/dv0 in FP32"}
    sim.close()
    return res


def e2e_run(mp, args, rank, world, dist, mesh_max):
    """End to end through the public API with host buffers: a fresh engine
    from the same configuration and seed (the engine is deterministic, so
    after the same warm-up it steps through the same frames as the timed
    region), then `e2e_steps` steps (default: as many as the timed ones),
    each uploading its host inputs (random table and nucleation cells) from
    pinned memory and downloading the three extracted meshes into host
    buffers sized from `mesh_max` (the largest vertex and index counts of the
    timed steps). Wall clock around the steps, max over ranks."""
    import numpy as np
    import torch
    import ctypes as C
    steps = args.e2e_steps if args.e2e_steps > 0 else args.steps
    sim = mp.Sim.from_config(args.config, args.n, replica_seed(args.seed, rank))
    p = sim.params
    for _ in range(args.warmup):
        sim.bubblesim()
    torch.cuda.synchronize()
    rf, seeds = mp.scene_tables(p, args.config, replica_seed(args.seed, rank))
    rf_pin = torch.empty(rf.size, dtype=torch.float32, pin_memory=True).numpy(); rf_pin[:] = rf
    sd_pin = torch.empty(max(seeds.size, 1), dtype=torch.int32, pin_memory=True).numpy()[:seeds.size]; sd_pin[:] = seeds
    # twice the largest mesh of the timed steps, which were the same frames
    # when e2e_steps <= steps (the download reports a capacity error if a
    # mesh were larger)
    cap_v = min(p.mc_max_verts, max(2 * mesh_max[0], 1024))
    cap_i = min(3 * p.mc_max_tris, max(2 * mesh_max[1], 3072))
    vbuf = torch.empty((cap_v, 3), dtype=torch.float32, pin_memory=True).numpy()
    nbuf = torch.empty((cap_v, 3), dtype=torch.float32, pin_memory=True).numpy()
    ibuf = torch.empty(cap_i, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    h2d = rf_pin.nbytes + sd_pin.nbytes
    d2h = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.set_tables(rf_pin, sd_pin)
        sim.bubblesim()
        st = sim.state()
        for s in range(3):
            nv, ni = st.mc_verts[s], st.mc_indices[s]
            rc = sim.lib.mp_mc_download(sim.ctx, s, vbuf.ctypes.data_as(C.c_void_p), nbuf.ctypes.data_as(C.c_void_p),
                                        ibuf.ctypes.data_as(C.c_void_p), cap_v, cap_i)
            if rc:
                raise RuntimeError(f"mesh download failed {rc}")
            d2h += 24 * nv + 4 * ni
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * steps / e2e_s, "unit": "steps/s",
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h / max(steps, 1))}
    sim.close()
    return e2e


def main():
    args = parse()
    if args.profile_case:
        profile_case(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import importlib
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    mp = importlib.import_module("2017multiphase_b200")

    sim = mp.Sim.from_config(args.config, args.n, replica_seed(args.seed, rank))
    p = sim.params
    n = p.nx * p.ny * p.nz
    npart0 = int(sim.state().par_num_now)
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    for _ in range(args.warmup):
        sim.bubblesim()
    torch.cuda.synchronize()

    classes = [mp.KT_CG_STENCIL, mp.KT_CG_UPDATE, mp.KT_P2G, mp.KT_G2P, mp.KT_SORT, mp.KT_LEVELSET, mp.KT_MC_DENS,
               mp.KT_CORRECT]
    # the timed region runs with no per-kernel timing events (they would sit
    # between the launches); the per-class breakdown is a separate pass below
    sim.kernel_timing_reset()
    clocks = ClockSampler(local)
    clocks.start()
    cg_iters = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    mesh_max = [0, 0]
    for _ in range(args.steps):
        sim.bubblesim()
        st = sim.state()
        cg_iters += st.last_cg_iters
        mesh_max = [max(mesh_max[0], *st.mc_verts), max(mesh_max[1], *st.mc_indices)]
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = sim.launch_count()
    # per-class device time (CUDA events around every launch of a class) over
    # further steps of the same run
    class_steps = max(1, min(args.steps, args.class_steps))
    sim.kernel_timing_reset()
    for k in classes:
        sim.kernel_timing(k, True)
    for _ in range(class_steps):
        sim.bubblesim()
    kt = {k: sim.kernel_timing_read(k) for k in classes}
    work_counts = sim.work_counts()
    for k in classes:
        sim.kernel_timing(k, False)
    t_max = ms
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = aggregate_steps_per_s(world, args.steps, t_max)

    # roofline of the dominant kernel class (by device time in the timed
    # region); algorithmic bytes from the compulsory-traffic model (each byte
    # a launch must move, counted once; N_p particles, n cells), per unit of
    # work: a CG iteration for the CG passes (launches of an iteration batch
    # after the stop test are not counted), a call otherwise; a sort that
    # found the particles in cell order moves only positions and ranges
    peak, peak_kind = peaks()
    npart = int(sim.state().par_num_now)
    wc = work_counts
    model = {mp.KT_CG_STENCIL: ("k_cg_tma<PressOp,0> (direction p = r + beta p, A p, p.Ap)",
                                CG_DIR_BYTES_PER_CELL * n * wc["cg_iters"], wc["cg_iters"]),
             mp.KT_CG_UPDATE: ("k_cg_tma<PressOp,1> (A p, x and r update, r.r)",
                               CG_UPD_BYTES_PER_CELL * n * wc["cg_iters"], wc["cg_iters"]),
             mp.KT_P2G: ("k_p2g_water + k_p2g_air (water + air launches)", (29 * npart + 56 * n) * kt[mp.KT_P2G][1],
                         kt[mp.KT_P2G][1]),
             mp.KT_G2P: ("k_g2p", (37 * npart + 72 * n) * kt[mp.KT_G2P][1], kt[mp.KT_G2P][1]),
             mp.KT_SORT: ("hash sort (count, scan, scatter, segment sort, gather)",
                          (102 * npart + 8 * n) * wc["sort_full"] + (12 * npart + 8 * n) * wc["sort_fast"],
                          wc["sort_full"] + wc["sort_fast"]),
             mp.KT_LEVELSET: ("k_genlevelset", (13 * npart + 9 * n) * kt[mp.KT_LEVELSET][1], kt[mp.KT_LEVELSET][1]),
             mp.KT_MC_DENS: ("k_mc_density (fused fluid + gas fields at 2x)", (13 * npart + 64 * n) * kt[mp.KT_MC_DENS][1],
                             kt[mp.KT_MC_DENS][1]),
             # read each position record and neighbour mass, write the corrected record; cell ranges
             mp.KT_CORRECT: ("k_correct_pos (particle spacing spring)", (36 * npart + 4 * n) * kt[mp.KT_CORRECT][1],
                             kt[mp.KT_CORRECT][1])}
    dom = max(model, key=lambda k: kt[k][0])
    ms_k = kt[dom][0]
    units = max(model[dom][2], 1)
    per_unit_s = ms_k / 1e3 / units
    alg = model[dom][1] / units
    achieved = alg / per_unit_s / 1e9
    traffic = TRAFFIC_PER_LAUNCH.get(names_kt(mp)[dom])
    cg_ms = kt[mp.KT_CG_STENCIL][0] + kt[mp.KT_CG_UPDATE][0]
    pcg_gbs = (CG_DIR_BYTES_PER_CELL + CG_UPD_BYTES_PER_CELL) * n * max(wc["cg_iters"], 1) / (cg_ms / 1e3) / 1e9
    names = names_kt(mp)
    psrc = f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback"
    roof = {"kernel": model[dom][0], "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": psrc,
            "traffic": (traffic(n, npart) if traffic else None), "algorithmic_bytes_per_launch": alg,
            "avg_launch_ms": per_unit_s * 1e3}
    cls_table = {}
    for k, (nm, b, u) in model.items():
        ms_c, nl_c = kt[k]
        if nl_c and ms_c > 0:
            a = b / (ms_c / 1e3) / 1e9
            cls_table[names[k]] = {"ms": ms_c, "launches": nl_c, "work_units": u, "algorithmic_GBps": a,
                                   "frac": a / peak}
    cls_table["sort"]["calls_reordering"] = wc["sort_full"]
    cls_table["sort"]["calls_in_order"] = wc["sort_fast"]
    cls_table["steps"] = class_steps
    cls_table["note"] = ("device time per class from CUDA events around its launches over the steps after the "
                         "timed region (frames differ from the timed ones); ms are totals over those steps")

    st = sim.state()
    out = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 (CG dots, alpha/beta in f64)", "data": "synthetic",
           "config": workload_config(p, npart0, args.seed, world),
           "roofline": roof, "pcg_hbm_gbs": pcg_gbs,
           "pcg_roofline": {"achieved": pcg_gbs, "peak": peak, "unit": "GB/s", "frac": pcg_gbs / peak,
                            "note": "both CG passes, 34 B/cell/iteration algorithmic, per CG iteration"},
           "cg_iters_per_step": cg_iters / max(args.steps, 1),
           "mesh": {"verts": [int(v) for v in st.mc_verts], "triangles": [int(v) // 3 for v in st.mc_indices]},
           "kernel_classes": cls_table,
           "e2e": None, "gpu_launches": int(launches), "clocks": clk}
    nx = p.nx
    if args.precision_steps > 0:
        out["precision"] = precision_report(sim, mp, stream, args.precision_steps)
        out["pressure_rel_err"] = out["precision"]["projection"]["mixed"]["pressure_rel_err"]
    sim.close()
    out["e2e"] = e2e_run(mp, args, rank, world, dist, mesh_max)
    if args.adj_steps > 0:
        out["fwd_adjoint"] = fwd_adjoint(args, nx, local, dist)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(args.config, nx, args.seed)
        except Exception as e:   # the baseline is reported, not required
            out["cpu_baseline"] = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
                                   "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
