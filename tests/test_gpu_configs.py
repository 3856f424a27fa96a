"""GPU-vs-oracle parity at the configurations' own grids, on non-cubic grids,
and over the configurations' step counts (bubblesim, spray.cpp:979-1233).

* One whole step at the configuration's grid: pool boiling at 64^3 and
  melting/freezing at 128^3 (about 8M particles), float fields within 1e-5
  relative of the oracle.
* Every stage of the step on a 32 x 24 x 30 grid, whose k-rows do not split
  into groups of four (the CG's plane-marching path) and whose extents differ
  (the kernels index the three separately): bit-exact or 1e-5 as in the 32^3
  stage tests.
* Drift over many steps. The GPU and the oracle add the CG's FP64 dot
  products in different orders, so their pressures differ in the last bits;
  over many steps those differences grow through the advection and through
  threshold decisions (cell marks, gas generation, melting). The stated bounds
  below are relative L2 errors of the grid fields and of the particle
  attributes, the fraction of differing cell marks, and the relative
  difference of the particle counts, after the configurations' step counts:
  20 steps of the rising bubble (32^3, its own grid), 100 steps of pool
  boiling and 200 steps of melting/freezing, on a 32^3 grid so that the
  oracle's run takes seconds.
"""
import numpy as np
import pytest

from parity_util import (bubblesim_stages, check_one_step, compare, drift, grid_params, make_pair, rel_err,
                         snapshot, transplant)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("config,n", [(2, 64), (3, 128)])
def test_one_step_at_configuration_grid(mp, oracle_mod, config, n):
    sim, orc = make_pair(mp, oracle_mod, config, n, 2017_200 + config)
    check_one_step(sim, orc, config)
    sim.close()


SHAPE = (32, 24, 30)
TOLERANT = {"project_CG_bubble", "updateTemperature", "GenerateGasParticle", "updateSoloAirParticle"}


@pytest.mark.parametrize("config", [1, 2, 3])
@pytest.mark.parametrize("k", range(38))
def test_stage_non_cubic(mp, oracle_mod, config, k):
    p = grid_params(mp, config, *SHAPE)
    stages = bubblesim_stages(p, 0)
    if k >= len(stages):
        pytest.skip("step has fewer stages")
    sim, orc = make_pair(mp, oracle_mod, config, SHAPE[0], 2017_400 + config, params=p)
    for st in stages[:k]:
        getattr(sim, st[0])(*st[1:])
    transplant(sim, orc)
    st = stages[k]
    getattr(sim, st[0])(*st[1:])
    getattr(orc, st[0])(*st[1:])
    tolerant = st[0] in TOLERANT or (st[0] == "solidmotion" and not sim.params.b_fix_solid)
    bad = compare(snapshot(sim), snapshot(orc), exact=not tolerant, rtol=1e-5)
    assert not bad, f"config {config} stage {k} {st}: {bad}"
    sim.close()


@pytest.mark.parametrize("config", [1, 2, 3])
def test_one_step_non_cubic(mp, oracle_mod, config):
    p = grid_params(mp, config, *SHAPE)
    sim, orc = make_pair(mp, oracle_mod, config, SHAPE[0], 2017_500 + config, params=p)
    check_one_step(sim, orc, config)
    sim.close()


# The stated drift. The GPU and the oracle agree bit for bit until the first
# FP32 rounding of a CG scalar or of an SPH force sum falls the other way
# (step 2 of the rising bubble, step ~75 of pool boiling, never in 200 steps
# of melting/freezing at 32^3); from there the difference grows at the flow's
# own rate -- about x10 per step in the rising bubble, whose solo-air SPH
# particles make it chaotic -- so per-particle and per-cell fields
# decorrelate within ~10 steps while whole-domain quantities stay close.
# configuration: grid, steps, and per checked step {quantity: bound}
# (quantities of parity_util.drift; agg_* are relative differences of
# parity_util.aggregates). The bounds are 3-10x the measured drift.
DRIFT_CASES = {
    1: (32, 20, {
        4: {"press": 1e-5, "lsmerge": 1e-5, "waterux": 1e-4, "wateruy": 1e-4, "wateruz": 1e-4, "airux": 1e-4,
            "airuy": 1e-4, "airuz": 1e-4, "mark": 0.0, "count": 0.0, "pos": 1e-3, "vel": 1e-2},
        20: {"agg_kinetic": 2e-2, "agg_gas_z": 5e-3, "agg_liquid_z": 2e-4, "agg_fluid_cells": 2e-2,
             "agg_gas_cells": 5e-2, "count": 0.0, "mark": 0.05},
    }),
    2: (32, 100, {
        60: "exact",
        100: {"agg_kinetic": 0.5, "agg_temp": 1e-2, "agg_gas_z": 0.2, "agg_liquid_z": 2e-3,
              "agg_fluid_cells": 2e-2, "count": 1e-2, "mark": 0.1},
    }),
    3: (32, 200, {200: "exact"}),
}


@pytest.mark.parametrize("config", sorted(DRIFT_CASES))
def test_drift_over_steps(mp, oracle_mod, config):
    n, steps, checks = DRIFT_CASES[config]
    sim, orc = make_pair(mp, oracle_mod, config, n, 2017_300 + config)
    for s in range(1, steps + 1):
        sim.bubblesim()
        orc.bubblesim()
        if s not in checks:
            continue
        g, r = snapshot(sim), snapshot(orc)
        if checks[s] == "exact":
            # the solid-velocity faces are not gathered by the step when no
            # cell holds a SOLID particle (the collision reads them only near
            # a solid); the oracle fills them anyway. Solubility and gas
            # content take expf, whose CUDA and host results may differ in the
            # last bit (the stage tests compare them at 1e-5)
            bad = compare(g, r, exact=True, skip=("solidux", "soliduy", "soliduz", "solubility", "gascontain"))
            assert rel_err(g["solubility"], r["solubility"]) <= 1e-5
            assert rel_err(g["gascontain"], r["gascontain"]) <= 1e-5
            assert not bad, f"config {config} step {s}: not bit-identical: {bad[:3]}"
            continue
        d = drift(g, r)
        for q, b in checks[s].items():
            assert d[q] <= b, f"config {config} after {s} steps: {q} drift {d[q]:.3e} > {b:.1e}"
    sim.close()
