"""The CUDA path against the reference's own kernels, through the pinned
digests (tests/golden/refhost_pin.json, made with the reference's kernels
compiled for the host).  From the same inputs, the GPU runs bubblesim's first
frame stage by stage and its whole state must hash to the reference's after
every stage up to the projection: those stages are bit-exact on the GPU.
From the projection on, the GPU's FP64 reductions add in another order than
the pinned definition (compared at 1e-5 against the oracle instead, in
tests/test_gpu_stages.py), so the digests end there."""
import json
import os

import numpy as np
import pytest

from parity_util import CELL_FIELDS, FACE_FIELDS, bubblesim_stages, state_digest
from test_refhost_stages import reference_mode

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "refhost_pin.json")) as _f:
    PIN = json.load(_f)
FIRST_INEXACT = "project_CG_bubble"


@pytest.mark.parametrize("config", sorted(PIN["configs"], key=int))
def test_gpu_stages_hash_to_the_reference_kernels(mp, config):
    pin = PIN["configs"][config]
    p, parts, rf, seeds = reference_mode(mp, int(config), PIN["n"], pin["seed"])
    sim = mp.Sim(p)
    sim.upload_particles(**parts)
    sim.set_tables(rf, seeds)
    for f in CELL_FIELDS + FACE_FIELDS:        # the reference run starts from zeroed fields
        sim.set_field(f, np.zeros_like(sim.get_field(f)))
    st = sim.state()
    st.frame = 0
    st.n_real_solpoint = int((np.asarray(parts["flag"]) == mp.TYPESOLID).sum())
    sim.set_state(st)
    checked = 0
    for stage, row in zip(bubblesim_stages(p, 0), pin["stages"]):
        if stage[0] == FIRST_INEXACT:
            break
        assert row[:2] == [0, " ".join(str(x) for x in stage)]
        getattr(sim, stage[0])(*stage[1:])
        assert state_digest(sim) == row[2], f"config {config}: GPU state differs from the reference after {row[1]}"
        checked += 1
    assert checked >= 12
    sim.close()
