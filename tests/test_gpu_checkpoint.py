"""Checkpoint / resume: a context that loads a checkpoint and steps reproduces
the steps of the context that saved it, bit for bit."""
import numpy as np
import pytest

from parity_util import CELL_FIELDS, FACE_FIELDS

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("config", [1, 2])
def test_resume_is_bit_exact(mp, config):
    a = mp.Sim.from_config(config, 32, 7100 + config)
    for _ in range(2):
        a.bubblesim()
    blob = a.checkpoint()
    for _ in range(3):
        a.bubblesim()
    b = mp.Sim(a.params)
    b.restore(blob)
    assert b.state().frame == 2
    for _ in range(3):
        b.bubblesim()
    sa, sb = a.state(), b.state()
    assert sa.frame == sb.frame and sa.par_num_now == sb.par_num_now
    pa, pb = a.download_particles(), b.download_particles()
    for k in pa:
        assert np.array_equal(pa[k].view(np.uint8), pb[k].view(np.uint8)), k
    for f in CELL_FIELDS + FACE_FIELDS:
        if f.startswith("solidu"):
            continue
        assert np.array_equal(a.get_field(f).view(np.uint8), b.get_field(f).view(np.uint8)), f
    a.close(); b.close()


def test_load_rejects_other_parameters(mp):
    a = mp.Sim.from_config(1, 32, 7101)
    blob = a.checkpoint()
    p = mp.scene_params(1, 32)
    p.dt = p.dt * 0.5
    b = mp.Sim(p)
    with pytest.raises(mp.MPError, match="other parameters"):
        b.restore(blob)
    with pytest.raises(mp.MPError, match="format"):
        b.restore(b"x" * len(blob))
    a.close(); b.close()
