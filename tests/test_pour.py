"""Pouring emitter lattices (mp_scene_pour) against the restatement of
CompPouringParam_Freezing / _Ineraction / _Ineraction2 in oracle/pour_ref.py,
at the reference scenes' constants (spray.cpp:261-264, 299-302, 340-344,
379-383). Host code only: runs without a GPU."""
import numpy as np
import pytest

from oracle import pour_ref

SS = 0.5 / 64   # samplespace of the reference scenes

CASES = [
    (0, 0.035, (0.6, 0.45, 0.75), (0.0, 0.0, -0.5), None),       # MELTINGPOUR
    (0, 0.035, (0.60, 0.48, 0.75), (0.0, 0.0, -0.5), None),      # FREEZING
    (2, 0.05, (0.27, 0.25, 0.05), (0.0, 0.0, 1.1), (0.45, 0.25, 0.05)),   # INTERACTION
    (1, 0.060, (0.25, 0.25, 0.05), (0.0, 0.0, 1.5), None),       # INTERACTION_HIGHRES
    (1, 0.001, (0.5, 0.5, 0.5), (0.0, 0.0, 1.0), None),          # radius below the spacing: the centre only
]


@pytest.mark.parametrize("variant,radius,center,vel,center2", CASES)
def test_emitter_lattice_matches_reference(mp, variant, radius, center, vel, center2):
    pos, v = mp.scene_pour(variant, SS, radius, center, vel, center2=center2)
    rpos, rv = pour_ref.emitter(variant, SS, radius, center, vel, center2)
    assert pos.shape == rpos.shape and len(pos) > 0
    assert np.array_equal(pos.view(np.uint32), rpos.view(np.uint32))
    assert np.array_equal(v, rv)
    # every point within the radius of its disc, in the disc's plane
    assert np.all(pos[:, 2] == np.float32(center[2]))


def test_emitter_arguments(mp):
    with pytest.raises(mp.MPError):
        mp.scene_pour(2, SS, 0.05, (0.2, 0.2, 0.1), (0, 0, 1))        # two discs need a second centre
    with pytest.raises(mp.MPError):
        mp.scene_pour(5, SS, 0.05, (0.2, 0.2, 0.1), (0, 0, 1))
