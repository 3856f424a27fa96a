"""The oracle's own scene inputs (oracle/scene.py, the reference arm of the
benchmark) equal the product's: the same parameters byte for byte, the same
seeded particles, tables and fixed-heat field, the same case tables, and the
same field ids and state layout, so both arms start from identical inputs."""
import ctypes as C

import numpy as np
import pytest


@pytest.fixture(scope="module")
def scene(oracle_mod):
    from oracle import scene
    return scene


def test_field_ids_and_state_layout(mp, scene):
    assert scene.FIELDS == mp.FIELDS
    assert C.sizeof(scene.State) == C.sizeof(mp.MPState)
    for (na, ta), (nb, tb) in zip(scene.State._fields_, mp.MPState._fields_):
        assert na == nb and getattr(scene.State, na).offset == getattr(mp.MPState, nb).offset


@pytest.mark.parametrize("config,n", [(1, 32), (2, 24), (3, 32), (4, 16), (5, 48)])
def test_scene_equals_product(mp, scene, config, n):
    po, pp = scene.scene_params(config, n), mp.scene_params(config, n)
    assert C.sizeof(po) == C.sizeof(pp)
    assert C.string_at(C.addressof(po), C.sizeof(po)) == C.string_at(C.addressof(pp), C.sizeof(pp))
    a, b = scene.scene_particles(po, config, 2017), mp.scene_particles(pp, config, 2017)
    for k in b:
        assert np.array_equal(a[k], b[k]), k
    for x, y in zip(scene.scene_tables(po, config, 2017), mp.scene_tables(pp, config, 2017)):
        assert np.array_equal(x, y)
    assert np.array_equal(scene.scene_fixed_heat(po, config), mp.scene_fixed_heat(pp, config))


def test_mc_tables_equal_product(mp, scene):
    for x, y in zip(scene.mc_tables(), mp.mc_tables()):
        assert np.array_equal(x, y)
