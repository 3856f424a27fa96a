"""Per-frame file writers (mp_write_mesh, mp_write_particles) against the
restatement of the reference's writers in oracle/export_ref.py: byte-equal
POV-Ray and OBJ text, byte-equal BOBJ payload inside a valid gzip stream,
with the reference's edge cases (empty mesh, NaN vertices, infinities, every
colour band of mapColorBlue2Red_h). Host code only: runs without a GPU."""
import gzip
import os

import numpy as np
import pytest

from oracle import export_ref


def _mesh(rng, nv, ntri):
    v = rng.uniform(-2, 2, (nv, 3)).astype(np.float32)
    n = rng.standard_normal((nv, 3)).astype(np.float32)
    ix = rng.integers(0, max(nv, 1), 3 * ntri).astype(np.uint32) if nv else np.zeros(0, np.uint32)
    return v, n, ix


def _read(path):
    with open(path, "rb") as f:
        return f.read()


@pytest.mark.parametrize("nv,ntri", [(0, 0), (1, 0), (7, 5), (500, 900)])
def test_mesh_formats_match_reference_writers(mp, tmp_path, nv, ntri):
    rng = np.random.default_rng(2250 + nv)
    v, n, ix = _mesh(rng, nv, ntri)
    if nv > 3:
        # verifyfloat3 replaces a vertex with a NaN component by (0,0,0);
        # infinities pass and print as "inf"
        v[1, 2] = np.nan
        n[2, 0] = np.nan
        v[3, 0] = np.inf
        n[3, 1] = -np.inf
        v[0] = [1e-7, -0.0, 123456.789]
    pov, obj, bobj = (str(tmp_path / f) for f in ("m.pov", "m.obj", "m.bobj.gz"))
    mp.write_mesh(mp.OUT_POV_MESH, pov, v, n, ix, object_name="gas")
    mp.write_mesh(mp.OUT_OBJ_MESH, obj, v, n, ix)
    mp.write_mesh(mp.OUT_BOBJ_GZ, bobj, v, n, ix)
    assert _read(pov) == export_ref.pov_mesh(v, n, ix, "gas")
    assert _read(obj) == export_ref.obj_mesh(v, n, ix)
    raw = _read(bobj)
    assert raw[:2] == b"\x1f\x8b"            # a gzip stream even when empty
    assert gzip.decompress(raw) == export_ref.bobj_payload(v, n, ix)


def test_mesh_header_layout(mp, tmp_path):
    v = np.array([[0.5, 0.25, 1.0], [1, 0, 0], [0, 1, 0]], np.float32)
    ix = np.array([0, 1, 2], np.uint32)
    p = str(tmp_path / "t.pov")
    mp.write_mesh(mp.OUT_POV_MESH, p, v, v, ix, object_name="water")
    txt = _read(p).decode()
    assert txt.startswith("#declare watermesh=mesh2{\nvertex_vectors{\n3,\n< 0.500000, 0.250000, 1.000000 >,\n")
    assert "face_indices{\n1,\n<0, 1, 2>,\n}\n " in txt
    assert txt.endswith("object{ watermesh material{water_material} }\n ")
    o = str(tmp_path / "t.obj")
    mp.write_mesh(mp.OUT_OBJ_MESH, o, v, v, ix)
    assert _read(o).decode().endswith("#face_indices\nf  1 2 3\n")
    b = str(tmp_path / "t.bobj.gz")
    mp.write_mesh(mp.OUT_BOBJ_GZ, b, v, v, ix)
    pay = gzip.decompress(_read(b))
    # vertex count, 3 vertices, normal count, 3 normals, INDEX count (3), 3 indices
    assert len(pay) == 4 + 36 + 4 + 36 + 4 + 12
    assert np.frombuffer(pay[-16:-12], np.int32)[0] == 3


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_particle_spheres_match_reference_writers(mp, tmp_path, kind):
    rng = np.random.default_rng(2440 + kind)
    n = 2000
    pos = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    flag = rng.integers(0, 6, n).astype(np.int8)
    # temperatures over and beyond [t_min, t_max]: every band, below (blue) and above (red)
    T = rng.uniform(250.0, 400.0, n).astype(np.float32)
    T[:8] = [273.0, 373.0, 289.6666, 306.3333, 323.0, 339.6666, 356.3333, 372.9999]
    p = str(tmp_path / f"p{kind}.pov")
    mp.write_particles(kind, p, pos, flag=flag, temperature=T, t_min=273.0, t_max=373.0)
    assert _read(p) == export_ref.particles(kind, pos, flag, T, 273.0, 373.0)


def test_color_bands(mp):
    # the oracle's colour map itself: band edges as mapColorBlue2Red_h defines them
    assert export_ref.blue2red(-0.5) == (0, 0, 1)
    assert export_ref.blue2red(0.0) == (0, 0, 1)
    assert export_ref.blue2red(2.0) == (0, 1, 1)
    assert export_ref.blue2red(4.0) == (1, 1, 0)
    assert export_ref.blue2red(6.0) == (1, 0, 0)
    assert export_ref.blue2red(9.0) == (1, 0, 0)


def test_writer_errors(mp, tmp_path):
    v = np.zeros((3, 3), np.float32)
    with pytest.raises(mp.MPError) as e:
        mp.write_mesh(mp.OUT_POV_MESH, str(tmp_path / "no_such_dir" / "m.pov"), v, v, np.array([0, 1, 2], np.uint32))
    assert e.value.code == mp.MP_ERR_IO
    with pytest.raises(mp.MPError) as e:       # an index past the last vertex
        mp.write_mesh(mp.OUT_OBJ_MESH, str(tmp_path / "m.obj"), v, v, np.array([0, 1, 3], np.uint32))
    assert e.value.code == mp.MP_ERR_ARG
    with pytest.raises(mp.MPError) as e:       # not whole triangles
        mp.write_mesh(mp.OUT_OBJ_MESH, str(tmp_path / "m.obj"), v, v, np.array([0, 1], np.uint32))
    assert e.value.code == mp.MP_ERR_ARG
    with pytest.raises(mp.MPError) as e:
        mp.write_mesh(7, str(tmp_path / "m.x"), v, v, np.array([0, 1, 2], np.uint32))
    assert e.value.code == mp.MP_ERR_ARG
    with pytest.raises(mp.MPError) as e:       # flags are needed for the AIR / AIRSOLO kinds
        mp.write_particles(mp.OUT_PARTICLES_AIR, str(tmp_path / "p.pov"), v)
    assert e.value.code == mp.MP_ERR_ARG
    assert not os.path.exists(str(tmp_path / "m.x"))
