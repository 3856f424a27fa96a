"""Per-frame files of the step (mp_set_output): the names, cadence and contents
bubblesim and runMC_smooth give them, checked against the restated writers of
oracle/export_ref.py applied to the meshes and particles the context holds."""
import gzip
import os

import numpy as np
import pytest

from oracle import export_ref

pytestmark = pytest.mark.gpu

NAMES = {0: "solid", 1: "water", 2: "gas"}   # runMC_solid / runMC_fluid / runMC_gas


def _read(path):
    with open(path, "rb") as f:
        return f.read()


def _dirs(root):
    for sub in ("waterdata", "waterOBJdata", "waterBOBJdata", "gasBOBJdata", "solidBOBJdata"):
        os.makedirs(os.path.join(root, sub), exist_ok=True)


@pytest.mark.parametrize("config", [1, 2])
def test_step_writes_the_reference_files(mp, tmp_path, config):
    sim = mp.Sim.from_config(config, 32, 7300 + config)
    root = str(tmp_path) + "/"
    _dirs(root)
    tmin, tmax = 273.0, 373.0
    sim.set_output(root, pov=True, obj=True, colored_particles=True, t_render_min=tmin, t_render_max=tmax)
    every = sim.params.mc_every
    assert every >= 1
    for _ in range(every + 1):
        frame = sim.state().frame
        before = {os.path.join(dp, f) for dp, _, fs in os.walk(root) for f in fs}
        sim.bubblesim()
        after = {os.path.join(dp, f) for dp, _, fs in os.walk(root) for f in fs}
        if frame % every:
            assert after == before, "files written off the output cadence"
            continue
        F = frame // every
        parts = sim.download_particles()
        for s, nm in NAMES.items():
            v, n, ix = sim.mc_mesh(s)
            assert _read(f"{root}waterdata/{nm}{F:05d}.pov") == export_ref.pov_mesh(v, n, ix, nm)
            if len(v) == 0:
                assert _read(f"{root}waterOBJdata/{nm}{F:05d}.obj") == b""
            else:
                gz = f"{root}{nm}BOBJdata/fluidsurface_final_{F - 1:04d}.bobj.gz"
                assert gzip.decompress(_read(gz)) == export_ref.bobj_payload(v, n, ix)
        assert len(sim.mc_mesh(1)[0]) > 0
        assert _read(f"{root}waterdata/allparticles{F:05d}.pov") == export_ref.particles(
            0, parts["pos"], parts["flag"], parts["temp"], tmin, tmax)
        solo = f"{root}waterdata/solobubble{F:05d}.pov"
        if sim.params.scene == mp.scene_params(2, 32).scene:     # boiling: the AIR spheres
            assert _read(solo) == export_ref.particles(2, parts["pos"], parts["flag"], parts["temp"], tmin, tmax)
        else:
            assert not os.path.exists(solo)
    sim.close()


def test_context_exporters_and_missing_directory(mp, tmp_path):
    sim = mp.Sim.from_config(2, 32, 7310)
    sim.bubblesim()                       # frame 0 extracts the meshes
    parts = sim.download_particles()
    for kind in (0, 1, 2):
        p = str(tmp_path / f"k{kind}.pov")
        sim.export_particles(kind, p, 273.0, 373.0)
        assert _read(p) == export_ref.particles(kind, parts["pos"], parts["flag"], parts["temp"], 273.0, 373.0)
    v, n, ix = sim.mc_mesh(1)
    for fmt, ref in ((mp.OUT_POV_MESH, export_ref.pov_mesh(v, n, ix, "water")),
                     (mp.OUT_OBJ_MESH, export_ref.obj_mesh(v, n, ix))):
        p = str(tmp_path / f"m{fmt}")
        sim.export_mesh(1, fmt, p)
        assert _read(p) == ref
    # the directories are the caller's, as in the reference: a missing one is
    # MP_ERR_IO, and the step itself still completes and advances the frame
    sim.set_output(str(tmp_path / "absent") + "/", pov=True, obj=False)
    f0 = sim.state().frame
    while sim.state().frame % sim.params.mc_every:
        sim.bubblesim()
    with pytest.raises(mp.MPError) as e:
        sim.bubblesim()
    assert e.value.code == mp.MP_ERR_IO
    assert sim.state().frame > f0
    sim.set_output(None)
    sim.bubblesim()
    sim.close()


def test_kept_solid_surface_is_written_as_text_obj(mp, tmp_path):
    """runMC_interaction's kept-surface branch writes the solid mesh with
    outputOBJwater (a text OBJ), not as BOBJ."""
    sim = mp.Sim.from_config(3, 32, 7320, scene=mp.SCENE_MELTANDBOIL, b_run_mc_solid=0, b_fix_solid=0, b_melt=0,
                             b_freeze=0, mc_every=2)
    root = str(tmp_path) + "/"
    _dirs(root)
    sim.set_output(root, pov=False, obj=True, colored_particles=False)
    for _ in range(3):                    # frames 0, 1, 2: extraction at 0, kept surface at 2
        sim.bubblesim()
    v, n, ix = sim.mc_mesh(mp.MC_SOLID)
    assert len(v) > 0
    assert _read(f"{root}waterOBJdata/solid00001.obj") == export_ref.obj_mesh(v, n, ix)
    assert os.path.exists(f"{root}solidBOBJdata/fluidsurface_final_-001.bobj.gz")   # frame 0: extracted
    assert not os.path.exists(f"{root}solidBOBJdata/fluidsurface_final_0000.bobj.gz")
    sim.close()


def test_water_mode_writes_the_fluid_surface(mp, tmp_path):
    """watersim reaches runMC_fluid's writers too: the water surface only."""
    sim = mp.Sim.from_config(4, 32, 7330, b_run_mc=1, b_correct_position=1)
    root = str(tmp_path) + "/"
    _dirs(root)
    sim.set_output(root, pov=True, obj=True, colored_particles=True)
    sim.watersim()                        # frame 0
    v, n, ix = sim.mc_mesh(mp.MC_FLUID)
    assert len(v) > 0
    assert _read(f"{root}waterdata/water00000.pov") == export_ref.pov_mesh(v, n, ix, "water")
    assert gzip.decompress(_read(f"{root}waterBOBJdata/fluidsurface_final_-001.bobj.gz")) == \
        export_ref.bobj_payload(v, n, ix)
    files = {f for _, _, fs in os.walk(root) for f in fs}
    assert files == {"water00000.pov", "fluidsurface_final_-001.bobj.gz"}
    sim.close()
