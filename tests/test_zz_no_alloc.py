"""mp_pressure_cg_static: the pressure solve that allocates no device memory.

Some callers cannot allocate while they run: a host application that owns a
fixed device budget, or a frame loop that cudaFree's device-wide
synchronisation would stall. They call mp_pressure_cg_static, which keeps all
its working vectors in one fixed array inside the library. Its pressure must be
the one mp_project computes from the same marks and divergence, call after
call (the array keeps the previous call's contents, so a second call checks
that nothing stale leaks into the next solve).

Three cases cover its two solver paths: a 32^3 grid with 16-byte aligned
arrays (four cells per thread), the same grid with the pressure array one
float off alignment, and a 32 x 24 x 30 grid whose k-rows do not split into
groups of four (both the plane-marching path).

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from parity_util import bubblesim_stages, grid_params, rel_err

TOL = 1e-5   # the relative tolerance of the CG parity tests


def _until_projection(sim):
    for st in bubblesim_stages(sim.params, sim.state().frame):
        if st[0] == "project_CG_bubble":
            return
        getattr(sim, st[0])(*st[1:])


@pytest.mark.gpu
@pytest.mark.parametrize("shape,offset", [((32, 32, 32), 0), ((32, 32, 32), 1), ((32, 24, 30), 0)],
                         ids=["aligned", "pressure-off-alignment", "nz-not-multiple-of-4"])
def test_static_pressure_cg_matches_project(mp, shape, offset):
    import torch
    p = grid_params(mp, 1, *shape)
    sim = mp.Sim.from_config(1, shape[0], 2017001, params=p)
    _until_projection(sim)
    it_ref, res_ref, rc_ref = sim.project_CG_bubble()
    assert rc_ref == 0 and it_ref > 0
    press = sim.get_field("press")
    div = sim.get_field("div")
    mark = sim.get_field("mark")
    n = p.nx * p.ny * p.nz
    dev = torch.device("cuda", 0)
    d_mark = torch.from_numpy(np.ascontiguousarray(mark).view(np.int8)).to(dev)
    d_div = torch.from_numpy(np.ascontiguousarray(div, np.float32)).to(dev)
    d_buf = torch.empty(n + offset, dtype=torch.float32, device=dev)
    d_out = d_buf[offset:]
    lib = mp.load_library()
    for call in range(2):
        d_buf.fill_(float("nan"))   # the call must write every cell
        torch.cuda.synchronize()
        it, res = C.c_int(), C.c_double()
        rc = lib.mp_pressure_cg_static(p.nx, p.ny, p.nz, C.c_float(p.cellsize), C.c_void_p(d_mark.data_ptr()),
                                       C.c_void_p(d_div.data_ptr()), C.c_void_p(d_out.data_ptr()), p.cg_max_iter,
                                       p.cg_tol_mode, C.c_float(p.cg_tol), None, C.byref(it), C.byref(res))
        assert rc == 0, f"call {call}: rc {rc}"
        out = d_out.cpu().numpy()
        assert it.value == it_ref, f"call {call}: {it.value} iterations, mp_project took {it_ref}"
        assert abs(res.value - res_ref) <= TOL * max(abs(res_ref), 1e-300)
        assert rel_err(out, press) <= TOL, f"call {call}: rel err {rel_err(out, press)}"
    sim.close()


def test_static_pressure_cg_rejects_large_grids(mp):
    """Grids beyond the fixed scratch are refused before any GPU work."""
    lib = mp.load_library()
    it, res = C.c_int(), C.c_double()
    rc = lib.mp_pressure_cg_static(65, 64, 64, C.c_float(1 / 64), C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                                   10, mp.TOL_REL, C.c_float(1e-6), None, C.byref(it), C.byref(res))
    assert rc == mp.MP_ERR_CAPACITY
    buf = C.create_string_buffer(256)
    lib.mp_last_error(None, buf, 256)
    assert b"262144-cell limit" in buf.value
