"""The CPU oracle checked on its own: known answers where the reference's math
fixes them, structural properties elsewhere. No GPU."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

UNDEF = 0xFFFFFFFF


def _oracle(mp, oracle_mod, config, n, seed=11, **over):
    p = mp.scene_params(config, n)
    for k, v in over.items():
        setattr(p, k, v)
    o = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    parts = mp.scene_particles(p, config, seed)
    o.upload_particles(**parts)
    rf, seeds = mp.scene_tables(p, config, seed)
    o.set_tables(rf, seeds)
    o.set_field("fixedheat", mp.scene_fixed_heat(p, config))
    return o, p, parts


def test_hash_sort_is_a_stable_cell_sort(mp, oracle_mod):
    """thrust::sort_by_key semantics (spray_thrust.cu:12-17): keys ascending,
    equal keys keep their pre-sort order; cellStart/cellEnd bracket each cell."""
    o, p, parts = _oracle(mp, oracle_mod, 5, 16)
    rng = np.random.default_rng(3)
    perm = rng.permutation(len(parts["flag"]))
    shuffled = {k: v[perm] for k, v in parts.items()}
    shuffled["mass"] = np.arange(len(perm), dtype=np.float32)      # pre-sort index as a tag
    o.upload_particles(**shuffled)
    o.hashAndSortParticles()
    pos = o.get_field("pos").reshape(-1, 3)
    tag = o.get_field("mass")
    h = p.cellsize
    ijk = np.floor(pos / h).astype(np.int64)
    key = (ijk[:, 0] * p.ny + ijk[:, 1]) * p.nz + ijk[:, 2]
    assert (np.diff(key) >= 0).all()
    same = np.diff(key) == 0
    assert (np.diff(tag)[same] > 0).all(), "not stable within a cell"
    cs, ce = o.get_field("cellstart"), o.get_field("cellend")
    counts = np.bincount(key, minlength=p.nx * p.ny * p.nz)
    assert ((cs == UNDEF) == (counts == 0)).all()
    ne = counts > 0
    assert np.array_equal(ce[ne] - cs[ne], counts[ne])


def test_hash_out_of_range_axis_maps_to_zero(mp, oracle_mod):
    """getijkfrompos (spray_k.cu:51-57): an axis outside the grid hashes to index 0."""
    p = mp.scene_params(1, 16)
    o = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState)
    pos = np.array([[0.51, 0.52, 0.53], [-0.1, 0.52, 0.53], [0.51, 1.5, 0.53], [0.51, 0.52, -2.0]], np.float32)
    o.upload_particles(pos=pos, flag=np.zeros(4, np.int8), mass=np.ones(4, np.float32))
    o.hashAndSortParticles()
    cs = o.get_field("cellstart")
    nz = np.nonzero(cs != UNDEF)[0]
    i, j, k = 8, 8, 8
    expect = {i * 256 + j * 16 + k, 0 * 256 + j * 16 + k, i * 256 + 0 * 16 + k, i * 256 + j * 16 + 0}
    assert set(nz.tolist()) == expect


def _laplacian(mark, nx, ny, nz, h, types=(0, 1)):
    """computeAx_bubble (spray_k.cu:3423-3447) as a sparse matrix over FLUID/AIR
    cells; with types=(0,) computeAx (spray_k.cu:2300-2322) over FLUID cells."""
    idx = lambda i, j, k: (i * ny + j) * nz + k
    unk = np.isin(mark, types)
    rows, cols, vals = [], [], []
    for c in np.nonzero(unk)[0]:
        i, j, k = c // (ny * nz), (c // nz) % ny, c % nz
        diag = -6.0
        for di, dj, dk in ((1, 0, 0), (0, 1, 0), (0, 0, 1), (-1, 0, 0), (0, -1, 0), (0, 0, -1)):
            q = idx(i + di, j + dj, k + dk)
            if mark[q] == 2:
                diag += 1.0
            elif unk[q]:
                rows.append(c); cols.append(q); vals.append(1.0)
        rows.append(c); cols.append(c); vals.append(diag)
    n = nx * ny * nz
    A = sp.csr_matrix((np.array(vals) / (h * h), (rows, cols)), shape=(n, n))
    return A, unk


@pytest.mark.parametrize("config", [1, 5])
def test_projection_solves_the_reference_laplacian(mp, oracle_mod, config):
    """The FP64 projection's pressure solves the reference's 7-point system
    (BOUNDARY neighbours Neumann, other non-fluid neighbours zero) to 1e-7."""
    o, p, _ = _oracle(mp, oracle_mod, config, 16, precision=mp.PREC_FP64, cg_tol=1e-12, cg_max_iter=10000)
    o.hashAndSortParticles(); o.addexternalforce(); o.computeLevelset(0.0); o.sweepLSAndMardGrid()
    o.mapvelp2g_bubble()
    for ph in (1, 0):
        o.sweepPhi(ph); o.sweepU(ph)
    o.setWaterBoundaryU(1); o.setWaterBoundaryU(0)
    it, res, rc = o.project_CG_bubble()
    assert rc == 0
    mark = o.get_field("mark")
    b = o.get_field("div").astype(np.float64)
    x = o.get_field("press").astype(np.float64)
    A, unk = _laplacian(mark, p.nx, p.ny, p.nz, p.cellsize)
    sub = np.nonzero(unk)[0]
    As = A[sub][:, sub]
    xd = spla.spsolve(As.tocsc(), b[sub])
    assert np.linalg.norm(x[sub] - xd) / np.linalg.norm(xd) < 1e-6
    assert (x[~unk] == 0).all()


def _to_projection(o):
    o.hashAndSortParticles(); o.addexternalforce(); o.computeLevelset(0.0); o.sweepLSAndMardGrid()
    o.markSoloAirParticle(); o.computesurfacetension()
    o.mapvelp2g_bubble(); o.enforceDragForce()
    for ph in (1, 0):
        o.sweepPhi(ph); o.sweepU(ph)
    o.setWaterBoundaryU(1); o.setWaterBoundaryU(0)


def test_gfm_at_unit_density_ratio_is_the_reference_projection(mp, oracle_mod):
    """With rho_liquid = rho_air every face weight is 1 and the ghost-fluid
    projection is the reference's constant-coefficient one."""
    out = []
    for over in ({"precision": mp.PREC_FP64, "cg_tol": 1e-13, "cg_max_iter": 20000},
                 {"coef_mode": 1, "density_ratio": 1.0}):
        o, p, _ = _oracle(mp, oracle_mod, 1, 32, **over)
        _to_projection(o)
        it, res, rc = o.project_CG_bubble()
        assert rc == 0
        out.append({f: o.get_field(f).astype(np.float64) for f in ("press", "waterux", "airuz")})
    for f in out[0]:
        a, b = out[0][f], out[1][f]
        assert np.abs(a - b).max() <= 1e-6 * np.abs(a).max(), f


def test_gfm_projection_leaves_single_phase_interiors_divergence_free(mp, oracle_mod):
    """At a 1000:1 density ratio the projected faces satisfy D u = 0 wherever
    the divergence reads one phase only (cells whose six neighbours are of
    their own type), i.e. D beta G is the matrix that was solved."""
    o, p, _ = _oracle(mp, oracle_mod, 1, 32, coef_mode=1, density_ratio=1000.0)
    _to_projection(o)
    b = None
    it, res, rc = o.project_CG_bubble()
    assert rc == 0 and it > 0
    b = o.get_field("div").astype(np.float64)
    n, h = p.nx, p.cellsize
    mark = o.get_field("mark").reshape(n, n, n)
    w = [o.get_field(f).astype(np.float64) for f in ("waterux", "wateruy", "wateruz")]
    a = [o.get_field(f).astype(np.float64) for f in ("airux", "airuy", "airuz")]
    w = [w[0].reshape(n + 1, n, n), w[1].reshape(n, n + 1, n), w[2].reshape(n, n, n + 1)]
    a = [a[0].reshape(n + 1, n, n), a[1].reshape(n, n + 1, n), a[2].reshape(n, n, n + 1)]
    checked = 0
    worst = 0.0
    for t, u in ((mp.TYPEFLUID, w), (mp.TYPEAIR, a)):
        c = mark[1:-1, 1:-1, 1:-1] == t
        for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            c &= np.roll(mark, (-d[0], -d[1], -d[2]), axis=(0, 1, 2))[1:-1, 1:-1, 1:-1] == t
        div = ((u[0][2:-1, 1:-1, 1:-1] - u[0][1:-2, 1:-1, 1:-1]) + (u[1][1:-1, 2:-1, 1:-1] - u[1][1:-1, 1:-2, 1:-1]) +
               (u[2][1:-1, 1:-1, 2:-1] - u[2][1:-1, 1:-1, 1:-2])) / h
        checked += int(c.sum())
        if c.any():
            worst = max(worst, float(np.abs(div[c]).max()))
    assert checked > 1000
    # face velocities are stored in FP32 after the FP64 solve
    assert worst <= 1e-5 * float(np.abs(b).max())


def test_oracle_is_thread_count_independent(mp, oracle_mod):
    a, _, _ = _oracle(mp, oracle_mod, 2, 16, seed=5)
    oracle_mod.load().or_set_threads(1)
    a.bubblesim()
    r1 = {f: a.get_field(f) for f in ("press", "tp", "lsmerge", "pos", "flag")}
    b, _, _ = _oracle(mp, oracle_mod, 2, 16, seed=5)
    oracle_mod.load().or_set_threads(4)
    b.bubblesim()
    for f, v in r1.items():
        assert np.array_equal(v, b.get_field(f), equal_nan=True), f


def _water_to_projection(o):
    o.hashAndSortParticles(); o.sweepPhi(0); o.computeLevelset(0.0); o.sweepLSAndMardGrid()
    o.flipMark_sphere(); o.computesurfacetension(); o.mapvelp2g()
    o.sweepU(0); o.setWaterBoundaryU(0)


def test_water_projection_solves_the_single_phase_laplacian(mp, oracle_mod):
    """project_CG of the water mode: FLUID unknowns, AIR cells (the flipped
    vacuum) at zero pressure, BOUNDARY neighbours Neumann; the FP32 CG reaches
    the direct solve to the accuracy its vectors allow, and the divergence is
    cptdivergence's over FLUID cells."""
    o, p, _ = _oracle(mp, oracle_mod, 4, 16, cg_tol_mode=mp.TOL_REL, cg_tol=1e-7, cg_max_iter=10000)
    _water_to_projection(o)
    mark = o.get_field("mark")
    assert not (mark == 3).any() and (mark == 1).any()          # no VACUUM left, AIR present
    ux, uy, uz = (o.get_field(f).astype(np.float64) for f in ("waterux", "wateruy", "wateruz"))
    it, res, rc = o.project_CG()
    assert rc == 0 and it > 0
    n = p.nx
    ux = ux.reshape(n + 1, n, n); uy = uy.reshape(n, n + 1, n); uz = uz.reshape(n, n, n + 1)
    div = ((ux[1:] - ux[:-1]) + (uy[:, 1:] - uy[:, :-1]) + (uz[:, :, 1:] - uz[:, :, :-1])).reshape(-1) / p.cellsize
    b = o.get_field("div").astype(np.float64)
    fl = mark == 0
    assert np.allclose(b[fl], div[fl], rtol=1e-5, atol=1e-3) and (b[~fl] == 0).all()
    x = o.get_field("press").astype(np.float64)
    A, unk = _laplacian(mark, n, n, n, p.cellsize, types=(0,))
    sub = np.nonzero(unk)[0]
    xd = spla.spsolve(A[sub][:, sub].tocsc(), b[sub])
    assert np.linalg.norm(x[sub] - xd) / np.linalg.norm(xd) < 1e-4
    assert (x[~unk] == 0).all()


def test_oracle_modes_are_thread_count_independent(mp, oracle_mod):
    runs = []
    for th in (1, 4):
        oracle_mod.load().or_set_threads(th)
        o, _, _ = _oracle(mp, oracle_mod, 4, 16, seed=6)
        o.watersim(); o.watersim()
        h, ph, _ = _oracle(mp, oracle_mod, 1, 16, seed=6)
        h.initheat_grid(); h.heatsim(); h.heatsim()
        runs.append({"pos": o.get_field("pos"), "press": o.get_field("press"), "tp": h.get_field("tp")})
    for f in runs[0]:
        assert np.array_equal(runs[0][f], runs[1][f]), f


def test_oracle_pouring_matches_the_numpy_restatement(mp, oracle_mod):
    """The oracle's pouring stage appends exactly what oracle/pour_ref.py's
    restatement of pouringwater gives, with the reference's per-type values."""
    from oracle import pour_ref
    o, p, parts = _oracle(mp, oracle_mod, 1, 16, seed=8)
    rf, _ = mp.scene_tables(p, 1, 8)
    ppos, pvel = pour_ref.emitter(0, p.samplespace, 0.05, (0.5, 0.5, 0.5), (0.0, 0.0, -0.5))
    o.set_pour(ppos, pvel)
    np0 = o.state().par_num_now
    o.pouring()                                       # frame 0: 0 % 4 == 0
    d = o.download_particles()
    assert len(d["pos"]) == np0 + len(ppos)
    rpos, rvel = pour_ref.pour(ppos, pvel, rf, p.pos_rand_param, p.vel_rand_param, p.samplespace)
    t = slice(np0, None)
    assert np.array_equal(d["pos"][t].view(np.uint32), rpos.view(np.uint32))
    assert np.array_equal(d["vel"][t].view(np.uint32), rvel.view(np.uint32))
    assert (d["flag"][t] == mp.TYPEFLUID).all() and (d["mass"][t] == np.float32(p.m0)).all()
    st = o.state(); st.frame = 1; o.set_state(st)
    o.pouring()                                       # not a pouring frame
    assert o.state().par_num_now == np0 + len(ppos)


def test_scene_configurations(mp):
    p = mp.scene_params(1, 32)
    parts = mp.scene_particles(p, 1, 1)
    pos, flag = parts["pos"], parts["flag"]
    assert (pos[:, 2] < 0.6).all() and pos.min() >= p.cellsize and pos.max() <= 1 - p.cellsize
    r = np.linalg.norm(pos - np.array([0.5, 0.5, 0.25]), axis=1)
    assert np.array_equal(flag == mp.TYPEAIR, r < 0.15)
    # 8 particles per liquid cell
    ijk = np.floor(pos / p.cellsize).astype(int)
    _, counts = np.unique(ijk, axis=0, return_counts=True)
    assert counts.max() == 8 and np.median(counts) == 8
    p4 = mp.scene_params(4, 32)
    v = mp.scene_particles(p4, 4, 2)["vel"]
    assert abs(v.std() - 0.1) < 0.01 and abs(v.mean()) < 0.01
    p3 = mp.scene_params(3, 32)
    f3 = mp.scene_particles(p3, 3, 3)
    sol = f3["flag"] == mp.TYPESOLID
    assert sol.any() and (f3["temp"][sol] == p3.default_solid_T).all()
    fh = mp.scene_fixed_heat(p3, 3).reshape(32, 32, 32)
    assert (fh[5, 5, -4:] == np.float32(0.6)).all() and (fh[5, 5, :-4] == -10000.0).all()
    p2 = mp.scene_params(2, 32)
    rf, seeds = mp.scene_tables(p2, 2, 9)
    assert rf.size == 10000 and 0 <= rf.min() and rf.max() < 1 and len(set(seeds.tolist())) == 16
    assert ((seeds % 32) == 2).all()


@pytest.mark.parametrize("smooth", [0, 1])
def test_marching_cubes_on_the_reference_sphere_field(mp, oracle_mod, smooth):
    """The extraction on genSphereDensfield's analytic sphere (spray_k.cu:1827):
    a closed, consistently oriented surface whose vertices lie on the sphere
    (to the linear interpolation's error; Taubin's lambda step pulls them in by
    less than a fifth of a 2x cell) with normals along the radius."""
    p = mp.scene_params(1, 16)
    p.b_smooth_mc = smooth
    o = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    c, r = np.array([0.5, 0.48, 0.52]), 0.3
    assert o.runMC_sphere(1, c, r) == 0
    v, n, ix = o.mc_mesh(1)
    assert len(v) > 100 and len(ix) % 3 == 0
    hm = p.cellsize / 2
    d = np.linalg.norm(v.astype(np.float64) - c, axis=1)
    tol = 0.2 * hm if smooth else 0.02 * hm
    assert np.abs(d - r).max() < tol, np.abs(d - r).max() / hm
    radial = (v.astype(np.float64) - c) / d[:, None]
    cosang = np.sum(radial * n, axis=1)
    assert (np.abs(np.linalg.norm(n, axis=1) - 1) < 1e-5).all()
    assert (np.abs(cosang) > 0.9).all() and (np.sign(cosang) == np.sign(cosang[0])).all()
    tri = ix.reshape(-1, 3)
    edges = {}
    for t in tri:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            edges[(a, b)] = edges.get((a, b), 0) + 1
    # closed and consistently wound: every directed edge once, its reverse once
    assert all(cnt == 1 and edges.get((b, a), 0) == 1 for (a, b), cnt in edges.items())
