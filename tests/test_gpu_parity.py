"""Parity of the sm_100a path (through the C ABI) with the FP64 oracle.

Tolerances:
  FP64 storage:  fields 1e-12 absolute, Cd and L2 1e-11 relative, per step
                 (operation order differs from the oracle only by FMA contraction);
  FP32 (f - w):  relative L2 of u and of rho <= 1e-5, Cd <= 1e-4 relative;
  FP16 (f - w):  relative L2 of u <= 5e-3, Cd <= 5e-3 relative (stated error of
                 the half-precision storage form; measured 2.5e-3 and 3.0e-3).
"""
import numpy as np
import pytest

import make_ref

pytestmark = pytest.mark.gpu


def rel_l2(geo, fo, fm, key):
    num = den = 0.0
    for a in range(geo.layout.number_area):
        m = geo.Areas[a].m
        if key == "u":
            num += (np.sum((fo[a]["ux"] - fm[a]["ux"]) ** 2) + np.sum((fo[a]["uy"] - fm[a]["uy"]) ** 2)) / m
            den += (np.sum(fo[a]["ux"] ** 2) + np.sum(fo[a]["uy"] ** 2)) / m
        else:
            num += np.sum((fo[a][key] - fm[a][key]) ** 2) / m
            den += np.sum(fo[a][key] ** 2) / m
    return float(np.sqrt(num / den))


def all_fields(sim, geo):
    return [sim.fields(a) for a in range(geo.layout.number_area)]


def make_pair(mb, orc, name, prec="f64", graph=True):
    L, cfg, _ = make_ref.case(name)
    g = mb.geo_init(L, cfg)
    o = orc.Oracle(g)
    o.init()
    m = mb.MultiBlockLBM(g, prec, graph=graph)
    m.init()
    return g, o, m


@pytest.mark.parametrize("graph", [True, False, "program"])
@pytest.mark.parametrize("name", make_ref.GOLDEN)
def test_f64_stepwise(mb, orc, cuda_device, name, graph):
    g, o, m = make_pair(mb, orc, name, "f64", graph)
    cds_o, cds_m = [], []
    for _ in range(25):
        o.evolution(1)
        m.evolution(1)
        cds_o.append(o.getDrag_block()[2])
        cds_m.append(m.getDrag_block()[2])
        lo, lm = o.error_L2(), m.error_L2()
        assert lm == pytest.approx(lo, rel=1e-11)
    scale = max(abs(v) for v in cds_o)
    assert np.abs(np.array(cds_o) - np.array(cds_m)).max() <= 1e-11 * scale
    for fo, fm in zip(all_fields(o, g), all_fields(m, g)):
        assert (fo["solid"] == fm["solid"]).all()
        for k in ("rho", "ux", "uy", "F"):
            np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-12, err_msg=f"{name} {k}")


@pytest.mark.parametrize("name", ["g25", "n3", "g49"])
def test_f64_multi_step_plans(mb, orc, cuda_device, name):
    """mb_step(n) replays cached multi-step graphs; 13 = 2 x 6 + 1 steps."""
    g, o, m = make_pair(mb, orc, name, "f64", True)
    o.evolution(13)
    m.evolution(13)
    assert m.getDrag_block()[2] == pytest.approx(o.getDrag_block()[2], rel=1e-11)
    assert m.error_L2() == pytest.approx(o.error_L2(), rel=1e-11)
    for fo, fm in zip(all_fields(o, g), all_fields(m, g)):
        for k in ("rho", "ux", "uy", "F"):
            np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-12)


def test_drag_links_match(mb, orc, cuda_device):
    for name in make_ref.GOLDEN:
        g, o, m = make_pair(mb, orc, name)
        assert m.drag_links() == len(o.drag_links())


def _randomise(g, o, m, seed):
    """Same random near-equilibrium state in both (F and rho/u of every cell)."""
    rng = np.random.default_rng(seed)
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    for a in range(g.layout.number_area):
        A = g.Areas[a]
        F = w[:, None, None] * (1 + 0.05 * rng.standard_normal((9, A.ny, A.nx)))
        rho = 1 + 0.01 * rng.standard_normal((A.ny, A.nx))
        ux = 0.05 + 0.01 * rng.standard_normal((A.ny, A.nx))
        uy = 0.01 * rng.standard_normal((A.ny, A.nx))
        o.set_fields(a, rho, ux, uy, F, None)
        m.set_fields(a, rho, ux, uy, F)


def _stale_f_init(g, o, orc):
    """The oracle's post-stream array starts as feq(rho0, U0) (init_General), which
    is what a block-edge solid cell keeps for off-block directions."""
    c = g.config
    fe = np.array([orc.feq(k, c.rho0, c.U0[0], c.U0[1]) for k in range(9)])
    for a in range(g.layout.number_area):
        A = g.Areas[a]
        o.set_fields(a, f=np.broadcast_to(fe[:, None, None], (9, A.ny, A.nx)).copy())


@pytest.mark.parametrize("name", ["g25", "n3", "g49"])
def test_block_step_random_state(mb, orc, cuda_device, name):
    g, o, m = make_pair(mb, orc, name)
    _randomise(g, o, m, 1)
    _stale_f_init(g, o, orc)
    for a in range(g.layout.number_area):
        o.block_step(a)
        m.block_step(a)
    for a, (fo, fm) in enumerate(zip(all_fields(o, g), all_fields(m, g))):
        np.testing.assert_allclose(fm["F"], fo["F"], rtol=0, atol=1e-14, err_msg=f"block {a}")
        fl = fo["solid"] == 0
        for k in ("rho", "ux", "uy"):
            np.testing.assert_allclose(fm[k][fl], fo[k][fl], rtol=0, atol=1e-14)


@pytest.mark.parametrize("name", ["g25", "n3", "g49"])
def test_interface_ops_random_state(mb, orc, cuda_device, name):
    """c_c, spline, rotation, temporal, c_f and f_c one call at a time."""
    g, o, m = make_pair(mb, orc, name)
    _randomise(g, o, m, 2)
    L = g.layout
    for c in range(L.number_line2):
        o.c_c_boundary_transfer(c)
        m.c_c_boundary_transfer(c)
    for b in range(L.number_line):
        o.space_interpolation(b)
        m.space_interpolation(b)
        o.rotate_markers(b)
        m.rotate_markers(b)
    for b in range(L.number_line):
        o.temporal_interpolation(b, 0.5)
        m.temporal_interpolation(b, 0.5)
    check = lambda tol: [np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=tol, err_msg=f"{k}")
                         for fo, fm in zip(all_fields(o, g), all_fields(m, g)) for k in ("rho", "ux", "uy", "F")]
    check(1e-13)
    for b in range(L.number_line):
        o.c_f_boundary_transfer(b)
        m.c_f_boundary_transfer(b)
        o.f_c_boundary_transfer(b)
        m.f_c_boundary_transfer(b)
    check(1e-13)


@pytest.mark.parametrize("prec,tol_u,tol_cd", [("f32", 1e-5, 1e-4), ("f16s", 5e-3, 5e-3), ("f16c", 2e-3, 2e-3)])
def test_reduced_precision_error(mb, orc, cuda_device, prec, tol_u, tol_cd):
    """Config-1 layout (400x160, Re=40) for 2000 coarse steps against the oracle."""
    g = mb.config1_geometry()
    o = orc.Oracle(g)
    o.init()
    m = mb.MultiBlockLBM(g, prec)
    m.init()
    o.evolution(2000)
    m.evolution(2000)
    fo, fm = all_fields(o, g), all_fields(m, g)
    eu, er = rel_l2(g, fo, fm, "u"), rel_l2(g, fo, fm, "rho")
    cdo, cdm = o.getDrag_block()[2], m.getDrag_block()[2]
    print(f"{prec}: relL2 u {eu:.3e} rho {er:.3e} Cd {cdm:.8f} vs {cdo:.8f}")
    assert eu <= tol_u and er <= tol_u
    assert abs(cdm - cdo) <= tol_cd * abs(cdo)


def test_graph_equals_direct_bitwise(mb, cuda_device):
    g = mb.geo_init(*make_ref.case("n3")[:2])
    a = mb.MultiBlockLBM(g, "f32", graph=True)
    b = mb.MultiBlockLBM(g, "f32", graph=False)
    for s in (a, b):
        s.init()
        s.evolution(20)
    for k in range(g.layout.number_area):
        fa, fb = a.fields(k), b.fields(k)
        for key in ("rho", "ux", "uy", "F"):
            assert np.array_equal(fa[key], fb[key])
    assert a.getDrag_block() == b.getDrag_block()


def test_deterministic(mb, cuda_device):
    g = mb.config1_geometry()
    res = []
    for _ in range(2):
        s = mb.MultiBlockLBM(g, "f32")
        s.init()
        s.evolution(50)
        res.append((s.getDrag_block(), s.error_L2(), s.fields(4)["F"].copy()))
        s.close()
    assert res[0][0] == res[1][0] and res[0][1] == res[1][1]
    assert np.array_equal(res[0][2], res[1][2])


def test_config2_f64_two_steps_match_oracle(mb, orc, cuda_device):
    """The 3-level 4096x1024 workload itself, FP64, against the oracle."""
    g = mb.config2_geometry()
    o = orc.Oracle(g)
    o.init()
    m = mb.MultiBlockLBM(g, "f64")
    m.init()
    o.evolution(2)
    m.evolution(2)
    assert m.getDrag_block()[2] == pytest.approx(o.getDrag_block()[2], rel=1e-11)
    for a in (0, 4, 8):
        fo, fm = o.fields(a), m.fields(a)
        for k in ("rho", "ux", "F"):
            np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-13)


def test_config2_f32_properties(mb, cuda_device):
    """Full-size properties: finite state, plausible drag, graph = direct bitwise."""
    g = mb.config2_geometry()
    a = mb.MultiBlockLBM(g, "f32", graph=True)
    b = mb.MultiBlockLBM(g, "f32", graph=False)
    for s in (a, b):
        s.init()
        s.evolution(7)
    assert a.check_finite() == 0
    fa, fb = a.fields(8), b.fields(8)
    assert np.array_equal(fa["F"], fb["F"]) and np.array_equal(fa["ux"], fb["ux"])
    a.evolution(100)
    cd = a.getDrag_block()[2]
    assert 0.5 < cd < 5.0
    st = a.stats()
    assert st["updates_per_coarse_step"] == 6986527
    assert st["kernels_per_coarse_step"] > 0


def test_tecplot_writer_matches_oracle(mb, orc, cuda_device, tmp_path):
    g, o, m = make_pair(mb, orc, "g25", "f64")
    o.evolution(10)
    m.evolution(10)
    o.output(str(tmp_path / "o.dat"))
    m.output(str(tmp_path / "m.dat"))
    lo = (tmp_path / "o.dat").read_text().splitlines()
    lm = (tmp_path / "m.dat").read_text().splitlines()
    assert len(lo) == len(lm) and lo[:3] == lm[:3]
    for x, y in zip(lo[3:], lm[3:]):
        if x.startswith("ZONE"):
            assert x == y
            continue
        vx, vy = x.split("\t"), y.split("\t")
        assert vx[2] == vy[2] and len(vx) == len(vy) == 6
        # %g prints values near 1e-17 (zero up to rounding) differently
        np.testing.assert_allclose([float(v) for v in vx[:2] + vx[3:]], [float(v) for v in vy[:2] + vy[3:]],
                                   rtol=2e-6, atol=1e-12)


def test_error_codes(mb, cuda_device):
    g = mb.config1_geometry()
    s = mb.MultiBlockLBM(g, "f32")
    with pytest.raises(mb.MBError) as e:
        s.evolution(1)
    assert e.value.code == -8  # step before init
    with pytest.raises(mb.MBError):
        s.lib.mb_copy_fields(s.h, 99, None, None, None, None, None, None) and mb._check(-1, "x")
    assert s.lib.mb_copy_fields(s.h, 99, None, None, None, None, None, None) == -1
    import ctypes as C

    h = C.c_void_p()
    assert mb.load().mb_create(C.byref(g), 7, C.byref(h)) == -1


@pytest.mark.parametrize("name", ["g25", "n3", "g49"])
def test_interior_rim_split(mb, orc, cuda_device, name):
    """Every level stepped as separate interior and rim nodes (threshold 0):
    FP64 equals the oracle and FP32 equals the unsplit run bitwise."""
    g, o, m = make_pair(mb, orc, name, "f64", True)
    m.set_split_cells(0)
    o.evolution(14)
    m.evolution(14)
    assert m.getDrag_block()[2] == pytest.approx(o.getDrag_block()[2], rel=1e-11)
    for fo, fm in zip(all_fields(o, g), all_fields(m, g)):
        for k in ("rho", "ux", "uy", "F"):
            np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-12)
    a = mb.MultiBlockLBM(g, "f32")
    b = mb.MultiBlockLBM(g, "f32")
    b.set_split_cells(0)
    for s in (a, b):
        s.init()
        s.evolution(14)
    for k in range(g.layout.number_area):
        assert np.array_equal(a.fields(k)["F"], b.fields(k)["F"])


@pytest.mark.parametrize("split", [0, 10**12])
@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("prec", ["f32", "f16s", "f64", "f16c"])
def test_quad_kernel_equals_cell_kernel(mb, cuda_device, prec, variant, split):
    """Every block-step variant gives bitwise the same state, on whole levels
    and on split (interior + rim) levels."""
    g = mb.geo_init(*make_ref.case("n3")[:2])
    a = mb.MultiBlockLBM(g, prec)
    b = mb.MultiBlockLBM(g, prec)
    for lvl in range(g.layout.LEVEL):
        a.set_stb_variant(lvl, 0)
        b.set_stb_variant(lvl, variant)
    b.set_split_cells(split)
    for s in (a, b):
        s.init()
        s.evolution(9)
    for k in range(g.layout.number_area):
        fa, fb = a.fields(k), b.fields(k)
        for key in ("F", "rho", "ux", "uy"):
            assert np.array_equal(fa[key], fb[key]), (k, key)


@pytest.mark.parametrize("name", ["n3", "g49"])
def test_programmatic_edges_bitwise(mb, cuda_device, name):
    """Graphs with programmatic kernel-to-kernel edges give the same state."""
    g = mb.geo_init(*make_ref.case(name)[:2])
    sims = [mb.MultiBlockLBM(g, "f32", graph=mode) for mode in (False, True, "pdl")]
    for s in sims:
        s.set_split_cells(0)
        s.init()
        s.evolution(19)
    ref = [sims[0].fields(k) for k in range(g.layout.number_area)]
    for s in sims[1:]:
        for k in range(g.layout.number_area):
            f = s.fields(k)
            for key in ("F", "ux"):
                assert np.array_equal(f[key], ref[k][key]), (k, key)
        assert s.getDrag_block() == sims[0].getDrag_block()


def test_checkpoint_restart_bitwise(mb, cuda_device, tmp_path):
    """Save after 7 steps, run 11 more; a fresh context restored from the file
    and run 11 steps ends bitwise equal, drag included."""
    g = mb.geo_init(*make_ref.case("n3")[:2])
    a = mb.MultiBlockLBM(g, "f32")
    a.init()
    a.evolution(7)
    (tmp_path / "ck.bin").write_bytes(a.checkpoint())
    a.evolution(11)
    b = mb.MultiBlockLBM(g, "f32")
    b.restore((tmp_path / "ck.bin").read_bytes())
    b.evolution(11)
    for k in range(g.layout.number_area):
        fa, fb = a.fields(k), b.fields(k)
        for key in ("F", "rho", "ux", "uy"):
            assert np.array_equal(fa[key], fb[key])
    assert a.getDrag_block() == b.getDrag_block()
    assert a.error_L2() == b.error_L2()
    c = mb.MultiBlockLBM(g, "f64")
    with pytest.raises(mb.MBError):
        c.restore((tmp_path / "ck.bin").read_bytes())


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("split", [10**12, 0])
@pytest.mark.parametrize("prec", ["f32", "f64", "f16s", "f16c"])
def test_step_diag_equals_step_by_step(mb, cuda_device, prec, split, graph):
    """mb_step_diag (plans of several steps with the drag and the L2 change of
    each step beside the next) gives the values of mb_step(1), mb_drag and
    mb_error_L2 called in turn, bitwise, and the same final state, over two
    calls in a row."""
    g = mb.geo_init(*make_ref.case("n3")[:2])
    a = mb.MultiBlockLBM(g, prec, graph=graph)
    b = mb.MultiBlockLBM(g, prec, graph=graph)
    for s in (a, b):
        s.set_split_cells(split)
        s.init()
    ref = []
    for _ in range(17):
        a.evolution(1)
        _, _, cd, cl = a.getDrag_block()
        ref.append((cd, cl, a.error_L2()))
    cd1, cl1, err1 = b.evolution_diag(13)
    cd2, cl2, err2 = b.evolution_diag(4)
    cd, cl, err = np.concatenate([cd1, cd2]), np.concatenate([cl1, cl2]), np.concatenate([err1, err2])
    assert np.array_equal(cd, [r[0] for r in ref])
    assert np.array_equal(cl, [r[1] for r in ref])
    assert np.array_equal(err, [r[2] for r in ref])
    for k in range(g.layout.number_area):
        fa, fb = a.fields(k), b.fields(k)
        for key in ("F", "rho", "ux", "uy"):
            assert np.array_equal(fa[key], fb[key])


@pytest.mark.parametrize("graph", [True, False, "program"])
@pytest.mark.parametrize("split,variant", [(10**12, 0), (0, 0), (10**12, 4), (0, 4), (0, 3), (0, 5), (0, 6)])
@pytest.mark.parametrize("name,prec", [("n3", "f32"), ("g49", "f64"), ("g25", "f16s"), ("n3", "f16c")])
def test_fused_copies_bitwise(mb, cuda_device, name, prec, split, variant, graph):
    """Same-level copies done inside the block step (mb_set_fusion bit 0),
    temporal interpolations done by the splines (bits 1 and 2), f_c points
    inside the fine steps (bit 3) and record launches split by what they wait
    for (bit 4), alone and together, give bitwise the state of separate
    launches."""
    g = mb.geo_init(*make_ref.case(name)[:2])
    sims = []
    for fuse in (0, 1, 2, 3, 4, 5, 7, 9, 17, 25, 31):
        s = mb.MultiBlockLBM(g, prec, graph=graph)
        s.set_fusion(fuse)
        s.set_split_cells(split)
        for lvl in range(g.layout.LEVEL):
            s.set_stb_variant(lvl, variant)
        s.init()
        s.evolution(13)
        sims.append(s)
    cd0, l20 = sims[0].getDrag_block()[2], sims[0].error_L2()
    for other in sims[1:]:
        for k in range(g.layout.number_area):
            fa, fb = sims[0].fields(k), other.fields(k)
            for key in ("F", "rho", "ux", "uy"):
                assert np.array_equal(fa[key], fb[key]), (k, key)
        assert cd0 == other.getDrag_block()[2]
        assert l20 == other.error_L2()


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_fused_tskip_options_kernel_bitwise(mb, cuda_device, prec, graph):
    """With a collision option on, every block step runs the options kernel
    (k_block_step_x); the splines' next temporal interpolation (fusion bit 2,
    with the fine substep in between leaving those edge cells alone) still
    gives bitwise the state of separate launches."""
    g = mb.geo_init(*make_ref.case("n3")[:2])
    sims = []
    for fuse in (0, 4, 5, 7):
        s = mb.MultiBlockLBM(g, prec, graph=graph)
        s.set_fusion(fuse)
        s.set_body_force(1e-6, 0.0)
        s.init()
        s.evolution(13)
        sims.append(s)
    for other in sims[1:]:
        for k in range(g.layout.number_area):
            fa, fb = sims[0].fields(k), other.fields(k)
            for key in ("F", "rho", "ux", "uy"):
                assert np.array_equal(fa[key], fb[key]), (k, key)
        assert sims[0].getDrag_block()[2] == other.getDrag_block()[2]


@pytest.mark.parametrize("prec", ["f32", "f16c"])
def test_shift_modes(mb, orc, cuda_device, prec):
    """Both shifts of the stored words (f - w and f - feq(rho0, U0)) give the
    scheme: every field within the precision's bound of the FP64 oracle after
    300 steps of the 3-level nested layout; a checkpoint of one shift does not
    load into a context of the other."""
    g = mb.geo_init(*make_ref.case("n3")[:2])
    o = orc.Oracle(g)
    o.init()
    o.evolution(300)
    fo = all_fields(o, g)
    tol = 2e-5 if prec == "f32" else 2e-3
    ck = {}
    for shift in ("w", "feq0"):
        m = mb.MultiBlockLBM(g, prec, shift=shift)
        m.init()
        m.evolution(300)
        fm = all_fields(m, g)
        eu, er = rel_l2(g, fo, fm, "u"), rel_l2(g, fo, fm, "rho")
        print(f"{prec} shift {shift}: relL2 u {eu:.3e} rho {er:.3e}")
        assert eu <= tol and er <= tol
        ck[shift] = m.checkpoint()
        m.close()
    other = mb.MultiBlockLBM(g, prec, shift="w")
    with pytest.raises(mb.MBError):
        other.restore(ck["feq0"])
    other.restore(ck["w"])
    other.close()


@pytest.mark.parametrize("prec", ["f16c", "f16s"])
@pytest.mark.parametrize("split", [0, 10**12])
def test_stochastic_rounding_variants_bitwise(mb, orc, cuda_device, split, prec):
    """16-bit storage with stochastic rounding: every block-step variant and execution
    mode gives bitwise the same state (the dither is a function of the cell and
    its inputs), the state differs from round-to-nearest's and stays within
    the 16-bit bound of the FP64 oracle; the other precisions refuse it."""
    g = mb.geo_init(*make_ref.case("n3")[:2])
    steps = 60
    sims = []
    for variant, graph in ((0, True), (1, True), (3, True), (5, False), (2, "program"), (6, True), (6, False)):
        s = mb.MultiBlockLBM(g, prec, graph=graph, rounding="stochastic")
        for lvl in range(g.layout.LEVEL):
            s.set_stb_variant(lvl, variant)
        s.set_split_cells(split)
        s.init()
        s.evolution(steps)
        sims.append(s)
    ref = [sims[0].fields(k) for k in range(g.layout.number_area)]
    for s in sims[1:]:
        for k in range(g.layout.number_area):
            f = s.fields(k)
            for key in ("F", "rho", "ux", "uy"):
                assert np.array_equal(f[key], ref[k][key]), (k, key)
    rn = mb.MultiBlockLBM(g, prec, rounding="nearest")
    rn.init()
    rn.evolution(steps)
    assert any(not np.array_equal(rn.fields(k)["F"], ref[k]["F"]) for k in range(g.layout.number_area))
    o = orc.Oracle(g)
    o.init()
    o.evolution(steps)
    fo = all_fields(o, g)
    for s in (rn, sims[0]):
        fm = all_fields(s, g)
        eu, er = rel_l2(g, fo, fm, "u"), rel_l2(g, fo, fm, "rho")
        print(f"{prec} {'stochastic' if s is sims[0] else 'nearest'}: relL2 u {eu:.3e} rho {er:.3e}")
        assert eu <= (2e-3 if prec == "f16c" else 5e-3) and er <= (2e-3 if prec == "f16c" else 5e-3)
    for s in sims + [rn]:
        s.close()
    f32 = mb.MultiBlockLBM(g, "f32")
    with pytest.raises(mb.MBError):
        f32.set_rounding("stochastic")
    f32.set_rounding("nearest")
    f32.close()


@pytest.mark.parametrize("name,prec,variant,split,graph", [
    ("n3", "f32", 0, None, True), ("n3", "f32", 1, 0, True), ("n3", "f16s", 4, None, True),
    ("n3", "f16c", 3, 0, False), ("n3", "f64", 0, None, True), ("g49", "f32", 5, 0, True),
    ("c1", "f32", 0, None, True), ("g25", "f16s", 4, 0, False), ("n3", "f32u", 0, None, True),
    ("n3", "f32u", 2, None, True), ("n3", "f16s", 6, None, True), ("g25", "f16c", 6, 0, False)])
def test_fc_fusion_bitwise(mb, cuda_device, name, prec, variant, split, graph):
    """f_c points done inside the fine level's last block step (mb_set_fusion
    bit 3) give bitwise the state, drag and L2 series of the record launches,
    for every block-step kernel; the plan of the nested layout carries them."""
    g = mb.geo_init(*make_ref.case(name)[:2])
    sims = []
    for flags in (1, 9, 25):
        s = mb.MultiBlockLBM(g, prec, graph=graph)
        s.set_fusion(flags)
        for lvl in range(g.layout.LEVEL):
            s.set_stb_variant(lvl, variant)
        if split is not None:
            s.set_split_cells(split)
        s.init()
        s.evolution(13)
        sims.append(s)
    if name == "n3" and split is None:  # split fine levels keep f_c sources in their bulk interiors: records
        # the two-cell kernel (variant 2) computes cells in its own paired code: records
        # and in unshifted FP32 the per-cell code compiled into k_fc_pull rounds differently: records
        assert (" ; fc " in sims[1].plan_description(6)) == (variant != 2 and prec != "f32u")
        assert " ; fc " not in sims[0].plan_description(6)
    a = sims[0]
    for b in sims[1:]:
        for k in range(g.layout.number_area):
            fa, fb = a.fields(k), b.fields(k)
            for key in ("F", "rho", "ux", "uy"):
                assert np.array_equal(fa[key], fb[key]), (k, key)
    da = a.evolution_diag(8)
    for b in sims[1:]:
        db = b.evolution_diag(8)
        for x, y in zip(da, db):
            assert np.array_equal(x, y)
        for k in range(g.layout.number_area):
            assert np.array_equal(a.fields(k)["F"], b.fields(k)["F"]), k
    for s in sims:
        s.close()


def test_fc_fusion_after_cell_type_change(mb, cuda_device):
    """Cell types changed through mb_set_cell_types keep the f_c source marks:
    fused and record f_c points still agree bitwise."""
    g = mb.geo_init(*make_ref.case("n3")[:2])
    sims = []
    for flags in (1, 9):
        s = mb.MultiBlockLBM(g, "f32")
        s.set_fusion(flags)
        s.init()
        a = g.layout.number_area - 1
        A = g.Areas[a]
        t = s.fields(a)["solid"].copy()
        t[A.ny // 2, A.nx // 2 - 3] = 1  # one more solid cell inside the finest block
        s.set_cell_types(a, t)
        s.init()
        s.evolution(11)
        sims.append(s)
    for k in range(g.layout.number_area):
        assert np.array_equal(sims[0].fields(k)["F"], sims[1].fields(k)["F"]), k
    for s in sims:
        s.close()
