"""The persistent plan executor (graph mode "program") against the CUDA-graph
path and the FP64 oracle.

Every cell update is computed by the same device code in both modes, so the
executor must reproduce the graph path bitwise, whatever the work-item sizes
and the order in which CTAs claim items; in FP64 it must match the oracle to
the tolerances of the other parity tests (fields 1e-12 absolute, Cd 1e-11
relative).  The timeout test makes the executor's bounded wait run out on a
node that nothing makes ready and checks that the error reaches the host and
that the context keeps working.
"""
import numpy as np
import pytest

import make_ref

pytestmark = pytest.mark.gpu

MB_ERR_TIMEOUT = -7


def run(mb, g, prec, graph, steps, split=None, items=None):
    s = mb.MultiBlockLBM(g, prec, graph=graph)
    if split is not None:
        s.set_split_cells(split)
    if items is not None:
        s.set_program_shape(*items)
    s.init()
    s.evolution(steps)
    return s


def assert_same_state(g, a, b):
    for k in range(g.layout.number_area):
        fa, fb = a.fields(k), b.fields(k)
        for key in ("F", "rho", "ux", "uy"):
            assert np.array_equal(fa[key], fb[key]), (k, key)
    assert a.getDrag_block() == b.getDrag_block()


@pytest.mark.parametrize("prec", ["f32", "f16s", "f64", "f32u", "f16c"])
@pytest.mark.parametrize("name", ["n3", "g49", "c1"])
def test_program_equals_graph_bitwise(mb, cuda_device, name, prec):
    g = mb.geo_init(*make_ref.case(name)[:2])
    a = run(mb, g, prec, True, 19)
    b = run(mb, g, prec, "program", 19)
    assert_same_state(g, a, b)


@pytest.mark.parametrize("name", ["n3", "g25"])
def test_program_split_levels_bitwise(mb, cuda_device, name):
    """Interior nodes of every level are bulk work of the executor."""
    g = mb.geo_init(*make_ref.case(name)[:2])
    a = run(mb, g, "f32", True, 14, split=0)
    b = run(mb, g, "f32", "program", 14, split=0)
    assert_same_state(g, a, b)


@pytest.mark.parametrize("items", [(32, 32, 1, 0), (100, 7, 3, 5), (4096, 2048, 2, 64), (512, 256, 2, 1)])
def test_program_item_sizes_bitwise(mb, cuda_device, items):
    g = mb.geo_init(*make_ref.case("n3")[:2])
    a = run(mb, g, "f32", True, 13, split=0)
    b = run(mb, g, "f32", "program", 13, split=0, items=items)
    assert_same_state(g, a, b)


@pytest.mark.parametrize("name", ["g25", "n3", "g49"])
def test_program_f64_matches_oracle(mb, orc, cuda_device, name):
    L, cfg, _ = make_ref.case(name)
    g = mb.geo_init(L, cfg)
    o = orc.Oracle(g)
    o.init()
    m = mb.MultiBlockLBM(g, "f64", graph="program")
    m.init()
    for n in (1, 13, 1):  # single steps and a multi-step plan
        o.evolution(n)
        m.evolution(n)
        assert m.getDrag_block()[2] == pytest.approx(o.getDrag_block()[2], rel=1e-11)
        assert m.error_L2() == pytest.approx(o.error_L2(), rel=1e-11)
    for a in range(g.layout.number_area):
        fo, fm = o.fields(a), m.fields(a)
        for k in ("rho", "ux", "uy", "F"):
            np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-12, err_msg=f"{name} {k}")


def test_program_config2_bitwise(mb, cuda_device):
    """The 3-level 4096 x 1024 case with split coarse level, 13 steps."""
    g = mb.config2_geometry()
    a = run(mb, g, "f32", True, 13)
    b = run(mb, g, "f32", "program", 13)
    assert_same_state(g, a, b)
    assert a.error_L2() == b.error_L2()


def test_program_timeout_reaches_host(mb, cuda_device):
    g = mb.geo_init(*make_ref.case("n3")[:2])
    s = mb.MultiBlockLBM(g, "f32", graph="program")
    s.init()
    s.set_program_timeout(0.05)
    assert s.program_selftest(0) == 0
    assert s.program_selftest(1) == MB_ERR_TIMEOUT
    # reported once; the context stays usable
    assert s.program_selftest(0) == 0
    s.sync()
    s.evolution(7)
    s.sync()
    ref = run(mb, g, "f32", True, 7)
    assert_same_state(g, ref, s)


def test_program_trace(mb, cuda_device):
    """Tracing records every executed item and leaves the results unchanged."""
    g = mb.geo_init(*make_ref.case("n3")[:2])
    a = run(mb, g, "f32", "program", 6)
    b = mb.MultiBlockLBM(g, "f32", graph="program")
    b.set_program_trace(1 << 16)
    b.init()
    b.evolution(6)
    tr = b.program_trace()
    assert len(tr) > 0
    assert (tr["t_pick"] <= tr["t_start"]).all() and (tr["t_start"] <= tr["t_end"]).all()
    assert len(np.unique(tr["launch"])) >= 2  # 5 single steps + the final step are separate launches
    # every (launch, node, item) ran exactly once
    keys = np.stack([tr["launch"], tr["plan_node"], tr["item"]], axis=1)
    assert len(np.unique(keys, axis=0)) == len(tr)
    assert_same_state(g, a, b)
    assert len(b.program_trace()) == 0  # emptied by the read


@pytest.mark.parametrize("prec", ["f32", "f16s", "f64", "f16c"])
@pytest.mark.parametrize("name,split", [("n3", 0), ("g49", 0), ("c1", 0), ("n3", None)])
def test_hybrid_equals_graph_bitwise(mb, cuda_device, name, split, prec):
    """Graph mode "hybrid": the chain as executor launches between the bulk
    interior kernels (split levels) gives the graph path's state bitwise, with
    single steps, multi-step plans and the diagnostics loop."""
    g = mb.geo_init(*make_ref.case(name)[:2])
    a = run(mb, g, prec, True, 19, split=split)
    b = run(mb, g, prec, "hybrid", 19, split=split)
    assert_same_state(g, a, b)
    da = a.evolution_diag(7)
    db = b.evolution_diag(7)
    for x, y in zip(da, db):
        assert np.array_equal(x, y)
    assert_same_state(g, a, b)


@pytest.mark.parametrize("per_sm", [1, 3])
def test_hybrid_grid_caps_bitwise(mb, cuda_device, per_sm):
    g = mb.geo_init(*make_ref.case("n3")[:2])
    a = run(mb, g, "f32", True, 13, split=0)
    b = mb.MultiBlockLBM(g, "f32", graph="hybrid")
    b.set_hybrid_ctas(per_sm)
    b.set_split_cells(0)
    b.init()
    b.evolution(13)
    assert_same_state(g, a, b)
