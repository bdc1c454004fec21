"""Parity of the options kernel (k_block_step_x: MRT, body force, free-slip and
half-way bounce-back walls) with the FP64 oracle, through the C ABI.

Tolerances: FP64 storage 1e-12 absolute on the fields and 1e-10 relative on
Cd after 20 coarse steps (FMA contraction is the only difference in operation
order); a single block step from a random state 1e-14.  FP32 storage:
relative L2 of u <= 2e-5; Cd <= 1e-4 relative for f - w storage, 5e-4 for
unshifted f (measured 1.1e-4 at 20 steps with every option on).
"""
import numpy as np
import pytest

import make_ref
from test_gpu_parity import _randomise, _stale_f_init, all_fields, rel_l2

pytestmark = pytest.mark.gpu

FLUID, SBB, SLIP, HBB = 0, 1, 2, 3


def hbb_cylinder(sim, g):
    a = g.layout.number_area - 1
    t = sim.fields(a)["solid"].copy()
    t[t == SBB] = HBB
    return a, t


def slip_rows(sim, g):
    t = sim.fields(0)["solid"].copy()
    ny = t.shape[0]
    t[3, 1:-1] = SLIP
    t[ny - 4, 1:-1] = SLIP
    return 0, t


OPTIONS = {
    "mrt": dict(coll=(1, 1.1, 1.2, 1.3)),
    "mrt_bgk_rates": dict(coll=(1, 0.0, 0.0, 0.0)),
    "force": dict(force=(2e-5, -1e-5)),
    "mrt_force": dict(coll=(1, 1.4, 1.0, 1.2), force=(1e-5, 3e-6)),
    "hbb": dict(types=hbb_cylinder),
    "slip": dict(types=slip_rows),
    "all": dict(coll=(1, 1.1, 1.2, 1.3), force=(1e-5, 0.0), types=hbb_cylinder, types2=slip_rows),
}


def apply(sim, g, opt):
    if "coll" in opt:
        sim.set_collision(*opt["coll"])
    if "force" in opt:
        sim.set_body_force(*opt["force"])
    for key in ("types", "types2"):
        if key in opt:
            a, t = opt[key](sim, g)
            sim.set_cell_types(a, t)


def make(mb, orc, name, prec, opt, graph=True):
    L, cfg, _ = make_ref.case(name)
    g = mb.geo_init(L, cfg)
    o = orc.Oracle(g)
    o.init()
    apply(o, g, opt)
    m = mb.MultiBlockLBM(g, prec, graph=graph)
    m.init()
    apply(m, g, opt)
    return g, o, m


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("name", ["n2", "g25"])
@pytest.mark.parametrize("which", list(OPTIONS))
def test_f64_options_match_oracle(mb, orc, cuda_device, which, name, graph):
    g, o, m = make(mb, orc, name, "f64", OPTIONS[which], graph)
    assert m.drag_links() == len(o.drag_links())
    for _ in range(4):
        o.evolution(5)
        m.evolution(5)
        dm, do = m.getDrag_block(), o.getDrag_block()
        assert dm[2] == pytest.approx(do[2], rel=1e-10)
        assert dm[3] == pytest.approx(do[3], rel=1e-8, abs=1e-12)
        assert m.error_L2() == pytest.approx(o.error_L2(), rel=1e-10)
    for fo, fm in zip(all_fields(o, g), all_fields(m, g)):
        assert (fo["solid"] == fm["solid"]).all()
        for k in ("rho", "ux", "uy", "F"):
            np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-12, err_msg=f"{which} {k}")


@pytest.mark.parametrize("which", ["mrt_force", "all"])
def test_f64_options_block_step_random_state(mb, orc, cuda_device, which):
    g, o, m = make(mb, orc, "g25", "f64", OPTIONS[which])
    _randomise(g, o, m, 3)
    _stale_f_init(g, o, orc)
    for a in range(g.layout.number_area):
        o.block_step(a)
        m.block_step(a)
    for a, (fo, fm) in enumerate(zip(all_fields(o, g), all_fields(m, g))):
        np.testing.assert_allclose(fm["F"], fo["F"], rtol=0, atol=1e-14, err_msg=f"block {a}")
        fl = fo["solid"] == 0
        for k in ("rho", "ux", "uy"):
            np.testing.assert_allclose(fm[k][fl], fo[k][fl], rtol=0, atol=1e-14)


@pytest.mark.parametrize("prec", ["f32", "f32u"])
@pytest.mark.parametrize("which", ["mrt", "force", "all"])
def test_f32_options_match_oracle(mb, orc, cuda_device, which, prec):
    g, o, m = make(mb, orc, "n2", prec, OPTIONS[which])
    o.evolution(20)
    m.evolution(20)
    fo, fm = all_fields(o, g), all_fields(m, g)
    assert rel_l2(g, fo, fm, "u") <= 2e-5
    # unshifted FP32 storage rounds f itself (|f| up to 0.45), 10x coarser than f - w
    assert m.getDrag_block()[2] == pytest.approx(o.getDrag_block()[2], rel=1e-4 if prec == "f32" else 5e-4)


def test_options_off_again_is_the_plain_step(mb, orc, cuda_device):
    """Switching every option off again returns to the standard kernels,
    bitwise the step of a context that never had options."""
    L, cfg, _ = make_ref.case("g25")
    g = mb.geo_init(L, cfg)
    ref = mb.MultiBlockLBM(g, "f32")
    ref.init()
    m = mb.MultiBlockLBM(g, "f32")
    m.init()
    a = g.layout.number_area - 1
    orig = m.fields(a)["solid"].copy()
    apply(m, g, OPTIONS["all"])
    m.evolution(3)
    m.set_collision(0)
    m.set_body_force(0.0, 0.0)
    m.set_cell_types(a, orig)
    m.set_cell_types(0, np.where(m.fields(0)["solid"] == SLIP, FLUID, m.fields(0)["solid"]))
    m.init()
    ref.evolution(7)
    m.evolution(7)
    for fr, fm in zip(all_fields(ref, g), all_fields(m, g)):
        assert np.array_equal(fr["F"], fm["F"])
        assert (fr["solid"] == fm["solid"]).all()


def test_options_refused_by_executor_and_batches(mb, cuda_device):
    L, cfg, _ = make_ref.case("g25")
    g = mb.geo_init(L, cfg)
    m = mb.MultiBlockLBM(g, "f32", graph="program")
    m.init()
    m.set_body_force(1e-5, 0.0)
    with pytest.raises(mb.MBError):
        m.evolution(1)
    with pytest.raises(mb.MBError):
        mb.Batch([m])
    with pytest.raises(mb.MBError):
        m.set_collision(1, 2.5, 1.0, 1.0)
    bad = m.fields(1)["solid"].copy()
    bad[bad == 9] = FLUID
    with pytest.raises(mb.MBError):
        m.set_cell_types(1, bad)
