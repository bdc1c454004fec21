"""The oracle's collision and boundary options that the reference declares but
never uses: MRT (lbm/lbm.h:53-75, lbm/assit_func.h:10-22), the body-force term
of stb3 (multi/FH/evolution_block.h:97-108), free slip (slip_gpu,
lbm/lbm.h:51) and half-way bounce-back (SOLID_HBB, lbm/lbm.h:28).

With no reference kernel to compare against, the checks are the identities
each option must satisfy: MRT with every rate at 1/tau is BGK, the force term
adds dt (1 - tau^-1/2) F of momentum per step and no mass, half-way
bounce-back conserves the mass of a closed cavity, and a free-slip wall
leaves a uniform stream parallel to it unchanged.
"""
import numpy as np
import pytest

import make_ref

FLUID, SBB, SLIP, HBB, CB = 0, 1, 2, 3, 9
BGK, MRT = 0, 1


def oracle(mb, orc, name):
    L, cfg, _ = make_ref.case(name)
    g = mb.geo_init(L, cfg)
    o = orc.Oracle(g)
    return g, o


def fields(o, g):
    return [o.fields(a) for a in range(g.layout.number_area)]


def test_mrt_at_bgk_rates_is_bgk(mb, orc):
    g, a = oracle(mb, orc, "n2")
    _, b = oracle(mb, orc, "n2")
    a.init()
    b.set_collision(MRT, 0.0, 0.0, 0.0)  # every rate at the block's 1/tau
    b.init()
    a.evolution(20)
    b.evolution(20)
    for fa, fb in zip(fields(a, g), fields(b, g)):
        assert np.abs(fa["F"] - fb["F"]).max() < 1e-13
        assert np.abs(fa["ux"] - fb["ux"]).max() < 1e-13
    assert a.getDrag_block()[2] == pytest.approx(b.getDrag_block()[2], rel=1e-10)


def test_mrt_rates_change_the_flow_but_keep_it_bounded(mb, orc):
    g, a = oracle(mb, orc, "n2")
    _, b = oracle(mb, orc, "n2")
    a.init()
    b.set_collision(MRT, 1.1, 1.2, 1.3)
    b.init()
    a.evolution(30)
    b.evolution(30)
    diff = max(np.abs(fa["ux"] - fb["ux"]).max() for fa, fb in zip(fields(a, g), fields(b, g)))
    assert 1e-7 < diff < 1e-2
    with pytest.raises(ValueError):
        b.set_collision(7)


def test_body_force_adds_momentum_not_mass(mb, orc):
    g, o = oracle(mb, orc, "g11")
    fx, fy = 3e-5, -2e-5
    o.set_body_force(fx, fy)
    o.init()
    A = g.Areas[0]
    o.block_step(0)
    f = o.fields(0)
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
    ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
    F = f["F"]
    # interior cells away from the cylinder and the block edge: pulled
    # equilibrium at (rho0, U0), so F carries that plus the force term
    sl = (slice(2, 5), slice(30, 40))
    rho = F.sum(axis=0)[sl]
    jx = np.tensordot(ex, F, axes=1)[sl]
    jy = np.tensordot(ey, F, axes=1)[sl]
    k = (1.0 / A.m) * (1.0 - 0.5 * A.rv_tau)
    assert np.abs(rho - 1.0).max() < 1e-15
    assert np.abs(jx - (0.1 + k * fx)).max() < 1e-15
    assert np.abs(jy - k * fy).max() < 1e-15
    # block-edge FLUID cells: stb3 collides the equilibrium, so they also
    # carry the term (evolution_block.h:90-111 runs for every FLUID cell)
    jx_edge = np.tensordot(ex, F, axes=1)[0, 20]
    assert jx_edge == pytest.approx(0.1 + k * fx, abs=1e-15)


def cavity_types(o, a, box):
    """Cell types of block a with the cylinder removed and a closed ring of
    HBB cells on the border of box = (i0, i1, j0, j1)."""
    t = o.fields(a)["solid"].copy()
    t[t == SBB] = FLUID
    i0, i1, j0, j1 = box
    t[j0:j1 + 1, i0] = HBB
    t[j0:j1 + 1, i1] = HBB
    t[j0, i0:i1 + 1] = HBB
    t[j1, i0:i1 + 1] = HBB
    return t


def test_halfway_bounce_back_closed_cavity_keeps_its_mass(mb, orc):
    g, o = oracle(mb, orc, "g11")
    o.init()
    box = (10, 30, 4, 18)
    o.set_cell_types(0, cavity_types(o, 0, box))
    f = o.fields(0)
    rng = np.random.default_rng(5)
    F = f["F"].copy()
    i0, i1, j0, j1 = box
    F[:, j0 + 1:j1, i0 + 1:i1] *= 1.0 + 0.02 * rng.standard_normal((9, j1 - j0 - 1, i1 - i0 - 1))
    o.set_fields(0, F=F)
    m0 = F[:, j0 + 1:j1, i0 + 1:i1].sum()
    for _ in range(60):
        o.block_step(0)
    F1 = o.fields(0)["F"]
    assert F1[:, j0 + 1:j1, i0 + 1:i1].sum() == pytest.approx(m0, rel=1e-13)
    # the drag sum runs over the links of HBB cells as over SBB ones
    assert o.drag_links().shape[0] > 0


def test_halfway_bounce_back_cylinder_drag_is_close_to_on_node(mb, orc):
    g, a = oracle(mb, orc, "g11")
    _, b = oracle(mb, orc, "g11")
    a.init()
    b.init()
    t = b.fields(0)["solid"].copy()
    t[t == SBB] = HBB
    b.set_cell_types(0, t)
    assert a.drag_links().shape == b.drag_links().shape
    a.evolution(200)
    b.evolution(200)
    cda, cdb = a.getDrag_block()[2], b.getDrag_block()[2]
    assert cda != cdb
    assert cdb == pytest.approx(cda, rel=0.15)


def test_free_slip_walls_keep_a_parallel_stream(mb, orc):
    g, o = oracle(mb, orc, "g11")
    _, s = oracle(mb, orc, "g11")
    for sim, wall in ((o, SLIP), (s, SBB)):
        sim.init()
        t = sim.fields(0)["solid"].copy()
        t[t == SBB] = FLUID
        ny = t.shape[0]
        t[4, 1:-1] = wall
        t[ny - 5, 1:-1] = wall
        sim.set_cell_types(0, t)
        for _ in range(40):
            sim.block_step(0)
    ny = o.fields(0)["ux"].shape[0]
    slip = o.fields(0)["ux"][5:ny - 5, 1:-1]
    noslip = s.fields(0)["ux"][5:ny - 5, 1:-1]
    assert np.abs(slip - 0.1).max() < 1e-13
    assert np.abs(noslip - 0.1).max() > 1e-3


def test_cell_types_reject_interface_cells(mb, orc):
    g, o = oracle(mb, orc, "n2")
    o.init()
    t = o.fields(1)["solid"].copy()
    assert (t == CB).any()
    bad = t.copy()
    bad[t == CB] = FLUID
    with pytest.raises(ValueError):
        o.set_cell_types(1, bad)
    bad = t.copy()
    bad[t == FLUID] = 5
    with pytest.raises(ValueError):
        o.set_cell_types(1, bad)


def test_channel_walls_of_config1(mb, orc):
    """mblbm.channel_walls marks the domain's bottom and top rows (inlet and
    outlet columns excepted) free-slip and the cylinder half-way bounce-back;
    the oracle then runs the config-1 case with those boundaries."""
    g = mb.config1_geometry()
    o = orc.Oracle(g)
    o.init()
    mb.channel_walls(o, g)
    cfg = g.config
    for a in range(g.layout.number_area):
        A = g.Areas[a]
        t = o.fields(a)["solid"]
        y = A.base_y + np.arange(A.ny) / A.m
        x = A.base_x + np.arange(A.nx) / A.m
        for j in range(A.ny):
            wall = y[j] in (0.0, cfg.LY - 1.0)
            for i in (1, A.nx // 2):
                if wall and x[i] not in (0.0, cfg.LX - 1.0):
                    assert t[j, i] == SLIP
        assert not (t == SBB).any()
    assert (o.fields(g.layout.number_area - 1)["solid"] == HBB).sum() > 0
    o.evolution(20)
    assert np.isfinite(o.getDrag_block()[2])
