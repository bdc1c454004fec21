"""geo_init / Line_init (geo/init_geo.h:17-165): product vs oracle vs the
reference's own tables (dumped by its geo_init into the golden fixtures)."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN

import make_ref


BUILTIN_CASES = [(n, LX, LY) for n in ("1_1", "2_2", "2_5", "4_9") for (LX, LY) in ((768, 320), (64, 32), (200, 80), (86, 38))]


@pytest.mark.parametrize("name,LX,LY", BUILTIN_CASES)
def test_builtin_layouts_product_equals_oracle(mb, orc, name, LX, LY):
    L = mb.layout_builtin(name)
    cfg = mb.make_config(LX, LY, 3, LX // 4, LY // 2)
    g1 = mb.geo_init(L, cfg)
    g2 = orc.geo_init(L, cfg)
    assert bytes(g1) == bytes(g2)
    assert mb.coverage(g1) == 0


def test_reference_default_2_5_extents(mb):
    """The numbers geo_init gives for the shipped parameters.h (LX=768, LY=320)."""
    g = mb.geo_init(mb.layout_builtin("2_5"), mb.make_config(768, 320, 10, 160, 160, U0=(0.1, 0.0), Re=10.0))
    ext = [(g.AreaDefine[a].xstart, g.AreaDefine[a].xend, g.AreaDefine[a].ystart, g.AreaDefine[a].yend) for a in range(5)]
    assert ext == [(0, 767, 238, 319), (0, 767, 0, 80), (0, 144, 79, 239), (238, 767, 79, 239), (143, 239, 79, 239)]
    assert (g.Areas[4].nx, g.Areas[4].ny, g.Areas[4].m) == (193, 321, 2)
    nu = 0.1 * 2 * 10 / 10.0
    assert g.Areas[0].tau == pytest.approx(0.5 + 3 * nu, rel=0, abs=1e-15)
    assert g.Areas[4].tau == pytest.approx(0.5 + 2 * (3 * nu), rel=0, abs=1e-15)
    l0 = g.Line_Inf_C[0]
    assert (l0.areac_n, l0.areaf_n, l0.Nc, l0.Nf) == (0, 4, 97, 193)


@pytest.mark.parametrize("name", make_ref.GOLDEN)
def test_tables_equal_reference_geo_init(mb, name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    z = np.load(path)
    L, cfg, _ = make_ref.case(name)
    g = mb.geo_init(L, cfg)
    raw = bytes(z["geometry_raw"])
    # the reference dumps AreaDefine, Areas, Line_Inf_C/F/CC sized by its own tables
    na, nl, nl2 = L.number_area, max(1, L.number_line), max(1, L.number_line2)
    ours = (bytes((mb.P4 * na)(*g.AreaDefine[:na])) + bytes((mb.Area * na)(*g.Areas[:na]))
            + bytes((mb.Line * nl)(*g.Line_Inf_C[:nl])) + bytes((mb.Line * nl)(*g.Line_Inf_F[:nl]))
            + bytes((mb.Line * nl2)(*g.Line_Inf_CC[:nl2])))
    assert len(raw) == len(ours)
    assert raw == ours


def test_benchmark_layouts(mb, orc):
    g1 = mb.config1_geometry()
    assert [(g1.Areas[a].nx, g1.Areas[a].ny) for a in range(5)] == [(400, 41), (400, 42), (62, 81), (261, 81), (161, 161)]
    assert mb.updates_per_coarse_step(g1) == 111205
    g2 = mb.config2_geometry()
    assert g2.layout.LEVEL == 3 and g2.layout.number_area == 9
    assert mb.updates_per_coarse_step(g2) == 6986527
    for g in (g1, g2):
        assert mb.coverage(g) == 0
        assert bytes(orc.geo_init(g.layout, g.config)) == bytes(g)
    # tau per level from nu = |U0| D / Re (init_geo.h:101-109)
    nu = 0.04 * 32 / 100.0
    taus = [0.5 + 3 * nu]
    for _ in range(2):
        taus.append(0.5 + 2 * (taus[-1] - 0.5))
    assert [g2.Areas[a].tau for a in (0, 4, 8)] == pytest.approx(taus, abs=1e-15)


@pytest.mark.parametrize("boxes", [[(1, 10, 5, 20)], [(10, 90, 10, 20), (11, 12, 11, 12)], [(10, 398, 10, 50)]])
def test_nested_layout_rejects_bad_boxes(mb, boxes):
    with pytest.raises(mb.MBError) as e:
        mb.layout_nested(400, 60, boxes)
    assert e.value.code == -4


def test_geo_init_rejects_bad_tables(mb):
    L = mb.layout_builtin("2_5")
    L.NeborCF[0].nc = 77
    with pytest.raises(mb.MBError):
        mb.geo_init(L, mb.make_config(64, 32, 3, 15, 15))
    L = mb.layout_builtin("2_5")
    L.number_line2 = 7  # same-level lines come in pairs
    with pytest.raises(mb.MBError):
        mb.geo_init(L, mb.make_config(64, 32, 3, 15, 15))
