"""Periodic level-0 domains (mb_config.periodic) on the GPU against the FP64
oracle, and the 2-level Taylor-Green vortex on 1024^2 coarse cells with a
256^2-cell refined patch (512^2 fine cells), u0 = 0.01, tau = 0.6, 5000
coarse steps, in FP16-shifted and FP32 storage.

Tolerances: FP64 storage 1e-12 absolute on the fields and 1e-11 relative on
the L2 change, as for the non-periodic parity.  After 200 steps of the small
vortex: relative L2 of u <= 1e-5 for FP32 (f - w), 5e-5 for unshifted FP32,
5e-3 for FP16 (f - w).  Full size: the FP64 amplitudes after 1000 and 5000
steps within 1e-9 relative of the oracle's (tests/golden/tgv_1024.json), and
within 0.1% of u0 exp(-2 nu k^2 t) (the oracle is 1.7e-4 below it: the
refinement interfaces add a little dissipation); FP32 within 5e-4 and FP16S
within 2e-3 of the FP64 run's amplitude (measured 1.6e-4 and 3.4e-4: FP32
arithmetic on f rounds at 1e-8 absolute per step, which 5000 steps
accumulate).
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from test_gpu_parity import all_fields, rel_l2
from test_periodic import CASES, poiseuille, poiseuille_profile_error, poiseuille_walls

pytestmark = pytest.mark.gpu


def pair(mb, orc, name, prec="f64", graph=True, tgv=None, split=None, variant=None):
    g = CASES[name](mb)
    o = orc.Oracle(g)
    o.init()
    m = mb.MultiBlockLBM(g, prec, graph=graph)
    if split is not None:
        m.set_split_cells(split)
    if variant is not None:
        for lvl in range(g.layout.LEVEL):
            m.set_stb_variant(lvl, variant)
    m.init()
    if tgv if tgv is not None else name.startswith("tgv"):
        mb.tgv_init(o, g)
        mb.tgv_init(m, g)
    return g, o, m


@pytest.mark.parametrize("graph", [True, False, "program"])
@pytest.mark.parametrize("name", list(CASES))
def test_f64_periodic_matches_oracle(mb, orc, cuda_device, name, graph):
    g, o, m = pair(mb, orc, name, "f64", graph)
    for _ in range(12):
        o.evolution(1)
        m.evolution(1)
        assert m.error_L2() == pytest.approx(o.error_L2(), rel=1e-11)
    if name == "channel_x":
        assert m.getDrag_block()[2] == pytest.approx(o.getDrag_block()[2], rel=1e-11)
    for fo, fm in zip(all_fields(o, g), all_fields(m, g)):
        assert (fo["solid"] == fm["solid"]).all()
        for k in ("rho", "ux", "uy", "F"):
            np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-12, err_msg=f"{name} {k}")


@pytest.mark.parametrize("split,variant", [(0, 1), (0, 3), (10**12, 0), (10**12, 5), (0, 5)])
def test_f64_periodic_kernel_variants(mb, orc, cuda_device, split, variant):
    g, o, m = pair(mb, orc, "tgv2", "f64", True, split=split, variant=variant)
    o.evolution(9)
    m.evolution(9)
    for fo, fm in zip(all_fields(o, g), all_fields(m, g)):
        for k in ("rho", "ux", "uy", "F"):
            np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-12, err_msg=k)


def test_fused_ghost_copies_bitwise(mb, cuda_device):
    """Ghost copies done beside the block step (the default), and temporal
    interpolations done by the splines (fusion bits 1 and 2), equal separate
    launches bitwise."""
    g = CASES["tgv2"](mb)
    out = []
    for fuse in (0, 1, 2, 4, 5):
        s = mb.MultiBlockLBM(g, "f32")
        s.set_fusion(fuse)
        s.init()
        mb.tgv_init(s, g)
        s.evolution(13)
        out.append([s.fields(a) for a in range(g.layout.number_area)])
    for other in out[1:]:
        for fa, fb in zip(out[0], other):
            for key in ("F", "rho", "ux", "uy"):
                assert np.array_equal(fa[key], fb[key])


@pytest.mark.parametrize("prec,tol", [("f32", 1e-5), ("f32u", 6e-5), ("f16s", 5e-3), ("f16c", 2e-3)])
def test_reduced_precision_periodic(mb, orc, cuda_device, prec, tol):
    g, o, m = pair(mb, orc, "tgv2", prec)
    o.evolution(200)
    m.evolution(200)
    fo, fm = all_fields(o, g), all_fields(m, g)
    eu = rel_l2(g, fo, fm, "u")
    print(f"{prec}: relL2 u {eu:.3e}")
    assert eu <= tol
    assert mb.tgv_amplitude(m, g, fm) == pytest.approx(mb.tgv_amplitude(o, g, fo), rel=tol)


def test_tgv_1024_two_levels_decay(mb, cuda_device):
    """The 2-level vortex of the FP16-shifted workload: 1024^2 coarse cells,
    a centred 256^2-cell refined patch, 5000 coarse steps, against the
    oracle's amplitudes (tests/golden/tgv_1024.json) and the exact decay."""
    with open(os.path.join(GOLDEN, "tgv_1024.json")) as f:
        gold = json.load(f)
    g = mb.tgv_geometry(n=1024, patch=256, u0=0.01, tau=0.6, levels=2)
    nu = (g.Areas[0].tau - 0.5) / 3.0
    k = 2 * np.pi / 1024
    amp = {}
    for prec in ("f64", "f32", "f16s", "f16c"):
        s = mb.MultiBlockLBM(g, prec)
        s.init()
        mb.tgv_init(s, g)
        a0 = mb.tgv_amplitude(s, g)
        s.evolution(1000)
        a1000 = mb.tgv_amplitude(s, g)
        s.evolution(4000)
        assert s.check_finite() == 0
        amp[prec] = mb.tgv_amplitude(s, g)
        print(f"{prec}: amplitude {a1000:.10e} {amp[prec]:.10e}")
        if prec == "f64":
            assert a0 == pytest.approx(gold["a0"], rel=1e-12)
            assert a1000 == pytest.approx(gold["amplitude"]["1000"], rel=1e-9)
            assert amp[prec] == pytest.approx(gold["amplitude"]["5000"], rel=1e-9)
        s.close()
    exact = gold["a0"] * np.exp(-2 * nu * k * k * 5000)
    assert amp["f64"] == pytest.approx(exact, rel=1e-3)
    assert amp["f32"] == pytest.approx(amp["f64"], rel=5e-4)
    assert amp["f16s"] == pytest.approx(amp["f64"], rel=2e-3)
    assert amp["f16c"] == pytest.approx(amp["f64"], rel=1e-3)


@pytest.mark.parametrize("levels", [1, 2])
def test_poiseuille_matches_oracle(mb, orc, cuda_device, levels):
    """Body force, on-node walls and x-periodic ghosts together (the options
    kernel with ghost copies), to the steady state: FP64 fields within 1e-12
    of the oracle, FP32's profile error within 5e-3 of u_max of the oracle's
    (measured 1.5e-3 with the patch: FP32 arithmetic adds force increments
    of 1e-7 to f near 0.1, whose spacing is 7.5e-9)."""
    g, fx = poiseuille(mb, levels)
    o = orc.Oracle(g)
    o.init()
    poiseuille_walls(o, g, fx)
    o.evolution(12000)
    for prec in ("f64", "f32"):
        m = mb.MultiBlockLBM(g, prec)
        m.init()
        poiseuille_walls(m, g, fx)
        m.evolution(12000)
        if prec == "f64":
            for fo, fm in zip(all_fields(o, g), all_fields(m, g)):
                for k in ("rho", "ux", "uy", "F"):
                    np.testing.assert_allclose(fm[k], fo[k], rtol=0, atol=1e-12, err_msg=k)
        assert poiseuille_profile_error(m, g, fx) == pytest.approx(poiseuille_profile_error(o, g, fx), abs=5e-3)
        m.close()


def test_periodic_cases_in_a_batch(mb, cuda_device):
    """Vortices of different sizes and amplitudes advanced as one batch equal
    each case advanced alone, bitwise."""
    geos = [mb.tgv_geometry(n=64, patch=32), mb.tgv_geometry(n=96, patch=40), mb.tgv_geometry(n=64, patch=24)]
    amps = (0.01, 0.02, 0.005)
    sims = [mb.MultiBlockLBM(g, "f32") for g in geos]
    alone = [mb.MultiBlockLBM(g, "f32") for g in geos]
    for g, s, a, u0 in zip(geos, sims, alone, amps):
        for x in (s, a):
            x.init()
            mb.tgv_init(x, g, u0)
    batch = mb.Batch(sims)
    batch.evolution(13)
    for g, s, a in zip(geos, sims, alone):
        a.evolution(13)
        for k in range(g.layout.number_area):
            fs, fa = s.fields(k), a.fields(k)
            for key in ("F", "rho", "ux", "uy"):
                assert np.array_equal(fs[key], fa[key]), (k, key)
    batch.close()
