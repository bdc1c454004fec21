"""Batches of independent cases (mb_batch_*): every case advanced in a batch
equals the same case advanced alone, bitwise (the batched launches run the
single-case device code on each case's parameters), whatever the interface
work shape the autotuner picks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cases(mb, ids, levels, d_range=(10.0, 14.0)):
    return [mb.batch_case(i, levels=levels, d_range=d_range)[0] for i in ids]


def assert_same(geo, a, b):
    for k in range(geo.layout.number_area):
        fa, fb = a.fields(k), b.fields(k)
        for key in ("F", "rho", "ux", "uy"):
            assert np.array_equal(fa[key], fb[key]), (k, key)


@pytest.mark.parametrize("levels", [2, 3])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_batch_equals_single_cases(mb, cuda_device, levels, prec):
    geos = cases(mb, range(5), levels)
    sims = [mb.MultiBlockLBM(g, prec) for g in geos]
    alone = [mb.MultiBlockLBM(g, prec) for g in geos]
    for s in sims + alone:
        s.init()
    batch = mb.Batch(sims)
    batch.evolution(13)
    cd, cl = batch.drag()
    for g, s, a, c1, c2 in zip(geos, sims, alone, cd, cl):
        a.evolution(13)
        assert_same(g, s, a)
        _, _, acd, acl = a.getDrag_block()
        assert c1 == acd and c2 == acl
    batch.close()


def test_batch_autotune_keeps_results(mb, cuda_device):
    geos = cases(mb, range(4), 3)
    sims = [mb.MultiBlockLBM(g, "f32") for g in geos]
    alone = [mb.MultiBlockLBM(g, "f32") for g in geos]
    for s in sims + alone:
        s.init()
    batch = mb.Batch(sims)
    choice = batch.autotune(steps=3)
    assert choice["rec_points"] in (32, 64) and 1 <= choice["spline_segments"] <= 4 and choice["ms_per_step"] > 0
    assert choice["stb_ctas_per_sm"] in (0, 2, 4, 8) and choice["stb_kernel"] in (0, 1)
    batch.evolution(5)
    # 7 kernel/schedule pairs + 4 interface shapes, each (one untimed chunk of
    # period + 1 = 7 steps, then 3 timed), then 5 more
    steps_done = 11 * (7 + 3) + 5
    for g, a, s in zip(geos, alone, sims):
        a.evolution(steps_done)
        assert_same(g, s, a)
    batch.close()


def test_batch_rejects_diverged_state(mb, cuda_device):
    geos = cases(mb, range(2), 2)
    sims = [mb.MultiBlockLBM(g, "f32") for g in geos]
    for s in sims:
        s.init()
    batch = mb.Batch(sims)
    sims[0].evolution(1)
    with pytest.raises(mb.MBError):
        batch.evolution(1)
    batch.close()


@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("sched", [0, 1, 2, 4, 8])
@pytest.mark.parametrize("prec", ["f32", "f64", "f16s"])
def test_batch_persistent_schedule_bitwise(mb, cuda_device, prec, sched, kernel):
    """The persistent block-step schedule (k CTAs per SM over equal shares of
    the 256-cell tiles of all cases), and the cell-pair kernel on such a grid,
    give the state of one CTA per tile of one cell per thread."""
    if prec == "f64" and sched > 4:
        pytest.skip("FP64 block steps run at most 4 CTAs per SM")
    if kernel == 0 and sched == 0:
        pytest.skip("the reference schedule itself")
    geos = cases(mb, range(6), 3, d_range=(10.0, 30.0))
    a = [mb.MultiBlockLBM(g, prec) for g in geos]
    b = [mb.MultiBlockLBM(g, prec) for g in geos]
    for s in a + b:
        s.init()
    ba, bb = mb.Batch(a), mb.Batch(b)
    bb.set_schedule(sched)
    bb.set_kernel(kernel)
    ba.evolution(9)
    bb.evolution(9)
    for g, x, y in zip(geos, a, b):
        assert_same(g, x, y)
    ba.close()
    bb.close()


@pytest.mark.parametrize("levels", [2, 3])
def test_batch_f64_matches_oracle_full_ranges(mb, orc, cuda_device, levels):
    """FP64 batches of the batched workload's cases over its full ranges
    (D in [10, 40], Re in [20, 200], ellipses of aspect 1-3 at any angle)
    against the FP64 C oracle, every field after 12 coarse steps and the
    drag."""
    ids = [3, 17, 42] if levels == 2 else [12, 14]
    drawn = [mb.batch_case(i, levels=levels) for i in ids]
    geos = [g for g, _ in drawn]
    assert max(p["D"] for _, p in drawn) > 25 and min(p["Re"] for _, p in drawn) < 150
    sims = [mb.MultiBlockLBM(g, "f64") for g in geos]
    for s in sims:
        s.init()
    batch = mb.Batch(sims)
    batch.set_schedule(4)
    batch.set_interface_shape(64, 2)
    n = 0
    batch.evolution(12)
    cd, _ = batch.drag()
    for g, s, c in zip(geos, sims, cd):
        o = orc.Oracle(g)
        o.init()
        o.evolution(n + 12)
        for k in range(g.layout.number_area):
            fo, fm = o.fields(k), s.fields(k)
            for key in ("rho", "ux", "uy", "F"):
                np.testing.assert_allclose(fm[key], fo[key], rtol=0, atol=1e-12, err_msg=f"block {k} {key}")
        assert c == pytest.approx(o.getDrag_block()[2], rel=1e-10)
        o.close()
    batch.close()
