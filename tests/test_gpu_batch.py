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
    batch.evolution(5)
    # 5 candidates x (one untimed chunk of period + 1 = 7 steps, then 3 timed), then 5 more
    steps_done = 5 * (7 + 3) + 5
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
