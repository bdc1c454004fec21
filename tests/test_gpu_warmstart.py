"""Learned warm start end to end at a small scale: snapshots from the batched
solver, a few hundred Adam steps of the surrogate, and a warm start of two
held-out cases.  The warm-started state must step stably, and its drag after
one coarse step must be closer to the developed drag of the cold-started run
than the cold start's own first-step drag."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 1500
D_RANGE = (10.0, 12.0)


def test_warm_start_pipeline(mb, cuda_device):
    import torch
    from mblbm import surrogate as sg

    h, w = 64, 128
    x, t, m, ids = sg.generate(range(16), STEPS / D_RANGE[1], "f32", h, w, d_range=D_RANGE)
    assert len(ids) >= 12 and np.isfinite(t).all()
    X, T, M = (torch.from_numpy(a).cuda() for a in (x, t, m))
    net = mb.UNet(h, w, max_batch=4, seed=3)
    hist = sg.train(net, X, T, M, epochs=60, batch=4, lr=2e-3)
    assert hist[-1] < 0.5 * hist[0]
    for cid in (100, 101):
        g, prm = mb.batch_case(cid, d_range=D_RANGE)
        cold = mb.MultiBlockLBM(g, "f32")
        cold.init()
        cold.evolution(1)
        cd_cold1 = cold.getDrag_block()[2]
        cold.evolution(STEPS - 1)
        cd_dev = cold.getDrag_block()[2]
        xin, _ = sg.case_inputs(g, h, w)
        pred = sg.predict(net, torch.from_numpy(xin[None]).cuda())[0].cpu().numpy()
        warm = mb.MultiBlockLBM(g, "f32")
        warm.init()
        sg.warm_start(warm, g, pred)
        warm.evolution(1)
        cd_warm1 = warm.getDrag_block()[2]
        warm.evolution(200)
        assert warm.check_finite() == 0
        assert abs(cd_warm1 - cd_dev) < abs(cd_cold1 - cd_dev), (cid, cd_warm1, cd_cold1, cd_dev)
        cold.close()
        warm.close()
    net.close()


def _steady_ids(lo, hi, d_range, re_max=47.0):
    """Case ids in [lo, hi) of the batched distribution whose Re is below
    re_max (steady wakes)."""
    import mblbm

    return [i for i in range(lo, hi) if mblbm.batch_case(i, d_range=d_range)[1]["Re"] < re_max]


def test_warm_start_reaches_cd_band_sooner(mb, cuda_device):
    """On held-out steady cases, the warm start from a surrogate trained on
    developed snapshots settles within 0.5 % of the converged drag (the cold
    run's final value) in fewer coarse steps than the cold start."""
    import torch
    from mblbm import surrogate as sg

    h, w = 64, 128
    d_range = (10.0, 12.0)
    train_ids = _steady_ids(0, 200, d_range)[:32]
    x, t, m, ids = sg.generate(train_ids, 600.0, "f32", h, w, d_range=d_range)
    assert len(ids) >= 24
    X, T, M = (torch.from_numpy(a).cuda() for a in (x, t, m))
    net = mb.UNet(h, w, max_batch=8, seed=5)
    hist = sg.train(net, X, T, M, epochs=80, batch=8, lr=2e-3)
    assert hist[-1] < 0.2 * hist[0]
    held = [i for i in _steady_ids(1000, 1200, d_range) if mb.batch_case(i, d_range=d_range)[1]["levels"] == 2][:3]
    n = 8000
    gains = []
    for cid in held:
        g, _ = mb.batch_case(cid, d_range=d_range)
        cold = mb.MultiBlockLBM(g, "f32")
        cold.init()
        cd_c, _, _ = cold.evolution_diag(n)
        ref = float(np.mean(cd_c[-500:]))
        assert abs(cd_c[-1] / ref - 1) < 1e-3  # converged
        xin, _ = sg.case_inputs(g, h, w)
        pred = sg.predict(net, torch.from_numpy(xin[None]).cuda())[0].cpu().numpy()
        warm = mb.MultiBlockLBM(g, "f32")
        warm.init()
        sg.warm_start(warm, g, pred)
        cd_w, _, _ = warm.evolution_diag(n)
        assert warm.check_finite() == 0
        sc, sw = mb.settle_step(cd_c, ref), mb.settle_step(cd_w, ref)
        print(f"case {cid}: cold settles at {sc}, warm at {sw} (Cd {ref:.5f})")
        gains.append((sc, sw))
        cold.close()
        warm.close()
    net.close()
    assert len(gains) == 3
    assert all(sw < sc for sc, sw in gains), gains
    assert sum(sw for _, sw in gains) < 0.8 * sum(sc for sc, _ in gains), gains
