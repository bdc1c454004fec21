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
