"""mb_error_L2_noalloc against mb_error_L2, through the C ABI.

The no-allocation entry point is for callers that cannot allocate device
memory (an application that owns the device through its own pool, or a loop
that must not pay the synchronisation of cudaMalloc/cudaFree).  It must give
the result of the context's mb_error_L2 on the same velocities, on two calls
in a row: the second call sees the shared scratch as the first left it and
the previous velocity the first call wrote.  This file is collected last."""
import numpy as np
import pytest

import make_ref

pytestmark = pytest.mark.gpu


def test_noalloc_l2_matches_context_l2_twice(mb, cuda_device):
    import torch

    g = mb.geo_init(*make_ref.case("n3")[:2])
    sim = mb.MultiBlockLBM(g, "f64")
    sim.init()
    nblk = g.layout.number_area
    # the caller's own device arrays: u_prev starts at U0, as mb_init sets it
    c = g.config
    up = []
    for a in range(nblk):
        n = g.Areas[a].nx * g.Areas[a].ny
        up.append((torch.full((n,), c.U0[0], dtype=torch.float64, device=cuda_device),
                   torch.full((n,), c.U0[1], dtype=torch.float64, device=cuda_device)))
    out = torch.zeros(3, dtype=torch.float64, device=cuda_device)
    for call in range(2):
        sim.evolution(7)
        ref = sim.error_L2()  # the context's entry point (its own scratch)
        cur = []
        for a in range(nblk):
            f = sim.fields(a)
            cur.append((torch.from_numpy(f["ux"].ravel().copy()).to(cuda_device),
                        torch.from_numpy(f["uy"].ravel().copy()).to(cuda_device)))
        segs = [(cur[a][0].data_ptr(), cur[a][1].data_ptr(), up[a][0].data_ptr(), up[a][1].data_ptr(),
                 cur[a][0].numel(), 1.0 / g.Areas[a].m) for a in range(nblk)]
        assert mb.error_L2_noalloc(segs, out.data_ptr()) == 0
        torch.cuda.synchronize()
        e = float(out[2])
        assert e == pytest.approx(ref, rel=1e-12), (call, e, ref)
        for a in range(nblk):  # u_prev <- u
            assert torch.equal(up[a][0], cur[a][0]) and torch.equal(up[a][1], cur[a][1])


def test_noalloc_l2_rejects_too_many_segments(mb, cuda_device):
    import torch

    x = torch.zeros(4, dtype=torch.float64, device=cuda_device)
    out = torch.zeros(3, dtype=torch.float64, device=cuda_device)
    seg = (x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(), 4, 1.0)
    assert mb.error_L2_noalloc([seg] * (mb.MB_L2_NOALLOC_MAX_SEGMENTS + 1), out.data_ptr()) == -5
