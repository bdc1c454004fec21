"""Host side of the learned warm start: the wake kick that warm_start adds to
the surrogate's prediction of a shedding case (surrogate.wake_kick)."""
import numpy as np


def _case(mb, want_shedding):
    from mblbm import surrogate as sg
    for i in range(200):
        g, prm = mb.batch_case(i)
        if (prm["Re"] >= sg.RE_SHEDDING) == want_shedding:
            return g
    raise AssertionError("no such case among the first 200")


def test_wake_kick_shape(mb):
    from mblbm import surrogate as sg
    g = _case(mb, True)
    c = g.config
    h, w = 64, 128
    v = sg.wake_kick(c, h, w, 0.5)
    assert v.shape == (h, w)
    # peak kick * U0 at the grid point nearest (CX + 3R, CY), a Gaussian of radius R
    gx, gy = (c.LX - 1.0) / (w - 1), (c.LY - 1.0) / (h - 1)
    j, i = np.unravel_index(np.argmax(v), v.shape)
    assert abs(i * gx - (c.CX + 3 * c.R)) <= gx and abs(j * gy - c.CY) <= gy
    assert 0.5 * c.U0[0] * np.exp(-1.0) < v.max() <= 0.5 * c.U0[0]
    assert v.min() >= 0.0
    # far from the wake (upstream of the obstacle) it vanishes
    assert v[:, : int((c.CX - 2 * c.R) / gx)].max() < 1e-6 * c.U0[0]


def test_wake_kick_off(mb):
    from mblbm import surrogate as sg
    steady = _case(mb, False)
    shedding = _case(mb, True)
    assert not sg.wake_kick(steady.config, 32, 64, 0.5).any()
    assert not sg.wake_kick(shedding.config, 32, 64, 0.0).any()
