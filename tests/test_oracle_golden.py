"""Pins the FP64 oracle to the reference's own CUDA build.

tests/golden/<case>.npz were produced by running the reference (its kernels,
geo_init, evolution, error_L2 and getDrag_block, compiled unmodified from its
sources by oracle/ref_harness/make_ref.py) on a B200 for the case's step
count (oracle/ref_harness/make_golden.py).  The oracle must reproduce them at
FP64 rounding level."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

import make_ref

TOL_FIELD = 1e-11   # abs, rho ~ 1, |u| ~ 0.1
TOL_DRAG = 1e-10    # relative, per step


@pytest.fixture(scope="module")
def runs(mb, orc):
    out = {}
    for name in make_ref.GOLDEN:
        L, cfg, steps = make_ref.case(name)
        g = mb.geo_init(L, cfg)
        o = orc.Oracle(g)
        o.init()
        drag, l2 = [], []
        for _ in range(steps):
            o.evolution(1)
            l2.append(o.error_L2())
            drag.append(o.getDrag_block()[:2])
        out[name] = (g, o, np.array(drag), np.array(l2))
    return out


@pytest.mark.parametrize("name", make_ref.GOLDEN)
def test_fields(runs, name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    g, o, _, _ = runs[name]
    for a in range(g.layout.number_area):
        f = o.fields(a)
        assert (f["solid"] == z[f"solid_{a}"]).all()
        for k in ("rho", "ux", "uy"):
            np.testing.assert_allclose(f[k], z[f"{k}_{a}"], rtol=0, atol=TOL_FIELD, err_msg=f"{name} block {a} {k}")
        np.testing.assert_allclose(f["F"].sum(axis=(1, 2)), z[f"Fsum_{a}"], rtol=1e-12, err_msg=f"{name} F {a}")
        np.testing.assert_allclose(f["f"].sum(axis=(1, 2)), z[f"fsum_{a}"], rtol=1e-12, err_msg=f"{name} f {a}")


@pytest.mark.parametrize("name", make_ref.GOLDEN)
def test_drag_series(runs, name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    _, _, drag, _ = runs[name]
    ref = z["drag"]
    assert drag.shape == ref.shape
    scale = np.abs(ref[:, 0]).max()
    assert np.abs(drag - ref).max() <= TOL_DRAG * scale


@pytest.mark.parametrize("name", make_ref.GOLDEN)
def test_l2_series(runs, name):
    """error_L2.dat holds %g values: 6 significant digits."""
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    _, _, _, l2 = runs[name]
    np.testing.assert_allclose(l2, z["l2"], rtol=6e-6, atol=1e-300)


@pytest.mark.parametrize("name", make_ref.GOLDEN)
def test_ring_slots(runs, name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    g, o, _, _ = runs[name]
    for b in range(g.layout.number_line):
        assert o.markers(b) == list(z["markers"][b])
        np.testing.assert_allclose(o.slots(b).sum(axis=2), z["slotsum"][b], rtol=1e-12)


def test_tecplot_format(runs, tmp_path):
    """output() (output/output.h:2-38) text, compared value by value."""
    z = np.load(os.path.join(GOLDEN, "g11.npz"))
    _, o, _, _ = runs["g11"]
    p = tmp_path / "steady.dat"
    o.output(str(p))
    ours = p.read_text().splitlines()
    ref = bytes(z["tecplot"]).decode().splitlines()
    assert len(ours) == len(ref)
    assert ours[:3] == ref[:3]
    for a, b in zip(ours[3:], ref[3:]):
        va, vb = a.split("\t"), b.split("\t")
        assert len(va) == len(vb) == 6
        assert va[2] == vb[2]
        np.testing.assert_allclose([float(v) for v in va[:2] + va[3:]], [float(v) for v in vb[:2] + vb[3:]], rtol=1e-5)
