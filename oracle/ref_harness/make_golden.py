"""Runs the reference's own CUDA build on small cases and packs golden fixtures.

TEST INFRASTRUCTURE ONLY.  Needs a CUDA device and the binaries built by
make_ref.py (oracle/_ref/ref_<case>).  For every case of make_ref.GOLDEN it
runs `ref_<case> golden <steps>` in a scratch directory and writes
<out>/<case>.npz with:
  areas, lines_C, lines_F, lines_CC   geometry tables from geo_init()
  drag        (steps, 2)  force[] of getDrag_block after every step, FP64
  l2          (steps,)    error_L2.dat values (the reference prints %g)
  rho_<a>, ux_<a>, uy_<a>, up_<a>     final fields of block a, FP64
  solid_<a>, Fsum_<a>, fsum_<a>       cell types and per-direction sums
  markers, slotsum                    ring markers and per-slot sums per line
  tecplot                             steady_<steps>.dat text (case g11 only)
With --long CASE STEPS it runs one benchmark case (c1: the 400x160 2-level
cylinder at Re=40) for STEPS coarse steps and writes <out>/<CASE>_<STEPS>.npz
with the final rho/ux/uy of every block and the drag and error_L2 series
sampled every --every steps (pack_long).
The committed fixtures in tests/golden/ were produced by
    python oracle/ref_harness/make_ref.py && python oracle/ref_harness/make_golden.py --out <dir>
on a B200 and copied from <dir>.
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_ref  # noqa: E402
import mblbm  # noqa: E402  (path set by make_ref)


def pack(name, wd, geo, steps):
    L = geo.layout
    out = {}
    raw = open(os.path.join(wd, "geometry.bin"), "rb").read()
    out["geometry_raw"] = np.frombuffer(raw, dtype=np.uint8)
    out["drag"] = np.fromfile(os.path.join(wd, "drag.bin"), dtype=np.float64).reshape(steps, 2)
    l2 = [float(line.split()[1]) for line in open(os.path.join(wd, "error_L2.dat")) if line.strip()]
    out["l2"] = np.array(l2)
    buf = open(os.path.join(wd, "fields.bin"), "rb").read()
    off = 0
    for a in range(L.number_area):
        nx, ny = geo.Areas[a].nx, geo.Areas[a].ny
        N = nx * ny
        solid = np.frombuffer(buf, dtype=np.int32, count=N, offset=off).reshape(ny, nx)
        off += 4 * N
        arr = np.frombuffer(buf, dtype=np.float64, count=25 * N, offset=off).reshape(25, ny, nx)
        off += 8 * 25 * N
        up = np.frombuffer(buf, dtype=np.float64, count=2 * N, offset=off).reshape(2, ny, nx)
        off += 8 * 2 * N
        out[f"solid_{a}"] = solid.astype(np.int8)
        out[f"rho_{a}"] = arr[2].copy()
        out[f"ux_{a}"] = arr[3].copy()
        out[f"uy_{a}"] = arr[4].copy()
        out[f"up_{a}"] = up.copy()
        out[f"fsum_{a}"] = arr[7:16].sum(axis=(1, 2))
        out[f"Fsum_{a}"] = arr[16:25].sum(axis=(1, 2))
    markers, slotsum = [], []
    for b in range(L.number_line):
        m = np.frombuffer(buf, dtype=np.int32, count=3, offset=off)
        off += 12
        Nf = geo.Line_Inf_C[b].Nf
        sl = np.frombuffer(buf, dtype=np.float64, count=27 * Nf, offset=off).reshape(3, 9, Nf)
        off += 8 * 27 * Nf
        markers.append(m.copy())
        slotsum.append(sl.sum(axis=2))
    out["markers"] = np.array(markers, dtype=np.int32).reshape(-1, 3)
    out["slotsum"] = np.array(slotsum).reshape(-1, 3, 9)
    assert off == len(buf), (off, len(buf))
    if name == "g11":
        out["tecplot"] = np.frombuffer(open(os.path.join(wd, f"steady_{steps}.dat"), "rb").read(), dtype=np.uint8)
    return out


def pack_long(wd, geo, steps, every):
    """A long run of a benchmark case, kept small: the final rho, ux, uy of
    every block (FP64), the cell types, and the drag and error_L2 series
    sampled every `every` steps plus the last step."""
    L = geo.layout
    out = {}
    drag = np.fromfile(os.path.join(wd, "drag.bin"), dtype=np.float64).reshape(steps, 2)
    l2 = np.array([float(line.split()[1]) for line in open(os.path.join(wd, "error_L2.dat")) if line.strip()])
    idx = np.unique(np.r_[np.arange(every - 1, steps, every), steps - 1])
    out["sample_steps"] = idx + 1
    out["drag"] = drag[idx]
    out["l2"] = l2[idx]
    buf = open(os.path.join(wd, "fields.bin"), "rb").read()
    off = 0
    for a in range(L.number_area):
        nx, ny = geo.Areas[a].nx, geo.Areas[a].ny
        N = nx * ny
        out[f"solid_{a}"] = np.frombuffer(buf, dtype=np.int32, count=N, offset=off).reshape(ny, nx).astype(np.int8)
        off += 4 * N
        arr = np.frombuffer(buf, dtype=np.float64, count=25 * N, offset=off).reshape(25, ny, nx)
        off += 8 * 27 * N
        out[f"rho_{a}"] = arr[2].copy()
        out[f"ux_{a}"] = arr[3].copy()
        out[f"uy_{a}"] = arr[4].copy()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--long", nargs=2, metavar=("CASE", "STEPS"),
                    help="one long run of a benchmark case (e.g. c1 20000), packed as <out>/<CASE>_<STEPS>.npz")
    ap.add_argument("--every", type=int, default=20, help="--long: drag and L2 sample interval")
    ap.add_argument("names", nargs="*")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.long:
        name, steps = a.long[0], int(a.long[1])
        L, cfg, _ = make_ref.case(name)
        geo = mblbm.geo_init(L, cfg)
        exe = os.path.join(make_ref.OUT, f"ref_{name}")
        wd = tempfile.mkdtemp(prefix=f"ref_{name}_")
        r = subprocess.run([exe, "golden", str(steps)], cwd=wd, capture_output=True, text=True, timeout=3000)
        print(name, steps, r.returncode, r.stdout.strip(), r.stderr.strip()[-500:], flush=True)
        if r.returncode != 0:
            return 1
        np.savez_compressed(os.path.join(a.out, f"{name}_{steps}.npz"), steps=steps,
                            **pack_long(wd, geo, steps, a.every))
        return 0
    for name in a.names or make_ref.GOLDEN:
        L, cfg, steps = make_ref.case(name)
        geo = mblbm.geo_init(L, cfg)
        exe = os.path.join(make_ref.OUT, f"ref_{name}")
        wd = tempfile.mkdtemp(prefix=f"ref_{name}_")
        r = subprocess.run([exe, "golden", str(steps)], cwd=wd, capture_output=True, text=True, timeout=600)
        print(name, r.returncode, r.stdout.strip(), r.stderr.strip()[-500:], flush=True)
        if r.returncode != 0:
            return 1
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), steps=steps, **pack(name, wd, geo, steps))
    return 0


if __name__ == "__main__":
    sys.exit(main())
