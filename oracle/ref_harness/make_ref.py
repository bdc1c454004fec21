"""Builds the reference's own CUDA code into oracle/_ref/ (test infrastructure).

The reference (zhangya9741/Multi-block-LBM-GPU) takes its physical constants
from parameters.h and its block tables from geo/geometry.h at compile time.
For each named case this script writes one header with both (same names and
types as those files) into oracle/_ref/cfg_<name>.h and compiles

    nvcc -O3 -arch=sm_100a -I<reference> -include cfg_<name>.h ref_main.cu -lcusparse

so every kernel, geo_init, evolution, error_L2 and getDrag_block come from the
unmodified reference sources where they lie; nothing is copied into the
repository.  The binaries run on a GPU box only (oracle/_ref travels with the
snapshot).  Usage: python make_ref.py [--ref DIR] [names...]; the reference
tree is DIR, else $MBLBM_REFERENCE_DIR, else reference_dir()'s default.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
REPO = os.path.dirname(ORACLE)
OUT = os.path.join(ORACLE, "_ref")
sys.path.insert(0, os.path.join(REPO, "multi-block-lbm-gpu_b200"))
import mblbm  # noqa: E402  (layout tables of the product, host-only functions)

# name -> (layout factory, config kwargs, golden steps)
CASES = {
    "g11": (lambda: mblbm.layout_builtin("1_1"), dict(LX=48, LY=24, R=4, CX=16, CY=12, U0=(0.1, 0.0), Re=10.0), 300),
    "g22": (lambda: mblbm.layout_builtin("2_2"), dict(LX=48, LY=24, R=3, CX=14, CY=17, U0=(0.1, 0.0), Re=10.0), 300),
    "g25": (lambda: mblbm.layout_builtin("2_5"), dict(LX=64, LY=32, R=3, CX=15, CY=15, U0=(0.1, 0.0), Re=10.0), 300),
    "g49": (lambda: mblbm.layout_builtin("4_9"), dict(LX=86, LY=38, R=3, CX=16, CY=18, U0=(0.1, 0.0), Re=10.0), 200),
    "n2": (lambda: mblbm.layout_nested(100, 40, [(15, 35, 10, 30)]),
           dict(LX=100, LY=40, R=3, CX=25, CY=20, U0=(0.05, 0.0), Re=40.0), 300),
    "n3": (lambda: mblbm.layout_nested(128, 64, [(30, 95, 15, 49), (46, 79, 24, 41)]),
           dict(LX=128, LY=64, R=3, CX=58, CY=32, U0=(0.04, 0.0), Re=20.0), 200),
    # benchmark workloads (reference arm of bench.py)
    "c1": (lambda: mblbm.layout_nested(400, 160, [(60, 140, 40, 120)]),
           dict(LX=400, LY=160, R=10, CX=100, CY=80, U0=(0.05, 0.0), Re=40.0), 0),
    "c2": (lambda: mblbm.layout_nested(4096, 1024, [(768, 1280, 384, 640), (896, 1152, 448, 576)]),
           dict(LX=4096, LY=1024, R=16, CX=960, CY=512, U0=(0.04, 0.0), Re=100.0), 0),
}
GOLDEN = ["g11", "g22", "g25", "g49", "n2", "n3"]


def case(name):
    lf, kw, steps = CASES[name]
    L = lf()
    cfg = mblbm.make_config(**kw)
    return L, cfg, steps


def header(L, cfg):
    r = repr
    o = ['#ifndef _DATA_MULTI', '#define _DATA_MULTI', '#include "multi/data_type_multi.h"', '#endif',
         '#define _D2Q9', '#define _BLOCKX 16', '#define _BLOCKY 16', '#define _BLOCK_1D (_BLOCKX*_BLOCKY)',
         '#define _BGK', '#define _LOOPS 1', '#define _T 1000',
         f'Lbd Re = {r(cfg.Re)};', f'Lbd rho0 = {r(cfg.rho0)};',
         f'Lbi LY = {cfg.LY};', f'Lbi LX = {cfg.LX};', f'Lbi R = {cfg.R};', f'Lbi CX = {cfg.CX};', f'Lbi CY = {cfg.CY};',
         f'__constant__ Lbi LY_gpu = {cfg.LY};', f'__constant__ Lbi LX_gpu = {cfg.LX};',
         f'__constant__ Lbi R_gpu = {cfg.R};', f'__constant__ Lbi CX_gpu = {cfg.CX};', f'__constant__ Lbi CY_gpu = {cfg.CY};',
         f'Lbd U0[2] = {{ {r(cfg.U0[0])}, {r(cfg.U0[1])} }};',
         'Lbd U0_2 = sqrt(U0[0] * U0[0] + U0[1] * U0[1]);',
         f'__constant__ Lbd rho0_gpu = {r(cfg.rho0)};',
         f'__constant__ Lbd U0_gpu[2] = {{ {r(cfg.U0[0])}, {r(cfg.U0[1])} }};',
         f'const Lbi LEVEL = {L.LEVEL};',
         'Lbi mi[LEVEL] = {' + ', '.join(str(L.mi[i]) for i in range(L.LEVEL)) + '};',
         f'const Lbi number_area = {L.number_area};',
         f'const Lbi number_line = {L.number_line};',
         f'const Lbi number_line2 = {L.number_line2};',
         'Lbi ASP[LEVEL+1] = {' + ', '.join(str(L.ASP[i]) for i in range(L.LEVEL + 1)) + '};']
    zones = []
    for a in range(L.number_area):
        z = L.AreaZone[a]
        zones.append(f'{{{{{r(z.reduced.xstart)}, {r(z.reduced.xend)}, {r(z.reduced.ystart)}, {r(z.reduced.yend)}}}, '
                     f'{{{z.move.xstart}, {z.move.xend}, {z.move.ystart}, {z.move.yend}}}}}')
    o.append('P4d4i AreaZone[number_area] = {' + ',\n  '.join(zones) + '};')
    for nm in ("LTCFFCP", "LS3CFFCP", "LCCP"):
        arr = getattr(L, nm)
        o.append(f'Lbi {nm}[LEVEL+1] = {{' + ', '.join(str(arr[i]) for i in range(L.LEVEL + 1)) + '};')
    cf = [f'{{{L.NeborCF[b].nc}, {L.NeborCF[b].nf}, {L.NeborCF[b].direction}}}' for b in range(L.number_line)]
    cc = [f'{{{L.NeborCC[c].nc}, {L.NeborCC[c].nf}, {L.NeborCC[c].direction}}}' for c in range(L.number_line2)]
    o.append(f'P3i NeborCF[{max(1, L.number_line)}] = {{' + ', '.join(cf) + '};')
    o.append(f'P3i NeborCC[{max(1, L.number_line2)}] = {{' + ', '.join(cc) + '};')
    o.append('#define _GEO')
    return '\n'.join(o) + '\n'


def race_notes(L, cfg):
    """Lines where the reference's own launches race: init_Spline3 reads
    neighbour points other CTAs write when Nc > 256, and init_tri_A's
    conditional stores collide when Nc - 1 is a multiple of 32."""
    g = mblbm.geo_init(L, cfg)
    notes = []
    for b in range(L.number_line):
        nc = g.Line_Inf_C[b].Nc
        if nc > 256:
            notes.append(f"line {b}: Nc={nc} > 256, init_Spline3 reads neighbours written by another CTA")
        if (nc - 1) % 32 == 0:
            notes.append(f"line {b}: Nc={nc}, init_tri_A writes l[Nc-1] from two warps")
    return notes


def reference_dir():
    """Where the reference sources lie: $MBLBM_REFERENCE_DIR, else the
    read-only checkout of the build machine."""
    return os.environ.get("MBLBM_REFERENCE_DIR", "/root/reference")


def build(name, ref):
    L, cfg, _ = case(name)
    os.makedirs(OUT, exist_ok=True)
    hdr = os.path.join(OUT, f"cfg_{name}.h")
    with open(hdr, "w") as f:
        f.write(header(L, cfg))
    exe = os.path.join(OUT, f"ref_{name}")
    cmd = ["nvcc", "-O3", "-arch=sm_100a", "-w", "-I", ref, "-include", hdr, os.path.join(HERE, "ref_main.cu"),
           "-o", exe, "-lcusparse"]
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    for n in race_notes(L, cfg):
        print(f"  [{name}] {n}")
    return exe


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference source tree (default: reference_dir())")
    ap.add_argument("names", nargs="*")
    a = ap.parse_args()
    a.ref = a.ref or reference_dir()
    if not os.path.isdir(a.ref):
        print(f"reference tree {a.ref} absent; nothing built")
        return 0
    for n in a.names or list(CASES):
        build(n, a.ref)
    return 0


if __name__ == "__main__":
    sys.exit(main())
