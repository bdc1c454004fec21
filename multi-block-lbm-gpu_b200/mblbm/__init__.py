"""Python host-side mirror of the mblbm C ABI (include/mblbm.h).

The names follow the reference program's host call surface
(zhangya9741/Multi-block-LBM-GPU): ``geo_init`` (geo/init_geo.h:89),
``evolution`` (evolution.h:2), ``error_L2`` (lbm/error_L2.h:57),
``getDrag_block`` (lbm/force_block.h:180) and ``output``
(output/output.h:2).  Everything runs through ``libmblbm.so``; there is no
Python or CPU fallback: constructing a :class:`MultiBlockLBM` without the
library or without a CUDA device raises.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmblbm.so")

MB_MAX_LEVEL = 8
MB_MAX_AREA = 64
MB_MAX_LINE = 128
MB_MAX_LINE2 = 128

MB_OK = 0
PREC_F64, PREC_F32, PREC_F16S, PREC_F32U, PREC_F16C = 0, 1, 2, 3, 4
# f32: FP32 storage of f - w (the product FP32 form); f32u: FP32 storage of f;
# f16s: IEEE FP16 storage of f - w; f16c: 16-bit storage of f - w with a
# 3-bit exponent and 12-bit fraction (a quarter of FP16's spacing for |f - w| < 1/4)
PRECISIONS = {"f64": PREC_F64, "f32": PREC_F32, "f16s": PREC_F16S, "f32u": PREC_F32U, "f16c": PREC_F16C}
SHIFT_W, SHIFT_FEQ0 = 0, 1  # mb_set_shift modes
ROUND_NEAREST, ROUND_STOCHASTIC = 0, 1  # mb_set_rounding modes
FLUID, SOLID_SBB, C_BOUNDARY = 0, 1, 9
OBST_CIRCLE, OBST_ELLIPSE, OBST_NONE = 0, 1, 2
PERIODIC_X, PERIODIC_Y, DIR_PERIODIC = 1, 2, 8  # mb_config.periodic bits, NeborCC code of ghost lines
MB_FLUID, MB_SOLID_SBB, MB_SOLID_SLIP, MB_SOLID_HBB, MB_C_BOUNDARY = 0, 1, 2, 3, 9
MB_COLL_BGK, MB_COLL_MRT = 0, 1  # cell kinds of mb_copy_fields' solid array


class P4(C.Structure):
    _fields_ = [("xstart", C.c_int), ("xend", C.c_int), ("ystart", C.c_int), ("yend", C.c_int)]


class P4d(C.Structure):
    _fields_ = [("xstart", C.c_double), ("xend", C.c_double), ("ystart", C.c_double), ("yend", C.c_double)]


class Zone(C.Structure):
    _fields_ = [("reduced", P4d), ("move", P4)]


class P3i(C.Structure):
    _fields_ = [("nc", C.c_int), ("nf", C.c_int), ("direction", C.c_int)]


class Layout(C.Structure):
    _fields_ = [
        ("LEVEL", C.c_int),
        ("mi", C.c_int * MB_MAX_LEVEL),
        ("number_area", C.c_int),
        ("number_line", C.c_int),
        ("number_line2", C.c_int),
        ("ASP", C.c_int * (MB_MAX_LEVEL + 1)),
        ("AreaZone", Zone * MB_MAX_AREA),
        ("LTCFFCP", C.c_int * (MB_MAX_LEVEL + 1)),
        ("LS3CFFCP", C.c_int * (MB_MAX_LEVEL + 1)),
        ("LCCP", C.c_int * (MB_MAX_LEVEL + 1)),
        ("NeborCF", P3i * MB_MAX_LINE),
        ("NeborCC", P3i * MB_MAX_LINE2),
    ]


class Config(C.Structure):
    _fields_ = [
        ("Re", C.c_double),
        ("rho0", C.c_double),
        ("LX", C.c_int),
        ("LY", C.c_int),
        ("R", C.c_int),
        ("CX", C.c_int),
        ("CY", C.c_int),
        ("U0", C.c_double * 2),
        ("obstacle", C.c_int),
        ("ell_cx", C.c_double),
        ("ell_cy", C.c_double),
        ("ell_a", C.c_double),
        ("ell_b", C.c_double),
        ("ell_angle", C.c_double),
        ("drag_area", C.c_int),
        ("periodic", C.c_int),
    ]


class Area(C.Structure):
    _fields_ = [
        ("m", C.c_int),
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("base_x", C.c_double),
        ("base_y", C.c_double),
        ("tau", C.c_double),
        ("rv_tau", C.c_double),
    ]


class Line(C.Structure):
    _fields_ = [("areac_n", C.c_int), ("Nc", C.c_int), ("line_C", P4), ("areaf_n", C.c_int), ("Nf", C.c_int), ("line_F", P4)]


class Geometry(C.Structure):
    _fields_ = [
        ("layout", Layout),
        ("config", Config),
        ("AreaDefine", P4 * MB_MAX_AREA),
        ("Areas", Area * MB_MAX_AREA),
        ("Line_Inf_C", Line * MB_MAX_LINE),
        ("Line_Inf_F", Line * MB_MAX_LINE),
        ("Line_Inf_CC", Line * MB_MAX_LINE2),
    ]


class L2Segment(C.Structure):
    """mb_l2_segment: device pointers of one segment for mb_error_L2_noalloc."""

    _fields_ = [("ux", C.c_void_p), ("uy", C.c_void_p), ("upx", C.c_void_p), ("upy", C.c_void_p),
                ("n", C.c_longlong), ("weight", C.c_double)]


MB_L2_NOALLOC_MAX_SEGMENTS = 64

# every symbol declared in include/mblbm.h, with its ctypes signature
_vp = C.c_void_p
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)
_pll = C.POINTER(C.c_longlong)
SIGNATURES = {
    "mb_version": ([], C.c_int),
    "mb_error_string": ([C.c_int], C.c_char_p),
    "mb_layout_builtin": ([C.c_char_p, C.POINTER(Layout)], C.c_int),
    "mb_layout_nested": ([C.c_int, C.c_int, C.c_int, _pi, C.POINTER(Layout)], C.c_int),
    "mb_geo_init": ([C.POINTER(Layout), C.POINTER(Config), C.POINTER(Geometry)], C.c_int),
    "mb_geo_check_coverage": ([C.POINTER(Geometry), _pi], C.c_int),
    "mb_create": ([C.POINTER(Geometry), C.c_int, C.POINTER(_vp)], C.c_int),
    "mb_destroy": ([_vp], C.c_int),
    "mb_init": ([_vp, _vp], C.c_int),
    "mb_step": ([_vp, C.c_int, _vp], C.c_int),
    "mb_set_graph_mode": ([_vp, C.c_int], C.c_int),
    "mb_set_split_cells": ([_vp, C.c_longlong], C.c_int),
    "mb_set_stb_variant": ([_vp, C.c_int, C.c_int], C.c_int),
    "mb_set_bulk_occupancy": ([_vp, C.c_int], C.c_int),
    "mb_set_collision": ([_vp, C.c_int, C.c_double, C.c_double, C.c_double], C.c_int),
    "mb_set_fusion": ([_vp, C.c_int], C.c_int),
    "mb_set_cta_spread": ([_vp, C.c_int, C.c_int], C.c_int),
    "mb_set_body_force": ([_vp, C.c_double, C.c_double], C.c_int),
    "mb_set_cell_types": ([_vp, C.c_int, _pi], C.c_int),
    "mb_set_stream_cells": ([_vp, C.c_longlong, C.c_int], C.c_int),
    "mb_set_interface_shape": ([_vp, C.c_int, C.c_int], C.c_int),
    "mb_set_split_levels": ([_vp, C.c_uint], C.c_int),
    "mb_set_program_timeout": ([_vp, C.c_double], C.c_int),
    "mb_set_program_shape": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
    "mb_sync": ([_vp, _vp], C.c_int),
    "mb_step_diag": ([_vp, C.c_int, _vp, _vp, _vp, _vp], C.c_int),
    "mb_sync_history": ([_vp, _vp], C.c_int),
    "mb_batch_create": ([C.POINTER(_vp), C.c_int, C.POINTER(_vp)], C.c_int),
    "mb_batch_destroy": ([_vp], C.c_int),
    "mb_batch_step": ([_vp, C.c_int, _vp], C.c_int),
    "mb_batch_drag": ([_vp, _vp, _vp, _vp], C.c_int),
    "mb_batch_prepare": ([_vp, C.c_int], C.c_int),
    "mb_unet_create": ([C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(_vp)], C.c_int),
    "mb_unet_destroy": ([_vp], C.c_int),
    "mb_unet_param_count": ([_vp, _pll], C.c_int),
    "mb_unet_get_params": ([_vp, _vp, C.c_longlong, C.c_int], C.c_int),
    "mb_unet_set_params": ([_vp, _vp, C.c_longlong], C.c_int),
    "mb_unet_forward": ([_vp, _vp, C.c_int, _vp, _vp], C.c_int),
    "mb_unet_set_gemm": ([_vp, C.c_int], C.c_int),
    "mb_unet_status": ([_vp, _vp], C.c_int),
    "mb_unet_train_step": ([_vp, _vp, _vp, _vp, C.c_int, C.c_float, C.c_int, C.POINTER(C.c_float), _vp], C.c_int),
    "mb_batch_stats": ([_vp, _pll, _pll, _pll], C.c_int),
    "mb_batch_set_interface_shape": ([_vp, C.c_int, C.c_int], C.c_int),
    "mb_batch_autotune": ([_vp, C.c_int, _vp, _pi, _pi, _pi, _pd, _pi], C.c_int),
    "mb_batch_set_schedule": ([_vp, C.c_int], C.c_int),
    "mb_batch_set_kernel": ([_vp, C.c_int], C.c_int),
    "mb_set_program_trace": ([_vp, C.c_longlong], C.c_int),
    "mb_program_trace": ([_vp, _vp, C.c_longlong, C.POINTER(C.c_longlong)], C.c_int),
    "mb_program_selftest": ([_vp, C.c_int, _vp], C.c_int),
    "mb_prepare": ([_vp, C.c_int], C.c_int),
    "mb_prepare_diag": ([_vp, C.c_int], C.c_int),
    "mb_set_bulk_spread": ([_vp, C.c_int], C.c_int),
    "mb_set_shift": ([_vp, C.c_int], C.c_int),
    "mb_set_rounding": ([_vp, C.c_int], C.c_int),
    "mb_set_l2_persist": ([_vp, C.c_int], C.c_int),
    "mb_set_plan_steps": ([_vp, C.c_int], C.c_int),
    "mb_set_hybrid_ctas": ([_vp, C.c_int], C.c_int),
    "mb_plan_describe": ([_vp, C.c_int, C.c_char_p, C.c_longlong, _pll], C.c_int),
    "mb_block_step": ([_vp, C.c_int, _vp], C.c_int),
    "mb_c_c_boundary_transfer": ([_vp, C.c_int, _vp], C.c_int),
    "mb_space_interpolation": ([_vp, C.c_int, _vp], C.c_int),
    "mb_temporal_interpolation": ([_vp, C.c_int, C.c_double, _vp], C.c_int),
    "mb_c_f_boundary_transfer": ([_vp, C.c_int, _vp], C.c_int),
    "mb_f_c_boundary_transfer": ([_vp, C.c_int, _vp], C.c_int),
    "mb_rotate_markers": ([_vp, C.c_int], C.c_int),
    "mb_drag": ([_vp, _pd, _pd, _pd, _vp], C.c_int),
    "mb_drag_link_count": ([_vp, _pi], C.c_int),
    "mb_error_L2": ([_vp, _pd, _vp], C.c_int),
    "mb_check_finite": ([_vp, _pll, _vp], C.c_int),
    "mb_copy_fields": ([_vp, C.c_int, _pd, _pd, _pd, _pd, _pi, _vp], C.c_int),
    "mb_set_fields": ([_vp, C.c_int, _pd, _pd, _pd, _pd, _vp], C.c_int),
    "mb_write_tecplot": ([_vp, C.c_char_p], C.c_int),
    "mb_append_drag": ([C.c_char_p, C.c_int, C.c_double, C.c_double], C.c_int),
    "mb_append_error_L2": ([C.c_char_p, C.c_int, C.c_double], C.c_int),
    "mb_stats": ([_vp, _pll, _pll, _pll], C.c_int),
    "mb_time_block_step": ([_vp, C.c_int, C.c_int, _vp, _pd, _pd, _pll], C.c_int),
    "mb_error_L2_noalloc": ([C.POINTER(L2Segment), C.c_int, C.c_void_p, _vp], C.c_int),
    "mb_checkpoint_size": ([_vp, _pll], C.c_int),
    "mb_checkpoint_save": ([_vp, C.c_void_p, C.c_longlong, _vp], C.c_int),
    "mb_checkpoint_load": ([_vp, C.c_void_p, C.c_longlong, _vp], C.c_int),
}

_lib = None


class MBError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        super().__init__(f"{what}: {load().mb_error_string(code).decode()} ({code})")


def load(path=LIB_PATH):
    """Loads libmblbm.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} not built; run multi-block-lbm-gpu_b200/build.py")
        lib = C.CDLL(path)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def _check(code, what):
    if code != MB_OK:
        raise MBError(code, what)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_pd)


# ---------------------------------------------------------------------------
# layouts and configurations
# ---------------------------------------------------------------------------
def layout_builtin(name):
    """Tables of geo/geometry.h for _GEO_<name> ("1_1", "2_2", "2_5", "4_9")."""
    L = Layout()
    _check(load().mb_layout_builtin(name.encode(), C.byref(L)), f"mb_layout_builtin({name})")
    return L


def layout_nested(LX, LY, boxes):
    """Nested-frame layout; boxes = [(xs, xe, ys, ye), ...] per refined level."""
    flat = (C.c_int * max(1, 4 * len(boxes)))(*[v for b in boxes for v in b])
    L = Layout()
    _check(load().mb_layout_nested(LX, LY, len(boxes) + 1, flat, C.byref(L)), "mb_layout_nested")
    return L


def make_config(LX, LY, R, CX, CY, U0=(0.1, 0.0), Re=10.0, rho0=1.0, drag_area=-1, ellipse=None,
                periodic=0, obstacle=True):
    c = Config()
    c.Re, c.rho0, c.LX, c.LY, c.R, c.CX, c.CY = float(Re), float(rho0), LX, LY, R, CX, CY
    c.U0[0], c.U0[1] = float(U0[0]), float(U0[1])
    c.obstacle = OBST_CIRCLE if obstacle else OBST_NONE
    c.drag_area = drag_area
    c.periodic = periodic
    if ellipse is not None:
        c.obstacle = OBST_ELLIPSE
        c.ell_cx, c.ell_cy, c.ell_a, c.ell_b, c.ell_angle = [float(v) for v in ellipse]
    return c


def geo_init(layout, config):
    """geo_init() (geo/init_geo.h:89-165) -> Geometry."""
    g = Geometry()
    _check(load().mb_geo_init(C.byref(layout), C.byref(config), C.byref(g)), "mb_geo_init")
    return g


def coverage(geo):
    n = C.c_int(0)
    _check(load().mb_geo_check_coverage(C.byref(geo), C.byref(n)), "mb_geo_check_coverage")
    return n.value


# Workloads of the benchmark configurations (coarse cells).
def config1_geometry():
    """2-level cylinder, Re=40: 400x160 coarse, fine box [60,140]x[40,120], D=20 at (100,80), U0=0.05."""
    L = layout_nested(400, 160, [(60, 140, 40, 120)])
    return geo_init(L, make_config(400, 160, 10, 100, 80, U0=(0.05, 0.0), Re=40.0))


def channel_walls(sim, geo, slip_walls=True, halfway_obstacle=True):
    """Channel boundaries for the 2-level cylinder at Re=40 in place of the
    reference's equilibrium edges and on-node walls: free-slip walls on the domain's
    bottom and top rows (MB_SOLID_SLIP, the reference's slip_gpu table) and
    half-way bounce-back on the obstacle (MB_SOLID_HBB).  The inlet and outlet
    columns keep their equilibrium."""
    cfg = geo.config
    for a in range(geo.layout.number_area):
        A = geo.Areas[a]
        t = sim.fields(a)["solid"].copy()
        x = A.base_x + np.arange(A.nx) / A.m
        y = A.base_y + np.arange(A.ny) / A.m
        if halfway_obstacle:
            t[t == MB_SOLID_SBB] = MB_SOLID_HBB
        if slip_walls:
            inner = (x != 0.0) & (x != cfg.LX - 1.0)
            for j in np.nonzero((y == 0.0) | (y == cfg.LY - 1.0))[0]:
                row = t[j]
                row[inner & (row == MB_FLUID)] = MB_SOLID_SLIP
        sim.set_cell_types(a, t)


def tgv_geometry(n=1024, patch=256, u0=0.01, tau=0.6, levels=2):
    """Taylor-Green vortex on a doubly periodic n x n coarse domain (nodes
    0..n+1, the outer ring being ghosts of the opposite side) with a centred
    refined patch of patch x patch coarse cells per finer level (each level
    halving the previous patch), no obstacle, relaxation time tau on level 0.
    The reference has no periodic boundary; this is the decay check of the
    multi-block step.  U0 = (u0, 0) is the vortex amplitude; R = 1 and Re
    are chosen so that geo_init's nu = |U0| 2R / Re gives tau."""
    nu = (tau - 0.5) / 3.0
    N = n + 2
    boxes = []
    w = patch
    for _ in range(levels - 1):
        lo = (N - 1 - w) // 2
        boxes.append((lo, lo + w, lo, lo + w))
        w //= 2
    L = layout_nested(N, N, boxes)
    cfg = make_config(N, N, 1, N // 2, N // 2, U0=(u0, 0.0), Re=u0 * 2.0 / nu, obstacle=False,
                      periodic=PERIODIC_X | PERIODIC_Y)
    return geo_init(L, cfg)


_EX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=np.float64)
_EY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=np.float64)
_WD = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def feq(rho, ux, uy):
    """feq of every direction (lbm/assit_func.h:2-9), arrays (9, ...)."""
    rho, ux, uy = np.asarray(rho, np.float64), np.asarray(ux, np.float64), np.asarray(uy, np.float64)
    eu = _EX.reshape((9,) + (1,) * ux.ndim) * ux + _EY.reshape((9,) + (1,) * uy.ndim) * uy
    uv = ux * ux + uy * uy
    return _WD.reshape((9,) + (1,) * rho.ndim) * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uv)


def tgv_mode(geo, a):
    """Phases of block a's nodes in the periodic frame: (s, c) with
    ux = u0 s, uy = u0 c for the initial vortex, k = 2 pi / (LX - 2)."""
    A, cfg = geo.Areas[a], geo.config
    kx, ky = 2.0 * np.pi / (cfg.LX - 2), 2.0 * np.pi / (cfg.LY - 2)
    X = (A.base_x + np.arange(A.nx) / A.m - 1.0) * kx
    Y = (A.base_y + np.arange(A.ny) / A.m - 1.0) * ky
    X, Y = np.meshgrid(X, Y)
    return np.sin(X) * np.cos(Y), -np.cos(X) * np.sin(Y), X, Y


def tgv_init(sim, geo, u0=None):
    """Sets every block to the equilibrium of the initial vortex,
    u = u0 (sin kx cos ky, -cos kx sin ky), rho = rho0 (1 - 3 u0^2/4 (cos 2kx
    + cos 2ky)), and re-derives the interface history (sync_history)."""
    cfg = geo.config
    u0 = cfg.U0[0] if u0 is None else u0
    for a in range(geo.layout.number_area):
        s, c, X, Y = tgv_mode(geo, a)
        ux, uy = u0 * s, u0 * c
        rho = cfg.rho0 * (1.0 - 0.75 * u0 * u0 * (np.cos(2 * X) + np.cos(2 * Y)))
        sim.set_fields(a, rho=rho, ux=ux, uy=uy, F=feq(rho, ux, uy))
    sim.sync_history()


def tgv_amplitude(sim, geo, fields=None):
    """Least-squares amplitude of the vortex mode in u over the FLUID cells
    of all blocks; u0 exp(-2 nu k^2 t) for the exact decay."""
    num = den = 0.0
    for a in range(geo.layout.number_area):
        f = fields[a] if fields is not None else sim.fields(a)
        s, c, _, _ = tgv_mode(geo, a)
        m = f["solid"] == MB_FLUID
        num += float((f["ux"][m] * s[m]).sum() + (f["uy"][m] * c[m]).sum())
        den += float((s[m] * s[m]).sum() + (c[m] * c[m]).sum())
    return num / den


def config2_geometry():
    """3-level cylinder, Re=100: 4096x1024 coarse, level-1 box 512x256, level-2 box 256x128,
    D=32 at (960,512), U0=0.04."""
    L = layout_nested(4096, 1024, [(768, 1280, 384, 640), (896, 1152, 448, 576)])
    return geo_init(L, make_config(4096, 1024, 16, 960, 512, U0=(0.04, 0.0), Re=100.0))


def _splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x, z ^ (z >> 31)


def batch_case(case_id, base_seed=20250, d_range=(10.0, 40.0), levels=None):
    """One case of the batched workload, drawn with splitmix64 from seed
    base_seed + case_id: obstacle extent D ~ U[d_range] coarse cells (the
    ellipse's major axis), aspect ~ U[1,3], angle ~ U[0,pi), Re ~ U[20,200],
    2 or 3 levels (unless given), domain 20D x 8D, U0 = 0.04.  The obstacle
    sits at (5D, 4D); level-1 box [CX-2D, CX+6D] x [CY-2D, CY+2D], level-2 box
    [CX-D, CX+3D] x [CY-D, CY+D].  Returns (geometry, parameters)."""
    state = (base_seed + case_id) & 0xFFFFFFFFFFFFFFFF
    u = []
    for _ in range(5):
        state, r = _splitmix64(state)
        u.append((r >> 11) / float(1 << 53))
    D = d_range[0] + (d_range[1] - d_range[0]) * u[0]
    aspect = 1.0 + 2.0 * u[1]
    angle = np.pi * u[2]
    Re = 20.0 + 180.0 * u[3]
    nlev = levels if levels is not None else (2 if u[4] < 0.5 else 3)
    Di = int(round(D))
    LX, LY = 20 * Di, 8 * Di
    CX, CY = 5 * Di, 4 * Di
    boxes = [(CX - 2 * Di, CX + 6 * Di, CY - 2 * Di, CY + 2 * Di)]
    if nlev == 3:
        boxes.append((CX - Di, CX + 3 * Di, CY - Di, CY + Di))
    a = D / 2.0
    b = a / aspect
    R = max(1, int(round(D / 2.0)))
    L = layout_nested(LX, LY, boxes)
    cfg = make_config(LX, LY, R, CX, CY, U0=(0.04, 0.0), Re=Re, ellipse=(CX, CY, a, b, angle))
    return geo_init(L, cfg), {"case": case_id, "D": D, "aspect": aspect, "angle": angle, "Re": Re, "levels": nlev,
                              "LX": LX, "LY": LY}


def updates_per_coarse_step(geo):
    L = geo.layout
    tot = 0
    for l in range(L.LEVEL):
        steps = 1
        for q in range(1, l + 1):
            steps *= L.mi[q]
        for a in range(L.ASP[l], L.ASP[l + 1]):
            tot += steps * geo.Areas[a].nx * geo.Areas[a].ny
    return tot


def error_L2_noalloc(segments, d_out, stream=None):
    """mb_error_L2_noalloc over [(ux, uy, upx, upy, n, weight), ...] device pointers;
    writes sum w|u-up|^2, sum w|u|^2 and their root ratio to the 3 doubles at d_out."""
    arr = (L2Segment * max(1, len(segments)))(*[L2Segment(*s) for s in segments])
    return load().mb_error_L2_noalloc(arr, len(segments), d_out, _stream_ptr(stream))


def _stream_ptr(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)  # torch.cuda.Stream


# ---------------------------------------------------------------------------
# the solver context
# ---------------------------------------------------------------------------
class MultiBlockLBM:
    """One multi-block simulation on the current CUDA device."""

    def __init__(self, geo, precision="f32", graph=True, shift=None, rounding=None):
        """graph: False launches kernels one by one, True replays CUDA graphs,
        "pdl" replays graphs with programmatic kernel-to-kernel edges,
        "program" runs each plan as one persistent executor launch, "hybrid" runs the
        fine-level chain as executor launches beside the bulk interior kernels.
        shift: "w" or "feq0" for the stored distributions of the shifted
        precisions (None: the precision's default, feq0 for f32 and f16c, w for f16s).
        rounding: "nearest" or "stochastic" (f16c, f16s) for the stored words (None: the
        precision's default, stochastic for f16c and f16s, nearest otherwise)."""
        self.lib = load()
        self.geo = geo
        self.precision = precision
        h = C.c_void_p()
        _check(self.lib.mb_create(C.byref(geo), PRECISIONS[precision], C.byref(h)), "mb_create")
        self.h = h
        mode = ({"pdl": 2, "program": 3, "hybrid": 4}.get(graph, 1 if graph else 0) if isinstance(graph, str)
                else (1 if graph else 0))
        if mode != 1:
            _check(self.lib.mb_set_graph_mode(self.h, mode), "mb_set_graph_mode")
        if shift is not None:
            _check(self.lib.mb_set_shift(self.h, {"w": SHIFT_W, "feq0": SHIFT_FEQ0}[shift]), "mb_set_shift")
        if rounding is not None:
            self.set_rounding(rounding)
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference call surface -------------------------------------------------
    def init(self, stream=None):
        _check(self.lib.mb_init(self.h, _stream_ptr(stream)), "mb_init")
        self.n = 0

    def evolution(self, n_coarse=1, stream=None):
        _check(self.lib.mb_step(self.h, int(n_coarse), _stream_ptr(stream)), "mb_step")
        self.n += n_coarse

    def set_split_cells(self, cells):
        """Levels with >= cells cells step interior and rim as separate graph nodes."""
        _check(self.lib.mb_set_split_cells(self.h, int(cells)), "mb_set_split_cells")

    def set_stb_variant(self, level, variant):
        """Block-step kernel of a level: 0 one cell per thread, 1 four cells per thread,
        2 two cells per thread, 3 cell ranges, 4 cell pairs, 5 bulk-copy row staging,
        6 eight cells per thread (16-bit stored forms; others run 0).  Results are identical."""
        _check(self.lib.mb_set_stb_variant(self.h, int(level), int(variant)), "mb_set_stb_variant")

    def set_split_levels(self, level_mask):
        """Split exactly the levels of level_mask (bit per level) into interior and rim nodes (0: threshold)."""
        _check(self.lib.mb_set_split_levels(self.h, int(level_mask)), "mb_set_split_levels")

    def set_interface_shape(self, rec_points=32, spline_segments=1):
        """Points per record CTA/item (32 or 64) and spline segments per CTA/item (1-4)."""
        _check(self.lib.mb_set_interface_shape(self.h, int(rec_points), int(spline_segments)),
               "mb_set_interface_shape")

    def set_stream_cells(self, cells, bulk=False):
        """Block steps over >= cells cells use evict-first cache hints (0: never);
        bulk=True also runs such whole levels as low-priority bulk work."""
        _check(self.lib.mb_set_stream_cells(self.h, int(cells), int(bool(bulk))), "mb_set_stream_cells")

    def set_bulk_occupancy(self, ctas_per_sm):
        """Cap interior block-step grids at ctas_per_sm CTAs per SM (0: uncapped)."""
        _check(self.lib.mb_set_bulk_occupancy(self.h, int(ctas_per_sm)), "mb_set_bulk_occupancy")

    def set_cta_spread(self, spline_kb, records_kb):
        """Minimum shared memory per spline / record CTA (KB): caps their CTAs per SM."""
        _check(self.lib.mb_set_cta_spread(self.h, int(spline_kb), int(records_kb)), "mb_set_cta_spread")

    def set_rounding(self, mode):
        """"nearest" or "stochastic" (f16c, f16s): how the collision rounds the stored words."""
        m = {"nearest": ROUND_NEAREST, "stochastic": ROUND_STOCHASTIC}[mode]
        _check(self.lib.mb_set_rounding(self.h, m), "mb_set_rounding")

    def set_hybrid_ctas(self, per_sm):
        """Executor CTAs per SM of the chain launches (graph="hybrid")."""
        _check(self.lib.mb_set_hybrid_ctas(self.h, int(per_sm)), "mb_set_hybrid_ctas")

    def set_plan_steps(self, n):
        """Coarse steps per replayed graph (rounded up to whole scheduler periods)."""
        _check(self.lib.mb_set_plan_steps(self.h, int(n)), "mb_set_plan_steps")

    def set_l2_persist(self, mb):
        """L2 set aside (MB) for the fine levels' state, kept resident for the chain kernels (0: off)."""
        _check(self.lib.mb_set_l2_persist(self.h, int(mb)), "mb_set_l2_persist")

    def set_bulk_spread(self, kb):
        """Unused shared memory (KB) reserved by each bulk (interior) block-step CTA (0: none)."""
        _check(self.lib.mb_set_bulk_spread(self.h, int(kb)), "mb_set_bulk_spread")

    def set_fusion(self, flags):
        """Plan fusions (bit 0: same-level copies inside the block step; bit 1: temporal
        interpolations inside the splines, moved to the interpolation's place; bit 2: the
        same at the spline's place, the fine substep in between leaving those edge cells
        alone; bit 3: f_c points inside the fine level's last block step; bit 4: record
        launches split by whether they wait for the latest block step); default 5 (bits 0
        and 2); results are identical."""
        _check(self.lib.mb_set_fusion(self.h, int(flags)), "mb_set_fusion")

    def set_collision(self, kind, s_e=0.0, s_eps=0.0, s_q=0.0):
        """MB_COLL_BGK, or MB_COLL_MRT with rates s_e, s_eps, s_q (<= 0: the block's 1/tau)."""
        _check(self.lib.mb_set_collision(self.h, int(kind), float(s_e), float(s_eps), float(s_q)), "mb_set_collision")

    def set_body_force(self, fx, fy):
        """Uniform body force (forcex, forcey of every cell, coarse lattice units)."""
        _check(self.lib.mb_set_body_force(self.h, float(fx), float(fy)), "mb_set_body_force")

    def set_cell_types(self, area, types):
        """Cell types of one block, an (ny, nx) array of MB_FLUID / MB_SOLID_SBB /
        MB_SOLID_SLIP / MB_SOLID_HBB codes (C_BOUNDARY cells unchanged)."""
        t = np.ascontiguousarray(types, dtype=np.int32)
        A = self.geo.Areas[area]
        if t.size != A.nx * A.ny:
            raise ValueError("types must have nx*ny entries")
        _check(self.lib.mb_set_cell_types(self.h, int(area), t.ctypes.data_as(_pi)), "mb_set_cell_types")

    def set_program_timeout(self, seconds):
        """Executor (graph="program"): give up after this long without ready work."""
        _check(self.lib.mb_set_program_timeout(self.h, float(seconds)), "mb_set_program_timeout")

    def set_program_shape(self, bulk_cells=512, urgent_cells=256, periods_per_launch=2, bulk_ctas=0):
        """Executor: cells per work item of interior and of other block-step
        nodes, scheduler periods per launch, and the cap on CTAs running bulk
        items at once (0: none)."""
        _check(self.lib.mb_set_program_shape(self.h, int(bulk_cells), int(urgent_cells), int(periods_per_launch),
                                             int(bulk_ctas)), "mb_set_program_shape")

    TRACE_DTYPE = np.dtype([("t_pick", "<u8"), ("t_start", "<u8"), ("t_end", "<u8"), ("plan_node", "<i4"),
                            ("item", "<i4"), ("sm", "<i4"), ("cta", "<i4"), ("launch", "<i4"), ("pad", "<i4")])

    def set_program_trace(self, capacity):
        """Executor: record every work item into a device buffer of capacity entries (0: off)."""
        _check(self.lib.mb_set_program_trace(self.h, int(capacity)), "mb_set_program_trace")

    def program_trace(self, max_records=1 << 22):
        """Recorded work items (numpy structured array) since the last call."""
        out = np.zeros(max_records, dtype=self.TRACE_DTYPE)
        n = C.c_longlong(0)
        _check(self.lib.mb_program_trace(self.h, out.ctypes.data_as(_vp), int(max_records), C.byref(n)),
               "mb_program_trace")
        return out[: n.value]

    def sync(self, stream=None):
        """Waits for the stream; raises MBError(MB_ERR_TIMEOUT) after an executor timeout."""
        _check(self.lib.mb_sync(self.h, _stream_ptr(stream)), "mb_sync")

    def program_selftest(self, stall, stream=None):
        """Raw status of one executor launch over an empty node (stall=1: never ready)."""
        return self.lib.mb_program_selftest(self.h, int(stall), _stream_ptr(stream))

    def prepare(self, n_coarse):
        """Compiles the plans and graphs that evolution(n_coarse) will replay."""
        _check(self.lib.mb_prepare(self.h, int(n_coarse)), "mb_prepare")

    def prepare_diag(self, n_coarse):
        """Compiles the plans and graphs that evolution_diag(n_coarse) will replay
        and sizes its result buffers."""
        _check(self.lib.mb_prepare_diag(self.h, int(n_coarse)), "mb_prepare_diag")

    def plan_description(self, n_coarse):
        """Text listing of the plan mb_step(n_coarse) starts with: one line per
        launch with its dependencies."""
        need = C.c_longlong()
        _check(self.lib.mb_plan_describe(self.h, int(n_coarse), None, 0, C.byref(need)), "mb_plan_describe")
        buf = C.create_string_buffer(need.value + 1)
        _check(self.lib.mb_plan_describe(self.h, int(n_coarse), buf, need.value + 1, C.byref(need)), "mb_plan_describe")
        return buf.value.decode()

    def block_step(self, area, stream=None):
        _check(self.lib.mb_block_step(self.h, area, _stream_ptr(stream)), "mb_block_step")

    def c_c_boundary_transfer(self, line, stream=None):
        _check(self.lib.mb_c_c_boundary_transfer(self.h, line, _stream_ptr(stream)), "mb_c_c_boundary_transfer")

    def space_interpolation(self, line, stream=None):
        _check(self.lib.mb_space_interpolation(self.h, line, _stream_ptr(stream)), "mb_space_interpolation")

    def temporal_interpolation(self, line, xm, stream=None):
        _check(self.lib.mb_temporal_interpolation(self.h, line, float(xm), _stream_ptr(stream)), "mb_temporal_interpolation")

    def c_f_boundary_transfer(self, line, stream=None):
        _check(self.lib.mb_c_f_boundary_transfer(self.h, line, _stream_ptr(stream)), "mb_c_f_boundary_transfer")

    def f_c_boundary_transfer(self, line, stream=None):
        _check(self.lib.mb_f_c_boundary_transfer(self.h, line, _stream_ptr(stream)), "mb_f_c_boundary_transfer")

    def rotate_markers(self, line):
        _check(self.lib.mb_rotate_markers(self.h, line), "mb_rotate_markers")

    def getDrag_block(self, stream=None):
        """Returns (Fx, Fy, Cd, Cl) as getDrag_block computes them."""
        f = (C.c_double * 2)()
        cd, cl = C.c_double(), C.c_double()
        _check(self.lib.mb_drag(self.h, f, C.byref(cd), C.byref(cl), _stream_ptr(stream)), "mb_drag")
        return f[0], f[1], cd.value, cl.value

    def evolution_diag(self, n_coarse, stream=None):
        """n coarse steps, each followed by getDrag_block and error_L2 on the
        device (mb_step_diag); returns numpy arrays (Cd, Cl, L2 change) of n values."""
        n = int(n_coarse)
        cd, cl, err = (np.zeros(n) for _ in range(3))
        _check(self.lib.mb_step_diag(self.h, n, cd.ctypes.data_as(_vp), cl.ctypes.data_as(_vp),
                                     err.ctypes.data_as(_vp), _stream_ptr(stream)), "mb_step_diag")
        self.n += n
        return cd, cl, err

    def drag_links(self):
        n = C.c_int()
        _check(self.lib.mb_drag_link_count(self.h, C.byref(n)), "mb_drag_link_count")
        return n.value

    def error_L2(self, stream=None):
        e = C.c_double()
        _check(self.lib.mb_error_L2(self.h, C.byref(e), _stream_ptr(stream)), "mb_error_L2")
        return e.value

    def check_finite(self, stream=None):
        bad = C.c_longlong()
        self.lib.mb_check_finite(self.h, C.byref(bad), _stream_ptr(stream))
        return bad.value

    def fields(self, area, stream=None, out=None):
        """Dict of FP64 host arrays rho, ux, uy (ny, nx), F (9, ny, nx), solid (ny, nx).
        out: a dict of preallocated C-contiguous arrays of those shapes (pinned
        host memory makes the copies direct) to fill instead; without an "F"
        entry the distributions are not copied."""
        A = self.geo.Areas[area]
        nx, ny = A.nx, A.ny
        if out is not None:
            rho, ux, uy, F, solid = (out.get(k) for k in ("rho", "ux", "uy", "F", "solid"))
            for k, shp, dt in (("rho", (ny, nx), np.float64), ("ux", (ny, nx), np.float64), ("uy", (ny, nx), np.float64),
                               ("F", (9, ny, nx), np.float64), ("solid", (ny, nx), np.int32)):
                a = out.get(k)
                if a is None and k == "F":
                    continue
                if a.size != int(np.prod(shp)) or a.dtype != dt or not a.flags.c_contiguous:
                    raise ValueError(f"out[{k!r}] must be a C-contiguous {dt.__name__} array of {shp}")
        else:
            rho = np.empty((ny, nx))
            ux = np.empty((ny, nx))
            uy = np.empty((ny, nx))
            F = np.empty((9, ny, nx))
            solid = np.empty((ny, nx), dtype=np.int32)
        _check(
            self.lib.mb_copy_fields(self.h, area, _dp(rho), _dp(ux), _dp(uy), None if F is None else _dp(F),
                                    solid.ctypes.data_as(_pi), _stream_ptr(stream)),
            "mb_copy_fields",
        )
        res = {"rho": rho, "ux": ux, "uy": uy, "F": F, "solid": solid}
        return res if F is not None else {k: v for k, v in res.items() if k != "F"}

    def macros(self, area, stream=None):
        """Dict of FP64 host arrays rho, ux, uy and solid (ny, nx), without the distributions."""
        A = self.geo.Areas[area]
        nx, ny = A.nx, A.ny
        rho, ux, uy = np.empty((ny, nx)), np.empty((ny, nx)), np.empty((ny, nx))
        solid = np.empty((ny, nx), dtype=np.int32)
        _check(self.lib.mb_copy_fields(self.h, area, _dp(rho), _dp(ux), _dp(uy), None, solid.ctypes.data_as(_pi),
                                       _stream_ptr(stream)), "mb_copy_fields")
        return {"rho": rho, "ux": ux, "uy": uy, "solid": solid}

    def set_fields(self, area, rho=None, ux=None, uy=None, F=None, stream=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (rho, ux, uy, F)]
        _check(self.lib.mb_set_fields(self.h, area, *[_dp(a) for a in arrs], _stream_ptr(stream)), "mb_set_fields")

    def sync_history(self, stream=None):
        """Ring slots <- fine edge F and u_prev <- u, after set_fields (mb_sync_history)."""
        _check(self.lib.mb_sync_history(self.h, _stream_ptr(stream)), "mb_sync_history")

    def checkpoint(self, stream=None):
        """The full device state as bytes (see mb_checkpoint_save)."""
        n = C.c_longlong()
        _check(self.lib.mb_checkpoint_size(self.h, C.byref(n)), "mb_checkpoint_size")
        buf = np.empty(n.value, dtype=np.uint8)
        _check(self.lib.mb_checkpoint_save(self.h, buf.ctypes.data, n.value, _stream_ptr(stream)), "mb_checkpoint_save")
        return buf.tobytes()

    def restore(self, data, stream=None):
        buf = np.frombuffer(data, dtype=np.uint8)
        _check(self.lib.mb_checkpoint_load(self.h, buf.ctypes.data, len(buf), _stream_ptr(stream)), "mb_checkpoint_load")

    def output(self, path):
        _check(self.lib.mb_write_tecplot(self.h, path.encode()), "mb_write_tecplot")

    def stats(self):
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(self.lib.mb_stats(self.h, C.byref(a), C.byref(b), C.byref(c)), "mb_stats")
        return {"kernels_last_call": a.value, "kernels_per_coarse_step": b.value, "updates_per_coarse_step": c.value}

    def time_block_step(self, level, n, stream=None):
        ms, by, cells = C.c_double(), C.c_double(), C.c_longlong()
        _check(self.lib.mb_time_block_step(self.h, level, n, _stream_ptr(stream), C.byref(ms), C.byref(by), C.byref(cells)),
               "mb_time_block_step")
        return ms.value, by.value, cells.value


# ---------------------------------------------------------------------------
# batches of independent cases
# ---------------------------------------------------------------------------
class Batch:
    """Independent cases of one precision and level count advanced together
    (mb_batch_*): each plan node is one launch over all cases."""

    def __init__(self, sims):
        self.lib = load()
        self.sims = list(sims)
        arr = (_vp * len(self.sims))(*[s.h.value for s in self.sims])
        h = _vp()
        _check(self.lib.mb_batch_create(arr, len(self.sims), C.byref(h)), "mb_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def evolution(self, n_coarse=1, stream=None):
        _check(self.lib.mb_batch_step(self.h, int(n_coarse), _stream_ptr(stream)), "mb_batch_step")
        for s in self.sims:
            s.n += n_coarse

    def prepare(self, n_coarse):
        """Compiles the plans and graphs that evolution(n_coarse) will replay."""
        _check(self.lib.mb_batch_prepare(self.h, int(n_coarse)), "mb_batch_prepare")

    def drag(self, stream=None):
        """(Cd, Cl) numpy arrays, one value per case."""
        n = len(self.sims)
        cd, cl = np.zeros(n), np.zeros(n)
        _check(self.lib.mb_batch_drag(self.h, cd.ctypes.data_as(_vp), cl.ctypes.data_as(_vp), _stream_ptr(stream)),
               "mb_batch_drag")
        return cd, cl

    def stats(self):
        u, k, n = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(self.lib.mb_batch_stats(self.h, C.byref(u), C.byref(k), C.byref(n)), "mb_batch_stats")
        return {"updates_per_step": u.value, "kernels_last_call": k.value, "steps_done": n.value}

    def set_split_levels(self, level_mask):
        """Split exactly the levels of level_mask (bit per level) into interior and rim nodes (0: threshold)."""
        _check(self.lib.mb_set_split_levels(self.h, int(level_mask)), "mb_set_split_levels")

    def set_interface_shape(self, rec_points=32, spline_segments=1):
        _check(self.lib.mb_batch_set_interface_shape(self.h, int(rec_points), int(spline_segments)),
               "mb_batch_set_interface_shape")

    def set_schedule(self, stb_ctas_per_sm):
        """Block-step schedule: 0 one CTA per 256-cell tile; k > 0 a persistent
        grid of k CTAs per SM over equal shares of the tiles."""
        _check(self.lib.mb_batch_set_schedule(self.h, int(stb_ctas_per_sm)), "mb_batch_set_schedule")

    def set_kernel(self, kernel):
        """Block-step kernel: 0 one cell per thread, 1 cell pairs on a persistent grid."""
        _check(self.lib.mb_batch_set_kernel(self.h, int(kernel)), "mb_batch_set_kernel")

    def autotune(self, steps=12, stream=None):
        """Times the block-step kernels and schedules, then the interface shapes; keeps the fastest."""
        r, sg, k, ms, kern = C.c_int(), C.c_int(), C.c_int(), C.c_double(), C.c_int()
        _check(self.lib.mb_batch_autotune(self.h, int(steps), _stream_ptr(stream), C.byref(r), C.byref(sg), C.byref(k),
                                          C.byref(ms), C.byref(kern)), "mb_batch_autotune")
        return {"rec_points": r.value, "spline_segments": sg.value, "stb_ctas_per_sm": k.value,
                "stb_kernel": kern.value, "ms_per_step": ms.value}


# ---------------------------------------------------------------------------
# post-processing of the Cd / Cl series
# ---------------------------------------------------------------------------
def settle_step(series, target, rel=0.005):
    """First index from which every later value lies within rel*|target| of
    target (len(series) when the series never settles)."""
    x = np.asarray(series, dtype=np.float64)
    bad = np.nonzero(np.abs(x - target) > rel * abs(target))[0]
    return 0 if len(bad) == 0 else int(bad[-1]) + 1


def strouhal(cl, D, U0, skip=0):
    """St = f D / U0 from the dominant frequency of the lift series (one value
    per coarse step, D and U0 in coarse lattice units); None without a clear
    oscillation.  f is the peak of the Hann-windowed spectrum of the series
    after `skip` steps, refined by a parabola through the peak and its
    neighbours (robust to the high-frequency noise of FP16 storage)."""
    x = np.asarray(cl[skip:], dtype=np.float64)
    if len(x) < 16:
        return None
    x = x - x.mean()
    if np.abs(x).max() < 1e-9:
        return None
    sp = np.abs(np.fft.rfft(x * np.hanning(len(x))))
    k = int(np.argmax(sp[1:])) + 1
    if k >= len(sp) - 1:
        return None
    a, b, c = np.log(sp[k - 1] + 1e-300), np.log(sp[k] + 1e-300), np.log(sp[k + 1] + 1e-300)
    den = a - 2 * b + c
    dk = 0.5 * (a - c) / den if den != 0 else 0.0
    f = (k + dk) / len(x)
    return f * D / U0


# ---------------------------------------------------------------------------
# learned warm start
# ---------------------------------------------------------------------------
class UNet:
    """The surrogate network (mb_unet_*).  Tensors are torch CUDA float32
    tensors (their device pointers go through the C ABI)."""

    def __init__(self, H=128, W=256, max_batch=16, seed=1):
        self.lib = load()
        self.H, self.W, self.max_batch = H, W, max_batch
        h = _vp()
        _check(self.lib.mb_unet_create(H, W, max_batch, seed, C.byref(h)), "mb_unet_create")
        self.h = h
        n = C.c_longlong()
        _check(self.lib.mb_unet_param_count(self.h, C.byref(n)), "mb_unet_param_count")
        self.nparam = n.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self, grads=False):
        out = np.zeros(self.nparam, dtype=np.float32)
        _check(self.lib.mb_unet_get_params(self.h, out.ctypes.data_as(_vp), self.nparam, int(grads)), "mb_unet_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self.lib.mb_unet_set_params(self.h, p.ctypes.data_as(_vp), self.nparam), "mb_unet_set_params")

    def set_gemm(self, kind):
        """3x3 convolutions on the tcgen05 tensor cores (1, default) or on mma.sync (0)."""
        _check(self.lib.mb_unet_set_gemm(self.h, int(kind)), "mb_unet_set_gemm")

    def status(self, stream=None):
        """Raises MBError(MB_ERR_TIMEOUT) if a tcgen05 kernel's bounded wait ran out."""
        _check(self.lib.mb_unet_status(self.h, _stream_ptr(stream)), "mb_unet_status")

    def forward(self, x, out, stream=None):
        _check(self.lib.mb_unet_forward(self.h, _vp(x.data_ptr()), x.shape[0], _vp(out.data_ptr()), _stream_ptr(stream)),
               "mb_unet_forward")
        return out

    def train_step(self, x, target, mask, lr, apply=True, stream=None):
        loss = C.c_float()
        _check(self.lib.mb_unet_train_step(self.h, _vp(x.data_ptr()), _vp(target.data_ptr()), _vp(mask.data_ptr()),
                                           x.shape[0], float(lr), int(apply), C.byref(loss), _stream_ptr(stream)),
               "mb_unet_train_step")
        return loss.value
