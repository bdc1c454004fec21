"""ctypes wrapper of the FP64 C oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the product package.  The oracle
restates the reference program (zhangya9741/Multi-block-LBM-GPU) in plain C;
see oracle.h for the function-by-function citations.

Parity status: pinned against outputs of the reference's own CUDA build
(tests/golden/, generated by oracle/ref_harness/make_golden.py on a B200).
"""
import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "multi-block-lbm-gpu_b200"))
from mblbm import Geometry, Layout, Config  # noqa: E402  (struct layouts of include/mblbm.h)

LIB_PATH = os.path.join(_HERE, "liboracle.so")
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)
_vp = C.c_void_p
_SIG = {
    "orc_geo_init": ([C.POINTER(Layout), C.POINTER(Config), C.POINTER(Geometry)], C.c_int),
    "orc_create": ([C.POINTER(Geometry)], _vp),
    "orc_destroy": ([_vp], None),
    "orc_set_threads": ([C.c_int], None),
    "orc_init": ([_vp], C.c_int),
    "orc_sync_history": ([_vp], None),
    "orc_evolution": ([_vp, C.c_int], None),
    "orc_error_L2": ([_vp], C.c_double),
    "orc_drag": ([_vp, _pd, _pd, _pd], None),
    "orc_drag_link_count": ([_vp], C.c_int),
    "orc_drag_links": ([_vp, _pi], None),
    "orc_block_step": ([_vp, C.c_int], None),
    "orc_c_c": ([_vp, C.c_int], None),
    "orc_space_interpolation": ([_vp, C.c_int], None),
    "orc_temporal": ([_vp, C.c_int, C.c_double], None),
    "orc_c_f": ([_vp, C.c_int], None),
    "orc_f_c": ([_vp, C.c_int], None),
    "orc_rotate_markers": ([_vp, C.c_int], None),
    "orc_gtsv": ([C.c_int, C.c_int, _pd, _pd, _pd, _pd, C.c_int], None),
    "orc_spline3_s": ([C.c_double] * 7, C.c_double),
    "orc_feq": ([C.c_int, C.c_double, C.c_double, C.c_double], C.c_double),
    "orc_get_fields": ([_vp, C.c_int, _pd, _pd, _pd, _pd, _pd, _pi], None),
    "orc_set_fields": ([_vp, C.c_int, _pd, _pd, _pd, _pd, _pd], None),
    "orc_get_slots": ([_vp, C.c_int, _pd], None),
    "orc_get_markers": ([_vp, C.c_int, _pi], None),
    "orc_write_tecplot": ([_vp, C.c_char_p], C.c_int),
    "orc_set_collision": ([_vp, C.c_int, C.c_double, C.c_double, C.c_double], C.c_int),
    "orc_set_body_force": ([_vp, C.c_double, C.c_double], None),
    "orc_set_cell_types": ([_vp, C.c_int, _pi], C.c_int),
}
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} not built; run multi-block-lbm-gpu_b200/build.py --oracle-only")
        lib = C.CDLL(LIB_PATH)
        for n, (a, r) in _SIG.items():
            f = getattr(lib, n)
            f.argtypes = a
            f.restype = r
        _lib = lib
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_pd)


def geo_init(layout, config):
    g = Geometry()
    rc = load().orc_geo_init(C.byref(layout), C.byref(config), C.byref(g))
    if rc != 0:
        raise RuntimeError(f"orc_geo_init failed ({rc})")
    return g


def set_threads(n):
    load().orc_set_threads(int(n))


class Oracle:
    """FP64 restatement of one reference simulation."""

    def __init__(self, geo):
        self.lib = load()
        self.geo = geo
        self.s = self.lib.orc_create(C.byref(geo))
        if not self.s:
            raise MemoryError("orc_create")

    def close(self):
        if self.s:
            self.lib.orc_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self):
        rc = self.lib.orc_init(self.s)
        if rc != 0:
            raise ValueError(f"orc_init failed ({rc})")

    def sync_history(self):
        """Ring slots <- fine edge F and u_prev <- u, after set_fields."""
        self.lib.orc_sync_history(self.s)

    def evolution(self, n=1):
        for _ in range(n):
            self.lib.orc_evolution(self.s, 0)

    def error_L2(self):
        return self.lib.orc_error_L2(self.s)

    def getDrag_block(self):
        f = (C.c_double * 2)()
        cd, cl = C.c_double(), C.c_double()
        self.lib.orc_drag(self.s, f, C.byref(cd), C.byref(cl))
        return f[0], f[1], cd.value, cl.value

    def drag_links(self):
        n = self.lib.orc_drag_link_count(self.s)
        out = np.zeros((max(n, 1), 3), dtype=np.int32)
        self.lib.orc_drag_links(self.s, out.ctypes.data_as(_pi))
        return out[:n]

    def set_collision(self, kind, s_e=0.0, s_eps=0.0, s_q=0.0):
        rc = self.lib.orc_set_collision(self.s, int(kind), float(s_e), float(s_eps), float(s_q))
        if rc:
            raise ValueError(f"orc_set_collision failed ({rc})")

    def set_body_force(self, fx, fy):
        self.lib.orc_set_body_force(self.s, float(fx), float(fy))

    def set_cell_types(self, a, types):
        t = np.ascontiguousarray(types, dtype=np.int32)
        rc = self.lib.orc_set_cell_types(self.s, int(a), t.ctypes.data_as(_pi))
        if rc:
            raise ValueError(f"orc_set_cell_types failed ({rc})")

    def block_step(self, a):
        self.lib.orc_block_step(self.s, a)

    def c_c_boundary_transfer(self, c):
        self.lib.orc_c_c(self.s, c)

    def space_interpolation(self, b):
        self.lib.orc_space_interpolation(self.s, b)

    def temporal_interpolation(self, b, xm):
        self.lib.orc_temporal(self.s, b, float(xm))

    def c_f_boundary_transfer(self, b):
        self.lib.orc_c_f(self.s, b)

    def f_c_boundary_transfer(self, b):
        self.lib.orc_f_c(self.s, b)

    def rotate_markers(self, b):
        self.lib.orc_rotate_markers(self.s, b)

    def fields(self, a):
        A = self.geo.Areas[a]
        nx, ny = A.nx, A.ny
        out = {k: np.empty((ny, nx)) for k in ("rho", "ux", "uy")}
        F = np.empty((9, ny, nx))
        f = np.empty((9, ny, nx))
        solid = np.empty((ny, nx), dtype=np.int32)
        self.lib.orc_get_fields(self.s, a, _dp(out["rho"]), _dp(out["ux"]), _dp(out["uy"]), _dp(F), _dp(f),
                                solid.ctypes.data_as(_pi))
        out.update(F=F, f=f, solid=solid)
        return out

    def set_fields(self, a, rho=None, ux=None, uy=None, F=None, f=None):
        arrs = [None if v is None else np.ascontiguousarray(v, dtype=np.float64) for v in (rho, ux, uy, F, f)]
        self.lib.orc_set_fields(self.s, a, *[_dp(v) for v in arrs])

    def slots(self, b):
        N = self.geo.Line_Inf_C[b].Nf
        out = np.empty((3, 9, N))
        self.lib.orc_get_slots(self.s, b, _dp(out))
        return out

    def markers(self, b):
        m = (C.c_int * 3)()
        self.lib.orc_get_markers(self.s, b, m)
        return list(m)

    def output(self, path):
        return self.lib.orc_write_tecplot(self.s, path.encode())


def gtsv(l, m, u, B):
    """Tridiagonal solve (column-major B with nrhs columns), in place copy."""
    n = len(m)
    Bc = np.array(B, dtype=np.float64, order="F", copy=True)
    nrhs = Bc.shape[1] if Bc.ndim == 2 else 1
    load().orc_gtsv(n, nrhs, _dp(np.ascontiguousarray(l, float)), _dp(np.ascontiguousarray(m, float)),
                    _dp(np.ascontiguousarray(u, float)), Bc.ctypes.data_as(_pd), n)
    return Bc


def spline3_s(xx, x_1, h, fi_1, fi, mi_1, mi):
    return load().orc_spline3_s(xx, x_1, h, fi_1, fi, mi_1, mi)


def feq(k, rh, ux, uy):
    return load().orc_feq(k, rh, ux, uy)
