"""TEST INFRASTRUCTURE — ctypes binding of the oracle (liboracle.so), the CPU
restatement of the reference Fortran.  Parity unpinned: the reference has no
golden vectors and cannot be compiled here (no Fortran compiler); see the
header of fdm_oracle.cpp.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or (
            os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "fdm_oracle.cpp"))):
        subprocess.run(["make", "-C", HERE, "-s", "-B" if force else "liboracle.so"],
                       check=True, env={**os.environ, "CXX": "g++"})
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, i64, i32, dp = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        i64p = ctypes.POINTER(ctypes.c_int64)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.c_void_p]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [vp, i32]
        L.orc_initial.argtypes = [vp, i32, dp, i32]
        L.orc_block_refine.argtypes = [vp, i32, dp, i32]
        L.orc_num_leaves.restype = i64
        L.orc_num_leaves.argtypes = [vp]
        L.orc_num_interior.restype = i64
        L.orc_num_interior.argtypes = [vp]
        L.orc_export_leaves.argtypes = [vp, i64, u64p, dp, dp]
        L.orc_import_leaves.argtypes = [vp, i64, u64p, dp]
        L.orc_set_T.argtypes = [vp, i64, dp]
        L.orc_get_scalars.argtypes = [vp, dp]
        L.orc_set_scalars.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, i64]
        for name in ("orc_step_control", "orc_time_advance_rk", "orc_solute_step", "orc_amr",
                     "orc_rot_div"):
            getattr(L, name).argtypes = [vp]
        L.orc_stage.argtypes = [vp, i32]
        L.orc_body_boundary.argtypes = [vp, i32]
        L.orc_step_control_global.argtypes = [vp, ctypes.c_double, ctypes.c_double, i32]
        L.orc_get_U.argtypes = [vp, i64, i64p, dp]
        L.orc_set_U.argtypes = [vp, i64, i64p, dp]
        L.orc_solute.argtypes = [vp, i64, i64p]
        L.orc_export_rot_div.argtypes = [vp, i64, dp, dp]
        L.orc_export_stencil.argtypes = [vp, i64, dp]
        L.orc_export_neighbors.argtypes = [vp, i64, u64p]
        L.orc_counters.argtypes = [vp, i64p]
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.orc_export_gather.argtypes = [vp, i64, i32p, u64p, dp, i32p, u64p]
        L.orc_residual.argtypes = [vp, dp, dp]
        L.orc_wcns_z3.argtypes = [dp, dp, dp, dp, dp]
        L.orc_eigen.argtypes = [ctypes.c_double, i32, dp, dp, dp]
        L.orc_brinv.argtypes = [i32, dp]
        L.orc_get_direction.argtypes = [ctypes.c_double] * 4
        L.orc_lxl_dir.argtypes = [ctypes.c_double, i32, ctypes.c_double, ctypes.c_double, dp, dp]
        L.orc_wls.argtypes = [ctypes.c_double, ctypes.c_double, i32, ctypes.c_double,
                              ctypes.c_double, ctypes.c_double, ctypes.c_double, i32, i32,
                              dp, dp, dp, dp]
        L.orc_wls.restype = i32
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


class Oracle:
    """One oracle solver instance (the reference's module globals + tree)."""

    def __init__(self, cfg, threads: int | None = None, initial: bool = True):
        self.cfg = cfg
        self.L = lib()
        self.h = self.L.orc_create(ctypes.byref(cfg.params))
        if threads:
            self.L.orc_set_threads(self.h, threads)
        if initial:
            if getattr(cfg, "block", None):
                lvl, box, buf = cfg.block
                bx = np.asarray(box, dtype=np.float64)
                if self.L.orc_block_refine(self.h, lvl, _dp(bx), buf):
                    raise ValueError("bad block refinement parameters")
            icp = np.asarray(cfg.ic_params if cfg.ic_params else [0.0], dtype=np.float64)
            self.L.orc_initial(self.h, cfg.ic_kind, _dp(icp), len(cfg.ic_params))

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state
    def num_leaves(self) -> int:
        return int(self.L.orc_num_leaves(self.h))

    def num_interior(self) -> int:
        return int(self.L.orc_num_interior(self.h))

    def leaves(self):
        n = self.num_leaves()
        keys = np.zeros(n, np.uint64)
        prim = np.zeros((n, 4), np.float64)
        T = np.zeros(n, np.float64)
        rc = self.L.orc_export_leaves(self.h, n, _u64p(keys), _dp(prim), _dp(T))
        assert rc == 0
        return keys, prim, T

    def set_leaves(self, keys, prim, T=None):
        keys = np.ascontiguousarray(keys, np.uint64)
        prim = np.ascontiguousarray(prim, np.float64)
        rc = self.L.orc_import_leaves(self.h, len(keys), _u64p(keys), _dp(prim))
        if rc:
            raise ValueError("orc_import_leaves failed")
        if T is not None:
            T = np.ascontiguousarray(T, np.float64)
            self.L.orc_set_T(self.h, len(T), _dp(T))

    def scalars(self) -> dict:
        out = np.zeros(17, np.float64)
        self.L.orc_get_scalars(self.h, _dp(out))
        return dict(lambda_x=out[0], lambda_y=out[1], tstep=out[2], tt=out[3], it=int(out[4]),
                    l_max=int(out[5]), res_max=out[6:10].copy(), res_rms=out[10:14].copy(),
                    srot=out[14], sdiv=out[15], ne=int(out[16]))

    def set_scalars(self, lambda_x, lambda_y, tstep, tt, it):
        self.L.orc_set_scalars(self.h, lambda_x, lambda_y, tstep, tt, int(it))

    def counters(self) -> dict:
        out = np.zeros(6, np.int64)
        self.L.orc_counters(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        return dict(singular=int(out[0]), wls_calls=int(out[1]), parent_interp=int(out[2]),
                    child_copy=int(out[3]), gm4_nonleaf=int(out[4]), regrids=int(out[5]))

    # ---- time loop
    def step_control(self):
        self.L.orc_step_control(self.h)

    def time_advance_rk(self):
        self.L.orc_time_advance_rk(self.h)

    def stage(self, krk: int):
        self.L.orc_stage(self.h, krk)

    def body_boundary(self, j: int):
        self.L.orc_body_boundary(self.h, j)

    # ---- strips of one mesh (halo exchange)
    def step_control_global(self, lambda_x, lambda_y, l_max):
        self.L.orc_step_control_global(self.h, float(lambda_x), float(lambda_y), int(l_max))
        return self.scalars()["tstep"]

    def get_U(self, idx):
        """U(1:7) of the leaves idx (positions in key order), shape (n, 7)."""
        idx = np.ascontiguousarray(idx, np.int64)
        out = np.zeros((len(idx), 7), np.float64)
        rc = self.L.orc_get_U(self.h, len(idx), idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _dp(out))
        if rc:
            raise IndexError("leaf index out of range")
        return out

    def set_U(self, idx, U):
        idx = np.ascontiguousarray(idx, np.int64)
        U = np.ascontiguousarray(U, np.float64)
        assert U.shape == (len(idx), 7)
        rc = self.L.orc_set_U(self.h, len(idx), idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _dp(U))
        if rc:
            raise IndexError("leaf index out of range")

    def solute_step(self) -> int:
        return int(self.L.orc_solute_step(self.h))

    def solute(self, nsteps: int) -> int:
        done = ctypes.c_int64(0)
        rc = self.L.orc_solute(self.h, nsteps, ctypes.byref(done))
        if rc:
            raise FloatingPointError(f"oracle NaN residual after {done.value} steps")
        return done.value

    def amr(self):
        self.L.orc_amr(self.h)

    def rot_div(self):
        self.L.orc_rot_div(self.h)
        n = self.num_interior()
        rot = np.zeros(n)
        div = np.zeros(n)
        self.L.orc_export_rot_div(self.h, n, _dp(rot), _dp(div))
        return rot, div

    def stencil(self):
        n = self.num_interior()
        out = np.zeros((n, 8, 4))
        self.L.orc_export_stencil(self.h, n, _dp(out))
        return out

    def gather(self):
        """Hanging-node stencil of every (interior leaf, entry): kind
        (0 leaf copy, 1 parent WLS, 2 parent interpA, 3 child WLS, 4 child
        copy), node key, target (xx, yy), (m1, m2) and member keys."""
        n = self.num_interior()
        kind = np.zeros((n, 8), np.int32)
        node = np.zeros((n, 8), np.uint64)
        xy = np.zeros((n, 8, 2))
        m12 = np.zeros((n, 8, 2), np.int32)
        mem = np.zeros((n, 8, 16), np.uint64)
        i32p = ctypes.POINTER(ctypes.c_int32)
        self.L.orc_export_gather(self.h, n, kind.ctypes.data_as(i32p), _u64p(node), _dp(xy),
                                 m12.ctypes.data_as(i32p), _u64p(mem))
        return dict(kind=kind, node=node, xy=xy, m12=m12, mem=mem)

    def neighbors(self):
        n = self.num_leaves()
        out = np.zeros((n, 8), np.uint64)
        self.L.orc_export_neighbors(self.h, n, _u64p(out))
        return out

    def residual(self):
        rmax = np.zeros(4)
        rrms = np.zeros(4)
        self.L.orc_residual(self.h, _dp(rmax), _dp(rrms))
        return rmax, rrms


# ---- numerics entry points (known-answer tests)
def wcns_z3(u1, u2, u3, R):
    u1, u2, u3 = (np.ascontiguousarray(a, np.float64) for a in (u1, u2, u3))
    R = np.ascontiguousarray(R, np.float64)
    out = np.zeros(4)
    lib().orc_wcns_z3(_dp(u1), _dp(u2), _dp(u3), _dp(R), _dp(out))
    return out


def eigen(gama, direction, U4):
    U4 = np.ascontiguousarray(U4, np.float64)
    R = np.zeros((4, 4))
    Ri = np.zeros((4, 4))
    lib().orc_eigen(gama, direction, _dp(U4), _dp(R), _dp(Ri))
    return R, Ri


def brinv(a):
    a = np.array(a, dtype=np.float64, order="C")
    n = a.shape[0]
    rc = lib().orc_brinv(n, _dp(a))
    return a, rc == 0


def get_direction(xx, yy, x, y):
    return int(lib().orc_get_direction(xx, yy, x, y))


def lxl_dir(gama, direction, lam, dxy, stencil5x4):
    st = np.ascontiguousarray(stencil5x4, np.float64)
    out = np.zeros(4)
    lib().orc_lxl_dir(gama, direction, lam, dxy, _dp(st), _dp(out))
    return out


def wls(h, xf, lvl, cx, cy, xx, yy, m1, m2, xs, ys, vals):
    xs = np.ascontiguousarray(xs, np.float64)
    ys = np.ascontiguousarray(ys, np.float64)
    vals = np.ascontiguousarray(vals, np.float64)
    out = np.zeros(4)
    nsing = lib().orc_wls(h, xf, lvl, cx, cy, xx, yy, m1, m2, _dp(xs), _dp(ys), _dp(vals), _dp(out))
    return out, nsing
