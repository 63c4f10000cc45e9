"""Host-side mirror of the reference's driver (program main / solute,
src/MAIN.F90:1-25, src/solution.F90:171-238) over the libfdm C-ABI.

The names follow the reference: ``creat_mesh`` builds the background grid
(src/mesh.F90:9-47), ``initial`` evaluates the initial state on the host
(src/solution.F90:9-69; the vortex formulas are evaluated with the C
library's exp/pow exactly as written there), ``solute`` runs the time loop,
``time_advance_rk`` / ``amr`` / ``step_control`` are the device calls.  There
is no CPU fallback: constructing a Solver without a CUDA device or without
libfdm.so raises.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

from . import params as P

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfdm.so")

FDM_OK = 0
FDM_ERR_NAN = 3
ERRORS = {1: "FDM_ERR_ARG", 2: "FDM_ERR_CUDA", 3: "FDM_ERR_NAN", 4: "FDM_ERR_TIMEOUT",
          5: "FDM_ERR_NOMEM", 6: "FDM_ERR_STATE", 7: "FDM_ERR_UNSUPPORTED"}

FACE_VARIANTS = 21   # FDM_FACE_VARIANTS of include/fdm.h

# every extern "C" symbol declared in include/fdm.h
EXPORTS = [
    "fdm_create", "fdm_destroy", "fdm_last_error", "fdm_upload_leaves", "fdm_num_leaves",
    "fdm_download_leaves", "fdm_set_values", "fdm_get_scalars", "fdm_set_scalars",
    "fdm_step_control", "fdm_time_advance_rk", "fdm_get_rkn", "fdm_solution_cells",
    "fdm_update_rk", "fdm_body_boundary", "fdm_residual", "fdm_solute_step", "fdm_solute",
    "fdm_advance", "fdm_amr", "fdm_get_counters", "fdm_debug_stencil", "fdm_debug_neighbors",
    "fdm_debug_requests",
    "fdm_debug_rot_div", "fdm_debug_ordered_sum", "fdm_device_state", "fdm_time_kernels", "fdm_fp64_peak", "fdm_autotune",
    "fdm_set_variant", "fdm_time_advance_rk_uniform_static", "fdm_gate_param_count", "fdm_gate_set",
    "fdm_gate_samples", "fdm_gate_train_step", "fdm_gate_eval", "fdm_gate_stats", "fdm_amr_phase_ms",
    "fdm_batch_create", "fdm_batch_destroy", "fdm_batch_last_error", "fdm_batch_advance", "fdm_batch_solute",
    "fdm_batch_sync", "fdm_batch_set_blocks_per_sm", "fdm_batch_set_wait_limit", "fdm_batch_set_face_flux", "fdm_batch_info", "fdm_batch_stream", "fdm_batch_phase_us",
    "fdm_set_values_async", "fdm_download_values_async", "fdm_io_sync",
    "fdm_leaf_slots", "fdm_pack_slots", "fdm_unpack_slots", "fdm_step_control_global",
    "fdm_download_internal", "fdm_set_internal", "fdm_set_async", "fdm_debug_barrier_timeout",
    "fdm_debug_fail_alloc", "fdm_solute_paired", "fdm_output_error", "fdm_download_keys_async",
    "fdm_readback_wait", "fdm_gate_set_jump_rule", "fdm_debug_nr_fallbacks",
]


class FdmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class FdmCounters(ctypes.Structure):
    _fields_ = [("n_leaves", ctypes.c_int64), ("n_interior", ctypes.c_int64),
                ("n_ghost", ctypes.c_int64), ("n_wls_requests", ctypes.c_int64),
                ("n_restrict_requests", ctypes.c_int64), ("n_faces_x", ctypes.c_int64),
                ("n_faces_y", ctypes.c_int64), ("n_singular", ctypes.c_int64),
                ("n_regrids", ctypes.c_int64), ("n_internal", ctypes.c_int64),
                ("n_gm1_iterations", ctypes.c_int64), ("n_gm4_visits", ctypes.c_int64),
                ("n_gm4_nonleaf", ctypes.c_int64), ("n_gm4_triggers", ctypes.c_int64),
                ("n_gm4_refines", ctypes.c_int64), ("n_gm4_steps", ctypes.c_int64),
                ("gm4_replay_us", ctypes.c_int64)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libfdm.so and declare the C signatures.  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run __graft_entry__.build() first")
    L = ctypes.CDLL(path)
    vp, i64, i32, dp = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L.fdm_create.argtypes = [ctypes.POINTER(P.FdmParams), ctypes.POINTER(vp)]
    L.fdm_destroy.argtypes = [vp]
    L.fdm_destroy.restype = None
    L.fdm_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    L.fdm_upload_leaves.argtypes = [vp, i64, u64p, dp]
    L.fdm_num_leaves.argtypes = [vp]
    L.fdm_num_leaves.restype = i64
    L.fdm_download_leaves.argtypes = [vp, i64, ctypes.POINTER(i64), u64p, dp]
    L.fdm_set_values.argtypes = [vp, i64, dp]
    L.fdm_set_values_async.argtypes = [vp, i64, dp]
    L.fdm_download_values_async.argtypes = [vp, i64, dp]
    L.fdm_io_sync.argtypes = [vp]
    L.fdm_get_scalars.argtypes = [vp, dp, dp, dp, dp, ctypes.POINTER(i64), ctypes.POINTER(i32)]
    L.fdm_set_scalars.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, i64]
    L.fdm_step_control.argtypes = [vp, dp, dp, dp, ctypes.POINTER(i32)]
    L.fdm_time_advance_rk.argtypes = [vp, ctypes.c_double]
    L.fdm_get_rkn.argtypes = [vp]
    L.fdm_solution_cells.argtypes = [vp, i32]
    L.fdm_update_rk.argtypes = [vp, i32]
    L.fdm_body_boundary.argtypes = [vp, i32]
    L.fdm_residual.argtypes = [vp, dp, dp]
    L.fdm_solute_step.argtypes = [vp]
    L.fdm_solute.argtypes = [vp, i64, ctypes.POINTER(i64)]
    L.fdm_advance.argtypes = [vp, i64]
    L.fdm_amr.argtypes = [vp]
    L.fdm_get_counters.argtypes = [vp, ctypes.POINTER(FdmCounters)]
    L.fdm_debug_stencil.argtypes = [vp, i64, dp]
    L.fdm_debug_neighbors.argtypes = [vp, i64, u64p]
    i32p = ctypes.POINTER(ctypes.c_int32)
    L.fdm_debug_requests.argtypes = [vp, i64, i32p, u64p, dp, i32p, u64p]
    L.fdm_debug_rot_div.argtypes = [vp, i64, dp, dp, dp]
    L.fdm_debug_ordered_sum.argtypes = [dp, dp, i64, dp]
    L.fdm_device_state.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(dp), ctypes.POINTER(i64)]
    L.fdm_time_kernels.argtypes = [vp, i32, dp]
    L.fdm_fp64_peak.argtypes = [dp]
    L.fdm_amr_phase_ms.argtypes = [vp, dp]
    L.fdm_autotune.argtypes = [vp, i32, ctypes.POINTER(i32), dp]
    L.fdm_set_variant.argtypes = [vp, i32]
    L.fdm_time_advance_rk_uniform_static.argtypes = [vp, vp, i32, i32, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                     ctypes.c_double, vp]
    L.fdm_batch_create.argtypes = [ctypes.POINTER(vp), i32, ctypes.POINTER(vp)]
    L.fdm_batch_destroy.argtypes = [vp]
    L.fdm_batch_destroy.restype = None
    L.fdm_batch_last_error.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
    L.fdm_batch_advance.argtypes = [vp, i64]
    L.fdm_batch_solute.argtypes = [vp, i64, ctypes.POINTER(i64)]
    L.fdm_batch_sync.argtypes = [vp]
    L.fdm_batch_set_blocks_per_sm.argtypes = [vp, i32]
    L.fdm_batch_set_wait_limit.argtypes = [vp, ctypes.c_double]
    L.fdm_batch_set_face_flux.argtypes = [vp, i32]
    L.fdm_batch_info.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i64)]
    L.fdm_batch_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.fdm_batch_phase_us.argtypes = [vp, dp]
    L.fdm_leaf_slots.argtypes = [vp, i64, i32p]
    L.fdm_download_internal.argtypes = [vp, i64, ctypes.POINTER(i64), u64p, dp]
    L.fdm_set_internal.argtypes = [vp, i64, u64p, dp]
    L.fdm_pack_slots.argtypes = [vp, i64, vp, vp]
    L.fdm_unpack_slots.argtypes = [vp, i64, vp, vp]
    L.fdm_step_control_global.argtypes = [vp, ctypes.c_double, ctypes.c_double, i32, dp]
    L.fdm_set_async.argtypes = [vp, i32]
    L.fdm_debug_barrier_timeout.argtypes = [dp]
    L.fdm_debug_fail_alloc.argtypes = [i64]
    L.fdm_solute_paired.argtypes = [vp, vp, i64, ctypes.POINTER(i64)]
    L.fdm_output_error.argtypes = [vp, dp, ctypes.POINTER(i64)]
    L.fdm_download_keys_async.argtypes = [vp, i64, u64p]
    L.fdm_readback_wait.argtypes = [vp]
    L.fdm_gate_set_jump_rule.argtypes = [vp, ctypes.c_float]
    L.fdm_debug_nr_fallbacks.argtypes = [vp, ctypes.POINTER(i64)]
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


# ------------------------------------------------------------ host mesh
def root_keys(m: int, n: int) -> np.ndarray:
    """Keys of the background cells, cell(1..m*n) (src/mesh.F90:15-37)."""
    return (np.arange(m * n, dtype=np.uint64) << np.uint64(34))


def node_centers(cfg: P.Config, keys: np.ndarray):
    """Centres by the reference's chain of operations: creat_mesh for the
    background cell, then one Refine_cell offset per level
    (src/mesh.F90:25-26, 205-248)."""
    p = cfg.params
    keys = np.asarray(keys, dtype=np.uint64)
    root = (keys >> np.uint64(34)).astype(np.int64)
    lvl = (keys & np.uint64(15)).astype(np.int64)
    path = ((keys >> np.uint64(4)) & np.uint64((1 << 30) - 1)).astype(np.int64)
    nj = (root % p.m + 1).astype(np.float64)
    ni = (root // p.m + 1 + p.window_row0).astype(np.float64)   # global row of a strip
    cx = 0.5 * (2.0 * nj - 1.0) * p.x_factor * p.h + p.xmin
    cy = (ni - 0.5) * p.h + p.ymin
    for k in range(1, int(lvl.max(initial=0)) + 1):
        act = lvl >= k
        q = (path >> (2 * (15 - k))) & 3
        qx = p.x_factor * p.h / float(1 << (k + 1))
        qy = p.h / float(1 << (k + 1))
        cx = np.where(act, np.where(q & 1, cx + qx, cx - qx), cx)
        cy = np.where(act, np.where(q & 2, cy + qy, cy - qy), cy)
    return cx, cy


def initial_state(cfg: P.Config, keys: np.ndarray) -> np.ndarray:
    """Initial primitive state (rho,u,v,p) per leaf (src/solution.F90:31-69
    for the vortex; quadrant and oblique-shock states for the extensions)."""
    p = cfg.params
    cx, cy = node_centers(cfg, keys)
    out = np.zeros((len(keys), 4))
    g = p.gama
    if cfg.ic_kind == P.IC_VORTEX:
        cc, pi = 5.0, 3.1415926535897932
        for i in range(len(keys)):
            x, y = float(cx[i]), float(cy[i])
            rr = (x - 5.0) * (x - 5.0) + (y - 5.0) * (y - 5.0)
            dT = -(g - 1.0) * (cc * cc) * math.exp(1.0 - rr) / (8.0 * g * pi * pi)
            out[i, 0] = 1.0 + math.pow(1.0 + dT, 1.0 / (g - 1.0)) - 1.0
            out[i, 1] = 1.0 - (y - 5.0) * cc / (2.0 * pi) * math.exp(0.5 * (1.0 - rr))
            out[i, 2] = 1.0 + (x - 5.0) * cc / (2.0 * pi) * math.exp(0.5 * (1.0 - rr))
            out[i, 3] = 1.0 + math.pow(1.0 + dT, g / (g - 1.0)) - 1.0
    elif cfg.ic_kind == P.IC_QUADRANTS:
        icp = cfg.ic_params
        st = np.asarray(icp[2:18], dtype=np.float64).reshape(4, 4)
        east = cx > icp[0]
        north = cy > icp[1]
        q = np.where(north, np.where(east, 0, 1), np.where(east, 3, 2))
        out[:] = st[q]
    else:
        x0, cot = cfg.ic_params[0], cfg.ic_params[1]
        post = np.array(list(p.dmr_post))
        pre = np.array(list(p.dmr_pre))
        xs = x0 + cy * cot
        out[:] = np.where((cx < xs)[:, None], post[None, :], pre[None, :])
    return out


class Solver:
    """One solver instance on the current CUDA device (a libfdm handle)."""

    def __init__(self, cfg: P.Config):
        self.cfg = cfg
        self.L = load_library()
        h = ctypes.c_void_p()
        rc = self.L.fdm_create(ctypes.byref(cfg.params), ctypes.byref(h))
        if rc:
            raise FdmError(rc, "fdm_create failed (no CUDA device, or inconsistent parameters)")
        self.h = h

    # ---- error handling
    def _check(self, rc: int):
        if rc:
            buf = ctypes.create_string_buffer(512)
            self.L.fdm_last_error(self.h, buf, 512)
            raise FdmError(rc, buf.value.decode(errors="replace"))

    def close(self):
        if getattr(self, "h", None):
            self.L.fdm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- mesh + state
    def creat_mesh_and_initial(self):
        """creat_mesh + initial (src/mesh.F90:9-47, src/solution.F90:9-29):
        background grid (with the static block refinement when the
        configuration has one), initial state, periodic/extension ghost
        fill."""
        if self.cfg.block:
            from .mesh import block_refined_keys
            keys = block_refined_keys(self.cfg)
        else:
            keys = root_keys(self.cfg.m, self.cfg.n)
        prim = initial_state(self.cfg, keys)
        self.upload(keys, prim)
        self.body_boundary(1)
        return keys

    def upload(self, keys, prim):
        keys = np.ascontiguousarray(keys, np.uint64)
        prim = np.ascontiguousarray(prim, np.float64)
        self._check(self.L.fdm_upload_leaves(self.h, len(keys), _u64p(keys), _dp(prim)))

    def set_values(self, prim):
        prim = np.ascontiguousarray(prim, np.float64)
        self._check(self.L.fdm_set_values(self.h, len(prim), _dp(prim)))

    def num_leaves(self) -> int:
        return int(self.L.fdm_num_leaves(self.h))

    def leaves(self):
        n = self.num_leaves()
        keys = np.zeros(n, np.uint64)
        prim = np.zeros((n, 4))
        nout = ctypes.c_int64()
        self._check(self.L.fdm_download_leaves(self.h, n, ctypes.byref(nout), _u64p(keys), _dp(prim)))
        return keys, prim

    def download_values(self, out):
        """Primitive values of all leaves, key order, into out (n x 4 float64,
        C-contiguous; pinned host memory makes the copy direct)."""
        n = self.num_leaves()
        assert out.shape == (n, 4) and out.dtype == np.float64 and out.flags["C_CONTIGUOUS"]
        nout = ctypes.c_int64()
        self._check(self.L.fdm_download_leaves(self.h, n, ctypes.byref(nout), None, _dp(out)))
        return out

    def set_values_async(self, prim):
        """Asynchronous fdm_set_values: prim must be pinned host memory
        (e.g. a torch pinned tensor's numpy view) kept until io_sync()."""
        assert prim.dtype == np.float64 and prim.flags["C_CONTIGUOUS"]
        self._check(self.L.fdm_set_values_async(self.h, len(prim), _dp(prim)))

    def download_values_async(self, out):
        """Asynchronous read-back of the current values into pinned out."""
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"]
        self._check(self.L.fdm_download_values_async(self.h, len(out), _dp(out)))

    def download_keys_async(self, out):
        """Asynchronous read-back of the leaf keys into pinned out (uint64)."""
        assert out.dtype == np.uint64 and out.flags["C_CONTIGUOUS"]
        self._check(self.L.fdm_download_keys_async(self.h, len(out), _u64p(out)))

    def output_error_device(self) -> dict:
        """output_error's density norms computed on the device (only the
        norms cross to the host)."""
        nm = np.zeros(9)
        ct = (ctypes.c_int64 * 3)()
        self._check(self.L.fdm_output_error(self.h, _dp(nm), ct))
        return dict(n_res=int(ct[0]), L1_rho=nm[0], L2_rho=nm[1], Loo_rho=nm[2], P1_rho=nm[3], P2_rho=nm[4],
                    Poo_rho=nm[5], n_0=int(ct[1]), n_patch=int(ct[2]), L1_rho0=nm[6], L2_rho0=nm[7],
                    Loo_rho0=nm[8])

    def readback_wait(self):
        """Wait for the queued read-backs only (safe from another thread)."""
        rc = self.L.fdm_readback_wait(self.h)
        if rc:
            raise FdmError(rc, "fdm_readback_wait failed")

    def io_sync(self):
        self._check(self.L.fdm_io_sync(self.h))

    def scalars(self) -> dict:
        lx, ly, dt, tt = (ctypes.c_double() for _ in range(4))
        it = ctypes.c_int64()
        lm = ctypes.c_int32()
        self._check(self.L.fdm_get_scalars(self.h, ctypes.byref(lx), ctypes.byref(ly), ctypes.byref(dt),
                                           ctypes.byref(tt), ctypes.byref(it), ctypes.byref(lm)))
        return dict(lambda_x=lx.value, lambda_y=ly.value, tstep=dt.value, tt=tt.value, it=it.value,
                    l_max=lm.value)

    def set_scalars(self, lambda_x, lambda_y, tstep, tt, it):
        self._check(self.L.fdm_set_scalars(self.h, lambda_x, lambda_y, tstep, tt, int(it)))

    def counters(self) -> dict:
        c = FdmCounters()
        self._check(self.L.fdm_get_counters(self.h, ctypes.byref(c)))
        return {k: getattr(c, k) for k, _ in FdmCounters._fields_ if k != "reserved"}

    # ---- time loop (reference names)
    def step_control(self):
        dt, lx, ly = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        lm = ctypes.c_int32()
        self._check(self.L.fdm_step_control(self.h, ctypes.byref(dt), ctypes.byref(lx), ctypes.byref(ly),
                                            ctypes.byref(lm)))
        return dt.value

    # ---- checkpoint/restart
    def internal_nodes(self):
        """Keys (sorted) and (rho,u,v,p) values of the internal nodes."""
        n = ctypes.c_int64()
        cnt = self.counters()["n_internal"]
        keys = np.zeros(cnt, np.uint64)
        vals = np.zeros((cnt, 4))
        self._check(self.L.fdm_download_internal(self.h, cnt, ctypes.byref(n), _u64p(keys), _dp(vals)))
        return keys, vals

    def set_internal(self, keys, vals):
        keys = np.ascontiguousarray(keys, np.uint64)
        vals = np.ascontiguousarray(vals, np.float64)
        self._check(self.L.fdm_set_internal(self.h, len(keys), _u64p(keys), _dp(vals)))

    def save_checkpoint(self, path: str):
        """The handle's whole state (leaves, internal-node values, scalars,
        and the parameters it runs with) into one .npz file."""
        keys, prim = self.leaves()
        ikeys, ivals = self.internal_nodes()
        sc = self.scalars()
        np.savez(path, params=np.frombuffer(bytes(self.cfg.params), np.uint8), keys=keys, prim=prim,
                 ikeys=ikeys, ivals=ivals,
                 scalars=np.array([sc["lambda_x"], sc["lambda_y"], sc["tstep"], sc["tt"]]),
                 it=np.array([sc["it"]], np.int64))

    def load_checkpoint(self, path: str):
        """Restore a state written by save_checkpoint into this handle (same
        parameters); the run then continues bit for bit."""
        with np.load(path) as z:
            if bytes(z["params"]) != bytes(self.cfg.params):
                raise ValueError("the checkpoint was written with other parameters")
            self.upload(z["keys"], z["prim"])
            self.set_internal(z["ikeys"], z["ivals"])
            lx, ly, dt, tt = (float(v) for v in z["scalars"])
            self.set_scalars(lx, ly, dt, tt, int(z["it"][0]))

    def step_control_info(self):
        """fdm_step_control: (tstep, lambda_x, lambda_y, l_max)."""
        dt, lx, ly = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        lm = ctypes.c_int32()
        self._check(self.L.fdm_step_control(self.h, ctypes.byref(dt), ctypes.byref(lx), ctypes.byref(ly),
                                            ctypes.byref(lm)))
        return dt.value, lx.value, ly.value, lm.value

    # ---- strips of one mesh (halo exchange)
    def step_control_global(self, lambda_x: float, lambda_y: float, l_max: int) -> float:
        """The time step from maxima taken over all strips of the mesh."""
        dt = ctypes.c_double()
        self._check(self.L.fdm_step_control_global(self.h, float(lambda_x), float(lambda_y), int(l_max),
                                                   ctypes.byref(dt)))
        return dt.value

    def set_async(self, on: bool):
        """Split-API calls and halo copies return once enqueued on the
        handle's stream (device_state()[0]) instead of waiting."""
        self._check(self.L.fdm_set_async(self.h, 1 if on else 0))

    def leaf_slots(self) -> np.ndarray:
        """State slot of every leaf, key order."""
        n = self.num_leaves()
        out = np.zeros(n, np.int32)
        self._check(self.L.fdm_leaf_slots(self.h, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return out

    def pack_slots(self, slots_dev: int, n: int, buf_dev: int):
        """Gather the latest stage's records at n slots (device int32 array)
        into a device buffer of n x 4 float64."""
        self._check(self.L.fdm_pack_slots(self.h, int(n), ctypes.c_void_p(slots_dev), ctypes.c_void_p(buf_dev)))

    def unpack_slots(self, slots_dev: int, n: int, buf_dev: int):
        self._check(self.L.fdm_unpack_slots(self.h, int(n), ctypes.c_void_p(slots_dev), ctypes.c_void_p(buf_dev)))

    def time_advance_rk(self, tstep: float):
        self._check(self.L.fdm_time_advance_rk(self.h, float(tstep)))

    def solution_cells(self, krk: int):
        self._check(self.L.fdm_solution_cells(self.h, krk))

    def update_rk(self, krk: int):
        self._check(self.L.fdm_update_rk(self.h, krk))

    def body_boundary(self, j: int):
        self._check(self.L.fdm_body_boundary(self.h, j))

    def residual(self):
        rmax = np.zeros(4)
        rrms = np.zeros(4)
        self._check(self.L.fdm_residual(self.h, _dp(rmax), _dp(rrms)))
        return rmax, rrms

    def solute_step(self):
        self._check(self.L.fdm_solute_step(self.h))

    def solute(self, nsteps: int) -> int:
        done = ctypes.c_int64()
        self._check(self.L.fdm_solute(self.h, int(nsteps), ctypes.byref(done)))
        return done.value

    def solute_paired(self, follower: "Solver", nsteps: int) -> int:
        """nsteps iterations of this solver and ``follower`` in lockstep: the
        follower takes this solver's time step and regrid decisions
        (fdm_solute_paired); returns the steps taken."""
        k = ctypes.c_int64()
        rc = self.L.fdm_solute_paired(self.h, follower.h, int(nsteps), ctypes.byref(k))
        if rc:
            buf = ctypes.create_string_buffer(512)
            self.L.fdm_last_error(follower.h, buf, 512)
            msg = buf.value.decode(errors="replace")
            self.L.fdm_last_error(self.h, buf, 512)
            raise FdmError(rc, f"follower: {msg}; leader: {buf.value.decode(errors='replace')}")
        return k.value

    def advance(self, nsteps: int):
        self._check(self.L.fdm_advance(self.h, int(nsteps)))

    def amr(self):
        self._check(self.L.fdm_amr(self.h))

    def stencil(self):
        n = self.counters()["n_interior"]
        out = np.zeros((n, 8, 4))
        self._check(self.L.fdm_debug_stencil(self.h, n, _dp(out)))
        return out

    def neighbors(self):
        n = self.num_leaves()
        out = np.zeros((n, 8), np.uint64)
        self._check(self.L.fdm_debug_neighbors(self.h, n, _u64p(out)))
        return out

    def requests(self):
        """Hanging-node stencils per (interior leaf, entry) in the oracle's
        gather encoding (see fdm_debug_requests)."""
        n = self.counters()["n_interior"]
        kind = np.zeros((n, 8), np.int32)
        node = np.zeros((n, 8), np.uint64)
        xy = np.zeros((n, 8, 2))
        m12 = np.zeros((n, 8, 2), np.int32)
        mem = np.zeros((n, 8, 16), np.uint64)
        i32p = ctypes.POINTER(ctypes.c_int32)
        self._check(self.L.fdm_debug_requests(self.h, n, kind.ctypes.data_as(i32p), _u64p(node), _dp(xy),
                                              m12.ctypes.data_as(i32p), _u64p(mem)))
        return dict(kind=kind, node=node, xy=xy, m12=m12, mem=mem)

    def rot_div(self):
        n = self.counters()["n_interior"]
        rot = np.zeros(n)
        div = np.zeros(n)
        sums = np.zeros(3)
        self._check(self.L.fdm_debug_rot_div(self.h, n, _dp(rot), _dp(div), _dp(sums)))
        return rot, div, sums

    def amr_phase_ms(self, total: bool = False) -> dict:
        """Device-timeline ms of the regrid phases: of the last regrid, or
        summed over all regrids of this solver."""
        a = np.zeros(10)
        self._check(self.L.fdm_amr_phase_ms(self.h, _dp(a)))
        v = a[5:] if total else a[:5]
        return dict(zip(("indicators", "flags", "gridmodify", "split", "tables"), v.tolist()))

    def time_kernels(self, reps: int = 10):
        """Average ms per launch: faces (x+y), cells, hanging nodes, ghosts."""
        ms = np.zeros(4)
        self._check(self.L.fdm_time_kernels(self.h, int(reps), _dp(ms)))
        return dict(faces=ms[0], cells=ms[1], requests=ms[2], ghosts=ms[3])

    def autotune(self, reps: int = 5):
        """Pick the fastest face-kernel launch shape for this leaf set."""
        best = ctypes.c_int32()
        ms = np.zeros(FACE_VARIANTS)
        self._check(self.L.fdm_autotune(self.h, int(reps), ctypes.byref(best), _dp(ms)))
        return best.value, ms

    def nr_fallbacks(self):
        """(x, y) faces of the current state whose branch-free division falls
        back to the compiler's."""
        out = (ctypes.c_int64 * 2)()
        self._check(self.L.fdm_debug_nr_fallbacks(self.h, out))
        return int(out[0]), int(out[1])

    def set_variant(self, v: int):
        self._check(self.L.fdm_set_variant(self.h, int(v)))

    def device_state(self):
        s = ctypes.c_void_p()
        p = ctypes.POINTER(ctypes.c_double)()
        n = ctypes.c_int64()
        self._check(self.L.fdm_device_state(self.h, ctypes.byref(s), ctypes.byref(p), ctypes.byref(n)))
        return s.value, ctypes.cast(p, ctypes.c_void_p).value, n.value

    # ---- diagnostics (output_error, src/output_ADT.F90:18-75)
    def output_error(self):
        """L1/L2/Linf density error of the interior leaves against the t = 0
        vortex, area-weighted as output_error does."""
        keys, prim = self.leaves()
        return vortex_error(self.cfg, keys, prim)


class Batch:
    """An ensemble of loaded solvers on one GPU advanced together: one
    persistent kernel launch per RK3 stage covers every member (libfdm's
    fdm_batch_*).  The solvers stay usable on their own between calls."""

    def __init__(self, solvers):
        self.L = load_library()
        self.members = list(solvers)
        arr = (ctypes.c_void_p * len(self.members))(*[s.h.value for s in self.members])
        b = ctypes.c_void_p()
        rc = self.L.fdm_batch_create(arr, len(self.members), ctypes.byref(b))
        if rc:
            raise FdmError(rc, "fdm_batch_create failed")
        self.b = b

    def _check(self, rc: int):
        if rc:
            buf = ctypes.create_string_buffer(512)
            self.L.fdm_batch_last_error(self.b, buf, 512)
            raise FdmError(rc, buf.value.decode(errors="replace"))

    def advance(self, nsteps: int):
        """nsteps steps of every unfinished member, no regrid, no host sync."""
        self._check(self.L.fdm_batch_advance(self.b, int(nsteps)))

    def solute(self, nsteps: int) -> int:
        """nsteps steps with the members' regrids when due; returns the steps taken."""
        k = ctypes.c_int64()
        self._check(self.L.fdm_batch_solute(self.b, int(nsteps), ctypes.byref(k)))
        return k.value

    def sync(self):
        self._check(self.L.fdm_batch_sync(self.b))

    def set_blocks_per_sm(self, k: int):
        """1 or 2 resident blocks per SM for the persistent kernel; 0: each
        member's own step graph on its own stream; 3: one launch per phase
        covering every member."""
        self._check(self.L.fdm_batch_set_blocks_per_sm(self.b, int(k)))

    def set_face_flux(self, branch_free: bool):
        """Face phases of the persistent kernel in the reference's order (False)
        or the split order with the branch-free division (True): same bits."""
        self._check(self.L.fdm_batch_set_face_flux(self.b, 1 if branch_free else 0))

    def set_wait_limit(self, seconds: float):
        """Wait limit of one grid barrier of the persistent kernel (default
        2 s); a wait that runs past it ends the step with FDM_ERR_TIMEOUT."""
        self._check(self.L.fdm_batch_set_wait_limit(self.b, float(seconds)))

    def info(self) -> dict:
        g, bps, sm = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        self._check(self.L.fdm_batch_info(self.b, ctypes.byref(g), ctypes.byref(bps), ctypes.byref(sm)))
        return {"grid": g.value, "blocks_per_sm": bps.value, "smem_bytes": sm.value}

    def phase_us(self):
        """Microseconds of each phase of the last step, shape (3 stages, 16)."""
        a = np.zeros(48)
        self._check(self.L.fdm_batch_phase_us(self.b, _dp(a)))
        return a.reshape(3, 16)

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.L.fdm_batch_stream(self.b, ctypes.byref(s)))
        return s.value or 0

    def close(self):
        if getattr(self, "b", None):
            self.L.fdm_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def vortex_error(cfg: P.Config, keys, prim):
    p = cfg.params
    root = (np.asarray(keys, np.uint64) >> np.uint64(34)).astype(np.int64)
    row, col = root // p.m, root % p.m
    inter = (row >= 3) & (row < p.n - 3) & (col >= 3) & (col < p.m - 3)
    lvl = (np.asarray(keys, np.uint64) & np.uint64(15)).astype(np.int64)
    cx, cy = node_centers(cfg, keys)
    g = p.gama
    rr = (cx - 5.0) ** 2 + (cy - 5.0) ** 2
    dT = -(g - 1.0) * 25.0 * np.exp(1.0 - rr) / (8.0 * g * math.pi ** 2)
    err = prim[:, 0] - (1.0 + dT) ** (1.0 / (g - 1.0))
    dy = p.h / (2.0 ** lvl)
    area = p.x_factor * dy * dy
    e, a = err[inter], area[inter]
    return dict(L1=float(np.sum(np.abs(e) * a) / np.sum(a)),
                L2=float(math.sqrt(np.sum(e * e * a) / np.sum(a))),
                Linf=float(np.max(np.abs(e))))


# ------------------------------------------------- static distance refinement
def distance_refined_keys(cfg: P.Config, lines, dist_by_level) -> np.ndarray:
    """Leaf keys of a statically refined mesh, in the manner of the
    reference's BlockDis_refi (src/mesh.F90:144-172): a leaf at level l is
    refined when its centre lies within dist_by_level[l] of any of the given
    axis-parallel lines ("x", c) / ("y", c).  Distances must shrink by at
    least two cells of the finer level per level so that the result keeps the
    2:1 balance.  Ghost background cells follow the same rule, so the balance
    also holds across the domain boundary (the reference's gridmodify refines
    ghost cells next to refined interior cells in the same way); a refined
    interior cell beside an unrefined ghost would break the hanging-node
    stencils there."""
    p = cfg.params
    m, n = cfg.m, cfg.n
    root = np.arange(m * n, dtype=np.int64)
    row, col = root // m, root % m
    lvl = np.zeros_like(root)
    ix = np.zeros_like(root)
    iy = np.zeros_like(root)
    inter = np.ones(m * n, dtype=bool)
    done_r, done_l, done_x, done_y = [], [], [], []
    cur_r, cur_l, cur_x, cur_y, cur_i = root, lvl, ix, iy, inter
    for L in range(len(dist_by_level) + 1):
        hx = p.x_factor * p.h / (1 << L)
        hy = p.h / (1 << L)
        cx = p.xmin + col_of(cur_r, m) * p.x_factor * p.h + (cur_x + 0.5) * hx
        cy = p.ymin + (cur_r // m) * p.h + (cur_y + 0.5) * hy
        refine = np.zeros(len(cur_r), bool)
        if L < len(dist_by_level):
            d = dist_by_level[L]
            for ax, c in lines:
                refine |= np.abs((cx if ax == "x" else cy) - c) < d
            refine &= cur_i
        keep = ~refine
        done_r.append(cur_r[keep]); done_l.append(cur_l[keep])
        done_x.append(cur_x[keep]); done_y.append(cur_y[keep])
        if not refine.any():
            break
        r, l, x, y, it = cur_r[refine], cur_l[refine], cur_x[refine], cur_y[refine], cur_i[refine]
        cur_r = np.repeat(r, 4)
        cur_l = np.repeat(l + 1, 4)
        q = np.tile(np.arange(4), len(r))
        cur_x = np.repeat(2 * x, 4) + (q & 1)
        cur_y = np.repeat(2 * y, 4) + (q >> 1)
        cur_i = np.repeat(it, 4)
    r = np.concatenate(done_r); l = np.concatenate(done_l)
    x = np.concatenate(done_x); y = np.concatenate(done_y)
    s = 15 - l
    path = morton(x << s, y << s)
    keys = (r.astype(np.uint64) << np.uint64(34)) | (path.astype(np.uint64) << np.uint64(4)) | l.astype(np.uint64)
    return np.sort(keys)


def col_of(r, m):
    return r % m


def morton(x, y):
    x = np.asarray(x, np.uint64)
    y = np.asarray(y, np.uint64)
    out = np.zeros_like(x)
    for b in range(15):
        out |= ((x >> np.uint64(b)) & np.uint64(1)) << np.uint64(2 * b)
        out |= ((y >> np.uint64(b)) & np.uint64(1)) << np.uint64(2 * b + 1)
    return out


def fp64_peak_tflops() -> float:
    """Measured FP64 FMA throughput of the current device."""
    L = load_library()
    v = ctypes.c_double()
    rc = L.fdm_fp64_peak(ctypes.byref(v))
    if rc:
        raise FdmError(rc, "fdm_fp64_peak failed")
    return v.value
