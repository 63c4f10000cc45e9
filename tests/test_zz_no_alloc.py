"""The no-allocation entry point fdm_time_advance_rk_uniform_static.

It serves callers that cannot allocate device memory (a host whose GPU heap
belongs to its own runtime, or one that runs under a budget fixed at
start-up): its scratch is a static device array inside libfdm.  This test
calls it through the C-ABI on device buffers the test owns and checks it
against the handle path (fdm_time_advance_rk on the same uniform periodic
grid) for two calls in a row.  It is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.solver import Solver, initial_state, load_library, root_keys

pytestmark = pytest.mark.gpu

REL = 1e-12   # the per-step tolerance of the parity tests


def test_uniform_static_matches_handle_path():
    import torch

    cfg = P.vortex(lvl_amr=0)             # 32 x 32 interior, periodic, no AMR
    p = cfg.params
    nx, ny = cfg.m - 6, cfg.n - 6
    keys = root_keys(cfg.m, cfg.n)
    g = Solver(cfg)
    g.upload(keys, initial_state(cfg, keys))
    g.body_boundary(1)                     # periodic ghosts of the initial state
    _, u0 = g.leaves()
    r, u, v, pr = u0[:, 0], u0[:, 1], u0[:, 2], u0[:, 3]
    c = np.sqrt(p.gama * pr / r)
    lx, ly = float(np.max(np.abs(u) + c)), float(np.max(np.abs(v) + c))
    dt = 0.01
    g.set_scalars(lx, ly, dt, 0.0, 0)

    L = load_library()
    fn = L.fdm_time_advance_rk_uniform_static
    dev = torch.device("cuda", 0)
    cur = torch.tensor(u0, dtype=torch.float64, device=dev).contiguous()
    for call in range(2):
        out = torch.empty_like(cur)
        stream = torch.cuda.current_stream(dev)
        rc = fn(cur.data_ptr(), out.data_ptr(), nx, ny, p.h, p.x_factor, p.gama, lx, ly, dt,
                ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize(dev)
        g.time_advance_rk(dt)              # the existing entry point
        _, ref = g.leaves()
        got = out.cpu().numpy()
        err = float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-14)))
        assert err <= REL, f"call {call}: max relative difference {err:.3e}"
        cur = out


def test_uniform_static_rejects_sizes_beyond_the_limit():
    L = load_library()
    fn = L.fdm_time_advance_rk_uniform_static
    import torch
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    # 300 x 300 exceeds FDM_STATIC_MAX_CELLS; 2 x 8 is below the minimum side
    for nx, ny in ((300, 300), (2, 8), (2000, 16)):
        assert fn(buf.data_ptr(), buf.data_ptr() + 64, nx, ny, 0.1, 1.0, 1.4, 1.0, 1.0, 0.01, None) == 1


def test_uniform_static_rejects_overlapping_buffers():
    L = load_library()
    fn = L.fdm_time_advance_rk_uniform_static
    import torch
    nx = ny = 3
    ngrid = (nx + 6) * (ny + 6)
    buf = torch.zeros(2 * ngrid * 4, dtype=torch.float64, device="cuda")
    base = buf.data_ptr()
    # out starts inside in, and in starts inside out: nothing is enqueued
    for a, b in ((base, base + 32 * 40), (base + 32 * 40, base), (base, base)):
        assert fn(a, b, nx, ny, 0.1, 1.0, 1.4, 1.0, 1.0, 0.01, None) == 1
