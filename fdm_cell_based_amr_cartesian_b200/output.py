"""The reference's diagnostic output (src/output_ADT.F90), on the host as in
the reference: output_Res (a console line and ./Output/Residual.dat) and
output_error (./Output/accuracy_error.dat: density error norms against the
isentropic vortex at its initial position).

Numbers are written with Fortran edit descriptors (Iw, Ew.d) so the files
read like the reference's.  The error norms follow output_error's loop over
cell_NS (interior leaves in key order): sequential sums, the vortex density
from the C library's exp and pow (as the Fortran's), Pi = 3.1415926535897932.
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import params as P

PI = 3.1415926535897932
PSTEP_RES = 100          # Pstep_Res of src/MAIN.F90:51


def fortran_i(v: int, w: int) -> str:
    """Iw: right-justified, all asterisks when it does not fit."""
    s = str(int(v))
    return s.rjust(w) if len(s) <= w else "*" * w


def fortran_e(x: float, w: int, d: int) -> str:
    """Ew.d: sign, 0., d digits, E+xx (or a three-digit exponent without
    the E), right-justified in w."""
    x = float(x)
    if math.isnan(x):
        return "NaN".rjust(w)
    if math.isinf(x):
        s = ("-" if x < 0 else "") + "Infinity"
        return s.rjust(w) if len(s) <= w else ("-Inf" if x < 0 else "Inf").rjust(w)
    if x == 0.0:
        digits, e = "0" * d, 0
    else:
        m = f"{abs(x):.{d - 1}e}"            # d significant digits, correctly rounded
        mant, ex = m.split("e")
        digits = mant.replace(".", "")
        e = int(ex) + 1
    ea = abs(e)
    exp = f"E{'+' if e >= 0 else '-'}{ea:02d}" if ea <= 99 else f"{'+' if e >= 0 else '-'}{ea:03d}"
    s = ("-" if x < 0 else "") + "0." + digits + exp
    if len(s) > w and s.startswith(("0.", "-0.")):
        s = s.replace("0.", ".", 1)          # the optional leading zero goes first
    return s.rjust(w) if len(s) <= w else "*" * w


def res_lines(it, n_res, tstep, tt, res_max, res_rms):
    """output_Res (src/output_ADT.F90:7-15): the console line (I8,I8,6E16.6)
    and the Residual.dat line (I8,I8,12E24.10)."""
    con = fortran_i(it, 8) + fortran_i(n_res, 8) + "".join(
        fortran_e(v, 16, 6) for v in [tstep, tt, *list(res_rms)[:4]])
    rec = fortran_i(it, 8) + fortran_i(n_res, 8) + "".join(
        fortran_e(v, 24, 10) for v in [tstep, tt, *list(res_max)[:4], *list(res_rms)[:4]])
    return con, rec


def error_norms(cfg: P.Config, keys, prim) -> dict:
    """The density error norms of output_error (src/output_ADT.F90:18-75)
    over the interior leaves: L1, L2, Loo over all of them and P1, P2, Poo
    over the refined ones (lvl /= 0), against the vortex of strength 5 at
    (5, 5).  Also the same norms over the level-0 leaves, which the second
    record of the file names but the reference never assigns."""
    from .solver import node_centers
    p = cfg.params
    keys = np.asarray(keys, np.uint64)
    root = (keys >> np.uint64(34)).astype(np.int64)
    row, col = root // p.m, root % p.m
    inter = (row >= 3) & (row < p.n - 3) & (col >= 3) & (col < p.m - 3)
    lvl = (keys & np.uint64(15)).astype(np.int64)
    cx, cy = node_centers(cfg, keys)
    g = p.gama
    cc1 = 5.0
    acc = {k: 0.0 for k in ("uni", "patch", "l1", "l2", "loo", "p1", "p2", "poo", "z", "z1", "z2", "zoo")}
    n0 = npatch = 0
    ios = False
    for i in np.nonzero(inter)[0]:
        dy = p.h / float(1 << int(lvl[i]))
        dx = p.x_factor * dy
        acc["uni"] = acc["uni"] + dx * dy
        rr = (cx[i] - 5.0) * (cx[i] - 5.0) + (cy[i] - 5.0) * (cy[i] - 5.0)
        dT = -(g - 1.0) * (cc1 * cc1) * math.exp(1.0 - rr) / (8.0 * g * PI * PI)
        r = float(prim[i, 0]) - math.pow(1.0 + dT, 1.0 / (g - 1.0))
        acc["l1"] = acc["l1"] + abs(r) * dx * dy
        acc["l2"] = acc["l2"] + r * r * dx * dy
        acc["loo"] = max(acc["loo"], abs(r))
        if lvl[i] != 0:
            ios = True
            npatch += 1
            acc["patch"] = acc["patch"] + dx * dy
            acc["p1"] = acc["p1"] + abs(r) * dx * dy
            acc["p2"] = acc["p2"] + r * r * dx * dy
            acc["poo"] = max(acc["poo"], abs(r))
        else:
            n0 += 1
            acc["z"] = acc["z"] + dx * dy
            acc["z1"] = acc["z1"] + abs(r) * dx * dy
            acc["z2"] = acc["z2"] + r * r * dx * dy
            acc["zoo"] = max(acc["zoo"], abs(r))
    out = dict(n_res=int(inter.sum()), L1_rho=acc["l1"] / acc["uni"], L2_rho=math.sqrt(acc["l2"] / acc["uni"]),
               Loo_rho=acc["loo"], P1_rho=0.0, P2_rho=0.0, Poo_rho=acc["poo"],
               n_0=n0, n_patch=npatch)
    if ios:
        out["P1_rho"] = acc["p1"] / acc["patch"]
        out["P2_rho"] = math.sqrt(acc["p2"] / acc["patch"])
    out["L1_rho0"] = acc["z1"] / acc["z"] if n0 else 0.0
    out["L2_rho0"] = math.sqrt(acc["z2"] / acc["z"]) if n0 else 0.0
    out["Loo_rho0"] = acc["zoo"]
    return out


def error_lines(it: int, e: dict, first: bool) -> list[str]:
    """The records output_error appends (src/output_ADT.F90:33-70)."""
    lines = []
    if first:
        lines.append(" nstep Ngrids L1_rho P1_rho L2_rho P2_rho Loo_rho Poo_rho ")
    lines.append(fortran_i(it, 8) + fortran_i(e["n_res"], 8) + "".join(
        fortran_e(e[k], 14, 6) for k in ("L1_rho", "P1_rho", "L2_rho", "P2_rho", "Loo_rho", "Poo_rho")))
    lines.append(fortran_i(it, 8) + fortran_i(e["n_res"], 8)
                 + "".join(fortran_e(e[k], 14, 6) for k in ("L1_rho", "L2_rho", "Loo_rho"))
                 + fortran_i(e["n_0"], 8)
                 + "".join(fortran_e(e[k], 14, 6) for k in ("L1_rho0", "L2_rho0", "Loo_rho0"))
                 + fortran_i(e["n_patch"], 8)
                 + "".join(fortran_e(e[k], 14, 6) for k in ("P1_rho", "P2_rho", "Poo_rho")))
    return lines


class Output:
    """The ./Output directory of a run: Residual.dat and accuracy_error.dat,
    appended as the reference appends them."""

    def __init__(self, directory: str = "Output"):
        self.dir = directory
        os.makedirs(directory, exist_ok=True)
        self._first_error = True

    def res(self, solver) -> str:
        """output_Res for a Solver; returns the console line."""
        sc = solver.scalars()
        rmax, rrms = solver.residual()
        con, rec = res_lines(sc["it"], solver.counters()["n_interior"], sc["tstep"], sc["tt"], rmax, rrms)
        with open(os.path.join(self.dir, "Residual.dat"), "a") as f:
            f.write(rec + "\n")
        return con

    def error(self, solver) -> dict:
        """output_error for a Solver (the vortex configurations): the norms
        are formed on the device (fdm_output_error), so no leaf crosses to
        the host."""
        e = solver.output_error_device()
        with open(os.path.join(self.dir, "accuracy_error.dat"), "a") as f:
            for line in error_lines(solver.scalars()["it"], e, self._first_error):
                f.write(line + "\n")
        self._first_error = False
        return e


class FieldDump:
    """Field dumps (no reference counterpart): the leaf keys and (rho, u, v,
    p) of a solver written as ``field_<it>.npz`` in ``directory``.  The
    read-back is queued on the solver's read-back stream into one of two
    pinned host buffers and a writer thread waits for it and writes the file,
    so the steps after a dump overlap its transfer and its file output.  A
    buffer is reused only after its file is written."""

    def __init__(self, directory: str):
        import threading
        self.dir = directory
        os.makedirs(directory, exist_ok=True)
        self._buf = [None, None]
        self._busy = [threading.Event(), threading.Event()]
        for e in self._busy:
            e.set()            # set: the buffer is free
        self._k = 0
        self._threads = []
        self.written = []

    def _pinned(self, b, n):
        import torch
        cur = self._buf[b]
        if cur is None or cur[0].shape[0] < n:
            keys = torch.empty(n, dtype=torch.int64, pin_memory=True)
            vals = torch.empty((n, 4), dtype=torch.float64, pin_memory=True)
            cur = (keys, vals)
            self._buf[b] = cur
        return cur

    def dump(self, solver):
        """Queue a dump of the solver's current leaves; returns at once."""
        import threading
        b = self._k % 2
        self._k += 1
        self._busy[b].wait()
        self._busy[b].clear()
        n = solver.num_leaves()
        kt, vt = self._pinned(b, n)
        keys = kt.numpy()[:n].view(np.uint64)
        vals = vt.numpy()[:n]
        solver.download_keys_async(keys)
        solver.download_values_async(vals)
        it = solver.scalars()["it"]
        path = os.path.join(self.dir, f"field_{it:08d}.npz")

        def write():
            solver.readback_wait()           # the read-back stream only
            np.savez(path, keys=keys.copy(), prim=vals.copy())
            self.written.append(path)
            self._busy[b].set()

        t = threading.Thread(target=write, daemon=True)
        t.start()
        self._threads.append(t)

    def close(self):
        for t in self._threads:
            t.join()
        self._threads = []
