"""One mesh split into horizontal strips of background rows, one solver per
strip, with the halo rows exchanged after every RK stage.

No reference counterpart: the reference advances its one tree in one OpenMP
process (src/solution.F90:267-298).  A strip holds its owned root rows plus
three rows on each side; on a side where the mesh is cut those three rows
are a halo that the owning neighbour's values overwrite after every stage
(pack -> send -> unpack).  The library places every strip at its global rows
(cell centres, neighbour classification), so each owned leaf is advanced by
the same arithmetic as in the whole mesh and the strips together reproduce
the whole-mesh run bit for bit.

Per step every strip makes the same calls in the same order:
  step_control (local lambda, l_max) -> max over strips -> step_control_global
  for krk = 1..3: solution_cells, update_rk, body_boundary(3), halo exchange
  tt + tstep, it + 1
The y sides that are cut must not be periodic and each strip owns at least
three rows.  With AMR on, the ghosts are refreshed after every step (and the
halos exchanged again), and a due regrid runs on a whole-mesh regrid host:
the strips' leaf values are gathered into it (without a table rebuild, so its
internal nodes keep the values the whole run gives them: they change only at
regrids), it regrids, and its new leaf set is split again (``StripRun``).

Engine: ``GpuStrip`` (a libfdm strip handle) with the regrid host
``GpuRegridHost``; any object with the same methods can stand in for them
(the tests drive the CPU restatement through this protocol).  Transports:
``LocalExchange`` (all strips in this process, e.g. on one GPU) and
``DistExchange`` (one strip per rank over torch.distributed: NCCL between
GPUs, gloo on CPU).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import params as P

HALO = 3          # ghost/halo rows of a strip side (the reference's ghost depth)


def key_rows(keys: np.ndarray, m: int) -> np.ndarray:
    """Root row (0-based) of every key."""
    return ((np.asarray(keys, np.uint64) >> np.uint64(34)) // np.uint64(m)).astype(np.int64)


def split_rows(keys: np.ndarray, m: int, n: int, nstrips: int) -> list[tuple[int, int]]:
    """Owned global row ranges [a, b) of nstrips strips covering the interior
    rows 3 .. n-4, contiguous, at least three rows each, balanced by the
    number of leaves per row."""
    rows = key_rows(keys, m)
    lo, hi = HALO, n - HALO
    if nstrips < 1 or (hi - lo) < HALO * nstrips:
        raise ValueError(f"{hi - lo} interior rows cannot hold {nstrips} strips of >= {HALO} rows")
    w = np.bincount(rows, minlength=n)[lo:hi].astype(np.float64)
    cum = np.concatenate([[0.0], np.cumsum(w)])
    cuts = [lo]
    for s in range(1, nstrips):
        target = cum[-1] * s / nstrips
        r = lo + int(np.searchsorted(cum, target))
        r = max(r, cuts[-1] + HALO)                      # this strip >= 3 rows
        r = min(r, hi - HALO * (nstrips - s))            # room for the rest
        cuts.append(r)
    cuts.append(hi)
    return [(cuts[s], cuts[s + 1]) for s in range(nstrips)]


@dataclass
class Strip:
    index: int
    own: tuple[int, int]          # owned global rows [a, b)
    row0: int                     # global row of local row 0
    rows: int                     # rows held (owned + 3 + 3)
    params: P.FdmParams
    sel: np.ndarray               # positions of the strip's leaves in the global key order
    keys: np.ndarray              # local keys (root relative to row0)
    # leaf ranges (positions in the strip's key order) sent to / received
    # from the strip below (index - 1) and above (index + 1)
    send_down: tuple[int, int] = (0, 0)
    send_up: tuple[int, int] = (0, 0)
    recv_down: tuple[int, int] = (0, 0)
    recv_up: tuple[int, int] = (0, 0)
    # leaves this strip reports in a gathered mesh: owned rows, plus the
    # mesh's own ghost rows at the bottom / top strip
    report: tuple[int, int] = (0, 0)


class StripPlan:
    """The strips of one mesh: windows, parameters, leaves and halo ranges."""

    def __init__(self, cfg: P.Config, keys: np.ndarray, nstrips: int):
        p = cfg.params
        if p.window_rows:
            raise ValueError("the configuration is already a strip")
        if nstrips > 1 and (p.kind_ymbc == P.BC_PERIODIC or p.kind_ypbc == P.BC_PERIODIC):
            raise ValueError("periodic y sides cannot be cut: the image of a ghost lies in another strip")
        self.cfg = cfg
        self.m, self.n = cfg.m, cfg.n
        keys = np.ascontiguousarray(keys, np.uint64)
        if np.any(keys[1:] <= keys[:-1]):
            raise ValueError("keys must be sorted and unique")
        self.keys = keys
        rows = key_rows(keys, self.m)
        self.strips: list[Strip] = []
        ranges = split_rows(keys, self.m, self.n, nstrips)
        for s, (a, b) in enumerate(ranges):
            row0, rows_held = a - HALO, (b - a) + 2 * HALO
            q = P.FdmParams.from_buffer_copy(p)
            if nstrips > 1:
                q.window_row0, q.window_rows = row0, rows_held
                if s > 0:
                    q.kind_ymbc = P.BC_EXCHANGE
                if s < nstrips - 1:
                    q.kind_ypbc = P.BC_EXCHANGE
            i0, i1 = np.searchsorted(rows, [row0, row0 + rows_held])
            sel = np.arange(i0, i1)
            shift = np.uint64((row0 * self.m) << 34) if nstrips > 1 else np.uint64(0)
            st = Strip(s, (a, b), row0, rows_held, q, sel, keys[i0:i1] - shift)
            lr = rows[i0:i1]

            def rng(r_lo, r_hi, lr=lr):
                j0, j1 = np.searchsorted(lr, [r_lo, r_hi])
                return int(j0), int(j1)

            st.send_down = rng(a, a + HALO)
            st.send_up = rng(b - HALO, b)
            st.recv_down = rng(a - HALO, a)
            st.recv_up = rng(b, b + HALO)
            st.report = rng(0 if s == 0 else a, self.n if s == nstrips - 1 else b)
            self.strips.append(st)
        for lo_s, hi_s in zip(self.strips[:-1], self.strips[1:]):
            # the same global leaves on both sides of every transfer
            assert hi_s.recv_down[1] - hi_s.recv_down[0] == lo_s.send_up[1] - lo_s.send_up[0]
            assert lo_s.recv_up[1] - lo_s.recv_up[0] == hi_s.send_down[1] - hi_s.send_down[0]
        cover = np.concatenate([st.sel[st.report[0]:st.report[1]] for st in self.strips])
        assert np.array_equal(cover, np.arange(len(keys))), "strips do not tile the mesh"

    def config(self, s: int) -> P.Config:
        c = self.cfg
        return P.Config(f"{c.name}_strip{s}", self.strips[s].params, c.ic_kind, list(c.ic_params), c.max_steps)

    def gather(self, parts) -> tuple[np.ndarray, np.ndarray]:
        """The whole mesh's (keys, values) from every strip's (local keys,
        values), each strip contributing the rows it owns."""
        ks, vs = [], []
        for st, (k, v) in zip(self.strips, parts):
            a, b = st.report
            shift = np.uint64((st.row0 * self.m) << 34) if len(self.strips) > 1 else np.uint64(0)
            ks.append(np.asarray(k, np.uint64)[a:b] + shift)
            vs.append(np.asarray(v)[a:b])
        return np.concatenate(ks), np.concatenate(vs)


# ------------------------------------------------------------------ engines
class GpuStrip:
    """A libfdm handle holding one strip on the current CUDA device.

    asynchronous=True: the stage calls and halo copies only enqueue on the
    handle's stream (``self.stream``); the exchange orders the strips with
    CUDA events.  The halo buffers live as long as the strip, so no copy in
    flight ever reads memory that was handed back."""

    width = 4   # (rho, u, v, p) per leaf

    def __init__(self, plan: StripPlan, s: int, values: np.ndarray, asynchronous: bool = False):
        import torch
        from .solver import Solver
        st = plan.strips[s]
        self.strip = st
        self.g = Solver(plan.config(s))
        self.g.upload(st.keys, np.ascontiguousarray(values[st.sel], np.float64))
        slots = self.g.leaf_slots()
        dev = torch.device("cuda", torch.cuda.current_device())
        self._slots = {name: torch.from_numpy(slots[r[0]:r[1]].copy()).to(dev)
                       for name, r in (("send_down", st.send_down), ("send_up", st.send_up),
                                       ("recv_down", st.recv_down), ("recv_up", st.recv_up))}
        self._bufs = {name: torch.empty((len(sl), 4), dtype=torch.float64, device=dev)
                      for name, sl in self._slots.items()}
        torch.cuda.synchronize(dev)
        self.device = dev
        self.stream = None
        if asynchronous:
            self.g.set_async(True)
            self.stream = torch.cuda.ExternalStream(self.g.device_state()[0], device=dev)

    def step_control(self):
        _, lx, ly, lm = self.g.step_control_info()
        return lx, ly, lm

    def step_control_global(self, lx, ly, lm):
        return self.g.step_control_global(lx, ly, lm)

    def stage(self, krk: int):
        self.g.solution_cells(krk)
        self.g.update_rk(krk)
        self.g.body_boundary(3)

    def buffer(self, name: str):
        return self._bufs[name]

    def pack(self, name: str, buf):
        sl = self._slots[name]
        if len(sl):
            self.g.pack_slots(sl.data_ptr(), len(sl), buf.data_ptr())

    def unpack(self, name: str, buf):
        sl = self._slots[name]
        if len(sl):
            self.g.unpack_slots(sl.data_ptr(), len(sl), buf.data_ptr())

    def end_step(self, lx, ly, tstep, tt, it):
        self.g.set_scalars(lx, ly, tstep, tt, it)

    def body_boundary(self, j: int):
        self.g.body_boundary(j)

    def leaves(self):
        return self.g.leaves()

    def values(self):
        return self.g.leaves()[1]

    def close(self):
        self.g.close()


class GpuRegridHost:
    """The whole mesh in one libfdm handle, used only at regrids.  It holds
    the mesh from the start of the run, so its internal nodes carry the
    values the whole run gives them (set at refinement / coarsening,
    src/mesh.F90:199-260, 397-408)."""

    def __init__(self, cfg: P.Config, keys: np.ndarray, values: np.ndarray):
        from .solver import Solver
        self.g = Solver(cfg)
        self.g.upload(keys, values)
        self.keys = np.asarray(keys, np.uint64)

    def regrid(self, keys, values, lx, ly, tstep, tt, it):
        if not np.array_equal(keys, self.keys):
            raise RuntimeError("the strips' leaf set differs from the regrid host's")
        self.g.set_values(values)                  # leaves only: no table rebuild
        self.g.set_scalars(lx, ly, tstep, tt, it)
        self.g.amr()
        self.g.body_boundary(1)
        self.keys, v = self.g.leaves()
        return self.keys, v

    def close(self):
        self.g.close()


# --------------------------------------------------------------- transports
class LocalExchange:
    """Every strip in this process: maxima by a loop, halos by buffer copies."""

    def __init__(self, engines):
        self.engines = engines

    def max3(self, vals):
        lx = max(v[0] for v in vals)
        ly = max(v[1] for v in vals)
        return lx, ly, max(v[2] for v in vals)

    def halos(self):
        e = self.engines
        if e and getattr(e[0], "stream", None) is not None:
            return self._halos_async()
        for lo, hi in zip(e[:-1], e[1:]):
            up = lo.buffer("send_up")
            lo.pack("send_up", up)
            hi.unpack("recv_down", up)
            down = hi.buffer("send_down")
            hi.pack("send_down", down)
            lo.unpack("recv_up", down)

    def _halos_async(self):
        """Every strip on its own stream: packs, an event per strip, the
        neighbours' unpacks after it, and a strip's next pack after the
        neighbours have read its buffers."""
        import torch
        e = self.engines
        pairs = list(zip(e[:-1], e[1:]))
        for lo, hi in pairs:
            lo.pack("send_up", lo.buffer("send_up"))
            hi.pack("send_down", hi.buffer("send_down"))
        packed = []
        for x in e:
            ev = torch.cuda.Event()
            ev.record(x.stream)
            packed.append(ev)
        for i, (lo, hi) in enumerate(pairs):
            hi.stream.wait_event(packed[i])
            hi.unpack("recv_down", lo.buffer("send_up"))
            lo.stream.wait_event(packed[i + 1])
            lo.unpack("recv_up", hi.buffer("send_down"))
        read = []
        for x in e:
            ev = torch.cuda.Event()
            ev.record(x.stream)
            read.append(ev)
        for i, (lo, hi) in enumerate(pairs):
            lo.stream.wait_event(read[i + 1])
            hi.stream.wait_event(read[i])


class DistExchange:
    """One strip per rank of the default torch.distributed group: the
    maxima by one all-reduce(max) of three values, the halos by paired
    send/recv with the neighbouring ranks (device buffers under NCCL)."""

    def __init__(self, engine, rank: int, world: int, device=None):
        import torch
        self.e = engine
        self.rank, self.world = rank, world
        self.device = device if device is not None else torch.device("cpu")

    def max3(self, vals):
        import torch
        import torch.distributed as dist
        (lx, ly, lm), = vals
        t = torch.tensor([lx, ly, float(lm)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t = t.cpu()
        return float(t[0]), float(t[1]), int(t[2])

    def _t(self, a):
        import torch
        return a if isinstance(a, torch.Tensor) else torch.from_numpy(a)

    def halos(self):
        import contextlib
        import torch
        # an asynchronous strip's copies are ordered on its own stream: the
        # transfers are issued on it and the waits make it (not the host)
        # wait for them, so its next pack cannot overwrite a buffer in flight
        st = getattr(self.e, "stream", None)
        with torch.cuda.stream(st) if st is not None else contextlib.nullcontext():
            self._halos()

    def _halos(self):
        import torch.distributed as dist
        e, r = self.e, self.rank
        ops, recvs = [], []
        if r + 1 < self.world:
            up = e.buffer("send_up")
            e.pack("send_up", up)
            rup = e.buffer("recv_up")
            ops += [dist.P2POp(dist.isend, self._t(up), r + 1), dist.P2POp(dist.irecv, self._t(rup), r + 1)]
            recvs.append(("recv_up", rup))
        if r > 0:
            down = e.buffer("send_down")
            e.pack("send_down", down)
            rdown = e.buffer("recv_down")
            ops += [dist.P2POp(dist.isend, self._t(down), r - 1), dist.P2POp(dist.irecv, self._t(rdown), r - 1)]
            recvs.append(("recv_down", rdown))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            # device buffers of a synchronous strip: the waits above only
            # hold torch's current stream, and the unpack runs on the
            # handle's own stream, so the host waits for the transfers
            if getattr(e, "stream", None) is None and any(
                    getattr(b, "is_cuda", False) for _, b in recvs):
                import torch
                torch.cuda.current_stream().synchronize()
        for name, buf in recvs:
            e.unpack(name, buf)


def step(engines, xchg, tt: float, it: int):
    """The RK3 step of one solute iteration on the strips (step control,
    three stages with the halo exchange, tt and it); returns the new
    (tt, it, tstep, lambda_x, lambda_y).  ``engines`` are this process's
    strips."""
    lx, ly, lm = xchg.max3([e.step_control() for e in engines])
    dts = [e.step_control_global(lx, ly, lm) for e in engines]
    tstep = dts[0]
    assert all(d == tstep for d in dts)
    for krk in (1, 2, 3):
        for e in engines:
            e.stage(krk)
        xchg.halos()
    tt = tt + tstep
    it = it + 1
    for e in engines:
        e.end_step(lx, ly, tstep, tt, it)
    return tt, it, tstep, lx, ly


def run(engines, xchg, nsteps: int, t_end: float, tt: float = 0.0, it: int = 0):
    """Up to nsteps RK3 steps on a fixed mesh, stopping at t_end
    (src/solution.F90:182); no ghost refresh or regrid between steps."""
    k = 0
    while k < nsteps and tt < t_end:
        tt, it, *_ = step(engines, xchg, tt, it)
        k += 1
    return tt, it, k


def amr_due(p: P.FdmParams, it: int) -> bool:
    """The regrid trigger of solute (it >= Nstep_Adapt, mod(it, Pstep_Adapt) == 1)."""
    return bool(p.iflag_amr) and it >= p.nstep_adapt and p.pstep_adapt != 0 and it % p.pstep_adapt == 1


class StripRun:
    """The time loop of solute (src/solution.F90:182-236, without file
    output) on strips: the RK3 step with halo exchanges, then with AMR on the
    ghost refresh of body_boundary_RK(1) and, when due, the regrid on the
    regrid host and a new split.

    make_engine(plan, s, values) builds strip s; make_host(keys, values)
    builds the regrid host (called on rank 0 only when ``comm`` is a
    torch.distributed world of one strip per rank; ``rank`` then names this
    process's strip)."""

    def __init__(self, cfg, keys, values, nstrips, make_engine, make_host=None, rank=None, device=None):
        self.cfg = cfg
        self.nstrips = nstrips
        self.make_engine = make_engine
        self.rank = rank                 # None: every strip in this process
        self.device = device
        self.tt, self.it = 0.0, 0
        self.steps = 0
        self.regrids = 0
        self.host = None
        if cfg.params.iflag_amr and (rank is None or rank == 0):
            if make_host is None:
                raise ValueError("AMR is on: a regrid host is needed")
            self.host = make_host(keys, values)
        self._split(keys, values)

    def _split(self, keys, values, scalars=None):
        self.plan = StripPlan(self.cfg, keys, self.nstrips)
        mine = range(self.nstrips) if self.rank is None else [self.rank]
        self.engines = [self.make_engine(self.plan, s, values) for s in mine]
        if scalars is not None:
            for e in self.engines:
                e.end_step(*scalars)
        if self.rank is None:
            self.xchg = LocalExchange(self.engines)
        else:
            self.xchg = DistExchange(self.engines[0], self.rank, self.nstrips, self.device)

    def _regrid(self, lx, ly, tstep):
        parts = [(e.strip.keys, e.values()) for e in self.engines]
        scal = (lx, ly, tstep, self.tt, self.it)
        if self.rank is None:
            keys, vals = self.plan.gather(parts)
            nk, nv = self.host.regrid(keys, vals, *scal)
        else:
            import torch.distributed as dist
            got = [None] * self.nstrips if self.rank == 0 else None
            dist.gather_object(parts[0], got, dst=0)
            box = [None]
            if self.rank == 0:
                keys, vals = self.plan.gather(got)
                box = [self.host.regrid(keys, vals, *scal)]
            dist.broadcast_object_list(box, src=0)
            nk, nv = box[0]
        for e in self.engines:
            e.close()
        self._split(nk, nv, scal)
        self.regrids += 1

    def solute_step(self):
        self.tt, self.it, tstep, lx, ly = step(self.engines, self.xchg, self.tt, self.it)
        self.steps += 1
        if self.cfg.params.iflag_amr:
            if amr_due(self.cfg.params, self.it):
                self._regrid(lx, ly, tstep)
            else:
                for e in self.engines:
                    e.body_boundary(1)
                self.xchg.halos()

    def solute(self, nsteps: int) -> int:
        k = 0
        while k < nsteps and self.tt < self.cfg.params.t_end:
            self.solute_step()
            k += 1
        return k

    def gather(self):
        """The whole mesh's (keys, values) from this process's strips (all
        strips of a LocalExchange run; rank 0 gets them in a distributed run,
        the other ranks None)."""
        parts = [(e.strip.keys, e.values()) for e in self.engines]
        if self.rank is None:
            return self.plan.gather(parts)
        import torch.distributed as dist
        got = [None] * self.nstrips if self.rank == 0 else None
        dist.gather_object(parts[0], got, dst=0)
        return self.plan.gather(got) if self.rank == 0 else None

    def close(self):
        for e in self.engines:
            e.close()
        if self.host is not None:
            self.host.close()
