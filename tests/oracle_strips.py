"""Strip engines and the regrid host backed by the oracle (the CPU
restatement): the checker side of the strip protocol in
fdm_cell_based_amr_cartesian_b200/strips.py, used only by the tests."""
import numpy as np

from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.strips import StripPlan


class OracleStrip:
    """The CPU restatement holding one strip (test infrastructure)."""

    width = 7   # U(1:7) per leaf

    def __init__(self, plan: StripPlan, s: int, values: np.ndarray, oracle_mod, threads=1):
        st = plan.strips[s]
        self.strip = st
        self.o = oracle_mod.Oracle(plan.config(s), threads=threads, initial=False)
        set_oracle_leaves(self.o, st.keys, values[st.sel])
        self._idx = {name: np.arange(*r, dtype=np.int64)
                     for name, r in (("send_down", st.send_down), ("send_up", st.send_up),
                                     ("recv_down", st.recv_down), ("recv_up", st.recv_up))}

    def step_control(self):
        self.o.step_control()
        sc = self.o.scalars()
        return sc["lambda_x"], sc["lambda_y"], sc["l_max"]

    def step_control_global(self, lx, ly, lm):
        return self.o.step_control_global(lx, ly, lm)

    def stage(self, krk: int):
        self.o.stage(krk)

    def buffer(self, name: str):
        return np.zeros((len(self._idx[name]), 7))

    def pack(self, name: str, buf):
        if len(self._idx[name]):
            buf[:] = self.o.get_U(self._idx[name])

    def unpack(self, name: str, buf):
        if len(self._idx[name]):
            self.o.set_U(self._idx[name], buf)

    def end_step(self, lx, ly, tstep, tt, it):
        self.o.set_scalars(lx, ly, tstep, tt, it)

    def body_boundary(self, j: int):
        self.o.body_boundary(j)

    def leaves(self):
        k, v, _ = self.o.leaves()
        return k, v

    def values(self):
        return self.o.get_U(np.arange(self.o.num_leaves()))

    def close(self):
        self.o.close()


def set_oracle_leaves(o, keys, values):
    """Leaves into an oracle instance from (rho, u, v, p) rows, or from full
    U(1:7) rows (which also carry T and the two unused slots)."""
    values = np.asarray(values, np.float64)
    if values.shape[1] == 7:
        o.set_leaves(keys, values[:, [0, 1, 2, 4]], values[:, 3])
        o.set_U(np.arange(len(keys)), values)
    else:
        o.set_leaves(keys, values)


class OracleRegridHost:
    """The CPU restatement's whole mesh, used only at regrids (tests)."""

    def __init__(self, cfg: P.Config, keys, values, oracle_mod, threads=1):
        self.o = oracle_mod.Oracle(cfg, threads=threads, initial=False)
        set_oracle_leaves(self.o, keys, values)
        self.keys = np.asarray(keys, np.uint64)

    def regrid(self, keys, values, lx, ly, tstep, tt, it):
        if not np.array_equal(keys, self.keys):
            raise RuntimeError("the strips' leaf set differs from the regrid host's")
        self.o.set_U(np.arange(len(keys)), values)  # leaves only
        self.o.set_scalars(lx, ly, tstep, tt, it)
        self.o.amr()                                # amr_core + body_boundary(1)
        self.keys = self.o.leaves()[0]
        return self.keys, self.o.get_U(np.arange(len(self.keys)))

    def close(self):
        self.o.close()
