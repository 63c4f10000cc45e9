"""Run parameters: the ctypes mirror of ``fdm_params`` (include/fdm.h) and
``set_parameter`` for the solver's workloads.

``set_parameter`` restates the reference's parameter routine
(src/MAIN.F90:29-71): the physical domain is padded by three ghost layers of
background cells, ``cv = 1/(gama (gama-1) Ma^2)``, and every value that the
Fortran writes as a default-REAL(4) literal (``gama = 1.4``, ``CFL = 0.45``,
``tstep = 1e-4``, the refine/coarsen goals 1.4 and 0.4) is passed as its
REAL(4) value promoted to REAL(8), which is what the Fortran computes with.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

BC_PERIODIC = 6       # BCcyc, src/module.F90:7
BC_TRANSMISSIVE = 2   # extension (no reference counterpart)
BC_WALL = 3           # extension
BC_INFLOW = 4         # extension
BC_DMR_BOTTOM = 5     # extension
BC_DMR_TOP = 7        # extension
BC_EXCHANGE = 8       # y side of a strip of the mesh: halo rows written by the caller

IC_VORTEX = 0         # src/solution.F90:31-69
IC_QUADRANTS = 1      # extension: four-quadrant Riemann problem
IC_OBLIQUE_SHOCK = 2  # extension: oblique shock (double Mach reflection)


def f32(x: float) -> float:
    """Value of a default-REAL(4) Fortran literal once promoted to REAL(8)."""
    return float(np.float32(x))


class FdmParams(ctypes.Structure):
    """Byte-for-byte mirror of ``struct fdm_params`` in include/fdm.h."""

    _fields_ = [
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
        ("ymin", ctypes.c_double), ("ymax", ctypes.c_double),
        ("h", ctypes.c_double), ("x_factor", ctypes.c_double),
        ("m", ctypes.c_int32), ("n", ctypes.c_int32),
        ("gama", ctypes.c_double), ("cv", ctypes.c_double), ("ma", ctypes.c_double),
        ("iflag_amr", ctypes.c_int32), ("lvl_amr", ctypes.c_int32),
        ("lvl_max", ctypes.c_int32), ("nstep_adapt", ctypes.c_int32),
        ("pstep_adapt", ctypes.c_int32),
        ("refine_goal_rot", ctypes.c_double), ("refine_goal_div", ctypes.c_double),
        ("coarse_goal_rot", ctypes.c_double), ("coarse_goal_div", ctypes.c_double),
        ("kind_xpbc", ctypes.c_int32), ("kind_xmbc", ctypes.c_int32),
        ("kind_ypbc", ctypes.c_int32), ("kind_ymbc", ctypes.c_int32),
        ("iflag_localdt", ctypes.c_int32),
        ("cfl", ctypes.c_double), ("tstep", ctypes.c_double), ("t_end", ctypes.c_double),
        ("bc_state", (ctypes.c_double * 4) * 4),
        ("dmr_x0", ctypes.c_double),
        ("dmr_post", ctypes.c_double * 4), ("dmr_pre", ctypes.c_double * 4),
        ("dmr_shock_speed", ctypes.c_double), ("dmr_angle_cot", ctypes.c_double),
        ("flux_variant", ctypes.c_int32),
        ("window_row0", ctypes.c_int32), ("window_rows", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 5),
    ]


@dataclass
class Config:
    """A workload: parameters, initial condition and step budget."""

    name: str
    params: FdmParams
    ic_kind: int
    ic_params: list = field(default_factory=list)
    max_steps: int = 10 ** 9
    # static block refinement of creat_mesh (src/mesh.F90:41-44):
    # (lvlBlock, Block_size(1:4) as set_parameter leaves it, BufferLayerLVL)
    block: tuple | None = None

    @property
    def m(self) -> int:
        return int(self.params.m)

    @property
    def n(self) -> int:
        return int(self.params.n)


def set_parameter(xmin: float, xmax: float, ymin: float, ymax: float, h: float, *,
                  gama: float = f32(1.4), x_factor: float = 1.0,
                  iflag_amr: bool = False, lvl_amr: int = 0, lvl_max: int = 0,
                  nstep_adapt: int = 0, pstep_adapt: int = 30,
                  refine_goal: float = f32(1.4), coarse_goal: float = f32(0.4),
                  bc=(BC_PERIODIC,) * 4, iflag_localdt: bool = False,
                  cfl: float = f32(0.45), tstep: float = f32(1e-4),
                  t_end: float = 10.0, ma: float = 1.0) -> FdmParams:
    """Restatement of set_parameter (src/MAIN.F90:29-71).

    ``bc`` = (kind_xmbc, kind_xpbc, kind_ymbc, kind_ypbc).
    """
    p = FdmParams()
    p.h = h
    p.x_factor = x_factor
    # ghost padding, src/MAIN.F90:55-56
    p.xmin = xmin - 3.0 * x_factor * h
    p.xmax = xmax + 3.0 * x_factor * h + 1.0e-10
    p.ymin = ymin - 3.0 * h
    p.ymax = ymax + 3.0 * h + 1.0e-10
    # background grid size, src/mesh.F90:15 (integer truncation)
    p.m = int((p.xmax - p.xmin) / (x_factor * h))
    p.n = int((p.ymax - p.ymin) / h)
    p.gama = gama
    p.ma = ma
    p.cv = 1.0 / (gama * (gama - 1.0) * ma * ma)
    p.iflag_amr = int(bool(iflag_amr))
    p.lvl_amr = lvl_amr
    p.lvl_max = lvl_max
    p.nstep_adapt = nstep_adapt
    p.pstep_adapt = pstep_adapt
    p.refine_goal_rot = refine_goal
    p.refine_goal_div = refine_goal
    p.coarse_goal_rot = coarse_goal
    p.coarse_goal_div = coarse_goal
    p.kind_xmbc, p.kind_xpbc, p.kind_ymbc, p.kind_ypbc = bc
    p.iflag_localdt = int(bool(iflag_localdt))
    p.cfl = cfl
    p.tstep = tstep
    p.t_end = t_end
    p.flux_variant = 0
    return p


def with_block(cfg: Config, lvlblock: int, block_size, buffer_layer_lvl: int = 0) -> Config:
    """The configuration with creat_mesh's static block refinement
    (Block_refine, src/mesh.F90:49-79): cells inside the box
    Block_size = (x1, x2, y1, y2) refined to lvlBlock, cells within
    BufferLayerLVL*h/2**(i-1) of it to level i, then lvlBlock-1 passes of the
    2:1 gridmodify.  set_parameter adds 1e-10 to the upper bounds
    (src/MAIN.F90:57)."""
    b = [float(v) for v in block_size]
    b[1] = b[1] + 1.0e-10
    b[3] = b[3] + 1.0e-10
    cfg.block = (int(lvlblock), tuple(b), int(buffer_layer_lvl))
    return cfg


def config_to_dict(cfg: Config) -> dict:
    """A configuration as plain data (JSON): every fdm_params field, the
    initial condition and the block refinement.  Floats keep every bit
    (JSON writes the shortest repr that reads back to the same double)."""
    p = cfg.params
    params = {}
    for name, ctype in FdmParams._fields_:
        v = getattr(p, name)
        if hasattr(ctype, "_length_"):
            params[name] = [list(r) if hasattr(r, "_length_") else r for r in v]
        else:
            params[name] = v
    return {"name": cfg.name, "ic_kind": int(cfg.ic_kind), "ic_params": [float(x) for x in cfg.ic_params],
            "max_steps": int(cfg.max_steps),
            "block": None if not cfg.block else [cfg.block[0], list(cfg.block[1]), cfg.block[2]],
            "params": params}


def config_from_dict(d: dict) -> Config:
    """The inverse of config_to_dict; fields left out keep their zero."""
    p = FdmParams()
    for name, ctype in FdmParams._fields_:
        if name not in d["params"]:
            continue
        v = d["params"][name]
        if hasattr(ctype, "_length_"):
            arr = getattr(p, name)
            for i, x in enumerate(v):
                if hasattr(arr[i], "_length_"):
                    for j, y in enumerate(x):
                        arr[i][j] = y
                else:
                    arr[i] = x
        else:
            setattr(p, name, v)
    cfg = Config(d["name"], p, int(d["ic_kind"]), list(d.get("ic_params", [])), int(d.get("max_steps", 10 ** 9)))
    if d.get("block"):
        lvl, box, buf = d["block"]
        cfg.block = (int(lvl), tuple(float(x) for x in box), int(buf))
    return cfg


def reference_default() -> Config:
    """The parameter set the reference ships (src/MAIN.F90:36-50): uniform
    h = 0.5 vortex, AMR and CFL stepping off, tstep = 1e-4, t_end = 10."""
    p = set_parameter(0.0, 10.0, 0.0, 10.0, 0.5)
    return Config("reference_default", p, IC_VORTEX)


def vortex(base: int = 32, lvl_amr: int = 2, steps: int = 200) -> Config:
    """Isentropic vortex advection: [0,10]^2 periodic, base 32^2, 2 AMR levels,
    regrid every 10 steps, CFL 0.5, 200 RK3 steps."""
    p = set_parameter(0.0, 10.0, 0.0, 10.0, 10.0 / base, iflag_amr=lvl_amr > 0,
                      lvl_amr=lvl_amr, lvl_max=lvl_amr, nstep_adapt=0, pstep_adapt=10,
                      iflag_localdt=True, cfl=0.5, t_end=1.0e30)
    return Config(f"vortex{base}", p, IC_VORTEX, [], steps)


RIEMANN4_STATES = [  # NE, NW, SW, SE (rho, u, v, p)
    (1.5, 0.0, 0.0, 1.5),
    (0.5323, 1.206, 0.0, 0.3),
    (0.138, 1.206, 1.206, 0.029),
    (0.5323, 0.0, 1.206, 0.3),
]


def riemann4(base: int = 128, lvl_amr: int = 4, t_end: float = 0.3,
             states=RIEMANN4_STATES, pstep_adapt: int = 10) -> Config:
    """Four-quadrant Riemann problem on [0,1]^2, split at (0.5, 0.5),
    transmissive boundaries (extension)."""
    p = set_parameter(0.0, 1.0, 0.0, 1.0, 1.0 / base, iflag_amr=lvl_amr > 0,
                      lvl_amr=lvl_amr, lvl_max=lvl_amr, pstep_adapt=pstep_adapt,
                      bc=(BC_TRANSMISSIVE,) * 4, iflag_localdt=True, t_end=t_end)
    icp = [0.5, 0.5]
    for s in states:
        icp.extend(float(v) for v in s)
    return Config(f"riemann4_{base}_l{lvl_amr}", p, IC_QUADRANTS, icp)


def random_quadrant_states(seed: int):
    """rho, p ~ U[0.1, 2]; u, v ~ U[-1, 1] per quadrant (numpy default_rng)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(4):
        rho, p = rng.uniform(0.1, 2.0, size=2)
        u, v = rng.uniform(-1.0, 1.0, size=2)
        out.append((float(rho), float(u), float(v), float(p)))
    return out


def random_riemann4(seed: int, base: int = 128, lvl_amr: int | None = None,
                    t_end: float = 0.25) -> Config:
    """One ensemble member: random quadrant states; when lvl_amr is None the
    maximum level is drawn from U{2..5} with the same generator."""
    rng = np.random.default_rng(seed)
    if lvl_amr is None:
        lvl_amr = int(rng.integers(2, 6))
    cfg = riemann4(base, lvl_amr, t_end, random_quadrant_states(seed))
    cfg.name = f"random4_s{seed}_l{lvl_amr}"
    return cfg


def double_mach(base_y: int = 64, lvl_amr: int = 4, t_end: float = 0.2) -> Config:
    """Oblique Mach-10 shock at 60 degrees through (1/6, 0) on [0,4]x[0,1]
    hitting a reflecting wall at y = 0 for x > 1/6 (extension)."""
    h = 1.0 / base_y
    post = (8.0, 8.25 * math.cos(math.pi / 6.0), -8.25 * math.sin(math.pi / 6.0), 116.5)
    pre = (1.4, 0.0, 0.0, 1.0)
    p = set_parameter(0.0, 4.0, 0.0, 1.0, h, iflag_amr=lvl_amr > 0, lvl_amr=lvl_amr,
                      lvl_max=lvl_amr, pstep_adapt=5,
                      bc=(BC_INFLOW, BC_TRANSMISSIVE, BC_DMR_BOTTOM, BC_DMR_TOP),
                      iflag_localdt=True, t_end=t_end)
    for k in range(4):
        p.bc_state[0][k] = post[k]
        p.dmr_post[k] = post[k]
        p.dmr_pre[k] = pre[k]
    p.dmr_x0 = 1.0 / 6.0
    p.dmr_angle_cot = 1.0 / math.sqrt(3.0)
    p.dmr_shock_speed = 20.0 / math.sqrt(3.0)
    return Config(f"double_mach_{base_y}_l{lvl_amr}", p, IC_OBLIQUE_SHOCK,
                  [1.0 / 6.0, 1.0 / math.sqrt(3.0)])


CONFIGS = {
    "reference_default": reference_default,
    "vortex": vortex,
    "riemann4": riemann4,
    "double_mach": double_mach,
}
