"""creat_mesh's static block refinement (Block_refine, src/mesh.F90:49-197):
the host generator of the package against the oracle's restatement of the
reference's pointer walk, leaf for leaf, and a few oracle steps on the
result."""
import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.mesh import block_refined_keys


def cases():
    return {
        # the reference's own box (src/MAIN.F90:45) on the vortex domain
        "vortex_box_l2": lambda: P.with_block(P.vortex(), 2, (2.5, 7.5, 2.5, 7.5), 2),
        "vortex_thin_box_l3": lambda: P.with_block(P.vortex(lvl_amr=3), 3, (4.0, 4.6, 2.0, 6.0), 3),
        "riemann4_l4": lambda: P.with_block(P.riemann4(base=32, lvl_amr=4), 4, (0.3, 0.55, 0.4, 0.45), 2),
        "double_mach_wall_l3": lambda: P.with_block(P.double_mach(base_y=16, lvl_amr=3), 3, (0.0, 0.5, 0.0, 0.2), 1),
        "no_buffer_l1": lambda: P.with_block(P.riemann4(base=32, lvl_amr=1), 1, (0.1, 0.2, 0.1, 0.9), 0),
    }


@pytest.mark.parametrize("name", sorted(cases()))
def test_generator_matches_oracle(oracle_mod, name):
    cfg = cases()[name]()
    keys = block_refined_keys(cfg)
    o = oracle_mod.Oracle(cfg, threads=2)
    ko, _, _ = o.leaves()
    o.close()
    assert np.array_equal(keys, ko)
    lvl = (keys & np.uint64(15)).astype(int)
    assert lvl.max() == cfg.block[0]


def test_no_block_is_the_root_grid():
    cfg = P.riemann4(base=32)
    keys = block_refined_keys(cfg)
    assert np.array_equal(keys, np.arange(cfg.m * cfg.n, dtype=np.uint64) << np.uint64(34))


def test_block_mesh_runs(oracle_mod):
    cfg = cases()["vortex_box_l2"]()
    o = oracle_mod.Oracle(cfg, threads=2)
    assert o.solute(3) == 3
    _, prim, _ = o.leaves()
    assert np.isfinite(prim).all() and prim[:, 0].min() > 0
    o.close()
