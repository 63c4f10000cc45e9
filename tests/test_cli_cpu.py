"""The command-line run's options map to the reference's configurations (no
GPU needed: only the parameter sets are built)."""
import argparse

from fdm_cell_based_amr_cartesian_b200.__main__ import config


def _args(**kw):
    base = dict(case="riemann4", base=128, lvl_amr=4, t_end=0.0, steps=0, gate=False, block=None, config=None)
    base.update(kw)
    return argparse.Namespace(**base)


def test_cli_configurations():
    c = config(_args())
    assert (c.m, c.n) == (134, 134)   # 128 + 3 ghost layers each side
    assert c.params.t_end == 0.3 and int(c.params.lvl_amr) == 4
    c = config(_args(case="riemann4", base=64, lvl_amr=3, t_end=0.1))
    assert c.params.t_end == 0.1 and int(c.params.lvl_amr) == 3
    c = config(_args(case="vortex", base=32, lvl_amr=2))
    assert int(c.params.lvl_amr) == 2
    c = config(_args(case="double_mach", base=16, lvl_amr=2))
    assert c.params.t_end == 0.2
    c = config(_args(case="reference"))
    assert c.name == "reference_default"


def test_cli_block_option():
    c = config(_args(case="vortex", base=32, lvl_amr=2, block=["2", "2.5", "7.5", "2.5", "7.5", "2"]))
    assert c.block == (2, (2.5, 7.5 + 1e-10, 2.5, 7.5 + 1e-10), 2)
    assert config(_args()).block is None


def test_cli_vortex_end_time():
    assert config(_args(case="vortex", base=32, lvl_amr=2, t_end=0.5)).params.t_end == 0.5


def test_cli_strips_refuse_periodic_y():
    import pytest
    from fdm_cell_based_amr_cartesian_b200.__main__ import run_strips
    args = _args(case="vortex", base=32, lvl_amr=2)
    args.strips = 2
    with pytest.raises(SystemExit):
        run_strips(args, config(args))


def test_configuration_files_round_trip(tmp_path):
    """Every named configuration written as JSON and read back gives the
    same fdm_params bytes, initial condition and block refinement."""
    from fdm_cell_based_amr_cartesian_b200 import params as P
    from fdm_cell_based_amr_cartesian_b200.__main__ import main
    cfgs = [P.vortex(), P.riemann4(base=64, lvl_amr=3), P.double_mach(base_y=32, lvl_amr=3),
            P.reference_default(), P.random_riemann4(1007, base=64),
            P.with_block(P.vortex(), 2, (2.5, 7.5, 2.5, 7.5), 2)]
    for c in cfgs:
        d = P.config_from_dict(P.config_to_dict(c))
        assert bytes(d.params) == bytes(c.params) and d.name == c.name
        assert d.ic_kind == c.ic_kind and d.ic_params == list(c.ic_params) and d.block == c.block
    path = str(tmp_path / "c.json")
    assert main(["--case", "double_mach", "--base", "32", "--lvl-amr", "3", "--save-config", path]) == 0
    c = config(_args(config=path))
    assert bytes(c.params) == bytes(P.double_mach(base_y=32, lvl_amr=3).params)


def test_config_file_refuses_configuration_options(tmp_path):
    """--config FILE fixes the configuration: --case/--base/--lvl-amr/--t-end/
    --block beside it are refused with a message, not silently ignored."""
    import pytest
    from fdm_cell_based_amr_cartesian_b200.__main__ import main
    path = str(tmp_path / "c.json")
    assert main(["--case", "vortex", "--base", "32", "--lvl-amr", "2", "--save-config", path]) == 0
    for extra in (["--base", "64"], ["--lvl-amr=3"], ["--t-end", "0.1"], ["--case", "riemann4"],
                  ["--block", "2", "2.5", "7.5", "2.5", "7.5", "2"]):
        with pytest.raises(SystemExit) as ei:
            main(["--config", path, *extra])
        assert ei.value.code == 2
    # the file alone, with --save-config, is accepted and round-trips
    path2 = str(tmp_path / "d.json")
    assert main(["--config", path, "--save-config", path2]) == 0
    assert open(path).read() == open(path2).read()
