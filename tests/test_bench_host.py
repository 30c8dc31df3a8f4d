"""Host logic of bench.py (no GPU): the JSON line's configuration labels, the secondary legs' error reporting,
the workload table, and the reference arm's fluid, which must be the state devinproj_b200.configs builds for the
same workload (the reference arm builds it with accusim's own API only)."""
import argparse

import numpy as np
import pytest

import bench


def _args(workload):
    return argparse.Namespace(workload=workload, record_every=100)


@pytest.mark.parametrize("world", [1, 4])
def test_config_labels(world):
    ens = bench.full_config(bench.workload_meta("ensemble"), _args("ensemble"), world)
    one = bench.full_config(bench.workload_meta("lj1m"), _args("lj1m"), world)
    if world == 1:
        assert ens["parallelism"] == "all replicas in one engine" and one["parallelism"] == "single system"
    else:
        assert ens["parallelism"] == f"replica shards x{world}"
        assert one["parallelism"] == f"independent replicas x{world}"
    assert one["l2"] == "inputs larger than L2" and one["atoms"] == 1048576 and one["record_every"] == 100
    assert bench.full_config(bench.workload_meta("argon864"), _args("argon864"), 1)["l2"].startswith("inputs resident")


def test_workload_table():
    for name in ("lj1m", "nacl4096", "argon864", "ensemble"):
        meta = bench.workload_meta(name)
        assert meta["workload"] and meta["atoms"] > 0
    with pytest.raises(SystemExit):
        bench.workload_meta("no_such_workload")


def test_secondary_leg_reports_errors():
    assert bench.secondary_leg(lambda x: {"value": x}, 3) == {"value": 3}

    def fails():
        raise RuntimeError("leg failed")

    out = bench.secondary_leg(fails)
    assert out == {"error": "RuntimeError: leg failed"}


def test_reference_fluid_is_the_workload_state():
    """bench.reference_lj_fluid (accusim's API only) and configs.lj_fluid give the same positions, velocities,
    masses, box and time step for the same seed."""
    from devinproj_b200 import configs
    accusim = bench.reference_package()
    sim = bench.reference_lj_fluid(accusim, 4, seed=3)
    s, lj = configs.lj_fluid(4, seed=3)
    assert np.array_equal(sim.system.pos, s.pos)
    assert np.array_equal(sim.system.vel, s.vel)
    assert np.allclose(sim.system.box, s.box, rtol=1e-15, atol=0)
    assert sim.system.species[0].mass == pytest.approx(s.species[0].mass, rel=1e-12)
    assert sim.dt == pytest.approx(0.005 * configs.AR_TAU, rel=1e-12)
    assert sim.forces[0].cutoff == lj.cutoff and sim.forces[0].skin == lj.skin
