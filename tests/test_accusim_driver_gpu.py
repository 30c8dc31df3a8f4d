"""The plug-ins inside accusim's own driver (accusim/simulation.py:95-112 Simulation.run, accusim/accuracy.py
AccuracyReport, accusim/io.py, accusim/analysis.py msd), and the device-resident `GpuSystem`.

Tolerances: a GpuSystem run and a run on accusim's plain System take the same kernels in the same order, so
their trajectories are bit-identical; the FP64 plug-in trajectory against the reference's own run to 1e-9 (the
device FP64 forces differ from NumPy's at round-off, tests/test_dropin_gpu.py)."""
import numpy as np
import pytest

from tests._helpers import rel_max
from tests.test_dropin_gpu import product_system

pytestmark = pytest.mark.gpu


def test_gpu_system_run_is_bit_identical_to_host_system_run(golden):
    """60 VelocityVerlet steps of the 864-atom argon case in accusim.Simulation.run: on a GpuSystem (state kept
    on the device between records) and on accusim's System (state copied every step) the records and the final
    state are identical bit for bit, and both follow the reference's own run."""
    import accusim

    from devinproj_b200 import GpuSystem, LennardJones, VelocityVerlet
    g = golden("argon864")
    out = {}
    for kind in ("host", "resident"):
        s = product_system(g, "0")
        if kind == "resident":
            s = GpuSystem.from_system(s)
        lj = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
        sim = accusim.Simulation(s, [lj], integrator=VelocityVerlet(), dt=float(g["dt"]))
        tr = sim.run(steps=int(g["steps"]), record_every=10, positions=True)
        out[kind] = (np.array(tr.kinetic), np.array(tr.potential), np.array(tr.momentum), s.pos.copy(), s.vel.copy(),
                     sim.force.copy(), sim.acc.copy(), lj.rebuilds, np.array(tr.positions))
    for a, b in zip(out["host"], out["resident"]):
        assert np.array_equal(a, b)
    assert rel_max(out["resident"][0], g["kinetic"][::10]) <= 1e-9
    d = out["resident"][3] - g["pos"]
    d -= g["box"] * np.round(d / g["box"])
    assert np.max(np.abs(d)) <= 1e-9 * g["box"][0]


def test_gpu_system_stays_on_the_device_between_records():
    """Inside Simulation.run with record_every = k the host arrays are read only at records: between them the
    device copy is authoritative, and the first host read brings back positions, velocities, forces and
    accelerations that equal a fresh FP64 evaluation."""
    import accusim

    from devinproj_b200 import GpuSystem, VelocityVerlet, configs
    s, forces, dt = configs.argon864(seed=2, gpu=True)
    assert isinstance(s, GpuSystem)
    sim = accusim.Simulation(s, forces, integrator=VelocityVerlet(), dt=dt)
    sim.run(steps=10, record_every=10, positions=False)
    sim.integrator.step(sim, dt)                   # one more step outside the recorder
    assert s._where == "device"
    F, U = forces[0].compute(s)                    # the force plug-in reads the resident copy
    assert s._where == "device"
    pos = s.pos                                    # first host read: synchronise
    assert s._where == "host"
    assert np.all((pos >= 0) & (pos < s.box))
    assert np.array_equal(sim.force, F) and sim.pe == U
    assert np.array_equal(sim.acc, F / s.masses[:, None])


def test_accuracy_report_rows_from_accusim_with_gpu_plugins(golden):
    """accusim's own AccuracyReport over a run of the GPU plug-ins on the 512-ion NaCl melt: its isinstance checks
    see the plug-ins (the 'DSF vs Ewald' row needs a DampedShiftedCoulomb, accusim/accuracy.py:149; the
    timescale row reads LennardJones._tables, accusim/advisor.py:36), and their values equal the reference
    report's to 1e-6."""
    import accusim

    from devinproj_b200 import DampedShiftedCoulomb, GpuSystem, LennardJones, VelocityVerlet
    g = golden("report_nacl512")
    s = GpuSystem.from_system(product_system(g))
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    forces = [LennardJones(params, cutoff=2.5), DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]))]
    sim = accusim.Simulation(s, forces, integrator=VelocityVerlet(), dt=float(g["dt"]))
    sim.run(steps=int(g["steps"]), record_every=1, positions=False)
    rep = {c.name: c for c in accusim.AccuracyReport.build(sim).checks}
    ref = {str(n): (str(st), float(v)) for n, st, v in zip(g["names"], g["statuses"], g["values"])}
    for name in ("DSF vs Ewald", "timestep vs physics", "energy"):
        assert rep[name].status == ref[name][0], name
        assert rep[name].value == pytest.approx(ref[name][1], rel=1e-6), name


def test_gpu_simulation_trajectory_through_accusim_io_and_msd(tmp_path):
    """A GpuSimulation trajectory is an accusim Trajectory: accusim.io saves and loads it unchanged, and
    accusim.analysis.msd reads it (same values before and after the round trip)."""
    from accusim import io
    from accusim.analysis import msd

    from devinproj_b200 import GpuSimulation, configs
    s, forces, dt = configs.argon864(seed=1)
    sim = GpuSimulation(s, forces, dt=dt)
    tr = sim.run(steps=40, record_every=10, positions=True)
    path = tmp_path / "traj.npz"
    io.save(tr, s, path)
    back, meta = io.load(path)
    assert [m["name"] for m in meta] == ["Ar"]
    assert np.array_equal(np.array(back.t), np.array(tr.t))
    assert np.array_equal(np.array(back.positions), np.array(tr.positions))
    assert np.array_equal(np.array(back.kinetic), np.array(tr.kinetic))
    t0, m0 = msd(tr, box=s.box)
    t1, m1 = msd(back, box=s.box)
    assert np.array_equal(t0, t1) and np.array_equal(m0, m1) and m0[-1] > 0
