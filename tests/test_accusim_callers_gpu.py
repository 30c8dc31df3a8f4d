"""The plug-ins under accusim's other callers of the force path, next to the reference's own NumPy forces on the
same systems:

* `analysis.pressure` (accusim/analysis.py:45-63) rescales the box and every position by (1 +- h)^(1/3) and calls
  `Force.compute` twice, so a plug-in that kept a neighbour list or cell grid across the box change would give a
  wrong dU/dV;
* `minimize` (accusim/minimize.py:11-47, FIRE) calls `Simulation.potential` every step after moving the host
  positions in place, and finishes with `update_forces`;
* `model.build` (accusim/model.py:102-135) makes a simulation from a JSON model with accusim's own classes, which
  `to_gpu` moves onto the plug-ins.

Each runs on accusim's plain `System` and on the device-resident `GpuSystem`. Tolerances: the FP64 plug-ins' forces
and energies differ from NumPy's at round-off (tests/test_dropin_gpu.py), which dU/dV's central difference with
h = 1e-6 lifts to about 1e-9 relative; FIRE's trajectory is damped, so 150 steps keep the positions within 1e-9 of
the box edge of the reference's."""
import numpy as np
import pytest

from tests.test_dropin_gpu import product_system

pytestmark = pytest.mark.gpu


def _pressures(make_system, make_forces_gpu, make_forces_ref, dt):
    import accusim
    from accusim import analysis

    from devinproj_b200 import GpuSystem
    ref = analysis.pressure(accusim.Simulation(make_system(), make_forces_ref(), dt=dt))
    out = {}
    for kind in ("host", "resident"):
        s = make_system()
        if kind == "resident":
            s = GpuSystem.from_system(s)
        sim = accusim.Simulation(s, make_forces_gpu(), dt=dt)
        box0, pos0 = s.box.copy(), s.pos.copy()
        out[kind] = analysis.pressure(sim)
        assert np.array_equal(s.box, box0) and np.array_equal(s.pos, pos0)   # pressure restores the state
        # the plug-ins see the restored box again: the energy equals a fresh evaluation on the original state
        U_after = sum(f.compute(s)[1] for f in sim.forces)
        U_ref = sum(f.compute(make_system())[1] for f in make_forces_ref())
        assert U_after == pytest.approx(U_ref, rel=1e-12)
    return ref, out


def test_pressure_lj_argon864(golden):
    import accusim

    from devinproj_b200 import LennardJones
    g = golden("argon864")
    params = {"Ar": (float(g["eps"]), float(g["sig"]))}
    ref, out = _pressures(lambda: product_system(g), lambda: [LennardJones(params, cutoff=2.5)],
                          lambda: [accusim.forces.LennardJones(params, cutoff=2.5)], float(g["dt"]))
    for kind, P in out.items():
        assert P == pytest.approx(ref, rel=1e-7), kind
    print(f"argon864 pressure {ref:.6e} Pa (reference forces), GPU plug-ins {out}")


def test_pressure_lj_dsf_nacl512(golden):
    import accusim

    from devinproj_b200 import DampedShiftedCoulomb, LennardJones
    g = golden("report_nacl512")
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    rc, al = float(g["rcut"]), float(g["alpha"])
    ref, out = _pressures(lambda: product_system(g),
                          lambda: [LennardJones(params, cutoff=2.5), DampedShiftedCoulomb(rcut=rc, alpha=al)],
                          lambda: [accusim.forces.LennardJones(params, cutoff=2.5),
                                   accusim.forces.DampedShiftedCoulomb(rcut=rc, alpha=al)], float(g["dt"]))
    for kind, P in out.items():
        assert P == pytest.approx(ref, rel=1e-7), kind
    print(f"nacl512 pressure {ref:.6e} Pa (reference forces), GPU plug-ins {out}")


def test_minimize_follows_the_reference_forces():
    """FIRE from a perturbed 500-atom argon lattice (the list path: N >= 400), 150 steps with the GPU LennardJones
    and with the reference's: the same energy, maximum force and positions."""
    import accusim
    from accusim.minimize import minimize

    from devinproj_b200 import GpuSystem, LennardJones, configs
    s0, _ = configs.lj_fluid(5, seed=3)
    rng = np.random.default_rng(3)
    s0.pos = (s0.pos + rng.normal(0.0, 0.08 * configs.AR_SIGMA, s0.pos.shape)) % s0.box
    params = {"Ar": (configs.AR_EPS, configs.AR_SIGMA)}
    dt = 5e-15
    s_ref = s0.copy()
    sim_ref = accusim.Simulation(s_ref, [accusim.forces.LennardJones(params, cutoff=2.5)], dt=dt)
    U0 = sim_ref.potential()[1]
    U_ref, f_ref, n_ref = minimize(sim_ref, max_steps=150)
    assert U_ref < U0
    for kind in ("host", "resident"):
        s = s0.copy()
        if kind == "resident":
            s = GpuSystem.from_system(s)
        sim = accusim.Simulation(s, [LennardJones(params, cutoff=2.5)], dt=dt)
        U, fmax, n = minimize(sim, max_steps=150)
        assert n == n_ref, kind
        assert U == pytest.approx(U_ref, rel=1e-10), kind
        assert fmax == pytest.approx(f_ref, rel=1e-6, abs=1e-9 * abs(f_ref)), kind
        d = s.pos - s_ref.pos
        d -= s.box * np.round(d / s.box)
        assert np.max(np.abs(d)) <= 1e-9 * s.box[0], kind
        assert np.all(s.vel == 0.0)
        assert np.allclose(sim.force, sim_ref.force, rtol=0, atol=1e-8 * np.max(np.abs(sim_ref.force))), kind


def _salt_model(field):
    """A 512-ion rock-salt model in accusim's JSON form (8^3 sites at 2.82 A, each ion displaced by a seeded 0.1 A
    so that the forces are not the lattice's zero, velocities at 1100 K): LJ (Lorentz-Berthelot) + DSF at 8 A,
    Nose-Hoover; with `field`, also a uniform electric field (a force without a GPU plug-in, which stays
    accusim's)."""
    n = np.stack(np.meshgrid(*[np.arange(8)] * 3, indexing="ij"), -1).reshape(-1, 3)
    odd = n.sum(1) % 2 == 1
    g = (n + 0.5) * 2.82e-10 + np.random.default_rng(7).normal(0.0, 0.1e-10, n.shape)
    forces = [{"type": "LennardJones", "params": {"Na": ["0.544 kJ/mol", "2.35 A"], "Cl": ["0.418 kJ/mol", "4.40 A"]},
               "cutoff": 2.5},
              {"type": "DampedShiftedCoulomb", "rcut": "8 A"}]
    if field:
        forces.append({"type": "UniformField", "E": [2e8, 0.0, -1e8]})
    return {"dim": 3, "box": "22.56 A", "periodic": True, "seed": 4, "temperature": "1100 K",
            "species": {"Na": {"mass": "22.99 u", "charge": "1 e"}, "Cl": {"mass": "35.45 u", "charge": "-1 e"}},
            "particles": [{"species": "Na", "pos": g[~odd].tolist()}, {"species": "Cl", "pos": g[odd].tolist()}],
            "forces": forces, "integrator": {"type": "NoseHoover", "temperature": "1100 K", "period": "0.1 ps"},
            "dt": "1 fs"}


@pytest.mark.parametrize("field", [False, True])
@pytest.mark.parametrize("resident", [True, False])
def test_model_built_simulation_moved_to_gpu(field, resident):
    """accusim.model.build makes the simulation from a JSON model; to_gpu swaps its LJ, DSF and Nose-Hoover for the
    GPU plug-ins (the field, without a plug-in, stays accusim's and runs through the host protocol). 30 steps then
    follow the same model run with the reference's own classes: energies, thermostat state and positions within
    1e-9, and accusim's report still finds the DSF force and the extended-energy row."""
    import copy

    import accusim
    from accusim.model import build

    import devinproj_b200 as b200
    model = _salt_model(field)
    ref, _ = build(copy.deepcopy(model))
    sim, _ = build(copy.deepcopy(model))
    b200.to_gpu(sim, resident=resident)
    assert type(sim.forces[0]) is b200.LennardJones and type(sim.forces[1]) is b200.DampedShiftedCoulomb
    assert type(sim.integrator) is b200.NoseHoover
    assert isinstance(sim.system, b200.GpuSystem) == resident
    if field:
        assert type(sim.forces[2]) is accusim.forces.UniformField
    assert np.allclose(sim.force, ref.force, rtol=0, atol=1e-10 * np.max(np.abs(ref.force)))
    tr_r = ref.run(steps=30, record_every=5, positions=False)
    tr = sim.run(steps=30, record_every=5, positions=False)
    E_r, E = np.asarray(tr_r.total_energy), np.asarray(tr.total_energy)
    assert np.max(np.abs(E - E_r)) <= 1e-9 * np.max(np.abs(E_r))
    assert sim.integrator.xi == pytest.approx(ref.integrator.xi, rel=1e-9, abs=1e-9 * abs(ref.integrator.xi) + 1e-30)
    d = sim.system.pos - ref.system.pos
    d -= ref.system.box * np.round(d / ref.system.box)
    assert np.max(np.abs(d)) <= 1e-9 * ref.system.box[0]
    names = {c.name for c in accusim.AccuracyReport.build(sim).checks}
    assert "extended energy" in names and "DSF vs Ewald" in names
