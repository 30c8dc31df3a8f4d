"""Device-resident engine (FP32-compensated pairs, FP64 integration) against the FP64 oracle and the
reference's golden vectors. Floating-point tolerances (FP32 pair arithmetic):
  force RMS error / force RMS   <= 1e-5   (LJ and LJ + DSF; FP32 images of offsets from cell origins)
  potential energy relative     <= 2e-6
  records vs host FP64 sums of the downloaded state: 1e-12 relative (same FP64 data)
  momentum drift (report metric max|P-P0| / sum m|v|) <= 1e-9 (the report's PASS grade)."""
import numpy as np
import pytest

from oracle import accusim_port as port
from tests._helpers import rel_max
from tests.test_dropin_gpu import product_system

pytestmark = pytest.mark.gpu


def rms_rel(F, Fref):
    return float(np.sqrt(np.mean(np.sum((F - Fref) ** 2, 1)) / np.mean(np.sum(Fref ** 2, 1))))


def energy_drift(tr):
    """The report's energy metric (the oracle's restatement of accusim/accuracy.py:70-76) of a trajectory."""
    return port.energy_drift(np.array(tr.total_energy), np.array(tr.kinetic), np.array(tr.potential))


def momentum_drift(tr, s):
    """The report's momentum metric (the oracle's restatement of accusim/accuracy.py:86-91)."""
    return port.momentum_drift(np.array(tr.momentum), s.masses, s.vel)


def oracle_of(s):
    return port.State(s.pos.copy(), s.vel.copy(), s.sp.copy(), s.ids.copy(), s.box.copy(), True,
                      [(x.name, x.mass, x.charge) for x in s.species])


def test_engine_lj_forces_fp32c_vs_oracle(golden):
    from devinproj_b200 import GpuSimulation, LennardJones
    g = golden("argon864")
    s = product_system(g)
    params = {"Ar": (float(g["eps"]), float(g["sig"]))}
    sim = GpuSimulation(s, [LennardJones(params, cutoff=2.5)], dt=float(g["dt"]))
    Fo, Uo = port.LennardJones(params, cutoff=2.5, skin=0.0).compute(oracle_of(s))
    e = rms_rel(sim.force, Fo)
    print(f"argon864 FP32c force RMS rel error {e:.2e}, energy rel error {abs(sim.pe - Uo) / abs(Uo):.2e}")
    assert e <= 1e-5
    assert abs(sim.pe - Uo) <= 2e-6 * abs(Uo)
    # exact antisymmetry: the net force is round-off of the per-atom sums only
    assert np.linalg.norm(sim.force.sum(0)) <= 1e-6 * np.sqrt(s.n) * np.sqrt(np.mean(np.sum(Fo ** 2, 1)))


def test_engine_nacl_lj_dsf_forces_vs_reference(golden):
    from devinproj_b200 import DampedShiftedCoulomb, GpuSimulation, LennardJones
    g = golden("nacl4096")
    s = product_system(g)
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    forces = [LennardJones(params, cutoff=2.5), DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]))]
    sim = GpuSimulation(s, forces, dt=float(g["dt"]))
    Fref = g["F_lj"] + g["F_dsf"]
    Uref = float(g["U_lj"] + g["U_dsf"])
    e = rms_rel(sim.force, Fref)
    print(f"nacl4096 FP32c force RMS rel error {e:.2e}, energy rel error {abs(sim.pe - Uref) / abs(Uref):.2e}")
    assert e <= 1e-5
    assert abs(sim.pe - Uref) <= 2e-6 * abs(Uref)


@pytest.mark.parametrize("tpa", [1, 32])
def test_engine_dsf_exclusions_match_fp64_plugins(golden, tpa):
    """DSF exclusions in the engine (accusim/forces.py:400, 418-426): 4096-ion NaCl with 600 close ion pairs
    excluded from the Coulomb term (LJ kept), against the FP64 plug-ins with the same exclusions (pinned to
    the reference by the exclusion golden test), on the start state and after 200 steps (rebuilds re-sort
    the atoms), with the list built by a warp per cell (1 thread per atom) and by a warp per atom (32)."""
    from devinproj_b200 import DampedShiftedCoulomb, GpuSimulation, LennardJones, cell_list_pairs
    g = golden("nacl4096")
    s = product_system(g)
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    i, j = cell_list_pairs(s, 3.2e-10)
    pick = np.random.default_rng(3).choice(len(i), 600, replace=False)
    exclude = [(int(s.ids[a]), int(s.ids[b])) for a, b in zip(i[pick], j[pick])]
    lj = LennardJones(params, cutoff=2.5)
    dsf = DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]), exclude=exclude)
    sim = GpuSimulation(s, [lj, dsf], dt=float(g["dt"]), tpa=tpa)
    for stage in ("start", "after 200 steps"):
        if stage != "start":
            sim.run(steps=200, record_every=100, positions=False)
        F64 = lj.compute(s)[0] + dsf.compute(s)[0]
        U64 = lj.compute(s)[1] + dsf.compute(s)[1]
        F_noex = lj.compute(s)[0] + DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"])).compute(s)[0]
        assert rms_rel(F_noex, F64) > 1e-2           # the exclusions matter at this tolerance
        e = rms_rel(sim.force, F64)
        print(f"nacl4096 with exclusions, tpa {tpa}, {stage}: force RMS rel error {e:.2e}")
        assert e <= 1e-5, stage
        assert abs(sim.pe - U64) <= 2e-6 * abs(U64), stage
    assert sim.rebuilds >= 2


def test_engine_dsf_exclusions_in_a_one_cell_box():
    """DSF exclusions through the list build for boxes with fewer than 3 list cells per edge (per-axis minimum
    image, a thread per atom): 1000-ion NaCl in a 31.5 A box, 150 close pairs excluded, against the FP64
    plug-ins with the same exclusions, at the start and after 200 steps."""
    from devinproj_b200 import DampedShiftedCoulomb, GpuSimulation, cell_list_pairs, configs
    s, (lj, _) = configs.nacl_melt(10, seed=4)
    s.pos = (s.pos + np.random.default_rng(4).normal(0, 0.1e-10, s.pos.shape)) % s.box
    i, j = cell_list_pairs(s, 3.2e-10)
    pick = np.random.default_rng(5).choice(len(i), 150, replace=False)
    exclude = [(int(s.ids[a]), int(s.ids[b])) for a, b in zip(i[pick], j[pick])]
    dsf = DampedShiftedCoulomb(rcut=12e-10, alpha=0.2e10, exclude=exclude)
    sim = GpuSimulation(s, [lj, dsf], dt=1e-15, tpa=1)
    for stage in ("start", "after 200 steps"):
        if stage != "start":
            sim.run(steps=200, record_every=100, positions=False)
        F64 = lj.compute(s)[0] + dsf.compute(s)[0]
        U64 = lj.compute(s)[1] + dsf.compute(s)[1]
        e = rms_rel(sim.force, F64)
        print(f"nacl1000 one-cell box with exclusions, {stage}: force RMS rel error {e:.2e}")
        assert e <= 1e-5, stage
        assert abs(sim.pe - U64) <= 2e-6 * abs(U64), stage


def test_engine_lj_species_without_parameters_do_not_interact():
    """accusim/forces.py:108-113, 144-155: a species absent from the LJ parameters has eps = 0 and no LJ
    interaction, and the list radius uses sigma_max over interacting pairs only. A 2048-atom Ar/Kr/tracer
    mixture (a third of the atoms a tracer species with no parameters), engine vs the FP64 plug-in, at the
    start and after 100 steps."""
    from accusim import System
    from devinproj_b200 import GpuSimulation, LennardJones, configs
    rng = np.random.default_rng(9)
    base, _ = configs.lj_fluid(8, seed=9)
    s = System(3, box=base.box.copy(), periodic=True)
    s.add_species("Ar", configs.AR_MASS)
    s.add_species("Kr", 83.798 * 1.66053906660e-27)
    s.add_species("X", 20.0 * 1.66053906660e-27)
    kind = rng.permutation(np.repeat([0, 1, 2], [1024, 512, 512]))
    pos = (base.pos + rng.normal(0, 0.05 * configs.AR_SIGMA, base.pos.shape)) % s.box
    for k, name in enumerate(("Ar", "Kr", "X")):
        s.add(name, pos[kind == k])
    s.maxwell_boltzmann(86.4, rng)
    lj = LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA), "Kr": (1.4 * configs.AR_EPS, 3.6e-10)}, cutoff=2.5)
    sim = GpuSimulation(s, [lj], dt=5e-15)
    for stage in ("start", "after 100 steps"):
        if stage != "start":
            sim.run(steps=100, record_every=50, positions=False)
        F64, U64 = lj.compute(s)
        assert np.all(F64[s.sp == 2] == 0)
        e = rms_rel(sim.force, F64)
        print(f"Ar/Kr/tracer mixture, {stage}: force RMS rel error {e:.2e}")
        assert e <= 1e-5, stage
        assert np.all(sim.force[s.sp == 2] == 0), stage
        assert abs(sim.pe - U64) <= 2e-6 * abs(U64), stage


@pytest.mark.parametrize("nz,tpa", [(6, 1), (6, 32), (12, 1)])
def test_engine_orthorhombic_boxes(nz, tpa):
    """Boxes with unequal edges: an LJ fluid on a perturbed 28 x 19 x nz lattice (spacing 1.06 sigma; box 29.7
    x 20.1 x 6.4 sigma has a one-cell axis, 12.7 sigma does not), engine vs the FP64 plug-in at the start and
    after 100 steps, through the list builds for a one-cell axis (a warp per atom), for >= 8 threads per atom (a
    warp per atom) and for >= 3 cells per axis (a warp per cell)."""
    from accusim import System
    from devinproj_b200 import GpuSimulation, LennardJones, configs
    rng = np.random.default_rng(nz + tpa)
    a = 1.06 * configs.AR_SIGMA
    n = np.array([28, 19, nz])
    s = System(3, box=n * a, periodic=True)
    s.add_species("Ar", configs.AR_MASS)
    g = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), -1).reshape(-1, 3)
    s.add("Ar", ((g + 0.5) * a + rng.normal(0, 0.05 * configs.AR_SIGMA, g.shape)) % s.box)
    s.maxwell_boltzmann(86.4, rng)
    lj = LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5)
    sim = GpuSimulation(s, [lj], dt=5e-15, tpa=tpa)
    for stage in ("start", "after 100 steps"):
        if stage != "start":
            sim.run(steps=100, record_every=50, positions=False)
        F64, U64 = lj.compute(s)
        e = rms_rel(sim.force, F64)
        print(f"box {np.round(s.box / configs.AR_SIGMA, 1)} sigma, tpa {tpa}, {stage}: force RMS rel error {e:.2e}")
        assert e <= 1e-5, stage
        assert abs(sim.pe - U64) <= 2e-6 * abs(U64), stage


def test_engine_box_smaller_than_twice_the_list_radius(golden):
    """108 argon atoms (a displaced fcc lattice) in a 17.3 A box, list radius 9.5 A: a pair's minimum image can
    change between rebuilds, so the engine rebuilds this replica's lists every step; forces against the FP64
    plug-in at the start and after 100 steps, one rebuild per step, and the energy drift of the 100 steps no
    more than 10x the reference's over its 60-step run of the undisplaced lattice."""
    from devinproj_b200 import GpuSimulation, LennardJones
    g = golden("report_argon108")
    s = product_system(g)
    assert 2 * 2.8 * float(g["sig"]) > s.box[0]
    # the fcc lattice's forces vanish by symmetry: displace every atom by a seeded 0.05 sigma first
    s.pos = (s.pos + np.random.default_rng(2).normal(0, 0.05 * float(g["sig"]), s.pos.shape)) % s.box
    lj = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    sim = GpuSimulation(s, [lj], dt=float(g["dt"]))
    rb0 = sim.rebuilds
    tr = None
    for stage in ("start", "after 100 steps"):
        if stage != "start":
            tr = sim.run(steps=100, record_every=1, positions=False)
        F64, U64 = lj.compute(s)
        e = rms_rel(sim.force, F64)
        print(f"argon108 small box, {stage}: force RMS rel error {e:.2e}")
        assert e <= 1e-5, stage
        assert abs(sim.pe - U64) <= 2e-6 * abs(U64), stage
    assert sim.rebuilds - rb0 >= 100
    ref = float(g["values"][list(g["names"]).index("energy")])
    print(f"energy drift {energy_drift(tr):.2e} (reference, 60 steps: {ref:.2e})")
    assert energy_drift(tr) <= 10 * ref


def test_gpu_simulation_report_matches_reference_rows(golden):
    """GpuSimulation's accuracy report (device run, batched FP32c Richardson runs) on the 512-ion NaCl melt of
    the reference's own report: the same rows; energy, momentum and relativity graded as the reference grades
    them; the timescale and DSF-vs-Ewald values to 1e-3 (the FP32c state differs from the FP64 one at ~1e-7)."""
    from devinproj_b200 import DampedShiftedCoulomb, GpuSimulation, LennardJones
    g = golden("report_nacl512")
    s = product_system(g)
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    forces = [LennardJones(params, cutoff=2.5), DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]))]
    sim = GpuSimulation(s, forces, dt=float(g["dt"]))
    sim.run(steps=int(g["steps"]), record_every=1, positions=False)
    rep = {c.name: c for c in sim.accuracy_report(convergence_duration=float(g["convergence_duration"])).checks}
    ref = {str(n): (str(st), float(v)) for n, st, v in zip(g["names"], g["statuses"], g["values"])}
    assert list(rep) == list(ref)
    for name in ("energy", "momentum", "relativity", "mass-energy", "charge"):
        assert rep[name].status == ref[name][0], name
    for name in ("timestep vs physics", "DSF vs Ewald", "relativity"):
        assert rep[name].value == pytest.approx(ref[name][1], rel=1e-3), name


def test_engine_trajectory_tracks_reference_and_conserves(golden):
    """60 steps of the 864-atom argon case: energy series against the reference's FP64 run."""
    from devinproj_b200 import GpuSimulation, LennardJones
    g = golden("argon864")
    s = product_system(g, "0")
    sim = GpuSimulation(s, [LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)],
                        dt=float(g["dt"]))
    tr = sim.run(steps=int(g["steps"]), positions=False)
    E = np.array(tr.kinetic) + np.array(tr.potential)
    Eref = g["kinetic"] + g["potential"]
    scale = max(abs(Eref[0]), np.max(np.abs(g["kinetic"])), np.max(np.abs(g["potential"])))
    assert np.max(np.abs(E - Eref)) <= 1e-5 * scale
    assert rel_max(np.array(tr.kinetic), g["kinetic"]) <= 1e-4
    assert momentum_drift(tr, s) <= 1e-9
    ref_drift = port.energy_drift(Eref, g["kinetic"], g["potential"])
    assert energy_drift(tr) <= 1.5 * ref_drift + 1e-6
    assert len(tr.t) == int(g["steps"]) + 1 and tr.t[-1] == pytest.approx(float(g["dt"]) * int(g["steps"]))


def test_engine_records_equal_host_sums_of_state():
    from devinproj_b200 import GpuSimulation, configs
    s, forces, dt = configs.argon864(seed=4)
    sim = GpuSimulation(s, forces, dt=dt)
    tr = sim.run(steps=37, record_every=10, positions=True)
    assert len(tr.t) == 1 + 3 + 1
    assert len(tr.positions) == len(tr.t)
    assert np.array_equal(tr.positions[-1], s.pos)
    assert tr.kinetic[-1] == pytest.approx(s.kinetic_energy(), rel=1e-12)
    assert np.allclose(tr.momentum[-1], s.momentum(), rtol=0, atol=1e-12 * np.sum(s.masses[:, None] * np.abs(s.vel)))
    L = s.angular_momentum()
    assert np.allclose(tr.angular_momentum[-1], L, rtol=1e-10, atol=1e-12 * np.abs(L).max())
    assert np.all(s.pos >= 0) and np.all(s.pos < s.box)


def test_engine_lists_stay_valid_across_rebuilds():
    """Hot argon: many rebuilds and re-sorts; forces at the end equal the FP64 oracle's on the same state."""
    from devinproj_b200 import GpuSimulation, configs
    s, forces, dt = configs.argon864(seed=1)
    s.maxwell_boltzmann(300.0, np.random.default_rng(1))
    sim = GpuSimulation(s, forces, dt=dt)
    sim.run(steps=300, record_every=100, positions=False)
    assert sim.rebuilds >= 10
    Fo, Uo = port.LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5, skin=0.0).compute(oracle_of(s))
    assert rms_rel(sim.force, Fo) <= 1e-5
    assert abs(sim.pe - Uo) <= 2e-6 * abs(Uo)


def test_engine_full_size_lj1m_pair_set_forces_and_net_force():
    """The headline system at full size (1,048,576-atom LJ fluid, fcc 64^3, rho* 0.8442, T* 0.72), through
    size-independent properties, on the displaced lattice and again on the state after 200 steps (about 20
    rebuilds): the engine's lists, decoded entry by entry, hold exactly the FP64 pair set at the list radius
    (the drop-in's cell_list_pairs, itself pinned to the reference's pair sets) on the positions of the last
    rebuild, each pair in both directions; FP32c forces within the force tolerance of the FP64 plug-in's on
    the same positions, energy within 2e-6, and the net force at round-off."""
    from accusim import System

    from devinproj_b200 import GpuSimulation, cell_list_pairs, configs
    from tests.test_engine_lists_gpu import compare_sets, engine_pairs
    s, forces, dt = configs.lj_large(64)
    assert s.n == 1_048_576
    # the lattice's forces vanish by symmetry: displace every atom by a seeded 0.02 sigma first
    s.pos = (s.pos + np.random.default_rng(7).normal(0, 0.02 * configs.AR_SIGMA, s.pos.shape)) % s.box
    sim = GpuSimulation(s, forces, dt=dt)
    for stage in ("initial", "after 200 steps"):
        if stage != "initial":
            sim.run(steps=200, record_every=100, positions=False)
            assert sim.rebuilds >= 10
        got, _, pos_build = engine_pairs(sim.engine)
        b = System(3, box=s.box, periodic=True)
        b.add_species("Ar", configs.AR_MASS)
        b.add("Ar", pos_build)
        i, j = cell_list_pairs(b, sim.rlist)
        compare_sets(got, np.sort(i * s.n + j), pos_build, s.box, sim.rlist, f"1M LJ {stage}")
        F64 = np.zeros_like(s.pos)
        U64 = 0.0
        for f in forces:
            Fi, Ui = f.compute(s)
            F64 += Fi
            U64 += Ui
        e = rms_rel(sim.force, F64)
        print(f"1M LJ {stage}: FP32c force RMS rel error {e:.2e}, energy rel error {abs(sim.pe - U64) / abs(U64):.2e}")
        assert e <= 1e-5, stage
        assert abs(sim.pe - U64) <= 2e-6 * abs(U64), stage
        frms = np.sqrt(np.mean(np.sum(F64 ** 2, 1)))
        assert np.linalg.norm(sim.force.sum(0)) <= 1e-6 * np.sqrt(s.n) * frms, stage


def test_batched_replicas_equal_single_runs_bitwise():
    """Replicas of different sizes and dt in one engine advance exactly as each would alone."""
    from devinproj_b200 import configs
    from devinproj_b200.engine import LEN, VEL, start_engine
    systems, dts = [], []
    for nc, T, dtf in [(4, 0.72, 1.0), (5, 1.0, 0.5), (6, 0.72, 0.25)]:
        s, lj = configs.lj_fluid(nc, T_star=T, seed=nc)
        systems.append(s)
        dts.append(0.005 * configs.AR_TAU * dtf)
    batch, _, _ = start_engine(systems, [lj], dts)
    batch.run(50, 0, True)
    bp, bv, _ = batch.get_state()
    bp, bv = bp.cpu().numpy(), bv.cpu().numpy()
    for k, (s, dt) in enumerate(zip(systems, dts)):
        eng, _, _ = start_engine([s], [lj], [dt], maxnb=batch.maxnb)
        eng.run(50, 0, True)
        p, v, _ = eng.get_state()
        sl = slice(batch.offsets[k], batch.offsets[k + 1])
        assert np.array_equal(p.cpu().numpy(), bp[sl])
        assert np.array_equal(v.cpu().numpy(), bv[sl])
    assert batch.status().rebuilds > 3


def test_batched_nose_hoover_replicas_equal_single_runs_bitwise():
    """Nose-Hoover keeps one thermostat per replica (its kinetic-energy sums, xi and eta): replicas of
    different sizes and dt under Nose-Hoover in one engine advance, thermostat state included, exactly as each
    would alone, across several graph blocks."""
    from devinproj_b200 import NoseHoover, configs
    from devinproj_b200.engine import nose_hoover_thermostat, start_engine
    th = nose_hoover_thermostat(NoseHoover(120.0, 0.2e-12))
    systems, dts = [], []
    for nc, T, dtf in [(4, 0.5, 1.0), (5, 1.0, 0.5), (6, 0.72, 0.25)]:
        s, lj = configs.lj_fluid(nc, T_star=T, seed=10 + nc)
        systems.append(s)
        dts.append(0.005 * configs.AR_TAU * dtf)
    batch, _, _ = start_engine(systems, [lj], dts, thermo=th)
    for _ in range(3):
        batch.run(20, 10, True)
    bp, bv, _ = batch.get_state()
    bp, bv, bnh = bp.cpu().numpy(), bv.cpu().numpy(), batch.nh_state()
    assert np.all(bnh[:, 0] != 0)
    for k, (s, dt) in enumerate(zip(systems, dts)):
        eng, _, _ = start_engine([s], [lj], [dt], maxnb=batch.maxnb, tpa=batch.tpa, thermo=th)
        for _ in range(3):
            eng.run(20, 10, True)
        p, v, _ = eng.get_state()
        sl = slice(batch.offsets[k], batch.offsets[k + 1])
        assert np.array_equal(p.cpu().numpy(), bp[sl]), k
        assert np.array_equal(v.cpu().numpy(), bv[sl]), k
        assert np.array_equal(eng.nh_state()[0], bnh[k]), k


def test_engine_rejects_unsupported_setups():
    from accusim import System
    from devinproj_b200 import DampedShiftedCoulomb, GpuSimulation, LennardJones
    s = System(3, box=None)
    s.add_species("Ar", 6.6e-26)
    s.add("Ar", np.random.default_rng(0).uniform(0, 3e-9, (50, 3)))
    with pytest.raises(ValueError):
        GpuSimulation(s, [LennardJones({"Ar": (1.6e-21, 3.4e-10)})], dt=1e-15)
    s2 = System(3, box=4e-9, periodic=True)    # two LennardJones forces
    s2.add_species("Ar", 6.6e-26)
    s2.add("Ar", [[0, 0, 0], [4e-10, 0, 0]])
    with pytest.raises(ValueError):
        GpuSimulation(s2, [LennardJones({"Ar": (1.6e-21, 3.4e-10)}), LennardJones({"Ar": (1.0e-21, 3.0e-10)})],
                      dt=1e-15)
    s3 = System(3, box=4e-9, periodic=True)
    s3.add_species("Na", 3.8e-26, charge=1.6e-19)
    s3.add("Na", [[0, 0, 0], [2e-10, 0, 0]])
    with pytest.raises(ValueError):   # one DampedShiftedCoulomb at most
        GpuSimulation(s3, [DampedShiftedCoulomb(rcut=1e-9), DampedShiftedCoulomb(rcut=1.1e-9)], dt=1e-15)


@pytest.mark.parametrize("seed", [0, 5])
def test_list_build_variants_agree(seed):
    """The warp-per-atom list build (>= 8 threads per atom) and the culled thread-per-atom build produce the
    same pair sets; both give FP64-oracle forces."""
    from devinproj_b200 import configs
    from devinproj_b200.engine import ACC, LEN, start_engine
    s, lj = configs.lj_fluid(6, seed=seed)
    s.maxwell_boltzmann(250.0, np.random.default_rng(seed))
    out = {}
    for tpa in (1, 8):
        eng, _, _ = start_engine([s], [lj], [0.005 * configs.AR_TAU], tpa=tpa)
        eng.run(40, 0, True)   # several rebuilds
        mx, total = eng.neighbor_stats()
        pairs = eng.count_pairs()
        p, v, a = eng.get_state()
        out[tpa] = (total, pairs, p.cpu().numpy() * LEN, a.cpu().numpy() * ACC, eng.status().rebuilds)
    assert out[1][4] > 1 and out[8][4] > 1
    for tpa in (1, 8):
        st = port.State(out[tpa][2], np.zeros_like(out[tpa][2]), s.sp.copy(), s.ids.copy(), s.box.copy(), True,
                        [("Ar", configs.AR_MASS, 0.0)])
        Fo, _ = port.LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5, skin=0.0).compute(st)
        assert rms_rel(out[tpa][3] * configs.AR_MASS, Fo) <= 1e-5
    # fresh engines on identical positions: identical pair sets (entry by entry) and pair counts
    from tests.test_engine_lists_gpu import engine_pairs
    s.pos = out[1][2]
    sets = []
    for tpa in (1, 8):
        eng, _, _ = start_engine([s], [lj], [0.005 * configs.AR_TAU], tpa=tpa)
        sets.append((engine_pairs(eng)[0], eng.count_pairs()))
    assert np.array_equal(sets[0][0], sets[1][0]) and sets[0][1] == sets[1][1]


@pytest.mark.parametrize("tpa", [1, 32])
def test_dense_cells_lists_match_oracle(tpa):
    """Dense cells: the 4096-ion melt's DSF list radius (13.8 A) gives 3 cells per edge and ~150 atoms per
    cell, so the warp-per-home-cell build (1 thread per atom) walks several home chunks and ~130 candidate
    batches per cell. Its list holds exactly the oracle's pairs within the list radius (each pair twice),
    and the forces match the FP64 oracle."""
    from devinproj_b200 import configs
    from devinproj_b200.engine import ACC, start_engine
    s, forces, dt = configs.nacl4096(seed=3)
    s.pos = (s.pos + np.random.default_rng(7).normal(0, 0.2e-10, s.pos.shape)) % s.box
    s.vel[:] = 0.0
    from tests._helpers import pair_keys
    from tests.test_engine_lists_gpu import compare_sets, engine_pairs
    eng, rlist, _ = start_engine([s], forces, [dt], tpa=tpa)
    eng.check("start")
    st = oracle_of(s)
    got, _, pos_build = engine_pairs(eng)
    bst = port.State(pos_build, np.zeros_like(pos_build), s.sp.copy(), s.ids.copy(), s.box.copy(), True,
                     [(x.name, x.mass, x.charge) for x in s.species])
    ref = pair_keys(*port.cell_list_pairs(bst, rlist), s.n)
    assert compare_sets(got, ref, pos_build, s.box, rlist, f"dense cells tpa {tpa}") == 0
    p, v, a = eng.get_state()
    Fo = sum(f.compute(st)[0] for f in (port.LennardJones(configs.NACL_LJ, cutoff=2.5, skin=0.0),
                                         port.DampedShiftedCoulomb(rcut=forces[1].rcut, alpha=forces[1].alpha,
                                                                   skin=0.0)))
    masses = np.array([x.mass for x in s.species])[s.sp][:, None]
    assert rms_rel(a.cpu().numpy() * ACC * masses, Fo) <= 1e-5


def test_engine_langevin_matches_oracle_with_the_same_draws():
    """BAOAB inside the engine (fused into the step kernel, counter-based Philox draws) against the FP64
    oracle's BAOAB fed the same draws (oracle/philox.py): 10 steps of the 864-atom argon case. Positions
    agree to FP32-force level (1e-9 of the box), velocities to 1e-6."""
    from devinproj_b200 import GpuSimulation, Langevin, configs
    from oracle import philox
    s, forces, dt = configs.argon864(seed=2)
    st = oracle_of(s)
    seed = 987654321
    sim = GpuSimulation(s, forces, integrator=Langevin(120.0, 5e12), dt=dt, seed=seed)
    sim.run(steps=10, record_every=5, positions=False)
    j = [0]

    def draws(shape):
        z = philox.normals(j[0], np.arange(shape[0]), 0, seed)
        j[0] += 1
        return z
    lj = port.LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5)
    port.Run(st, [lj], dt, integrator=port.LangevinBAOAB(120.0, 5e12, draws)).run(10)
    d = s.pos - st.pos
    d -= s.box * np.round(d / s.box)
    assert np.max(np.abs(d)) <= 1e-9 * s.box[0]
    assert rel_max(s.vel, st.vel) <= 1e-6


def test_engine_langevin_thermostats_and_zero_friction_is_verlet():
    """A 2000-step Langevin run from 60 K reaches the 120 K target (the report's thermostat row passes), and
    with zero friction the BAOAB step is VelocityVerlet: two half drifts round differently from one full
    drift, and a flipped FP32 image rounding moves forces by ~1e-7, so the 50-step trajectories agree to
    1e-9 of the box."""
    from devinproj_b200 import GpuSimulation, Langevin, VelocityVerlet, configs
    s, forces, dt = configs.argon864(seed=4)
    s.vel *= np.sqrt(60.0 / s.temperature())
    sim = GpuSimulation(s, forces, integrator=Langevin(120.0, 2e12), dt=dt, seed=7)
    sim.run(steps=2000, record_every=50, positions=False)
    row = {c.name: c for c in sim.accuracy_report().checks}["thermostat"]
    assert row.status == "PASS", row
    s1, forces1, _ = configs.argon864(seed=5)
    s2 = s1.copy()
    a = GpuSimulation(s1, forces1, integrator=Langevin(120.0, 0.0), dt=dt, seed=1)
    b = GpuSimulation(s2, forces1, integrator=VelocityVerlet(), dt=dt)
    a.run(steps=50, record_every=50, positions=False)
    b.run(steps=50, record_every=50, positions=False)
    d = s1.pos - s2.pos
    d -= s1.box * np.round(d / s1.box)
    assert np.max(np.abs(d)) <= 1e-9 * s1.box[0]


def test_engine_nose_hoover_matches_oracle():
    """Nose-Hoover inside the engine (step kernel -> chunked kinetic-energy sum -> thermostat scalars ->
    scale, kick and drift) against the FP64 oracle's Trotter half-steps: 20 steps of the 864-atom argon
    case with records every 5, run as several graph blocks. Trajectory (1e-8 of the box), thermostat state
    and bath energies (1e-6) agree to FP32-force level."""
    from devinproj_b200 import GpuSimulation, NoseHoover, configs
    s, forces, dt = configs.argon864(seed=6)
    s.vel *= np.sqrt(60.0 / s.temperature())
    st = oracle_of(s)
    nh = NoseHoover(120.0, 0.2e-12)
    sim = GpuSimulation(s, forces, integrator=nh, dt=dt)
    tr = sim.run(steps=20, record_every=5, positions=False)
    on = port.NoseHooverMTK(120.0, 0.2e-12)
    lj = port.LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5)
    run = port.Run(st, [lj], dt, integrator=on).run(20, 5)
    d = s.pos - st.pos
    d -= s.box * np.round(d / s.box)
    # FP32 pair forces (2e-6 relative) move positions by ~1e-17 m over 20 steps of 10 fs
    assert np.max(np.abs(d)) <= 1e-8 * s.box[0]
    assert rel_max(s.vel, st.vel) <= 1e-6
    assert abs(nh.xi - on.xi) <= 1e-6 * abs(on.xi) and abs(nh.eta - on.eta) <= 1e-6 * abs(on.eta)
    assert nh.Q == pytest.approx(on.Q, rel=1e-12)
    assert rel_max(np.array(tr.bath), np.array(run.bath)) <= 1e-6
    assert rel_max(np.array(tr.kinetic), np.array(run.kinetic)) <= 1e-6


def test_engine_nose_hoover_conserves_extended_energy():
    """The reference's own Nose-Hoover test (tests/test_nose_hoover.py:26-35) on the engine: heated from
    60 K to the 120 K target (thermostat row passes), extended-energy error below 1e-3, and that error is
    integration error: it shrinks by more than 2.5x when dt halves (second order)."""
    from devinproj_b200 import GpuSimulation, NoseHoover, configs

    def run(dt_fs, steps):
        s, forces, _ = configs.argon864(seed=8)
        s.vel *= np.sqrt(60.0 / s.temperature())
        sim = GpuSimulation(s, forces, integrator=NoseHoover(120.0, 0.2e-12), dt=dt_fs * 1e-15)
        sim.run(steps=steps, record_every=50, positions=False)
        return {c.name: c for c in sim.accuracy_report().checks}
    coarse, fine = run(10.0, 2000), run(5.0, 4000)
    assert coarse["thermostat"].status == "PASS", coarse["thermostat"]
    assert coarse["extended energy"].value < 1e-3
    assert coarse["extended energy"].value / fine["extended energy"].value > 2.5


def test_list_overflow_mid_run_regrows_and_continues():
    """The fcc argon lattice has exactly 78 neighbours per atom within the list radius, so a capacity of 80
    holds the first lists; once the crystal melts, some atom's list outgrows it during a run. The run goes on
    with a regrown engine from the block's start state, and the final forces match the FP64 oracle."""
    from devinproj_b200 import GpuSimulation, configs
    s, forces, dt = configs.argon864(seed=9)
    s.vel *= np.sqrt(300.0 / s.temperature())
    sim = GpuSimulation(s, forces, dt=dt, maxnb=80)
    assert sim.engine.maxnb == 80
    sim.run(steps=400, record_every=100, positions=False)
    assert getattr(sim, "regrowths", 0) >= 1 and sim.engine.maxnb > 80
    assert len(sim.trajectory.t) == 5
    Fo, _ = port.LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5, skin=0.0).compute(oracle_of(s))
    assert rms_rel(sim.force, Fo) <= 1e-5


def test_barrier_timeout_reports_and_returns():
    """A bounded device wait that runs out (no fault, no hang): an engine whose grid-barrier waits give up at
    once (barrier_wait_limit < 0) starts on a 32,000-atom fluid, so the first list build's cooperative kernel
    (125 blocks; block 0 arrives last at the first barrier, after its prefix scan) has blocks that stop
    waiting. The kernel returns, the status block carries ACS_FLAG_TIMEOUT, the host check raises
    ACS_ERR_TIMEOUT (the reference raises its errors as Python exceptions, accusim/simulation.py:96-97), and
    the engine's later kernels return at once. A new engine with the default limit then runs normally."""
    import torch

    from devinproj_b200 import _lib, configs
    from devinproj_b200.engine import _upload_state, build_engine, start_engine
    s, lj = configs.lj_fluid(20, seed=3)
    dt = 0.005 * configs.AR_TAU
    eng, _, _ = build_engine([dict(n=s.n, box=s.box, dt=dt)], [lj], s.species, barrier_wait_limit=-1)
    assert eng.launch_info()[1] >= 100
    _upload_state(eng, [s])            # set_state: the forced first rebuild
    torch.cuda.synchronize()           # returned: no wait outlived its limit
    assert eng.status().flags & _lib.FLAG_TIMEOUT
    with pytest.raises(_lib.AcsError) as err:
        eng.check("barrier timeout")
    assert err.value.code == _lib.ACS_ERR_TIMEOUT
    eng.run(5, 0, True)
    torch.cuda.synchronize()
    assert eng.status(clear=True).flags & _lib.FLAG_TIMEOUT
    assert eng.status().flags == 0
    del eng
    ok, _, _ = start_engine([s], [lj], [dt])
    ok.run(20, 10, True)
    ok.check("default barrier limit")
    assert np.all(np.isfinite(ok.records(2)))
