"""Batched replicas: Richardson triples and speculative calibrate_dt against their one-at-a-time forms
(accusim/accuracy.py:191-221, accusim/advisor.py:58-79)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_richardson_ensemble_equals_separate_runs():
    """Each trajectory of the batched triple is bit-identical to the same trajectory run alone."""
    from devinproj_b200 import configs
    from devinproj_b200.engine import LEN, start_engine
    from devinproj_b200.ensemble import richardson_ensemble
    s, lj = configs.lj_fluid(5, seed=2)
    dt = 0.005 * configs.AR_TAU
    T = 40 * dt
    checks, ens = richardson_ensemble([s], [lj], [dt], T, tpa=8)
    finals = []
    for k in (1, 2, 4):
        eng, _, _ = start_engine([s.copy()], [lj], [dt / k], maxnb=ens.engine.maxnb, tpa=8)
        eng.run(40 * k, 0, True)
        finals.append(eng.get_state()[0].cpu().numpy() * LEN)
    got = [p for p, _ in ens.state()]
    for a, b in zip(got, finals):
        assert np.array_equal(a, b)
    c = checks[0]
    assert c.name == "timestep error" and c.value is not None and c.value > 0


def test_richardson_order_matches_fp64_oracle():
    """Observed order and Richardson estimate against the reference's FP64 formulation (oracle)."""
    from devinproj_b200 import configs
    from devinproj_b200.ensemble import richardson_ensemble
    from oracle import accusim_port as port
    s, lj = configs.lj_fluid(4, T_star=0.72, seed=7)
    dt = 0.004 * configs.AR_TAU
    n = 25
    checks, _ = richardson_ensemble([s], [lj], [dt], n * dt, tpa=8)
    finals = []
    for k in (1, 2, 4):
        st = port.State(s.pos.copy(), s.vel.copy(), s.sp.copy(), s.ids.copy(), s.box.copy(), True,
                        [("Ar", configs.AR_MASS, 0.0)])
        run = port.Run(st, [port.LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5)], dt / k)
        run.run(n * k, record_every=10 ** 9)
        finals.append(st.pos.copy())
    status, est, p = port.richardson(finals, n)
    assert p is not None and abs(p - 2) < 0.3
    assert checks[0].value == pytest.approx(est, rel=0.05)


def test_calibrate_dt_ensemble_matches_sequential_fp64():
    from accusim import Simulation, calibrate_dt
    from devinproj_b200 import VelocityVerlet, configs
    from devinproj_b200.ensemble import calibrate_dt_ensemble
    s, lj = configs.lj_fluid(5, seed=1)
    dt0 = 0.04 * configs.AR_TAU
    T = 0.4 * configs.AR_TAU
    d_b, drift_b = calibrate_dt_ensemble(s, [lj], dt0, T, energy_tol=2e-4, tpa=8)
    sim = Simulation(s.copy(), [lj], integrator=VelocityVerlet(), dt=dt0)
    d_s, drift_s = calibrate_dt(sim, T, energy_tol=2e-4)
    assert d_b == d_s
    assert drift_b == pytest.approx(drift_s, rel=0.05, abs=2e-6)


def test_full_size_ensemble_forces_momentum_and_replica_independence():
    """The batched LJ ensemble at full size (256 replicas of 256..32000 atoms, each at dt*, dt*/2 and dt*/4:
    768 trajectories, 6.04M atoms in one engine), 100 steps: the smallest, median and largest trajectories'
    FP32c forces against the FP64 plug-in on their final states (force RMS error <= 1e-5), momentum drift
    (report metric) at PASS (<= 1e-9) for the median trajectory and within 1e-8 for all, and the largest
    trajectory run alone bit-identical to its run inside the batch."""
    from devinproj_b200 import configs
    from devinproj_b200.engine import ACC, LEN, MASS, VEL, start_engine
    from devinproj_b200.ensemble import ReplicaEnsemble
    nc = configs.replica_sizes(256, seed=0)
    systems, dts = [], []
    for k, c in enumerate(nc):
        s, lj = configs.lj_fluid(int(c), seed=k)
        for f in (1, 2, 4):
            systems.append(s.copy())
            dts.append(0.005 * configs.AR_TAU / f)
    assert len(systems) == 768 and sum(s.n for s in systems) == 6_038_184
    ens = ReplicaEnsemble(systems, [lj], dts)
    ens.run(100, record_every=50)
    pos, vel, acc = (t.cpu().numpy() for t in ens.engine.get_state())
    o = ens.engine.offsets
    sizes = np.array([s.n for s in systems])
    picks = [int(np.argmin(sizes)), int(np.argsort(sizes)[len(sizes) // 2]), int(np.argmax(sizes))]
    for r in picks:
        s = systems[r].copy()
        s.pos = pos[o[r]:o[r + 1]] * LEN
        s.vel = vel[o[r]:o[r + 1]] * VEL
        F32 = acc[o[r]:o[r + 1]] * ACC * configs.AR_MASS
        F64 = lj.compute(s)[0]
        e = float(np.sqrt(np.mean(np.sum((F32 - F64) ** 2, 1)) / np.mean(np.sum(F64 ** 2, 1))))
        print(f"replica {r} ({s.n} atoms, dt/{[1, 2, 4][r % 3]}): force RMS rel error {e:.2e}")
        assert e <= 1e-5, r
    drift = np.empty(len(systems))
    for r in range(len(systems)):
        P = np.array(ens.records[r])[:, 2:5]
        scale = float(np.sum(configs.AR_MASS * np.abs(vel[o[r]:o[r + 1]] * VEL)))
        drift[r] = np.max(np.linalg.norm(P - P[0], axis=1)) / scale
    small = sizes <= 500
    print(f"momentum drift: median {np.median(drift):.2e}, max {drift.max():.2e} "
          f"(<= 500 atoms: max {drift[small].max():.2e}; larger: max {drift[~small].max():.2e})")
    # FP32 round-off of the per-atom sums: the relative drift grows as 1/sqrt(N), so the smallest replicas
    # reach the report's WARN grade (<= 1e-6) while the typical one stays at PASS (<= 1e-9)
    assert np.median(drift) <= 1e-9 and drift.max() <= 1e-8
    big = picks[-1]
    solo, _, _ = start_engine([systems[big].copy()], [lj], [dts[big]], tpa=ens.engine.tpa, rec_cap=8)
    solo.run(100, 50, True)
    p1, v1, _ = (t.cpu().numpy() for t in solo.get_state())
    assert np.array_equal(p1, pos[o[big]:o[big + 1]]) and np.array_equal(v1, vel[o[big]:o[big + 1]])


def test_calibrate_dt_matches_reference(golden):
    """accusim/advisor.py:51-79 against the reference's own runs (108 argon atoms, 0.4 ps trials, tolerance
    1e-5): from dt = 40 fs the plug-in halves to the reference's dt, with its drift; with dt unset it starts
    from suggest_dt, as the reference does; the batched engine form reaches the same dt (in this 17 A box the
    list radius exceeds half the box, so the engine rebuilds its lists every step)."""
    from accusim import Simulation, calibrate_dt
    from devinproj_b200 import LennardJones, VelocityVerlet
    from devinproj_b200.ensemble import calibrate_dt_ensemble
    from tests.test_dropin_gpu import product_system
    g = golden("calibrate_argon108")
    lj = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    for tag, dt0 in (("from40fs", float(g["dt0"])), ("suggested", None)):
        sim = Simulation(product_system(g), [lj], integrator=VelocityVerlet(), dt=dt0)
        dt, drift = calibrate_dt(sim, float(g["trial"]), energy_tol=float(g["tol"]))
        assert dt == pytest.approx(float(g[f"{tag}_dt"]), rel=1e-12), tag
        assert drift == pytest.approx(float(g[f"{tag}_drift"]), rel=1e-6), tag
        assert sim.dt == dt
    d_b, _ = calibrate_dt_ensemble(product_system(g), [lj], float(g["dt0"]), float(g["trial"]),
                                   energy_tol=float(g["tol"]))
    assert d_b == pytest.approx(float(g["from40fs_dt"]), rel=1e-12)
