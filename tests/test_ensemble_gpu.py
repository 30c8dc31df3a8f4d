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
    from devinproj_b200 import Simulation, VelocityVerlet, calibrate_dt, configs
    from devinproj_b200.ensemble import calibrate_dt_ensemble
    s, lj = configs.lj_fluid(5, seed=1)
    dt0 = 0.04 * configs.AR_TAU
    T = 0.4 * configs.AR_TAU
    d_b, drift_b = calibrate_dt_ensemble(s, [lj], dt0, T, energy_tol=2e-4, tpa=8)
    sim = Simulation(s.copy(), [lj], integrator=VelocityVerlet(), dt=dt0)
    d_s, drift_s = calibrate_dt(sim, T, energy_tol=2e-4)
    assert d_b == d_s
    assert drift_b == pytest.approx(drift_s, rel=0.05, abs=2e-6)
