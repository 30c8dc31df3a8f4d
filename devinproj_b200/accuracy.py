"""The accuracy-report rows that read this path's reductions (accusim/accuracy.py:19-221) and the dt
calibration loop (accusim/advisor.py:58-79): energy drift, momentum drift, angular momentum,
mass and charge ledgers, and the Richardson dt / dt/2 / dt/4 timestep error. Thresholds and
formulas are the reference's."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .units import c_light, k_B

from .units import si

PASS, WARN, FAIL, NA = "PASS", "WARN", "FAIL", "n/a"


@dataclass
class Check:
    name: str
    status: str
    value: float | None
    detail: str

    def row(self):
        v = "" if self.value is None else f"{self.value:.2e}"
        return f"  [{self.status:>4}] {self.name:<22} {v:>10}  {self.detail}"


def _grade(x, good, ok):
    return PASS if x <= good else WARN if x <= ok else FAIL


def energy_drift(tr) -> float:
    """max|E - E0| / max(|E0|, max|KE|, max|PE|) (accusim/accuracy.py:70-76)."""
    E = tr.total_energy
    scale = max(abs(E[0]), np.max(np.abs(tr.kinetic)), np.max(np.abs(tr.potential)), 1e-300)
    return float(np.max(np.abs(E - E[0])) / scale)


def momentum_drift(tr, s) -> float:
    """max|P - P0| / sum m|v| (accusim/accuracy.py:86-91)."""
    P = np.array(tr.momentum)
    pscale = max(float(np.sum(s.masses[:, None] * np.abs(s.vel))), 1e-300)
    return float(np.max(np.linalg.norm(P - P[0], axis=1)) / pscale)


class AccuracyReport:
    def __init__(self, checks):
        self.checks = checks

    def __getitem__(self, name) -> Check:
        for c in self.checks:
            if c.name == name:
                return c
        raise KeyError(name)

    @property
    def ok(self) -> bool:
        return all(c.status != FAIL for c in self.checks)

    def __str__(self):
        nf = sum(c.status == FAIL for c in self.checks)
        nw = sum(c.status == WARN for c in self.checks)
        if nf:
            head = f"Accuracy report (PROBLEMS FOUND: {nf} failed, {nw} warnings)"
        elif nw:
            head = f"Accuracy report (no failures, {nw} warning{'s' * (nw != 1)})"
        else:
            head = "Accuracy report (all applicable checks passed)"
        return "\n".join([head] + [c.row() for c in self.checks])

    @classmethod
    def build(cls, sim, convergence_duration=None):
        tr, s = sim.trajectory, sim.system
        if len(tr.t) < 2:
            raise ValueError("run the simulation before asking for a report")
        checks = [Check("units", PASS, None, "every input was dimension-checked on entry")]
        integ = sim.integrator
        conservative = all(f.conservative for f in sim.forces) and not integ.thermostat
        external = any(f.external for f in sim.forces)
        walls = s.box is not None and not s.periodic
        central = all(f.central for f in sim.forces)
        if conservative:
            d = energy_drift(tr)
            checks.append(Check("energy", _grade(d, 1e-5, 1e-3), d,
                                "max |E(t)-E0| / energy scale (incl. reaction ledger)"))
        else:
            checks.append(Check("energy", NA, None, "not conserved by design"))
        if hasattr(integ, "bath_energy") and all(f.conservative for f in sim.forces) and len(tr.bath) == len(tr.t):
            # accusim/accuracy.py:81-84: the Nose-Hoover conserved quantity
            E = tr.total_energy
            scale = max(abs(E[0]), np.max(np.abs(tr.kinetic)), np.max(np.abs(tr.potential)), 1e-300)
            Ex = E + np.array(tr.bath)
            dx = float(np.max(np.abs(Ex - Ex[0])) / scale)
            checks.append(Check("extended energy", _grade(dx, 1e-5, 1e-3), dx,
                                "Nose-Hoover conserved quantity: E + thermostat energy"))
        if not external and not walls and not integ.thermostat:
            dp = momentum_drift(tr, s)
            checks.append(Check("momentum", _grade(dp, 1e-9, 1e-6), dp, "max |P(t)-P0| / sum m|v|"))
        else:
            checks.append(Check("momentum", NA, None, "external field, walls or thermostat"))
        if central and not external and s.box is None and not integ.thermostat and s.dim in (2, 3):
            Lm = np.array(tr.angular_momentum)
            lscale = max(float(np.sum(np.linalg.norm(np.cross(s.pos, s.masses[:, None] * s.vel), axis=-1)))
                         if s.dim == 3 else float(np.sum(np.abs(np.cross(s.pos, s.masses[:, None] * s.vel)))), 1e-300)
            dl = float(np.max(np.linalg.norm(Lm - Lm[0], axis=1)) / lscale)
            checks.append(Check("angular momentum", _grade(dl, 1e-9, 1e-6), dl, "max |L(t)-L0| / sum |r x p|"))
        else:
            checks.append(Check("angular momentum", NA, None, "needs central forces in open space"))
        M = np.array(tr.mass)
        dm = float(np.max(np.abs(M - M[0])) / M[0]) if M[0] else 0.0
        checks.append(Check("mass-energy", _grade(dm, 1e-12, 1e-9), dm, "rest mass + released/c^2"))
        Qc = np.array(tr.charge)
        qscale = max(float(np.sum(np.abs(s.charges))), 1e-300)
        dq = float(np.max(np.abs(Qc - Qc[0])) / qscale)
        checks.append(Check("charge", _grade(dq, 1e-12, 1e-9), dq, "total charge"))
        kind = type(integ).__name__
        if kind in ("Langevin", "NoseHoover") and len(tr.t) >= 4:
            # accusim/accuracy.py:112-123: mean temperature over the second half against the target
            half = len(tr.t) // 2
            kin = np.asarray(tr.kinetic[half:])
            n = np.array([sum(c.values()) for c in tr.counts[half:]], dtype=float)
            dof = s.dim * np.maximum(n - 1, 1) if kind == "NoseHoover" else s.dim * np.maximum(n, 1)
            T_meas = float(np.mean(2 * kin / (dof * k_B)))
            dev = abs(T_meas - integ.T) / integ.T
            tol = max(0.02, 3 * np.sqrt(2 / (s.dim * max(s.n, 1))))
            checks.append(Check("thermostat", PASS if dev <= tol else (WARN if dev <= 0.1 else FAIL), dev,
                                f"mean T over 2nd half {T_meas:.4g} K vs target {integ.T:.4g} K"))
        if kind != "Brownian":
            ts = timescales(sim)
            if ts:
                # accusim/accuracy.py:126-133
                tkind, tmin = min(ts.items(), key=lambda kv: kv[1])
                ratio = sim.dt / tmin
                checks.append(Check("timestep vs physics", _grade(ratio, 0.02, 0.1), ratio,
                                    f"dt / shortest timescale ({tkind}, {tmin:.3g} s) at end of run"))
        for f in [f for f in sim.forces if type(f).__name__ == "DampedShiftedCoulomb"]:
            # accusim/accuracy.py:148-161, with the device Ewald (pinned to the reference's)
            q = s.charges
            if not (s.periodic and s.dim == 3 and np.any(q)):
                continue
            if f.exclude or abs(q.sum()) > 1e-9 * np.sum(np.abs(q)) or s.n > 2000:
                checks.append(Check("DSF vs Ewald", NA, None, "needs a neutral system, no exclusions, n <= 2000"))
                continue
            from .ewald import Ewald
            F_d = f.compute(s)[0]
            F_e = Ewald(k=f.k).compute(s)[0]
            e = float(np.sqrt(np.mean(np.sum((F_d - F_e) ** 2, 1)) / np.mean(np.sum(F_e ** 2, 1))))
            checks.append(Check("DSF vs Ewald", _grade(e, 5e-2, 2e-1), e,
                                "RMS force error of the cutoff method vs Ewald, final snapshot (inflated for "
                                "near-crystalline states)"))
        # accusim/accuracy.py:176-182
        beta2 = float(np.max(np.sum(s.vel ** 2, axis=1)) / c_light ** 2) if s.n else 0.0
        checks.append(Check("relativity", _grade(beta2, 1e-4, 1e-2), beta2,
                            f"(v/c)^2 of fastest particle: Newtonian error ~ this size (v = {np.sqrt(beta2):.3g} c)"))
        if convergence_duration is not None:
            checks.append(timestep_convergence(sim, convergence_duration))
        return cls(checks)


def _closest_approach(s, max_rows=1500):
    """Smallest distance from the sampled atoms to any other atom (accusim/advisor.py:15-22: every atom for
    n <= max_rows, else max_rows atoms drawn by default_rng(0)), from the device cell list at a radius that
    doubles until some pair holds a sampled atom (any closer pair is then inside it too), instead of the
    reference's dense rows x n distance matrix."""
    from .forces import cell_list_pairs
    n = s.n
    sub = np.arange(n) if n <= max_rows else np.random.default_rng(0).choice(n, max_rows, replace=False)
    mark = np.zeros(n, dtype=bool)
    mark[sub] = True
    extent = s.box if s.box is not None else np.ptp(s.pos, axis=0)
    extent = np.maximum(np.asarray(extent, dtype=float), 1e-300)
    R = 2.0 * (float(np.prod(extent)) / n) ** (1.0 / 3.0)
    diameter = float(np.linalg.norm(extent))
    while True:
        i, j = cell_list_pairs(s, R)
        keep = mark[i] | mark[j]
        if np.any(keep) or R > 2.0 * diameter:
            break
        R *= 2.0
    if not np.any(keep):
        return np.inf
    d = s.pos[j[keep]] - s.pos[i[keep]]
    if s.periodic:
        d -= s.box * np.round(d / s.box)
    return float(np.sqrt(np.min(np.einsum("ij,ij->i", d, d))))


def timescales(sim) -> dict:
    """Shortest characteristic times (s) of the physics on this path (accusim/advisor.py:9-44): the
    Lennard-Jones time sigma_ii sqrt(m_i / eps_ii) of each interacting species, and the closest approach over
    the fastest speed."""
    s = sim.system
    out = {}
    if s.n < 2:
        return out
    for f in sim.forces:
        if type(f).__name__ == "LennardJones":
            eps_t, sig_t = f._tables(s)
            for i, sp in enumerate(s.species):
                if eps_t[i, i] > 0:
                    t = sig_t[i, i] * np.sqrt(sp.mass / eps_t[i, i])
                    out["Lennard-Jones"] = min(out.get("Lennard-Jones", np.inf), float(t))
    speed = float(np.max(np.linalg.norm(s.vel, axis=1)))
    if speed > 0 and any(not f.external for f in sim.forces):
        eps2 = max([getattr(f, "eps2", 0.0) for f in sim.forces] or [0.0])
        out["closest approach / speed"] = float(np.sqrt(_closest_approach(s) ** 2 + eps2) / speed)
    return out


def richardson_check(finals, n, order) -> Check:
    """Observed order and Richardson estimate from finals at dt, dt/2, dt/4 (accusim/accuracy.py:207-221)."""
    size = max(float(np.ptp(finals[2])), 1e-300)
    roundoff = 1e-13 * np.sqrt(n * 4)
    e1 = float(np.sqrt(np.mean((finals[0] - finals[1]) ** 2))) / size
    e2 = float(np.sqrt(np.mean((finals[1] - finals[2]) ** 2))) / size
    if e1 < 10 * roundoff:
        return Check("timestep error", PASS, e1, "converged to floating-point round-off")
    p = np.log2(e1 / e2)
    est = e1 * 2 ** p / (2 ** p - 1) if p > 0.2 else e1
    if p < 0.5 * order:
        return Check("timestep error", FAIL if est > 1e-2 else WARN, est,
                     f"observed order {p:.1f} (expected {order}): chaotic or dt too large; trust statistics, "
                     "not trajectories")
    return Check("timestep error", _grade(est, 1e-6, 1e-3), est,
                 f"est. position error at dt (relative to system size), observed order {p:.1f}/{order}")


def suggest_dt(sim, steps_per_timescale: int = 100) -> float:
    """accusim/advisor.py:51-55: the shortest physical timescale divided by `steps_per_timescale`."""
    ts = timescales(sim)
    if not ts:
        raise ValueError("no timescale found; choose dt manually")
    return min(ts.values()) / steps_per_timescale


def timestep_convergence(sim, duration, start=None) -> Check:
    """Re-run from the initial state at dt, dt/2, dt/4 and estimate the error at dt
    (accusim/accuracy.py:191-221)."""
    if sim.integrator.stochastic or sim.reactions:
        return Check("timestep error", NA, None, "stochastic run: compare ensemble statistics instead")
    if start is None and hasattr(sim, "engine"):
        # device-resident simulation: the three runs advance together as one batch of replicas
        from .ensemble import timestep_check
        return timestep_check(sim, duration)
    base = start or sim._initial
    T = si(duration, "s")
    n = max(int(round(T / sim.dt)), 1)
    finals = []
    for k in (1, 2, 4):
        c = base.clone(dt=sim.dt / k)
        c.run(steps=n * k, record_every=10 ** 9, positions=False)
        finals.append(c.system.pos.copy())
    return richardson_check(finals, n, sim.integrator.order)


def calibrate_dt(sim, trial_duration, energy_tol=1e-6, max_halvings=12):
    """Halve dt until a trial run conserves energy to `energy_tol`; sets and returns (sim.dt, drift)
    (accusim/advisor.py:58-79)."""
    if sim.integrator.stochastic or sim.integrator.thermostat or not all(f.conservative for f in sim.forces):
        raise ValueError("calibrate_dt needs conservative, deterministic physics")
    T = si(trial_duration, "s")
    dt = sim.dt if sim.dt is not None else suggest_dt(sim)
    drift = float("nan")
    for _ in range(max_halvings + 1):
        trial = sim.clone(dt=dt)
        n = max(int(round(T / dt)), 1)
        tr = trial.run(steps=n, record_every=max(1, n // 200), positions=False)
        drift = energy_drift(tr)
        if drift <= energy_tol:
            sim.dt = dt
            return dt, drift
        dt /= 2
    raise RuntimeError(f"energy drift {drift:.2e} still above {energy_tol:.0e} after {max_halvings} halvings")
