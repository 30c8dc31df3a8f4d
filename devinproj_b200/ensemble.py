"""Batched independent replicas: ensembles, `calibrate_dt` halvings and Richardson dt / dt/2 / dt/4 triples
(accusim/advisor.py:58-79, accusim/accuracy.py:191-221) advanced together.

Every replica is one periodic system with its own atom count, box and dt; they share the force field. All of
them advance in one engine: per step one fused force/kick/drift launch over every replica's atoms (warps
never straddle replicas) and one cooperative list-maintenance launch that rebuilds only the replicas whose
skin test fired, both captured in a CUDA graph. Replicas with fewer steps left are switched off between
blocks (`set_active`).
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np

from ._accusim import accuracy as _acc
from .engine import ENERGY, LEN, MASS, VEL, start_engine
from .units import si


def drift_of(KE, PE):
    """The energy-drift metric accusim grades and calibrates dt on, max|E - E0| / max(|E0|, max|KE|, max|PE|)
    (accusim/accuracy.py:70-76, accusim/advisor.py:72-74), of one replica's recorded energies."""
    E = np.asarray(KE) + np.asarray(PE)
    scale = max(abs(E[0]), np.max(np.abs(KE)), np.max(np.abs(PE)), 1e-300)
    return float(np.max(np.abs(E - E[0])) / scale)


class _FinishedRuns:
    """A start state whose runs at dt, dt/2 and dt/4 were already made on the device (in one batched engine):
    `clone(dt)` hands back the finished run with that time step and its `run` does nothing. Given as `start`
    to accusim's own `timestep_convergence` (accusim/accuracy.py:191-221), it lets the reference compute the
    observed order and the Richardson estimate from the batched final positions."""

    def __init__(self, finals):
        self._finals = finals   # {dt: final positions}

    def clone(self, dt=None):
        return SimpleNamespace(system=SimpleNamespace(pos=self._finals[dt]), run=lambda **kw: None)


def richardson_check(finals, dt, duration, integrator):
    """accusim's `timestep_convergence` check for a trajectory whose dt, dt/2, dt/4 final positions are
    `finals` (the three runs advanced together on the device)."""
    view = SimpleNamespace(dt=dt, integrator=integrator, reactions=None)
    start = _FinishedRuns({dt / k: f for k, f in zip((1, 2, 4), finals)})
    return _acc.timestep_convergence(view, duration, start=start)


class ReplicaEnsemble:
    """Independent periodic systems advanced together. `systems` are this package's (or accusim's)
    `System` objects sharing species; `forces` a LennardJones and/or DampedShiftedCoulomb list; `dts` one
    time step per replica (s)."""

    def __init__(self, systems, forces, dts, maxnb=None, rec_cap=256, tpa=None):
        if len(systems) != len(dts):
            raise ValueError("one dt per replica")
        self.systems = list(systems)
        self.forces = list(forces)
        self.dts = [float(si(dt, "s")) for dt in dts]
        self.engine, self.rlist, self.half_skin = start_engine(self.systems, self.forces, self.dts, maxnb=maxnb,
                                                               rec_cap=rec_cap, tpa=tpa)
        self.R = len(self.systems)
        self.active = np.ones(self.R, dtype=np.int32)
        self.steps_done = np.zeros(self.R, dtype=np.int64)
        init = self.engine.records(1)[0]
        self.records = [[self._rec_si(init[r])] for r in range(self.R)]
        self.record_steps = [[0] for _ in range(self.R)]

    @staticmethod
    def _rec_si(rec):
        return np.concatenate([[rec[0] * ENERGY, rec[1] * ENERGY], rec[2:5] * (MASS * VEL), rec[5:8] * (MASS * VEL * LEN)])

    def set_active(self, mask):
        self.active = np.asarray(mask, dtype=np.int32)
        self.engine.set_active(self.active)

    def run(self, steps, record_every=0):
        """Advance the active replicas by `steps`; records (SI: KE, PE, P[3], L[3]) every `record_every` steps
        of this call and after its last step."""
        eng = self.engine
        done = 0
        re = int(record_every)
        while done < steps:
            span = steps - done
            if re > 0:
                span = min(span, re * max(1, min(eng.rec_cap - 1, 4000 // re)))
            else:
                span = min(span, 4000)
            last = done + span == steps
            eng.run(span, re, True)
            marks = list(range(re, span + 1, re)) if re > 0 else []
            if not marks or marks[-1] != span:
                marks.append(span)
            recs = eng.records(len(marks))
            eng.check("ensemble run")
            for r in np.flatnonzero(self.active):
                for j, rec in zip(marks, recs[:, r, :]):
                    self.records[r].append(self._rec_si(rec))
                    self.record_steps[r].append(int(self.steps_done[r] + done + j))
            done += span
            del last
        self.steps_done[self.active.astype(bool)] += steps

    def state(self):
        """Per-replica (pos, vel) in SI, positions wrapped into the box."""
        pos, vel, _ = self.engine.get_state()
        pos = pos.cpu().numpy() * LEN
        vel = vel.cpu().numpy() * VEL
        o = self.engine.offsets
        return [(pos[o[r]:o[r + 1]], vel[o[r]:o[r + 1]]) for r in range(self.R)]

    def energy_series(self, r, every=None):
        """(steps, KE, PE) of replica r, optionally subsampled to multiples of `every` plus the final record."""
        steps = np.array(self.record_steps[r])
        rec = np.array(self.records[r])
        if every:
            keep = (steps % every == 0) | (steps == steps[-1])
            steps, rec = steps[keep], rec[keep]
        return steps, rec[:, 0], rec[:, 1]

    def drift(self, r, every=None):
        _, ke, pe = self.energy_series(r, every)
        return drift_of(ke, pe)


def richardson_ensemble(systems, forces, dts, duration, integrator=None, tpa=None):
    """Richardson timestep error for each (system, dt) at once: 3 trajectories per input at dt, dt/2, dt/4
    over the same duration (n, 2n, 4n steps), all in one engine (accusim/accuracy.py:191-221).
    Returns one accusim `Check` per input (computed by accusim's `timestep_convergence` from the finals) and
    the ensemble."""
    T = float(si(duration, "s"))
    triples, tdts, ns = [], [], []
    for s, dt in zip(systems, dts):
        n = max(int(round(T / dt)), 1)
        ns.append(n)
        for k in (1, 2, 4):
            triples.append(s.copy())
            tdts.append(dt / k)
    ens = ReplicaEnsemble(triples, forces, tdts, tpa=tpa)
    R = len(triples)
    # lock-step phases: all for n steps; dt/2 and dt/4 for n more; dt/4 for 2n more (same duration T)
    # (inputs with different n run in further phases of their own step counts)
    remaining = np.array([ns[r // 3] * (1, 2, 4)[r % 3] for r in range(R)])
    while np.any(remaining > 0):
        act = remaining > 0
        step = int(np.min(remaining[act]))
        ens.set_active(act.astype(np.int32))
        ens.run(step, record_every=0)
        remaining[act] -= step
    finals = [p for p, _ in ens.state()]
    if integrator is None:
        from .integrators import VelocityVerlet
        integrator = VelocityVerlet()
    return [richardson_check(finals[3 * q: 3 * q + 3], dts[q], duration, integrator)
            for q in range(len(systems))], ens


def calibrate_dt_ensemble(system, forces, dt, trial_duration, energy_tol=1e-6, max_halvings=12, per_batch=3,
                          tpa=None):
    """calibrate_dt (accusim/advisor.py:58-79) with the halvings tried speculatively `per_batch` at a time
    in one engine. Returns (dt, drift) of the first dt in halving order whose trial run conserves energy to
    `energy_tol` -- the reference's answer -- or raises RuntimeError like the reference."""
    T = float(si(trial_duration, "s"))
    cands = [dt / 2 ** k for k in range(max_halvings + 1)]
    drift = float("nan")
    for b0 in range(0, len(cands), per_batch):
        batch = cands[b0:b0 + per_batch]
        ns = [max(int(round(T / d)), 1) for d in batch]
        res = [max(1, n // 200) for n in ns]
        ens = ReplicaEnsemble([system.copy() for _ in batch], forces, batch, tpa=tpa)
        every = math.gcd(*res)
        remaining = np.array(ns)
        while np.any(remaining > 0):
            act = remaining > 0
            step = int(np.min(remaining[act]))
            if every > 0 and step > every:
                step = step // every * every
            ens.set_active(act.astype(np.int32))
            ens.run(step, record_every=every)
            remaining[act] -= step
        for k, d in enumerate(batch):
            drift = ens.drift(k, every=res[k])
            if drift <= energy_tol:
                return d, drift
    raise RuntimeError(f"energy drift {drift:.2e} still above {energy_tol:.0e} after {max_halvings} halvings")


def timestep_check(sim, duration, tpa=None):
    """`timestep_convergence` (accusim/accuracy.py:191-221) for one simulation from its initial state, the three
    runs batched in one engine."""
    if sim.integrator.stochastic or sim.reactions:
        return _acc.timestep_convergence(sim, duration)
    base = getattr(sim, "_initial", None)
    system = base.system if base is not None else sim.system
    checks, _ = richardson_ensemble([system], sim.forces, [sim.dt], duration, integrator=sim.integrator, tpa=tpa)
    return checks[0]


__all__ = ["ReplicaEnsemble", "richardson_ensemble", "calibrate_dt_ensemble", "timestep_check", "drift_of"]
