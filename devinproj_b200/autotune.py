"""Launch-shape autotuner for the engine: threads per atom in the pair kernel (1..32, which also fixes the
neighbour-list layout) and the step kernel's grid: one thread per slot (`grid_mult` 0), or k blocks per SM that
loop over the slots (`grid_mult` 4 or 8), which trades the last wave's tail for a loop.

`tune()` builds the engine for each candidate on the caller's own replicas, times a short eager run with
CUDA events around every kernel (`acs_engine_run_timed`), and keeps the fastest step + list-maintenance
time. Results are cached per workload signature (atom count and replica count buckets, list radius and
density) in a JSON file ($ACS_AUTOTUNE_CACHE, default ~/.cache/accusim_b200/autotune.json).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

CACHE = os.environ.get("ACS_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "accusim_b200",
                                                          "autotune.json"))


def forcefield_tag(forces):
    """The force terms a workload evaluates (they change the pair kernel's cost per entry): lj, dsf, and dsf with
    exclusions."""
    from ._accusim import forces as _af
    tags = []
    for f in forces:
        if isinstance(f, _af.LennardJones):
            tags.append("lj")
        elif isinstance(f, _af.DampedShiftedCoulomb):
            tags.append("dsfx" if f.exclude else "dsf")
    return "+".join(sorted(tags))


def device_tag():
    """The GPU the timings were taken on (a tuned launch shape is not carried over to another model)."""
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name().replace(" ", "-")
    except Exception:
        pass
    return "nodevice"


def signature(systems, rlist, forces=(), device=None):
    n = sum(s.n for s in systems)
    vol = sum(float(np.prod(s.box)) for s in systems)
    rho_nb = n / vol * 4.0 / 3.0 * math.pi * rlist ** 3     # neighbours per atom inside the list radius
    bucket = lambda x: float(f"{x:.2g}")                    # noqa: E731
    dev = device if device is not None else device_tag()
    return (f"n{bucket(n)}_r{len(systems)}_nb{bucket(rho_nb)}_sp{len(systems[0].species)}"
            f"_ff{forcefield_tag(forces) or 'none'}_{dev}")


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(db):
    try:
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        with open(CACHE + ".tmp", "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
        os.replace(CACHE + ".tmp", CACHE)
    except OSError:
        pass


def candidates(n_total, nb):
    tpas = [t for t in (1, 2, 4, 8, 16, 32) if t * 2 <= max(nb, 2)]   # at least two list entries per lane
    if n_total > 2_000_000:
        tpas = [t for t in tpas if t <= 4]
    grids = [0, 4, 8]
    return [(t, g) for t in tpas for g in grids]


def tune(systems, forces, dts, steps=30, use_cache=True, verbose=False):
    """Best (tpa, grid_mult) for these replicas. Runs the engine a few steps per candidate on the GPU."""
    from .engine import forcefield_from, start_engine
    _, rlist, _ = forcefield_from(forces, systems[0].species)
    key = signature(systems, rlist, forces)
    db = _load() if use_cache else {}
    if key in db:
        return tuple(db[key]["best"])
    n_total = sum(s.n for s in systems)
    vol = sum(float(np.prod(s.box)) for s in systems)
    nb = n_total / vol * 4.0 / 3.0 * math.pi * rlist ** 3
    results = {}
    for tpa, gm in candidates(n_total, nb):
        eng, _, _ = start_engine([s.copy() for s in systems], forces, dts, tpa=tpa, grid_mult=gm)
        eng.run(5, 0, True)
        k_ms, r_ms, tot = eng.run_timed(steps, 0)
        eng.check("autotune")
        results[f"{tpa},{gm}"] = tot / steps
        if verbose:
            print(f"autotune {key}: tpa={tpa} grid_mult={gm}: {tot / steps:.4f} ms/step "
                  f"(pair {k_ms:.4f}, list {r_ms:.4f})")
        del eng
    best = min(results, key=results.get)
    tpa, gm = (int(x) for x in best.split(","))
    db[key] = {"best": [tpa, gm], "ms_per_step": results}
    if use_cache:
        _store(db)
    return tpa, gm
