"""Launch-shape autotuner for the engine: threads per atom in the pair kernel (1..32, which also fixes the
neighbour-list layout), the step kernel's grid (one thread per slot, `grid_mult` 0, or k blocks per SM that
loop over the slots, `grid_mult` 4 or 8, which trades the last wave's tail for a loop), and the list build's
cell edge (`cell_scale` x the list radius: wider cells give a warp more home atoms per cell and more candidates
per stencil; on small boxes they leave axes with fewer than three cells, which the list build then walks a warp
per atom).

`tune()` builds the engine for each candidate on the caller's own replicas, times a short eager run with
CUDA events around every kernel (`acs_engine_run_timed`), and keeps the fastest step + list-maintenance
time: first every (threads per atom, step grid) pair at the narrowest cells, then the wider cell edges for the
best pair. Results are cached per workload signature (atom count and replica count buckets, list density, force
terms, GPU model) in a JSON file ($ACS_AUTOTUNE_CACHE, default ~/.cache/accusim_b200/autotune.json).
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


CELL_SCALES = (1.0, 1.25, 1.5)   # cell edge / list radius, searched after the (threads per atom, grid) pair


def candidates(n_total, nb):
    tpas = [t for t in (1, 2, 4, 8, 16, 32) if t * 2 <= max(nb, 2)]   # at least two list entries per lane
    if n_total > 2_000_000:
        tpas = [t for t in tpas if t <= 4]
    grids = [0, 4, 8]
    return [(t, g) for t in tpas for g in grids]


def _label(tpa, gm, cs):
    return f"{tpa},{gm},{cs:g}"


def _best(entry):
    """(tpa, grid_mult, cell_scale) of a cache entry (entries without a cell edge were tuned at 1)."""
    b = entry["best"]
    return int(b[0]), int(b[1]), float(b[2]) if len(b) > 2 else 1.0


def tune(systems, forces, dts, steps=30, use_cache=True, verbose=False):
    """Best (tpa, grid_mult, cell_scale) for these replicas. Runs the engine a few steps per candidate on the
    GPU."""
    from .engine import forcefield_from, start_engine
    _, rlist, _ = forcefield_from(forces, systems[0].species)
    key = signature(systems, rlist, forces)
    db = _load() if use_cache else {}
    if key in db:
        return _best(db[key])
    n_total = sum(s.n for s in systems)
    vol = sum(float(np.prod(s.box)) for s in systems)
    nb = n_total / vol * 4.0 / 3.0 * math.pi * rlist ** 3
    results = {}

    def measure(tpa, gm, cs):
        eng, _, _ = start_engine([s.copy() for s in systems], forces, dts, tpa=tpa, grid_mult=gm, cell_scale=cs)
        eng.run(5, 0, True)
        k_ms, r_ms, tot = eng.run_timed(steps, 0)
        eng.check("autotune")
        results[_label(tpa, gm, cs)] = tot / steps
        if verbose:
            print(f"autotune {key}: tpa={tpa} grid_mult={gm} cell_scale={cs:g}: {tot / steps:.4f} ms/step "
                  f"(pair {k_ms:.4f}, list {r_ms:.4f})")
        del eng
        return tot / steps

    shapes = {(tpa, gm): measure(tpa, gm, CELL_SCALES[0]) for tpa, gm in candidates(n_total, nb)}
    tpa, gm = min(shapes, key=shapes.get)
    for cs in CELL_SCALES[1:]:
        measure(tpa, gm, cs)
    best = min(results, key=results.get)
    t, g, c = best.split(",")
    db[key] = {"best": [int(t), int(g), float(c)], "ms_per_step": results}
    if use_cache:
        _store(db)
    return int(t), int(g), float(c)
