"""Benchmark: LJ/DSF atom-steps/s on one B200 at stated energy drift vs the FP64 path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload lj1m|nacl4096|argon864] [--impl ours|reference]

Default workload: 1,048,576-atom LJ fluid (fcc 64^3, rho* 0.8442, T* 0.72, rc 2.5 sigma, skin 0.3 sigma,
dt* 0.005), FP32-compensated pair forces with FP64 integration, the step loop as CUDA graphs. A step is
one VelocityVerlet step of the whole system (forces, both kicks, drift, skin test, list rebuilds when due).
Inputs (positions, velocities, 400+ MB of neighbour lists) exceed the 126 MB L2, so no flush is needed.
Under torchrun each rank advances its own independent system (replicas only; no collective in the step
loop), or, for the replica ensemble, its shard of the replicas; rank 0 prints one JSON line. The line also
carries the energy drift of a fixed 10^4-step window and the throughput of the plain FP64 plug-ins running
device-resident inside accusim's own Simulation.run (the denominator of the FP32c path's speed-up), and, for
the 1M-atom workload, the learned DSF->Ewald correction's step overhead and held-out accuracy (8000-ion melt).
`--impl reference` times the unmodified reference (accusim, installed under baseline/_ref) on this host's
cores (all of them, one process each) for the same metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LJ/DSF atom-steps/s on 1 B200 at stated energy drift vs FP64 oracle"
UNIT = "atom-steps/s"
BYTES_PER_ATOM_STEP = 128        # FP64 x, v read+write (96 B) + FP32 image write+read (32 B)
FLOP_PER_PAIR = {"lj": 40, "dsf": 70}
FALLBACK_HBM_GBS = 6650.0


def workload(name, seed=0):
    from devinproj_b200 import configs
    cfg = workload_meta(name)
    if name == "ensemble":
        nc = configs.replica_sizes(256, seed=seed)
        systems, dts = [], []
        for k, c in enumerate(nc):
            sys_k, lj = configs.lj_fluid(int(c), seed=1000 * seed + k)
            for f in (1, 2, 4):
                systems.append(sys_k.copy())
                dts.append(0.005 * configs.AR_TAU / f)
        return systems, [lj], dts, cfg
    if name == "lj1m":
        s, forces, dt = configs.lj_large(64, seed=seed)
    elif name == "nacl4096":
        s, forces, dt = configs.nacl4096(seed=seed)
    else:
        s, forces, dt = configs.argon864(seed=seed)
    return s, forces, dt, cfg


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": FALLBACK_HBM_GBS}, "fallback"


def reference_package():
    """accusim, the unmodified reference (pure Python), from the repository's offline install under
    baseline/_ref (baseline/install_reference.sh) or the environment."""
    ref = os.path.join(ROOT, "baseline", "_ref")
    if os.path.isdir(os.path.join(ref, "accusim")) and ref not in sys.path:
        sys.path.insert(0, ref)
    import accusim
    return accusim


def reference_lj_fluid(accusim, n_cells, seed=0, rho_star=0.8442, T_star=0.72):
    """The benchmark's LJ fluid built with accusim's own API only (no code of this repository): argon fcc
    n_cells^3 (basis of examples/rahman_argon.py:23-27), rho* 0.8442, Maxwell-Boltzmann at T* with
    default_rng(seed), LennardJones cutoff 2.5 skin 0.3, VelocityVerlet at dt* 0.005. The same state as
    devinproj_b200.configs.lj_fluid builds."""
    import numpy as np
    sig, eps_k, m = 3.4e-10, 120.0, accusim.Q(39.948, "u").value
    n = 4 * n_cells ** 3
    L = (n / rho_star) ** (1 / 3) * sig
    s = accusim.System(3, box=L, periodic=True)
    s.add_species("Ar", m)
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) + 0.25
    g = np.stack(np.meshgrid(*[np.arange(n_cells)] * 3, indexing="ij"), -1).reshape(-1, 1, 3)
    s.add("Ar", ((g + base[None]).reshape(-1, 3)) * L / n_cells)
    s.maxwell_boltzmann(T_star * eps_k, np.random.default_rng(seed))
    eps = eps_k * accusim.k_B.value
    lj = accusim.LennardJones({"Ar": (eps, sig)}, cutoff=2.5, skin=0.3)
    tau = sig * math.sqrt(m / eps)
    return accusim.Simulation(s, [lj], integrator=accusim.VelocityVerlet(), dt=0.005 * tau)


def _reference_seconds_per_atom_step():
    """The reference's NumPy cost per atom-step on this host, from 2 steps of a 2,048-atom sample (one core)."""
    accusim = reference_package()
    sim = reference_lj_fluid(accusim, 8, seed=1)
    sim.run(steps=1, record_every=10 ** 9, positions=False)
    t0 = time.perf_counter()
    sim.run(steps=2, record_every=10 ** 9, positions=False)
    return (time.perf_counter() - t0) / (2 * sim.system.n)


def cpu_baseline_reference(budget_s=15.0):
    """The unmodified reference (accusim's Simulation.run, NumPy FP64, one core) on a 32,000-atom sample of the
    same fluid, timed after one warm-up step."""
    accusim = reference_package()
    sim = reference_lj_fluid(accusim, 20, seed=0)
    sim.run(steps=1, record_every=10 ** 9, positions=False)
    t0 = time.perf_counter()
    sim.run(steps=1, record_every=10 ** 9, positions=False)
    t1 = time.perf_counter() - t0
    m = int(max(3, min(60, budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    sim.run(steps=m, record_every=10 ** 9, positions=False)
    dt = time.perf_counter() - t0
    return {"value": sim.system.n * m / dt, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"accusim (unmodified, baseline/_ref) Simulation.run, NumPy FP64 cell/Verlet list, 32000-atom "
                      f"fcc 20^3 at rho* 0.8442 T* 0.72, rc 2.5 skin 0.3, {m} steps after 2 warm-up steps, 1 process; "
                      f"the per-atom-step cost is nearly size-independent (8.4e4 atom-steps/s at 32k, 7.9e4 at 1M "
                      f"measured on one core)"}


def _ref_worker(args):
    nc, steps, warmup, seed = args
    accusim = reference_package()
    sim = reference_lj_fluid(accusim, nc, seed=seed)
    sim.run(steps=max(warmup, 1), record_every=10 ** 9, positions=False)
    t0 = time.perf_counter()
    sim.run(steps=steps, record_every=10 ** 9, positions=False)
    return sim.system.n * steps, time.perf_counter() - t0


def reference_arm(args, cfg):
    """The reference's own CPU path (accusim from baseline/_ref, unmodified, through Simulation.run) on all host
    cores: one process per core, each an independent fcc sample of the workload's fluid sized so that the
    --warmup + --steps steps take about 150 s. The NumPy cost per atom-step hardly depends on the size (8.4e4 vs
    7.9e4 atom-steps/s at 32k and 1M atoms on one core), so the summed atom-steps/s of the samples stand for the
    full-size run, which the reference cannot run 16 times at once (27 GB and 13 s per step each)."""
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    per_atom_step_s = _reference_seconds_per_atom_step()
    budget = 150.0
    n_target = budget / max(args.steps + args.warmup, 1) / per_atom_step_s
    nc = int(max(4, min(20, math.floor((n_target / 4) ** (1 / 3)))))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_ref_worker, [(nc, args.steps, args.warmup, 100 + k) for k in range(cores)])
    wall = time.perf_counter() - t0
    work = sum(r[0] for r in res)
    span = max(r[1] for r in res)
    value = work / span
    sample = (f"accusim (unmodified reference from baseline/_ref) Simulation.run, NumPy FP64, {cores} processes x "
              f"fcc {nc}^3 ({4 * nc ** 3} atoms, sized from a measured {per_atom_step_s * 1e6:.1f} us per atom-step) "
              f"at rho* 0.8442 T* 0.72, rc 2.5 skin 0.3, {args.steps} timed steps after {args.warmup} warm-up "
              f"(wall {wall:.0f} s); atom-steps/s of independent samples of the workload's fluid, summed")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * span / args.steps,
            "higher_is_better": True, "scaling": "strong" if args.workload == "ensemble" else "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bind_to_gpu_local_cores(local):
    """Run this process on the cores NVML reports as closest to its GPU, so that the pinned host buffers of the
    end-to-end leg (first touch) sit on the GPU's NUMA node. Affects this process only; returns the number of
    cores, or None when NVML cannot tell."""
    try:
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        words = pynvml.nvmlDeviceGetCpuAffinity(h, ((os.cpu_count() or 64) + 63) // 64)
        cpus = {64 * w + b for w, word in enumerate(words) for b in range(64) if (int(word) >> b) & 1}
        cpus &= set(os.sched_getaffinity(0))
        if not cpus:
            return None
        os.sched_setaffinity(0, cpus)
        return len(cpus)
    except Exception:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--workload", default="lj1m")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--record-every", type=int, default=100)
    ap.add_argument("--drift-steps", type=int, default=None,
                    help="length of the energy-drift window run after the timed region (default 10000; 2000 for the "
                         "ensemble; 0 skips it)")
    ap.add_argument("--drift-equil", type=int, default=2000,
                    help="steps run before the drift window opens (the fcc lattice start melts first)")
    ap.add_argument("--fp64-steps", type=int, default=300,
                    help="steps of the plain FP64 plug-ins (device-resident GpuSystem in accusim's Simulation.run) "
                         "timed for the speed-up denominator; 0 skips them")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--learned-snapshots", type=int, default=2000,
                    help="1M-atom line only: snapshots of the learned correction's held-out accuracy leg (8000-ion "
                         "melt, ~45 s); 0 skips it")
    ap.add_argument("--cell-order", type=int, default=1, choices=[0, 1],
                    help="slot order of the cells: 1 Morton (default), 0 row-major")
    ap.add_argument("--cell-scale", type=float, default=1.0,
                    help="cell edge of the list build in list radii (1..8; default 1, the narrowest complete stencil)")
    ap.add_argument("--tpa", default=None, help="threads per atom in the pair kernel: 1..32, 'auto' (timed "
                    "autotuner), default: size heuristic")
    ap.add_argument("--experiment", choices=["learned", "drift", "dropin", "correction_kernels", "autotune"],
                    default=None,
                    help="accuracy experiments (one JSON line each): the learned DSF->Ewald correction at full scale, "
                         "the 1e4-step energy drift of the 1M-atom run, the plain FP64 drop-in's throughput")
    ap.add_argument("--snapshots", type=int, default=2000)
    ap.add_argument("--train-configs", default="20:2e-3",
                    help="learned experiment: comma-separated epochs:learning-rate settings, chosen on a validation "
                         "split when there are several")
    ap.add_argument("--profile", action="store_true",
                    help="engine only: warm-up graph steps then --steps eager launches (for ncu), no timing legs")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.tpa not in (None, "auto"):
        args.tpa = int(args.tpa)
    if args.drift_steps is None:
        args.drift_steps = 2000 if args.workload == "ensemble" else 10000

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, full_config(workload_meta(args.workload), args, world))
        return
    if args.experiment:
        run_experiment(args)
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    host_cores = bind_to_gpu_local_cores(local) if not args.profile else None
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from devinproj_b200.engine import ACC, LEN, VEL, start_engine

    ensemble = args.workload == "ensemble"
    # the replica ensemble is one workload sharded over the ranks (largest replica first to the least-loaded
    # rank, no collective while stepping); the single-system workloads run one independent copy per rank
    s, forces, dt, cfg = workload(args.workload, seed=0 if ensemble else rank)
    systems, dts = (s, dt) if isinstance(s, list) else ([s], [dt])
    n_global = sum(x.n for x in systems)
    shard = list(range(len(systems)))
    if ensemble and world > 1:
        from devinproj_b200.sharding import shard_replicas
        shard = shard_replicas([x.n for x in systems], world)[rank]
        systems, dts = [systems[r] for r in shard], [dts[r] for r in shard]
    rec_cap = max(args.steps // args.record_every + 2, args.drift_steps // args.record_every + 2, 4)
    eng, rlist, hs = start_engine(systems, forces, dts, rec_cap=rec_cap, tpa=args.tpa, cell_order=args.cell_order,
                                  cell_scale=args.cell_scale)
    n = sum(x.n for x in systems)
    pairs_lj, pairs_dsf = eng.count_pairs()
    step_blocks, coop_blocks, slots = eng.launch_info()
    stream = torch.cuda.current_stream()
    if args.profile:
        eng.run(args.warmup, 0, True)
        torch.cuda.synchronize()
        rb0 = eng.status().rebuilds
        eng.phase_times(clear=True)
        k_ms, r_ms, tot = eng.run_timed(args.steps, 0)
        eng.check("profile")
        nreb = eng.status().rebuilds - rb0
        ph = {k: round(v / max(nreb, 1), 4) for k, v in eng.phase_times().items()}
        print(json.dumps({"profile": cfg["workload"], "tpa": eng.tpa, "cell_scale": eng.cell_scale,
                          "step_kernel_ms": k_ms, "list_kernel_ms": r_ms,
                          "rebuilds": nreb, "ms_per_rebuild_by_phase": ph, "pairs_lj": pairs_lj,
                          "pairs_dsf": pairs_dsf, "maxnb": eng.maxnb, "neighbors": eng.neighbor_stats()}))
        return

    # warm-up (also instantiates the timed graph's sibling shapes)
    eng.run(args.warmup, 0, True)
    torch.cuda.synchronize()
    eng.check("warm-up")

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world > 1:
            t = torch.tensor([x], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    # ---------------------------------------------------------------- timed region (device events)
    eng.run(args.steps, args.record_every, True)   # instantiate the graph outside the timed region
    torch.cuda.synchronize()
    eng.check("graph warm-up")
    rb0 = eng.status().rebuilds
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.25)
        barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e0.record(stream)
        eng.run(args.steps, args.record_every, True)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        wall = time.perf_counter() - w0
    ms = max_over_ranks(e0.elapsed_time(e1))
    st = eng.check("timed run")
    nrec = args.steps // args.record_every + (1 if args.steps % args.record_every else 0)
    recs_all = eng.records(nrec)                     # (records, replicas, 8), engine units
    rebuilds_timed = st.rebuilds - rb0
    # weak scaling: every rank advances its own copy; the ensemble: the ranks share one fixed set of replicas
    total_atoms = n_global if ensemble else n * world
    value = total_atoms * args.steps / (ms / 1e3)

    # momentum over the timed run (the report's metric), worst replica
    pos_d, vel_d, acc_d = eng.get_state()
    vel_np = vel_d.cpu().numpy() * VEL
    mom_drift = 0.0
    for r in range(len(systems)):
        sr = systems[r]
        o0, o1 = eng.offsets[r], eng.offsets[r + 1]
        m_r = np.array([x.mass for x in sr.species])[sr.sp]
        pscale = float(np.sum(m_r[:, None] * np.abs(vel_np[o0:o1])))
        P = recs_all[:, r, 2:5] * (1.66053906660e-27 * VEL)
        mom_drift = max(mom_drift, float(np.max(np.linalg.norm(P - P[0], axis=1)) / pscale))

    # ---------------------------------------------------------------- per-kernel timing (eager, events)
    k_step_ms, k_reb_ms, _ = eng.run_timed(min(args.steps, 1000), args.record_every)
    torch.cuda.synchronize()
    eng.check("timed eager run")

    # ---------------------------------------------------------------- accuracy vs the FP64 path
    # FP64 forces on the final state by the drop-in kernels (pinned to the reference to 1e-12); the largest
    # replica when there are several
    pos_d, vel_d, acc_d = eng.get_state()
    vel_np = vel_d.cpu().numpy() * VEL
    r_chk = int(np.argmax([x.n for x in systems]))
    sr = systems[r_chk].copy()
    o0, o1 = eng.offsets[r_chk], eng.offsets[r_chk + 1]
    sr.pos = pos_d.cpu().numpy()[o0:o1] * LEN
    sr.vel = vel_np[o0:o1]
    m_r = np.array([x.mass for x in sr.species])[sr.sp]
    F32 = acc_d.cpu().numpy()[o0:o1] * ACC * m_r[:, None]
    F64 = np.zeros_like(F32)
    for f in forces:
        Fi, _ = f.compute(sr)
        F64 += Fi
    f_err = float(np.sqrt(np.mean(np.sum((F32 - F64) ** 2, 1)) / np.mean(np.sum(F64 ** 2, 1))))

    # ---------------------------------------------------------------- energy drift over a fixed window
    # the report's metric max|E - E0| / max(|E0|, max|KE|, max|PE|) (accusim/accuracy.py:70-76) over
    # --drift-steps steps from the current state, E recorded at the window's start and every record_every steps
    drift = slope_rel = None
    drift_ms = None
    if args.drift_steps > 0:
        # steps taken so far: warm-up, graph warm-up, timed run, per-kernel timing; equilibrate up to --drift-equil
        done = args.warmup + 2 * args.steps + min(args.steps, 1000)
        eng.run(max(args.drift_equil - done, 0) + 1, 0, True)   # its last step is recorded: the window's start
        start = eng.records(1)[0].copy()
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        d0.record(stream)
        eng.run(args.drift_steps, args.record_every, True)
        d1.record(stream)
        torch.cuda.synchronize()
        eng.check("drift window")
        drift_ms = d0.elapsed_time(d1)
        nrec_d = args.drift_steps // args.record_every + (1 if args.drift_steps % args.record_every else 0)
        recs = np.concatenate([start[None], eng.records(nrec_d)])          # (1 + records, replicas, 8)
        steps_at = np.concatenate([[0], np.minimum(np.arange(1, nrec_d + 1) * args.record_every, args.drift_steps)])
        drift = slope_rel = 0.0
        for r in range(len(systems)):
            KE, PE = recs[:, r, 0], recs[:, r, 1]
            E = KE + PE
            scale = max(abs(E[0]), np.max(np.abs(KE)), np.max(np.abs(PE)))
            drift = max(drift, float(np.max(np.abs(E - E[0])) / scale))
            slope_rel = max(slope_rel, abs(float(np.polyfit(steps_at, E, 1)[0])) / scale)
        drift = max_over_ranks(drift)
        slope_rel = max_over_ranks(slope_rel)

    # ---------------------------------------------------------------- end to end (host buffers)
    pos_d, vel_d, _ = eng.get_state()          # the current state is the first step's input
    pos_h = (pos_d.cpu() * 1.0).pin_memory()
    vel_h = vel_d.cpu().pin_memory()
    out_p = torch.empty_like(pos_h).pin_memory()
    out_v = torch.empty_like(vel_h).pin_memory()
    dev_p = torch.empty_like(pos_d)
    dev_v = torch.empty_like(vel_d)
    eng.run(1, 0, True)
    torch.cuda.synchronize()
    barrier()
    w0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        dev_p.copy_(pos_h, non_blocking=True)
        dev_v.copy_(vel_h, non_blocking=True)
        eng.load_state(dev_p, dev_v)
        eng.run(1, 0, True)
        p, v, _ = eng.get_state()
        out_p.copy_(p, non_blocking=True)
        out_v.copy_(v, non_blocking=True)
        rec = eng.records(1)           # the step's energies: synchronises
        pos_h, out_p = out_p, pos_h
        vel_h, out_v = out_v, vel_h
    torch.cuda.synchronize()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - w0)
    e2e_val = total_atoms * args.e2e_steps / e2e_s
    eng.check("e2e")
    del rec

    # ---------------------------------------------------------------- the plain FP64 GPU drop-in
    fp64 = None
    if args.fp64_steps > 0 and not ensemble:
        fp64 = secondary_leg(fp64_dropin_device_resident, args, local, stream)
    learned = secondary_leg(learned_correction_cost, stream) if args.workload == "lj1m" and world == 1 else None
    learned_acc = (secondary_leg(learned_correction_accuracy, args.learned_snapshots)
                   if args.workload == "lj1m" and world == 1 and args.learned_snapshots > 0 else None)
    del eng

    peaks, peak_kind = measured_peaks()
    clocks = clk.summary()
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    mhz = clocks["sm_mhz"] or peaks.get("clocks_under_load", {}).get("sm_mhz_median") or 1965.0
    fp32_peak = sms * 128 * 2 * mhz * 1e6 / 1e12
    alg_bytes = BYTES_PER_ATOM_STEP * n
    achieved_gbs = alg_bytes / (k_step_ms / 1e3) / 1e9
    flops = FLOP_PER_PAIR["lj"] * pairs_lj + FLOP_PER_PAIR["dsf"] * pairs_dsf
    achieved_tf = flops / (k_step_ms / 1e3) / 1e12
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(cfg["workload"])
        except ValueError:
            traffic = None
    launches = 2 + 2 * args.steps
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if ensemble else "weak",
        "vs_baseline": None, "dtype": "fp32-pairs/f64-state", "data": "synthetic (seeded fcc lattice, MB velocities)",
        "config": full_config(cfg, args, world),
        "accuracy": {"force_rms_rel_err_vs_fp64": f_err,
                     "energy_drift_report_metric": drift, "energy_drift_window_steps": args.drift_steps,
                     "energy_drift_10k": drift if args.drift_steps == 10000 else None,
                     "energy_drift_window_start_step": max(args.drift_equil,
                                                           args.warmup + 2 * args.steps + min(args.steps, 1000)) + 1,
                     "energy_drift_linear_per_step_rel": slope_rel, "energy_drift_window_ms": drift_ms,
                     "drift_note": ("report metric max|E-E0|/scale over a fixed window that opens after the fcc "
                                    "lattice start has melted (window_start_step), E recorded at its start and every "
                                    f"{args.record_every} steps; from the lattice start the FP64 plug-ins drift as "
                                    "much as this path (bench.py --experiment drift); "
                                    + ("max over replicas and ranks" if len(systems) > 1 or world > 1
                                       else "single system")),
                     "momentum_drift_report_metric": mom_drift, "momentum_window_steps": args.steps,
                     "rebuilds_in_timed_region": int(rebuilds_timed)},
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved_gbs / peaks["hbm_gbs"], "traffic": traffic, "kernel": "k_step",
                     "kernel_ms": k_step_ms, "list_kernel_ms": k_reb_ms, "peak_source": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "fp32": {"achieved_tflops": achieved_tf, "peak_tflops": fp32_peak,
                              "frac": achieved_tf / fp32_peak, "pairs_lj": pairs_lj, "pairs_dsf": pairs_dsf,
                              "peak_basis": f"{sms} SMs x 128 FP32 lanes x 2 x {mhz:.0f} MHz (sampled median)"}},
        "clocks": clocks,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 48 * n, "d2h_bytes_per_step": 48 * n + 64,
                "steps": args.e2e_steps, "path": "pinned host pos/vel -> acs_engine_load_state -> 1 step graph -> "
                                                  "acs_engine_get_state -> pinned host + energy record",
                "host_cores": host_cores},
        "gpu_launches": launches,
        "wall_s_timed": wall,
    }
    if ensemble:
        line["sharding"] = {"replicas": len(shard) if world == 1 else None, "replicas_total": 768,
                            "this_rank_replicas": len(shard), "this_rank_atoms": n, "atoms_total": n_global,
                            "rule": "largest replica first to the least-loaded rank; no collective while stepping"}
    if fp64 is not None and "value" in fp64:
        fp64["fp32c_over_fp64"] = (value / world) / fp64["value"]
        line["fp64_dropin_device_resident"] = fp64
    if learned is not None:
        line["learned_correction_cost"] = learned
    if learned_acc is not None:
        line["learned_correction_accuracy"] = learned_acc
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = secondary_leg(cpu_baseline_reference)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def learned_correction_cost(stream, steps=200):
    """Step time of the 8000-ion NaCl melt (LJ + DSF, rc 10 A) in the graph, plain and with the learned
    DSF->Ewald correction (descriptors + tensor-core MLP) refreshed every step and every 10th step. The kernels'
    work does not depend on the weights, so an untrained network stands in for the trained one here; the
    correction's accuracy is the separate held-out leg (`learned_correction_accuracy`)."""
    import torch

    from devinproj_b200 import GpuSimulation, configs
    from devinproj_b200.learned import LearnedCorrection
    s, forces, dt = configs.nacl8000()
    plain = GpuSimulation(s.copy(), forces, dt=dt)
    corr = GpuSimulation(s.copy(), forces, dt=dt, correction=LearnedCorrection(seed=0), validate_every=0)

    def graph_ms(engine):
        engine.run(steps, 0, True)           # the block's graph is captured here
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        engine.run(steps, 0, True)
        b.record(stream)
        torch.cuda.synchronize()
        engine.check("learned correction timing")
        return a.elapsed_time(b) / steps

    out = {"ions": s.n, "plain_ms_per_step": graph_ms(plain.engine)}
    for stride in (1, 10):
        corr.engine.set_correction_stride(stride)
        out[f"corrected_ms_per_step_stride{stride}"] = graph_ms(corr.engine)
        out[f"overhead_stride{stride}"] = out[f"corrected_ms_per_step_stride{stride}"] / out["plain_ms_per_step"] - 1
    return out


def secondary_leg(fn, *args):
    """One of the line's secondary measurements (taken after the headline figures): an exception is reported in
    the line as {"error": ...}, with its traceback on stderr, instead of ending the run."""
    try:
        return fn(*args)
    except Exception as exc:   # noqa: BLE001 - any failure of a secondary leg is reported, not raised
        import traceback
        traceback.print_exc(file=sys.stderr)
        return {"error": f"{type(exc).__name__}: {exc}"[:300]}


def learned_correction_accuracy(snapshots, epochs=20, lr=2e-3):
    """Held-out accuracy of the learned DSF->Ewald correction on the 8000-ion NaCl melt, the same recipe
    as `--experiment learned` with one training setting: `snapshots` seeded snapshots (Langevin melt at 4000 K,
    cooled to 1300 K, sampled every 20 NVE steps, labels device Ewald minus FP64 DSF), trained on the first 90%
    and scored on the last 10%, which training never sees (RMS relative force error against Ewald)."""
    import numpy as np
    import torch

    from devinproj_b200.learned import LearnedCorrection, generate_dataset
    t0 = time.perf_counter()
    d = generate_dataset(snapshots, seed=0, n_sites=20, verbose=False)
    t_gen = time.perf_counter() - t0
    n_train = int(0.9 * snapshots)
    t0 = time.perf_counter()
    lc = LearnedCorrection(seed=0)
    hist = lc.train(d, np.arange(n_train), epochs=epochs, batch_tiles=64, lr=lr)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    e_dsf, e_corr = lc.errors(d, np.arange(n_train, snapshots))
    return {"ions": 8000, "snapshots": snapshots, "train_snapshots": n_train, "heldout_snapshots": snapshots - n_train,
            "epochs": epochs, "lr": lr, "train_loss_first_last": [hist[0], hist[-1]],
            "heldout_rms_rel_err_dsf": e_dsf, "heldout_rms_rel_err_corrected": e_corr, "error_ratio": e_dsf / e_corr,
            "dataset_s": t_gen, "train_s": t_train}


def fp64_dropin_device_resident(args, local, stream):
    """Throughput of the plain FP64 GPU plug-ins (LennardJones / DampedShiftedCoulomb / VelocityVerlet) inside
    accusim's own Simulation.run on a device-resident GpuSystem of the same workload: per step the FP64 kick,
    drift and wrap kernels, the FP64 pair kernel over the device Verlet list (rebuilt on the device when the
    skin test fires), the closing kick, and the potential-energy read-back that accusim's Simulation contract
    needs every step; the state crosses PCIe only at records (one at the end of the timed call). Timed with
    CUDA events and the wall clock around one Simulation.run call, SM clocks sampled."""
    import torch

    from devinproj_b200 import DampedShiftedCoulomb, LennardJones, VelocityVerlet
    from devinproj_b200._accusim import simulation as _asim
    s, forces, dt, _ = workload(args.workload, seed=0)
    from devinproj_b200 import GpuSystem
    g = GpuSystem.from_system(s)
    fresh = []
    for f in forces:   # plug-ins of their own (a Verlet list per force object)
        if isinstance(f, LennardJones):
            fresh.append(LennardJones(f.params, cutoff=f.cutoff, pairlist_threshold=f.pairlist_threshold, skin=f.skin))
        elif isinstance(f, DampedShiftedCoulomb):
            fresh.append(DampedShiftedCoulomb(f.rcut, alpha=f.alpha, k=f.k, pairlist_threshold=f.pairlist_threshold,
                                              exclude=f.exclude, skin=f.skin))
    sim = _asim.Simulation(g, fresh, integrator=VelocityVerlet(), dt=dt)
    sim.run(steps=3, record_every=10 ** 9, positions=False)          # warm-up (and the first upload)
    torch.cuda.synchronize()
    rb0 = fresh[0].rebuilds
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.2)
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        e0.record(stream)
        sim.run(steps=args.fp64_steps, record_every=10 ** 9, positions=False)
        e1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
    ms = e0.elapsed_time(e1)
    return {"value": g.n * args.fp64_steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.fp64_steps,
            "steps": args.fp64_steps, "wall_s": wall, "list_rebuilds": fresh[0].rebuilds - rb0,
            "path": "accusim.Simulation.run (unmodified, baseline/_ref) + devinproj_b200.GpuSystem (state resident on "
                    "the GPU) + FP64 LennardJones/DampedShiftedCoulomb/VelocityVerlet plug-ins; host sync of the "
                    "potential energy each step (accusim's contract), state at the final record only",
            "dtype": "f64", "clocks": clk.summary()}


WORKLOADS = {
    "lj1m": {"workload": "lj_fcc64_1048576", "atoms": 1048576, "rho_star": 0.8442, "T_star": 0.72,
             "cutoff_sigma": 2.5, "skin_sigma": 0.3, "dt_star": 0.005, "forces": "LennardJones"},
    "nacl4096": {"workload": "nacl_rocksalt16_4096", "atoms": 4096, "density_g_cm3": 1.55, "T_K": 1200,
                 "dsf_alpha_per_A": 0.2, "dsf_rc_A": 12.0, "dt_fs": 1.0, "forces": "LennardJones+DampedShiftedCoulomb"},
    "argon864": {"workload": "argon_fcc6_864", "atoms": 864, "box_sigma": 10.229, "T_K": 94.4, "dt_fs": 10.0,
                 "forces": "LennardJones"},
    "ensemble": {"workload": "lj_ensemble_256x3", "replicas": 256, "trajectories": 768, "atoms": 6038184,
                 "sizes": "log-uniform 256..32000 (fcc 4 nc^3, seed 0)", "rho_star": 0.8442, "T_star": 0.72,
                 "cutoff_sigma": 2.5, "skin_sigma": 0.3, "dt_star": [0.005, 0.0025, 0.00125],
                 "forces": "LennardJones"},
}


def run_experiment(args):
    """Accuracy experiments that back the design document's claims; each prints one JSON line."""
    import numpy as np
    import torch

    torch.cuda.set_device(0)
    if args.experiment == "learned":
        from devinproj_b200 import GpuSimulation, configs
        from devinproj_b200.learned import LearnedCorrection, generate_dataset
        t0 = time.perf_counter()
        d = generate_dataset(args.snapshots, seed=0, n_sites=20, verbose=False)
        t_gen = time.perf_counter() - t0
        n_train = int(0.9 * args.snapshots)
        # training settings chosen on a validation split (the last 10% of the training snapshots), the error
        # reported on the held-out 10% that no choice has seen
        configs_tried = [tuple(float(x) for x in c.split(":")) for c in args.train_configs.split(",")]
        n_fit = int(0.9 * n_train) if len(configs_tried) > 1 else n_train
        val_idx = np.arange(n_fit, n_train)
        trials = []
        best = None
        t0 = time.perf_counter()
        for epochs, lr in configs_tried:
            cand = LearnedCorrection(seed=0)
            hist_c = cand.train(d, np.arange(n_fit), epochs=int(epochs), batch_tiles=64, lr=lr)
            v = cand.errors(d, val_idx)[1] if len(val_idx) else float("nan")
            trials.append({"epochs": int(epochs), "lr": lr, "val_rms_rel_err": v, "train_loss_last": hist_c[-1]})
            if best is None or v < best[0]:
                best = (v, cand, hist_c)
        lc, hist = best[1], best[2]
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0
        e0, e1 = lc.errors(d, np.arange(n_train, args.snapshots))
        # floor of any pair-additive correction of range R (least squares on the same labels)
        from devinproj_b200.learned import pair_kernel_bound
        fit_idx = np.arange(min(n_train, 100))
        test_idx = np.arange(n_train, min(args.snapshots, n_train + 20))
        bound = {}
        for R in (10.0, 15.0, 20.0):
            b0, b1 = pair_kernel_bound(d, fit_idx, test_idx, R * 1e-10)
            bound[f"{R:g}A"] = {"err_dsf": b0, "err_fit": b1, "ratio": b0 / b1}
        # step-time overhead of the correction on the 8000-ion melt (eager per-kernel timing)
        s, forces, dt = configs.nacl8000()
        s.pos = d["pos"][-1].copy()
        plain = GpuSimulation(s.copy(), forces, dt=dt)
        plain.engine.run(20, 0, True)
        k0, r0, t_plain = plain.engine.run_timed(200, 0)
        corr = GpuSimulation(s.copy(), forces, dt=dt, correction=lc, validate_every=0)
        corr.engine.run(20, 0, True)
        k1, r1, t_c = corr.engine.run_timed(200, 0)
        c_ms = corr.engine.last_correction_ms()
        step_plain = t_plain / 200
        step_corr = step_plain + c_ms
        def graph_ms(engine, steps=200):
            engine.run(steps, 0, True)   # same block length as the timed run: its graph is captured here
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            engine.run(steps, 0, True)
            b.record()
            torch.cuda.synchronize()
            return a.elapsed_time(b) / steps

        graph_plain = graph_ms(plain.engine)
        graph_corr = {}
        for stride in (1, 5, 10, 25):
            corr.engine.set_correction_stride(stride)
            graph_corr[stride] = graph_ms(corr.engine)
        print(json.dumps({"experiment": "learned_dsf_correction", "ions": 8000, "snapshots": args.snapshots,
                          "train_snapshots": n_train, "dataset_s": t_gen, "train_s": t_train,
                          "train_loss_first_last": [hist[0], hist[-1]], "training_trials": trials,
                          "heldout_rms_rel_err_dsf": e0, "heldout_rms_rel_err_corrected": e1, "error_ratio": e0 / e1,
                          "pair_kernel_bound": bound,
                          "step_ms_plain": step_plain, "correction_ms": c_ms,
                          "overhead_frac": c_ms / step_plain, "step_ms_corrected": step_corr,
                          "graph_ms_per_step_plain": graph_plain,
                          "graph_ms_per_step_corrected": {f"stride{k}": v for k, v in graph_corr.items()},
                          "graph_overhead_frac": {f"stride{k}": v / graph_plain - 1.0 for k, v in graph_corr.items()}}),
              flush=True)
    elif args.experiment == "correction_kernels":
        # the correction's kernels inside the step loop on the 8000-ion melt (untrained weights: the kernels'
        # work does not depend on the weights); eager launches with per-kernel events
        from devinproj_b200 import GpuSimulation, configs
        from devinproj_b200.learned import LearnedCorrection
        s, forces, dt = configs.nacl8000()
        sim = GpuSimulation(s, forces, dt=dt, correction=LearnedCorrection(seed=0), validate_every=0)
        step_ms, list_ms, _ = sim.engine.run_timed(max(args.steps, 1), 0)
        print(json.dumps({"experiment": "correction_kernels", "ions": s.n, "steps": args.steps,
                          "step_kernel_ms": step_ms, "list_kernel_ms": list_ms,
                          "correction_ms": sim.engine.last_correction_ms()}), flush=True)
    elif args.experiment == "drift":
        # the report's energy-drift metric of the 1M-atom fluid: over a 10^4-step window after --drift-equil steps
        # from the fcc lattice start (the lattice melts first), and over the whole run from the lattice; the FP32c
        # engine, and the plain FP64 plug-ins inside accusim's Simulation.run on a device-resident GpuSystem from
        # the same state (the reference model's own drift at this dt, with no FP32 arithmetic)
        from devinproj_b200 import VelocityVerlet
        from devinproj_b200._accusim import simulation as _asim
        from devinproj_b200.engine import ENERGY, start_engine
        from devinproj_b200.ensemble import drift_of
        from devinproj_b200.state import GpuSystem
        steps, every, equil = args.drift_steps or 10000, 100, args.drift_equil
        s, forces, dt, cfg = workload("lj1m", seed=0)
        s64 = GpuSystem.from_system(s)
        eng, _, _ = start_engine([s], forces, [dt], rec_cap=max(steps, equil) // every + 2)
        init = eng.records(1)[0, 0].copy()
        eng.run(equil, every, True)
        r_eq = eng.records(equil // every)[:, 0, :].copy()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.run(steps, every, True)
        e1.record()
        torch.cuda.synchronize()
        eng.check("drift run")
        r_w = eng.records(steps // every)[:, 0, :]
        win = np.concatenate([r_eq[-1:], r_w]) * ENERGY              # SI, like the FP64 run's trajectory
        full = np.concatenate([init[None], r_eq, r_w]) * ENERGY

        def metrics(rec, ke, pe):
            E = ke + pe
            scale = max(abs(E[0]), np.max(np.abs(ke)), np.max(np.abs(pe)))
            return {"energy_drift_report_metric": drift_of(ke, pe),
                    "linear_drift_per_step_rel": float(np.polyfit(np.arange(len(E)) * every, E, 1)[0]) / scale}
        out = {"experiment": "energy_drift_lj1m", "window_steps": steps, "equilibration_steps": equil,
               "record_every": every,
               "fp32c": {"window": metrics(win, win[:, 0], win[:, 1]),
                         "from_lattice": metrics(full, full[:, 0], full[:, 1]),
                         "ms_per_step": e0.elapsed_time(e1) / steps, "rebuilds": eng.status().rebuilds}}
        del eng
        if args.fp64_steps > 0:
            sim = _asim.Simulation(s64, forces, integrator=VelocityVerlet(), dt=dt)
            t0 = time.perf_counter()
            sim.run(steps=equil, record_every=every, positions=False)
            n_eq = len(sim.trajectory.t)
            tr = sim.run(steps=steps, record_every=every, positions=False)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            KE, PE = np.array(tr.kinetic), np.array(tr.potential)
            out["fp64_dropin"] = {"window": metrics(None, KE[n_eq - 1:], PE[n_eq - 1:]),
                                  "from_lattice": metrics(None, KE, PE), "wall_s": wall,
                                  "path": "accusim.Simulation.run + GpuSystem + FP64 plug-ins"}
            E64 = KE + PE
            Ef = full[:, 0] + full[:, 1]
            n = min(len(E64), len(Ef))
            sc = max(abs(E64[0]), np.max(np.abs(KE)), np.max(np.abs(PE)))
            out["max_energy_difference_fp32c_vs_fp64_rel"] = float(np.max(np.abs(Ef[:n] - E64[:n])) / sc)
        print(json.dumps(out), flush=True)
    elif args.experiment == "autotune":
        # the tuned launch shape against the size rule on the ensemble's replica sizes: per bucket, 8 replicas of
        # one fcc size at dt*, every candidate (threads per atom x step grid) timed with per-kernel events, then the
        # wider cell edges for the fastest pair and for the size rule
        from devinproj_b200 import autotune, configs
        from devinproj_b200.engine import default_tpa, estimate_maxnb, forcefield_from, start_engine
        rows = []
        for nc in (4, 5, 6, 8, 10, 13, 16, 20):
            systems = []
            for k in range(8):
                sk, lj = configs.lj_fluid(nc, seed=k)
                systems.append(sk)
            dts = [0.005 * configs.AR_TAU] * len(systems)
            _, rlist, _ = forcefield_from([lj], systems[0].species)
            n_total = sum(x.n for x in systems)
            vol = sum(float(np.prod(x.box)) for x in systems)
            nb = n_total / vol * 4.0 / 3.0 * math.pi * rlist ** 3
            times = {}

            def timed(tpa, gm, cs):
                eng, _, _ = start_engine([x.copy() for x in systems], [lj], dts, tpa=tpa, grid_mult=gm, cell_scale=cs)
                eng.run(10, 0, True)
                k_ms, r_ms, tot = eng.run_timed(max(args.steps, 50), 0)
                eng.check("autotune experiment")
                times[autotune._label(tpa, gm, cs)] = tot / max(args.steps, 50)
                del eng

            for tpa, gm in autotune.candidates(n_total, nb):
                timed(tpa, gm, 1.0)
            cells = sum(int(np.prod([max(1, int(bx // rlist)) for bx in x.box])) for x in systems)
            rule = default_tpa(n_total, (estimate_maxnb(systems[0].n, systems[0].box, rlist) - 32) / 1.3, cells)
            narrow = {k: v for k, v in times.items() if k.endswith(",1")}
            pair = min(narrow, key=narrow.get).rsplit(",", 1)[0]
            for cs in autotune.CELL_SCALES[1:]:   # the tuner's second stage, and the same edges at the size rule
                timed(*(int(x) for x in pair.split(",")), cs)
                if f"{rule},0" != pair:
                    timed(rule, 0, cs)
            rule_key = autotune._label(rule, 0, 1.0)
            best = min(times, key=times.get)
            rows.append({"atoms_per_replica": systems[0].n, "replicas": len(systems), "rule": rule_key,
                         "rule_ms": times.get(rule_key), "best": best, "best_ms": times[best],
                         "gain": (times.get(rule_key) or float("nan")) / times[best],
                         "cells_per_axis": {f"{c:g}": int(systems[0].box[0] // (rlist * c)) for c in autotune.CELL_SCALES},
                         "ms_per_step": times})
            print(json.dumps(rows[-1]), flush=True)
        print(json.dumps({"experiment": "autotune_vs_size_rule", "rows": len(rows)}), flush=True)
    elif args.experiment == "dropin":
        # the FP64 plug-ins inside accusim's Simulation.run: on a device-resident GpuSystem (the honest FP64 GPU
        # figure) and on accusim's plain System (state copied to and from the host every step)
        from devinproj_b200 import VelocityVerlet
        from devinproj_b200._accusim import simulation as _asim
        from devinproj_b200.state import GpuSystem
        out = {}
        for kind in ("device_resident", "host_round_trip"):
            s, forces, dt, cfg = workload(args.workload, seed=0)
            if kind == "device_resident":
                s = GpuSystem.from_system(s)
            sim = _asim.Simulation(s, forces, integrator=VelocityVerlet(), dt=dt)
            sim.run(steps=3, record_every=10 ** 9, positions=False)
            torch.cuda.synchronize()
            n = max(args.steps, 5) if kind == "device_resident" else 5
            t0 = time.perf_counter()
            sim.run(steps=n, record_every=10 ** 9, positions=False)
            torch.cuda.synchronize()
            dt_s = time.perf_counter() - t0
            out[kind] = {"steps": n, "atom_steps_per_s": s.n * n / dt_s, "ms_per_step": 1e3 * dt_s / n}
        print(json.dumps({"experiment": "fp64_dropin_throughput", "workload": cfg["workload"], **out,
                          "path": "accusim.Simulation.run with the FP64 VelocityVerlet and force plug-ins"}), flush=True)


def workload_meta(name):
    """Workload description without building device state (for the reference arm)."""
    if name not in WORKLOADS:
        raise SystemExit(f"unknown workload {name}")
    return dict(WORKLOADS[name])


def full_config(cfg, args, world):
    if args.workload == "ensemble":   # one fixed set of trajectories, sharded over the ranks
        par = f"replica shards x{world}" if world > 1 else "all replicas in one engine"
    else:
        par = f"independent replicas x{world}" if world > 1 else "single system"
    return dict(cfg, l2="inputs larger than L2" if cfg["atoms"] >= 1 << 20 else "inputs resident in L2 (small system)",
                record_every=args.record_every, parallelism=par)


if __name__ == "__main__":
    main()
