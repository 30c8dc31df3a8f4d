"""Host side of the device-resident engine (include/accusim_b200_engine.h).

`GpuSimulation` runs `Simulation.run(duration, steps, record_every, positions)` of accusim
(accusim/simulation.py:95-112) with VelocityVerlet and LennardJones and/or DampedShiftedCoulomb as
CUDA-graph-captured step loops: FP32 pair terms with Kahan-compensated per-atom sums, FP64 positions,
velocities, integration and conserved-quantity sums. `Engine` is the thin ctypes wrapper; it also
advances batches of independent replicas (see `ensemble.py`).

Engine units: length A, mass u, energy kJ/mol per particle, charge e (time unit ~0.1 ps). The SI
conversion happens here, at the API edge; results are returned in SI.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._accusim import forces as _af
from ._accusim import integrators as _ai
from .device import require_cuda, stream_handle, to_dev
from .units import N_A, amu, e_charge, k_B, k_e

LEN = 1e-10
MASS = amu
ENERGY = 1e3 / N_A
TIME = LEN * math.sqrt(MASS / ENERGY)
VEL = LEN / TIME
ACC = VEL / TIME
CHARGE = e_charge
KE_ENGINE = k_e * CHARGE ** 2 / (ENERGY * LEN)

P = C.c_void_p


class Replica(C.Structure):
    _fields_ = [("n", C.c_int32), ("pad", C.c_int32), ("box", C.c_double * 3), ("dt", C.c_double),
                ("rlist", C.c_double), ("half_skin", C.c_double)]


class ForceField(C.Structure):
    _fields_ = [("n_species", C.c_int32), ("lj", C.c_int32), ("dsf", C.c_int32), ("pad", C.c_int32),
                ("mass", C.c_double * 8), ("lj_eps", C.c_double * 64), ("lj_sig", C.c_double * 64),
                ("lj_cutoff", C.c_double), ("dsf_alpha", C.c_double), ("dsf_rcut", C.c_double),
                ("dsf_k", C.c_double), ("q", C.c_double * 8)]


class Thermostat(C.Structure):
    _fields_ = [("kind", C.c_int32), ("pad", C.c_int32), ("kT", C.c_double), ("friction", C.c_double),
                ("seed", C.c_uint64), ("period", C.c_double)]


class EngineConfig(C.Structure):
    _fields_ = [("n_replicas", C.c_int32), ("maxnb", C.c_int32), ("rec_cap", C.c_int32), ("grid_mult", C.c_int32),
                ("tpa", C.c_int32), ("cell_order", C.c_int32), ("replicas", C.POINTER(Replica)), ("ff", ForceField),
                ("thermo", Thermostat), ("ex_start", C.POINTER(C.c_int32)), ("ex_ids", C.POINTER(C.c_int32)),
                ("n_ex_ids", C.c_int32), ("pad2", C.c_int32), ("barrier_wait_limit", C.c_int64),
                ("cell_scale", C.c_double)]


def langevin_thermostat(integrator, seed):
    """Engine thermostat block for a Langevin integrator (this package's or the reference's; SI T and
    friction) in engine units; seed None draws one."""
    if seed is None:
        seed = int(np.random.default_rng().integers(2 ** 63))
    return Thermostat(1, 0, k_B * float(integrator.T) / ENERGY, float(integrator.gamma) * TIME, int(seed) % 2 ** 64,
                      0.0)


def nose_hoover_thermostat(integrator):
    """Engine thermostat block for a Nose-Hoover integrator (this package's or the reference's: SI T and
    period) in engine units."""
    return Thermostat(2, 0, k_B * float(integrator.T) / ENERGY, 0.0, 0, float(integrator.tau) / TIME)


class DevStatusC(C.Structure):
    _fields_ = [("flags", C.c_int32), ("need_nbr", C.c_int32), ("rebuilds", C.c_int32), ("fail_step", C.c_int32),
                ("steps_done", C.c_int32), ("pad", C.c_int32 * 3)]


ENGINE_SIGNATURES = {
    "acs_engine_bytes": (C.c_size_t, [C.POINTER(EngineConfig)]),
    "acs_engine_create": (C.c_int, [C.POINTER(EngineConfig), P, C.c_size_t, C.POINTER(P)]),
    "acs_engine_set_state": (C.c_int, [P, P, P, P, P]),
    "acs_engine_get_state": (C.c_int, [P, P, P, P, P]),
    "acs_engine_set_active": (C.c_int, [P, P, P]),
    "acs_engine_run": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, P]),
    "acs_engine_records": (C.c_int, [P, P, C.c_int32, P]),
    "acs_engine_status": (C.c_int, [P, C.POINTER(DevStatusC), C.c_int, P]),
    "acs_engine_neighbor_stats": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int64), P]),
    "acs_engine_launch_info": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "acs_engine_load_state": (C.c_int, [P, P, P, P]),
    "acs_engine_count_pairs": (C.c_int, [P, P, P]),
    "acs_engine_dump_lists": (C.c_int, [P, P, C.c_longlong, P, P, P]),
    "acs_engine_run_timed": (C.c_int, [P, C.c_int32, C.c_int32, C.POINTER(C.c_float), P]),
    "acs_engine_phase_times": (C.c_int, [P, P, C.c_int]),
    "acs_engine_set_correction": (C.c_int, [P, P, P, P, P, P, P, C.c_float, P, P, P, P, C.c_int]),
    "acs_engine_last_correction_ms": (C.c_float, [P]),
    "acs_engine_nh_state": (C.c_int, [P, P, C.c_int32]),
    "acs_engine_bath_records": (C.c_int, [P, P, C.c_int32, P]),
    "acs_engine_set_correction_stride": (C.c_int, [P, C.c_int32]),
    "acs_engine_destroy": (C.c_int, [P]),
}
_lib.SIGNATURES.update(ENGINE_SIGNATURES)

REC_FIELDS = ("KE", "PE", "Px", "Py", "Pz", "Lx", "Ly", "Lz")


def forcefield_from(forces, species) -> tuple[ForceField, float, float]:
    """Engine force field from reference-shaped LennardJones / DampedShiftedCoulomb objects (SI).
    Returns (ff, list radius [m], half skin [m]) for the combined neighbour list: every pair within any
    force's cutoff stays listed until an atom has moved half of the smallest effective skin."""
    ff = ForceField()
    ns = len(species)
    if ns > 8:
        raise ValueError("the engine supports up to 8 species")
    ff.n_species = ns
    for a, sp in enumerate(species):
        ff.mass[a] = sp.mass / MASS
        ff.q[a] = sp.charge / CHARGE
    radii = []   # (cutoff_max, list radius) per force, SI
    lj = [f for f in forces if isinstance(f, _af.LennardJones)]
    dsf = [f for f in forces if isinstance(f, _af.DampedShiftedCoulomb)]
    if len(lj) + len(dsf) != len(forces) or len(lj) > 1 or len(dsf) > 1 or not forces:
        raise ValueError("the engine runs one LennardJones and/or one DampedShiftedCoulomb force")
    if lj:
        f = lj[0]
        eps, sig = f._tables(_SpeciesView(species))
        if not np.any(eps > 0):
            raise ValueError("LennardJones has no interacting species")
        ff.lj = 1
        ff.lj_cutoff = float(f.cutoff)
        for a in range(ns):
            for b in range(ns):
                ff.lj_eps[a * ns + b] = eps[a, b] / ENERGY
                ff.lj_sig[a * ns + b] = sig[a, b] / LEN
        smax = float(np.max(np.where(eps > 0, sig, 0)))
        radii.append((f.cutoff * smax, f.cutoff * smax + f.skin * smax))
    if dsf:
        f = dsf[0]
        ff.dsf = 1
        ff.dsf_alpha = f.alpha * LEN
        ff.dsf_rcut = f.rcut / LEN
        ff.dsf_k = f.k * CHARGE ** 2 / (ENERGY * LEN)
        radii.append((f.rcut, f.rcut + f.skin))
    rlist = max(r for _, r in radii)
    half_skin = 0.5 * min(rlist - c for c, _ in radii)
    return ff, rlist, half_skin


class _SpeciesView:
    def __init__(self, species):
        self.species = species


class Engine:
    """ctypes wrapper around one acs_engine; device memory is one torch allocation."""

    def __init__(self, replicas, ff: ForceField, maxnb: int, rec_cap: int = 64, grid_mult: int = 0, tpa: int = 1,
                 thermo=None, exclusions=None, barrier_wait_limit: int = 0, cell_order: int = 1,
                 cell_scale: float = 1.0):
        require_cuda()
        L = _lib.lib()
        for name, (res, args) in ENGINE_SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        self.L = L
        self.R = len(replicas)
        self._reps = (Replica * self.R)()
        for k, r in enumerate(replicas):
            self._reps[k].n = int(r["n"])
            for d in range(3):
                self._reps[k].box[d] = float(r["box"][d])
            self._reps[k].dt = float(r["dt"])
            self._reps[k].rlist = float(r["rlist"])
            self._reps[k].half_skin = float(r["half_skin"])
        self.tpa = int(tpa)
        self.cfg = EngineConfig(self.R, int(maxnb), int(rec_cap), int(grid_mult), self.tpa, 0, self._reps, ff,
                                thermo if thermo is not None else Thermostat())
        self.cfg.barrier_wait_limit = int(barrier_wait_limit)
        self.cfg.cell_order = int(cell_order)
        self.cell_order = int(cell_order)
        self.cfg.cell_scale = float(cell_scale)
        self.cell_scale = float(cell_scale)
        self._ex = exclusions   # (ex_start, ex_ids) int32 arrays, kept alive with the config
        if exclusions is not None:
            ex_start, ex_ids = exclusions
            self.cfg.ex_start = ex_start.ctypes.data_as(C.POINTER(C.c_int32))
            self.cfg.ex_ids = ex_ids.ctypes.data_as(C.POINTER(C.c_int32))
            self.cfg.n_ex_ids = len(ex_start) - 1
        nbytes = L.acs_engine_bytes(C.byref(self.cfg))
        if nbytes == 0:
            raise ValueError("engine configuration rejected (sizes, box, time step or too many replicas)")
        self.nbytes = int(nbytes)
        self.mem = torch.empty(self.nbytes + 256, dtype=torch.uint8, device="cuda")
        base = self.mem.data_ptr()
        off = (-base) % 256
        self.h = P()
        _lib.check(L.acs_engine_create(C.byref(self.cfg), base + off, self.nbytes, C.byref(self.h)),
                   "acs_engine_create")
        self.maxnb = int(maxnb)
        self.rec_cap = int(rec_cap)
        self.rlist_engine = float(replicas[0]["rlist"])
        self.correction = None
        self.counts = np.array([int(r["n"]) for r in replicas])
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)])
        self._rec_buf = torch.empty(rec_cap * self.R * 8, dtype=torch.float64, device="cuda")

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                self.L.acs_engine_destroy(h)
            except Exception:
                pass
            self.h = None

    def set_state(self, pos_d, vel_d, sp_d):
        _lib.check(self.L.acs_engine_set_state(self.h, pos_d.data_ptr(), vel_d.data_ptr(), sp_d.data_ptr(),
                                               stream_handle()), "acs_engine_set_state")

    def load_state(self, pos_d, vel_d):
        """Positions/velocities in caller order (engine units) replacing the current ones; lists kept."""
        _lib.check(self.L.acs_engine_load_state(self.h, pos_d.data_ptr(), vel_d.data_ptr(), stream_handle()),
                   "acs_engine_load_state")

    def count_pairs(self):
        """(LJ, DSF) unique pairs inside the physical cutoffs, counted on the device."""
        out = torch.zeros(2, dtype=torch.int64, device="cuda")
        _lib.check(self.L.acs_engine_count_pairs(self.h, out.data_ptr(), stream_handle()), "acs_engine_count_pairs")
        a, b = out.cpu().numpy()
        return int(a) // 2, int(b) // 2

    def list_entries(self):
        """The neighbour lists as they stand: (keys, positions) with keys an int64 device tensor of directed
        entries 2 (i n + j) + excluded over caller indices (sorted), and the FP64 positions (engine units,
        caller order) of the last rebuild, which the lists were built from."""
        n = int(self.offsets[-1])
        _, total = self.neighbor_stats()
        keys = torch.empty(max(total, 1), dtype=torch.int64, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        pos = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        _lib.check(self.L.acs_engine_dump_lists(self.h, keys.data_ptr(), int(keys.numel()), cnt.data_ptr(),
                                                pos.data_ptr(), stream_handle()), "acs_engine_dump_lists")
        m = int(cnt.item())
        if m != total:
            raise RuntimeError(f"list dump counted {m} entries, the lists hold {total}")
        return torch.sort(keys[:m]).values, pos

    def get_state(self):
        n = int(self.offsets[-1])
        pos = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        vel = torch.empty_like(pos)
        acc = torch.empty_like(pos)
        _lib.check(self.L.acs_engine_get_state(self.h, pos.data_ptr(), vel.data_ptr(), acc.data_ptr(),
                                               stream_handle()), "acs_engine_get_state")
        return pos, vel, acc

    def set_active(self, active):
        a = np.ascontiguousarray(np.asarray(active, dtype=np.int32))
        _lib.check(self.L.acs_engine_set_active(self.h, a.ctypes.data, stream_handle()), "acs_engine_set_active")
        torch.cuda.current_stream().synchronize()

    def run(self, steps: int, record_every: int = 0, record_last: bool = True):
        _lib.check(self.L.acs_engine_run(self.h, int(steps), int(record_every), 1 if record_last else 0,
                                         stream_handle()), "acs_engine_run")

    def set_correction(self, lc, enabled=True):
        """Attach (or detach) a LearnedCorrection: evaluated inside every force evaluation of later runs."""
        if not enabled or lc is None:
            _lib.check(self.L.acs_engine_set_correction(self.h, None, None, None, None, None, None, 0.0, None, None,
                                                        None, None, 0), "acs_engine_set_correction")
            self.correction = None
            return
        S = self.launch_info()[2]
        if lc.desc.p["rc"] > self.rlist_engine:
            raise ValueError("descriptor radius exceeds the engine's neighbour-list radius")
        self._cX = torch.zeros((S, 80), dtype=torch.bfloat16, device="cuda")
        self._cV = torch.zeros((S, 64, 3), dtype=torch.float32, device="cuda")
        self._cF = torch.zeros((S, 3), dtype=torch.float32, device="cuda")
        m = lc.mlp
        _lib.check(self.L.acs_engine_set_correction(self.h, lc.desc.params6.ctypes.data, lc.desc.mean.data_ptr(),
                                                    lc.desc.inv_std.data_ptr(), m._w5, m.b2.data_ptr(), m.b3.data_ptr(),
                                                    float(lc.scale), self._cX.data_ptr(), self._cV.data_ptr(),
                                                    self._cF.data_ptr(), m.status.ptr, 1), "acs_engine_set_correction")
        self.correction = lc

    def set_correction_stride(self, stride):
        _lib.check(self.L.acs_engine_set_correction_stride(self.h, int(stride)), "acs_engine_set_correction_stride")
        self.c_stride = int(stride)

    def last_correction_ms(self):
        return float(self.L.acs_engine_last_correction_ms(self.h))

    def run_timed(self, steps: int, record_every: int = 0):
        """Eager launches of one block with per-kernel CUDA events: (step ms avg, rebuild ms avg, total ms)."""
        out = (C.c_float * 4)()
        _lib.check(self.L.acs_engine_run_timed(self.h, int(steps), int(record_every), out, stream_handle()),
                   "acs_engine_run_timed")
        return out[0] / max(out[2], 1), out[1] / max(out[3], 1), out[0] + out[1]

    PHASES = {1: "flags", 2: "clear", 3: "bin", 4: "scan_a", 5: "scan_b", 6: "scan_c", 7: "scatter", 8: "sort",
              9: "gather", 10: "commit", 15: "list_build_block0"}

    def phase_times(self, clear=True):
        """List-maintenance phase times (ms, accumulated) from the device global timer."""
        out = np.zeros(16, dtype=np.uint64)
        _lib.check(self.L.acs_engine_phase_times(self.h, out.ctypes.data, 1 if clear else 0), "phase_times")
        return {name: float(out[k]) / 1e6 for k, name in self.PHASES.items()}

    def records(self, count: int) -> np.ndarray:
        """(count, R, 8) FP64 records [KE, PE, Px, Py, Pz, Lx, Ly, Lz] in engine units."""
        if count == 0:
            return np.zeros((0, self.R, 8))
        _lib.check(self.L.acs_engine_records(self.h, self._rec_buf.data_ptr(), int(count), stream_handle()),
                   "acs_engine_records")
        return self._rec_buf[: count * self.R * 8].view(count, self.R, 8).cpu().numpy()

    def bath_records(self, count: int) -> np.ndarray:
        """(count, R) thermostat energies at the records (Nose-Hoover; zero otherwise), engine units."""
        if count == 0:
            return np.zeros((0, self.R))
        buf = torch.empty(count * self.R, dtype=torch.float64, device="cuda")
        _lib.check(self.L.acs_engine_bath_records(self.h, buf.data_ptr(), int(count), stream_handle()),
                   "acs_engine_bath_records")
        return buf.view(count, self.R).cpu().numpy()

    def nh_state(self) -> np.ndarray:
        """(R, 2) Nose-Hoover (xi, eta) per replica, engine units."""
        out = np.zeros((self.R, 2))
        _lib.check(self.L.acs_engine_nh_state(self.h, out.ctypes.data, 0), "acs_engine_nh_state")
        return out

    def set_nh_state(self, xi_eta):
        arr = np.ascontiguousarray(np.asarray(xi_eta, dtype=np.float64).reshape(self.R, 2))
        _lib.check(self.L.acs_engine_nh_state(self.h, arr.ctypes.data, 1), "acs_engine_nh_state")

    def status(self, clear=False) -> DevStatusC:
        st = DevStatusC()
        _lib.check(self.L.acs_engine_status(self.h, C.byref(st), 1 if clear else 0, stream_handle()),
                   "acs_engine_status")
        return st

    def check(self, where="engine"):
        st = self.status()
        if st.flags & _lib.FLAG_OVERFLOW:
            raise _lib.ListOverflow(_lib.ACS_ERR_LIST_OVERFLOW, f"{where}: need {st.need_nbr} neighbours")
        if st.flags & _lib.FLAG_NONFINITE:
            raise _lib.AcsError(_lib.ACS_ERR_NONFINITE, where)
        if st.flags & _lib.FLAG_TIMEOUT:
            raise _lib.AcsError(_lib.ACS_ERR_TIMEOUT, where)
        return st

    def neighbor_stats(self):
        mx, sm = C.c_int32(), C.c_int64()
        _lib.check(self.L.acs_engine_neighbor_stats(self.h, C.byref(mx), C.byref(sm), stream_handle()))
        return mx.value, sm.value

    def launch_info(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int64()
        _lib.check(self.L.acs_engine_launch_info(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value


def estimate_maxnb(n, box, rlist):
    rho = n / float(np.prod(box))
    expected = rho * 4.0 / 3.0 * math.pi * rlist ** 3
    return int(min(expected * 1.3 + 32, 4096) + 7) // 8 * 8


def default_tpa(n_atoms_total, neighbors_per_atom, n_cells_total=None):
    """Threads per atom for the pair kernel, which also picks the list build (a warp per atom from 8 threads
    per atom, else a warp per cell). Measured on a B200 (LJ fcc fluids of 864 to 1M atoms, 4096-ion NaCl):
    with fewer than 512 cells the warp-per-cell build lacks parallelism, so 32 threads per atom (16 for long
    DSF lists) win; otherwise 1 to 4 threads per atom, enough for about 65k threads."""
    if n_cells_total is not None and n_cells_total < 512:
        return 16 if neighbors_per_atom > 200 else 32
    tpa = 1
    while tpa < 4 and n_atoms_total * tpa < 65536:
        tpa *= 2
    return tpa


def dsf_exclusions(forces, systems):
    """The DampedShiftedCoulomb exclusion id pairs as the engine takes them: CSR (ex_start, ex_ids) by atom
    index, both directions, ids mapped to indices through `system.ids` as accusim/forces.py:418-419 does
    (pairs with an id not in the system are dropped); None without exclusions. The engine applies one table
    to every replica, so the replicas must number their atoms alike."""
    dsf = [f for f in forces if isinstance(f, _af.DampedShiftedCoulomb)]
    if not dsf or not dsf[0].exclude:
        return None
    ids = np.asarray(systems[0].ids)
    for s in systems[1:]:
        if not np.array_equal(np.asarray(s.ids), ids):
            raise ValueError("DSF exclusions need the same atom ids in every replica")
    where = {int(pid): k for k, pid in enumerate(ids)}
    pairs = np.array([(where[a], where[b]) for a, b in dsf[0].exclude if a in where and b in where],
                     dtype=np.int64).reshape(-1, 2)
    if not len(pairs):
        return None
    a = np.concatenate([pairs[:, 0], pairs[:, 1]])
    b = np.concatenate([pairs[:, 1], pairs[:, 0]])
    order = np.argsort(a, kind="stable")
    ex_start = np.concatenate([[0], np.cumsum(np.bincount(a, minlength=len(ids)))]).astype(np.int32)
    return ex_start, np.ascontiguousarray(b[order], dtype=np.int32)


def build_engine(replicas_si, forces, species, maxnb=None, rec_cap=64, grid_mult=0, tpa=None, thermo=None,
                 exclusions=None, barrier_wait_limit=0, cell_order=1, cell_scale=1.0):
    """Create an engine for replicas given in SI [{n, box, dt}], sharing `forces`. Returns
    (engine, rlist, half_skin) with the radii in SI."""
    ff, rlist, half_skin = forcefield_from(forces, species)
    reps = [dict(n=r["n"], box=np.asarray(r["box"], float) / LEN, dt=r["dt"] / TIME, rlist=rlist / LEN,
                 half_skin=half_skin / LEN) for r in replicas_si]
    expect = max(estimate_maxnb(r["n"], r["box"], r["rlist"]) for r in reps)
    if maxnb is None:
        maxnb = expect
    if tpa is None:
        cells = sum(int(np.prod([max(1, int(bx // (r["rlist"] * cell_scale))) for bx in r["box"]])) for r in reps)
        tpa = default_tpa(sum(r["n"] for r in reps), (expect - 32) / 1.3, cells)
    return (Engine(reps, ff, maxnb, rec_cap=rec_cap, grid_mult=grid_mult, tpa=tpa, thermo=thermo,
                   exclusions=exclusions, barrier_wait_limit=barrier_wait_limit, cell_order=cell_order,
                   cell_scale=cell_scale), rlist,
            half_skin)


def _upload_state(engine, systems):
    ns = len(systems[0].species)
    for s in systems:
        if s.n and (s.sp.min() < 0 or s.sp.max() >= ns):
            raise ValueError("species index out of range")
        if not np.all(np.isfinite(s.pos)) or not np.all(np.isfinite(s.vel)):
            raise ValueError("non-finite positions or velocities")
    pos = np.concatenate([s.pos for s in systems]) / LEN
    vel = np.concatenate([s.vel for s in systems]) / VEL
    sp = np.concatenate([s.sp for s in systems]).astype(np.int32)
    engine.set_state(to_dev(pos), to_dev(vel), to_dev(sp))


def start_engine(systems, forces, dts, maxnb=None, rec_cap=64, grid_mult=0, tpa=None, thermo=None, cell_order=1,
                 cell_scale=1.0):
    """Engine over the given periodic 3-D systems (one replica each) with state loaded and lists built;
    grows the neighbour capacity once if the first build overflows."""
    for s in systems:
        if s.dim != 3 or not s.periodic:
            raise ValueError("the engine runs 3-dimensional periodic systems")
    species = systems[0].species
    if tpa == "auto":
        from .autotune import tune
        tpa, grid_mult, cell_scale = tune(systems, forces, dts)
    reps = [dict(n=s.n, box=s.box, dt=dt) for s, dt in zip(systems, dts)]
    ex = dsf_exclusions(forces, systems)
    for attempt in range(3):
        eng, rlist, hs = build_engine(reps, forces, species, maxnb=maxnb, rec_cap=rec_cap, grid_mult=grid_mult,
                                      tpa=tpa, thermo=thermo, exclusions=ex, cell_order=cell_order,
                                      cell_scale=cell_scale)
        _upload_state(eng, systems)
        st = eng.status()
        if st.flags & _lib.FLAG_OVERFLOW:
            maxnb = int(st.need_nbr * 1.2 + 16 + 7) // 8 * 8
            continue
        eng.check("engine start")
        mx, _ = eng.neighbor_stats()
        if mx * 1.15 + 8 > eng.maxnb and attempt == 0 and maxnb is None:
            maxnb = int(mx * 1.3 + 16 + 7) // 8 * 8
            continue
        return eng, rlist, hs
    raise _lib.ListOverflow(_lib.ACS_ERR_LIST_OVERFLOW, "engine start")


class GpuSimulation:
    """`Simulation` with the step loop on the device (accusim/simulation.py:40-131 interface).

    forces: [LennardJones] and/or [DampedShiftedCoulomb] (this package's or the reference's classes);
    integrator: VelocityVerlet, Langevin (BAOAB, counter-based draws keyed by `seed`) or NoseHoover (its xi,
    eta and Q kept in the integrator object, bath energy in the trajectory). `system.pos`/`vel` are
    synchronised from the device after every `run` call (and at records when positions=True)."""

    def __init__(self, system, forces=(), reactions=(), integrator=None, dt=None, seed=None, maxnb=None,
                 rec_cap=256, grid_mult=0, tpa=None, correction=None, validate_every=500, correction_stride=1):
        from ._accusim import simulation as _asim
        from .integrators import VelocityVerlet
        from .units import si
        Trajectory = _asim.Trajectory
        if reactions:
            raise NotImplementedError("reactions are not part of the accusim_b200 force-and-step path")
        kind = ("VelocityVerlet" if integrator is None or type(integrator) in (_ai.VelocityVerlet, VelocityVerlet)
                else "Langevin" if isinstance(integrator, _ai.Langevin)
                else "NoseHoover" if isinstance(integrator, _ai.NoseHoover) else None)
        if kind is None:
            raise ValueError("GpuSimulation integrates with VelocityVerlet, Langevin (BAOAB) or NoseHoover")
        thermo = (langevin_thermostat(integrator, seed) if kind == "Langevin"
                  else nose_hoover_thermostat(integrator) if kind == "NoseHoover" else None)
        self._thermo = thermo
        self._tpa, self._grid_mult = tpa, grid_mult
        self._nh = kind == "NoseHoover"
        self.system = system
        self.forces = list(forces)
        self.integrator = integrator or VelocityVerlet()
        self.dt = None if dt is None else si(dt, "s")
        self.seed = seed
        self.rng = np.random.default_rng(seed)
        self.reactions = None
        self.time = 0.0
        self.steps = 0
        self.trajectory = Trajectory()
        self._initial = None
        self.engine, self.rlist, self.half_skin = start_engine(
            [system], self.forces, [self.dt if self.dt is not None else 1e-15], maxnb=maxnb, rec_cap=rec_cap,
            grid_mult=grid_mult, tpa=tpa, thermo=thermo)
        if self._nh:   # continue the integrator's thermostat state; the initial record then carries its energy
            self.engine.set_nh_state([[float(self.integrator.xi) * TIME, float(self.integrator.eta)]])
            _upload_state(self.engine, [system])
            self.engine.check("thermostat state")
        self.correction = None
        self.validate_every = int(validate_every)
        self.validations = []
        self.engine.set_correction_stride(correction_stride)
        if correction is not None:
            self.set_correction(correction)
        self._last, self._last_bath = self._latest()
        self._pull()

    def _latest(self):
        """The engine's latest record and bath energy (engine units)."""
        return self.engine.records(1)[0, 0], (self.engine.bath_records(1)[0, 0] if self._nh else 0.0)

    def _sync_thermostat(self):
        """Nose-Hoover: the integrator object holds the run's (xi, eta) and Q, as the reference's does."""
        if not self._nh:
            return
        xi, eta = self.engine.nh_state()[0]
        it = self.integrator
        it.xi, it.eta = float(xi) / TIME, float(eta)
        if it.Q is None:
            nf = it.dof(self.system)
            it.Q = nf * (k_B * it.T) * it.tau ** 2

    def set_correction(self, lc, enabled=True):
        """Add a trained LearnedCorrection to the DSF forces (re-evaluates the current forces)."""
        self.engine.set_correction(lc, enabled)
        self.correction = lc if enabled else None
        _upload_state(self.engine, [self.system])
        self.engine.check("set_correction")
        self._last, self._last_bath = self._latest()
        self._pull()

    def validate(self):
        """Check the corrected electrostatic forces against the device Ewald on the current state; switch the
        correction off (fallback to plain DSF) unless it improves on DSF. Returns (err_dsf, err_corrected)."""
        from .ewald import Ewald
        dsf = [f for f in self.forces if isinstance(f, _af.DampedShiftedCoulomb)][0]
        Fd, _ = dsf.compute(self.system)
        Fe, _ = Ewald(k=dsf.k).compute(self.system)
        e0, e1, on = self.correction.validate(self.system, Fd, Fe)
        self.validations.append((self.steps, e0, e1, on))
        if not on:
            self.set_correction(None, enabled=False)
        return e0, e1

    # state ------------------------------------------------------------------------------------------
    def _pull(self):
        pos, vel, acc = self.engine.get_state()
        s = self.system
        s.pos = pos.cpu().numpy() * LEN
        s.vel = vel.cpu().numpy() * VEL
        self.acc = acc.cpu().numpy() * ACC
        self.force = self.acc * s.masses[:, None]
        self.pe = float(self._last[1] * ENERGY)

    @property
    def rebuilds(self):
        return int(self.engine.status().rebuilds)

    def _record(self, rec, positions, bath=0.0):
        s, tr = self.system, self.trajectory
        tr.t.append(self.time)
        tr.kinetic.append(float(rec[0] * ENERGY))
        tr.potential.append(float(rec[1] * ENERGY))
        tr.internal.append(float(np.sum(s.eint)))
        tr.released.append(0.0)
        tr.momentum.append(rec[2:5] * (MASS * VEL))
        tr.angular_momentum.append(rec[5:8] * (MASS * VEL * LEN))
        tr.mass.append(float(np.sum(s.masses)))
        tr.charge.append(float(np.sum(s.charges)))
        tr.counts.append(s.counts())
        tr.bath.append(float(bath * ENERGY))
        if positions:
            tr.positions.append(s.pos.copy())
            tr.velocities.append(s.vel.copy())
            tr.species.append(s.sp.copy())

    def run(self, duration=None, steps=None, record_every=1, positions=True):
        """Advance `steps` VelocityVerlet steps; record after every `record_every`-th step and the last
        (accusim/simulation.py:95-112). Blocks of steps run as one cached CUDA graph each; a block ends at
        every record when positions are recorded (they come back to the host there)."""
        from .units import si
        if self.dt is None:
            raise ValueError("set dt (or use accusim.advisor.suggest_dt)")
        if steps is None:
            steps = int(round(si(duration, "s") / self.dt))
        re = max(int(record_every), 1)
        if not self.trajectory.t:
            if self._initial is None:
                self._initial = _InitialState(self.system.copy(), self)
            self._record(self._last, positions, self._last_bath)
        eng = self.engine
        done = 0
        while done < steps:
            left = steps - done
            if self.correction is not None and self.validate_every > 0:
                left = min(left, self.validate_every - self.steps % self.validate_every)
            off = done % re
            if positions or off:
                block = min(re - off, left)       # up to the next record step
            else:
                block = min(re * max(1, min(eng.rec_cap - 1, 4000 // re)), left)
            periodic = 0 if (positions or off) else re
            snap = eng.get_state()[:2]            # device copy: the block is redone from here on overflow
            nh_snap = eng.nh_state() if self._nh else None
            eng.run(block, periodic, True)        # every block also records its last step
            local = list(range(periodic, block + 1, periodic)) if periodic else []
            if not local or local[-1] != block:
                local.append(block)
            try:
                eng.check("engine run")
            except _lib.ListOverflow:
                self._regrow(eng.status().need_nbr, snap, nh_snap)
                eng = self.engine
                continue
            recs = eng.records(len(local))[:, 0, :]
            baths = eng.bath_records(len(local))[:, 0] if self._nh else np.zeros(len(local))
            kept = [(j, rec, b) for j, rec, b in zip(local, recs, baths) if (done + j) % re == 0 or done + j == steps]
            if positions and kept:
                self._pull_positions()
            j0 = 0
            for j, rec, b in kept:
                for _ in range(j - j0):
                    self.time += self.dt
                j0 = j
                self._record(rec, positions, b)
            for _ in range(block - j0):
                self.time += self.dt
            self._last, self._last_bath = recs[-1], baths[-1]
            self.steps += block
            done += block
            if self.correction is not None and self.validate_every > 0 and self.steps % self.validate_every == 0:
                self._pull()
                self.validate()
        self._pull()
        self._sync_thermostat()
        return self.trajectory

    def _regrow(self, need, snap, nh_snap):
        """A neighbour list outgrew its capacity during a block (the engine stops its kernels then): build an
        engine with room for the largest list plus 20%, restore the block's start state and thermostat state,
        and let the caller redo the block. A Langevin run continues with the new engine's draws."""
        old = self.engine
        pos, vel = snap
        self.system.pos = np.mod(pos.cpu().numpy() * LEN, self.system.box)
        self.system.vel = vel.cpu().numpy() * VEL
        maxnb = int(max(need, old.maxnb) * 1.2 + 16 + 7) // 8 * 8
        self.engine, self.rlist, self.half_skin = start_engine(
            [self.system], self.forces, [self.dt], maxnb=maxnb, rec_cap=old.rec_cap, grid_mult=self._grid_mult,
            tpa=old.tpa, thermo=self._thermo)
        self.engine.set_correction_stride(getattr(old, "c_stride", 1))
        if nh_snap is not None:
            self.engine.set_nh_state(nh_snap)
            _upload_state(self.engine, [self.system])
        if self.correction is not None:
            self.engine.set_correction(self.correction, True)
            _upload_state(self.engine, [self.system])
        self.engine.check("regrown engine")
        self.regrowths = getattr(self, "regrowths", 0) + 1
        del old

    def _pull_positions(self):
        pos, vel, _ = self.engine.get_state()
        self.system.pos = pos.cpu().numpy() * LEN
        self.system.vel = vel.cpu().numpy() * VEL

    def update_forces(self):
        """Re-evaluate forces of the current host state on the device (after host-side edits)."""
        _upload_state(self.engine, [self.system])
        self.engine.check("update_forces")
        self._last, self._last_bath = self._latest()
        self._pull()

    def clone(self, dt=None):
        sim = GpuSimulation(self.system.copy(), self.forces, integrator=self.integrator,
                            dt=self.dt if dt is None else dt, seed=self.seed, maxnb=self.engine.maxnb,
                            rec_cap=self.engine.rec_cap, tpa=self.engine.tpa)
        return sim

    def accuracy_report(self, convergence_duration=None):
        """accusim's own AccuracyReport (accusim/accuracy.py:59-188) of this run. The timestep-error row, when
        asked for, comes from the dt, dt/2, dt/4 runs advanced together in one batched engine and graded by
        accusim's `timestep_convergence`."""
        from ._accusim import accuracy as _acc
        from .ensemble import timestep_check
        rep = _acc.AccuracyReport.build(self, None)
        if convergence_duration is not None:
            rep.checks.append(timestep_check(self, convergence_duration))
        return rep


class _InitialState:
    """Start state of a GpuSimulation run, kept on the host; `clone(dt)` makes a fresh simulation from it
    (the role of `Simulation._initial` in accusim/simulation.py:101-102 and accuracy.py:200-205)."""

    def __init__(self, system, sim):
        self.system = system
        self._sim = sim

    def clone(self, dt=None):
        s = self._sim
        return GpuSimulation(self.system.copy(), s.forces, integrator=s.integrator, dt=s.dt if dt is None else dt,
                             seed=s.seed, maxnb=s.engine.maxnb, rec_cap=s.engine.rec_cap, tpa=s.engine.tpa)
