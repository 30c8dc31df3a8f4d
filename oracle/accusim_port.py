"""NumPy FP64 restatement of accusim's short-range force-and-step path (test infrastructure only).

Each function names the reference file:line (paths inside the accusim project) it restates. The
arithmetic order follows the reference expression by expression, so results agree with the reference
to the last bits except where NumPy itself is not order-stable (np.add.at scatter order is kept;
einsum's r^2 is reproduced with einsum).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

K_B = 1.380649e-23          # accusim/units.py:229
K_E = 8987551792.261171     # accusim/units.py:232-233 (1 / (4 pi eps0), eps0 = 8.8541878128e-12)
AMU = 1.6605390666e-27      # accusim/units.py:154 (unit "u")
E_CHARGE = 1.602176634e-19  # accusim/units.py:231
N_A = 6.02214076e23         # accusim/units.py:230


@dataclass
class State:
    """Particle state in the layout of accusim/system.py:20-40 (flat float64 arrays, SI units)."""

    pos: np.ndarray
    vel: np.ndarray
    sp: np.ndarray
    ids: np.ndarray
    box: np.ndarray | None
    periodic: bool
    species: list = field(default_factory=list)   # [(name, mass, charge)]

    @property
    def n(self):
        return len(self.pos)

    @property
    def dim(self):
        return self.pos.shape[1]

    @property
    def masses(self):                       # accusim/system.py:83-85
        return np.array([s[1] for s in self.species])[self.sp] if self.n else np.zeros(0)

    @property
    def charges(self):                      # accusim/system.py:87-89
        return np.array([s[2] for s in self.species])[self.sp] if self.n else np.zeros(0)

    def copy(self):
        return State(self.pos.copy(), self.vel.copy(), self.sp.copy(), self.ids.copy(),
                     None if self.box is None else self.box.copy(), self.periodic, list(self.species))


def displacements(st: State) -> np.ndarray:
    """r_j - r_i for all pairs, minimum image: accusim/system.py:95-102."""
    d = st.pos[None, :, :] - st.pos[:, None, :]
    if st.periodic:
        d -= st.box * np.round(d / st.box)
    return d


def _pairs(st: State):
    """accusim/forces.py:24-28."""
    d = displacements(st)
    r2 = np.einsum("ijk,ijk->ij", d, d)
    np.fill_diagonal(r2, np.inf)
    return d, r2


def cell_list_pairs(st: State, rc: float):
    """All pairs i<j closer than rc: accusim/forces.py:279-321 (cells >= rc, 27-cell stencil, final
    minimum-image filter |d|^2 < rc^2)."""
    pos = st.pos
    if st.box is not None:
        lo, span = np.zeros(st.dim), st.box
    else:
        lo = pos.min(axis=0)
        span = np.maximum(pos.max(axis=0) - lo, rc)
    ncell = np.maximum((span // rc).astype(int), 1)
    if st.periodic:
        ncell = np.where(ncell < 3, 1, ncell)
    cell = np.minimum(((pos - lo) / span * ncell).astype(int), ncell - 1)
    cell = np.maximum(cell, 0)
    flat = np.ravel_multi_index(cell.T, ncell)
    order = np.argsort(flat, kind="stable")
    sorted_flat = flat[order]
    starts = np.searchsorted(sorted_flat, np.arange(np.prod(ncell)))
    ends = np.searchsorted(sorted_flat, np.arange(np.prod(ncell)), side="right")
    offsets = np.array(np.meshgrid(*[[-1, 0, 1]] * st.dim)).reshape(st.dim, -1).T
    I, J = [], []
    for c in range(int(np.prod(ncell))):
        a = order[starts[c]:ends[c]]
        if not len(a):
            continue
        cidx = np.array(np.unravel_index(c, ncell))
        neigh = cidx + offsets
        if st.periodic:
            neigh %= ncell
        else:
            neigh = neigh[np.all((neigh >= 0) & (neigh < ncell), axis=1)]
        nflat = np.unique(np.ravel_multi_index(neigh.T, ncell))
        b = np.concatenate([order[starts[k]:ends[k]] for k in nflat])
        ii, jj = np.meshgrid(a, b, indexing="ij")
        keep = ii < jj
        I.append(ii[keep])
        J.append(jj[keep])
    if not I:
        return np.zeros(0, int), np.zeros(0, int)
    i, j = np.concatenate(I), np.concatenate(J)
    d = pos[j] - pos[i]
    if st.periodic:
        d -= st.box * np.round(d / st.box)
    close = np.einsum("ij,ij->i", d, d) < rc ** 2
    return i[close], j[close]


class VerletList:
    """Skin list reused until max displacement^2 >= (skin/2)^2: accusim/forces.py:78-98."""

    def __init__(self):
        self._state = None
        self.rebuilds = 0

    def pairs(self, st: State, rc: float, skin: float):
        s = self._state
        if s is not None and s[3].shape == st.ids.shape and np.array_equal(s[3], st.ids) \
                and np.array_equal(s[4], st.box) and s[5] == rc and skin > 0:
            disp = st.pos - s[2]
            if st.periodic:
                disp -= st.box * np.round(disp / st.box)
            if float(np.max(np.einsum("ij,ij->i", disp, disp))) < (0.5 * skin) ** 2:
                return s[0], s[1]
        i, j = cell_list_pairs(st, rc + skin)
        self._state = (i, j, st.pos.copy(), st.ids.copy(), None if st.box is None else st.box.copy(), rc)
        self.rebuilds += 1
        return i, j


def lj_tables(species_names, params):
    """Lorentz-Berthelot tables: accusim/forces.py:144-155. params: {name: (eps J, sigma m)}."""
    n = len(species_names)
    eps = np.zeros((n, n))
    sig = np.ones((n, n))
    for i, a in enumerate(species_names):
        for j, b in enumerate(species_names):
            if a in params and b in params:
                ea, sa = params[a]
                eb, sb = params[b]
                eps[i, j] = np.sqrt(ea * eb)
                sig[i, j] = 0.5 * (sa + sb)
    return eps, sig


class LennardJones:
    """12-6 LJ, shifted energy at cutoff*sigma_ij, unshifted force: accusim/forces.py:101-175."""

    def __init__(self, params, cutoff=2.5, pairlist_threshold=400, skin=0.3):
        self.params = dict(params)
        self.cutoff = cutoff
        self.pairlist_threshold = pairlist_threshold
        self.skin = skin
        self._vl = VerletList()

    @property
    def rebuilds(self):
        return self._vl.rebuilds

    def tables(self, st):
        return lj_tables([s[0] for s in st.species], self.params)

    def list_radius(self, st):
        """(rc, skin) of the Verlet list: accusim/forces.py:121-123."""
        eps_t, sig_t = self.tables(st)
        smax = float(np.max(np.where(eps_t > 0, sig_t, 0)))
        return self.cutoff * smax, self.skin * smax

    def compute_pairlist(self, st):
        """accusim/forces.py:119-142."""
        eps_t, sig_t = self.tables(st)
        rc, skin = self.list_radius(st)
        i, j = self._vl.pairs(st, rc, skin)
        f = np.zeros_like(st.pos)
        if not len(i):
            return f, 0.0
        d = st.pos[j] - st.pos[i]
        if st.periodic:
            d -= st.box * np.round(d / st.box)
        r2 = np.einsum("ij,ij->i", d, d)
        eps = eps_t[st.sp[i], st.sp[j]]
        sig = sig_t[st.sp[i], st.sp[j]]
        mask = (r2 < (self.cutoff * sig) ** 2) & (eps > 0)
        d, r2, eps, sig, i, j = d[mask], r2[mask], eps[mask], sig[mask], i[mask], j[mask]
        sr6 = (sig ** 2 / r2) ** 3
        src6 = (1 / self.cutoff ** 2) ** 3
        U = float(np.sum(4 * eps * (sr6 ** 2 - sr6 - (src6 ** 2 - src6))))
        coef = -24 * eps * (2 * sr6 ** 2 - sr6) / r2
        fij = coef[:, None] * d
        np.add.at(f, i, fij)
        np.add.at(f, j, -fij)
        return f, U

    def compute_dense(self, st):
        """accusim/forces.py:162-175."""
        eps_t, sig_t = self.tables(st)
        eps = eps_t[st.sp[:, None], st.sp[None, :]]
        sig = sig_t[st.sp[:, None], st.sp[None, :]]
        d, r2 = _pairs(st)
        rc2 = (self.cutoff * sig) ** 2
        mask = (r2 < rc2) & (eps > 0)
        sr2 = np.where(mask, sig ** 2 / np.where(mask, r2, 1.0), 0.0)
        sr6 = sr2 ** 3
        src6 = (1 / self.cutoff ** 2) ** 3
        u = np.where(mask, 4 * eps * (sr6 ** 2 - sr6 - (src6 ** 2 - src6)), 0.0)
        coef = np.where(mask, -24 * eps * (2 * sr6 ** 2 - sr6) / np.where(mask, r2, 1.0), 0.0)
        f = np.einsum("ij,ijk->ik", coef, d)
        return f, 0.5 * float(np.sum(u))

    def compute(self, st):
        """accusim/forces.py:157-161."""
        if st.n < 2:
            return np.zeros_like(st.pos), 0.0
        if st.n >= self.pairlist_threshold:
            return self.compute_pairlist(st)
        return self.compute_dense(st)


def erfc(x):
    """accusim/forces.py:324-330 (scipy.special.erfc, math.erfc fallback)."""
    try:
        from scipy.special import erfc as _e
        return _e(x)
    except ImportError:  # pragma: no cover
        return np.vectorize(math.erfc)(x)


class DampedShiftedCoulomb:
    """Damped shifted force electrostatics (Fennell & Gezelter 2006): accusim/forces.py:391-452."""

    def __init__(self, rcut, alpha=None, k=K_E, pairlist_threshold=400, exclude=(), skin=None):
        self.pairlist_threshold = pairlist_threshold
        self.exclude = [tuple(p) for p in exclude]
        self.k = float(k)
        self.rcut = float(rcut)
        self.alpha = 2.0 / self.rcut if alpha is None else float(alpha)
        self.skin = 0.15 * self.rcut if skin is None else float(skin)
        self._vl = VerletList()

    def constants(self):
        """accusim/forces.py:413-416."""
        a, rc = self.alpha, self.rcut
        c = 2 * a / np.sqrt(np.pi)
        erc = float(erfc(np.array(a * rc)))
        fshift = erc / rc ** 2 + c * np.exp(-(a * rc) ** 2) / rc
        return c, erc, fshift

    def compute(self, st):
        """accusim/forces.py:408-452."""
        q = st.charges
        f = np.zeros_like(st.pos)
        if not np.any(q):
            return f, 0.0
        a, rc = self.alpha, self.rcut
        c, erc, fshift = self.constants()
        where = {pid: n for n, pid in enumerate(st.ids)} if self.exclude else {}
        ex = np.array([(where[x], where[y]) for x, y in self.exclude if x in where and y in where],
                      dtype=int).reshape(-1, 2)
        if st.n >= self.pairlist_threshold:
            i, j = self._vl.pairs(st, rc, self.skin)
            if len(ex):
                lo, hi = np.minimum(ex[:, 0], ex[:, 1]), np.maximum(ex[:, 0], ex[:, 1])
                keep = ~np.isin(i * st.n + j, lo * st.n + hi)
                i, j = i[keep], j[keep]
            d = st.pos[j] - st.pos[i]
            if st.periodic:
                d -= st.box * np.round(d / st.box)
            r = np.sqrt(np.einsum("ij,ij->i", d, d))
            inside = r < rc
            i, j, d, r = i[inside], j[inside], d[inside], r[inside]
            er = erfc(a * r)
            qq = q[i] * q[j]
            U = float(np.sum(qq * (er / r - erc / rc + fshift * (r - rc))))
            U -= float(np.sum(q ** 2)) * (erc / (2 * rc) + a / np.sqrt(np.pi))
            fv = (qq * ((er / r ** 2 + c * np.exp(-(a * r) ** 2) / r) - fshift) / r)[:, None] * d
            np.add.at(f, i, -fv)
            np.add.at(f, j, fv)
            return self.k * f, self.k * U
        d, r2 = _pairs(st)
        r = np.sqrt(r2)
        inside = r < rc
        rr = np.where(inside, r, 1.0)
        er = erfc(a * rr)
        qq = np.where(inside, q[:, None] * q[None, :], 0.0)
        if len(ex):
            qq[ex[:, 0], ex[:, 1]] = 0.0
            qq[ex[:, 1], ex[:, 0]] = 0.0
        U = 0.5 * float(np.sum(qq * (er / rr - erc / rc + fshift * (rr - rc))))
        U -= float(np.sum(q ** 2)) * (erc / (2 * rc) + a / np.sqrt(np.pi))
        fmag = qq * ((er / rr ** 2 + c * np.exp(-(a * rr) ** 2) / rr) - fshift) / rr
        f = -self.k * np.einsum("ij,ijk->ik", fmag, d)
        return f, self.k * U


class Ewald:
    """Ewald summation, the label oracle for the learned DSF correction: accusim/forces.py:333-388."""

    def __init__(self, k=K_E, alpha=None, rcut=None, kmax=12):
        self.k = float(k)
        self.alpha = alpha
        self.rcut = rcut
        self.kmax = kmax

    def kvectors(self, box, alpha):
        """accusim/forces.py:347-357."""
        n = np.arange(-self.kmax, self.kmax + 1)
        N = np.stack(np.meshgrid(n, n, n, indexing="ij"), -1).reshape(-1, 3)
        N = N[np.sum(N ** 2, axis=1) <= self.kmax ** 2]
        N = N[np.any(N != 0, axis=1)]
        kv = 2 * np.pi * N / box
        k2 = np.sum(kv ** 2, axis=1)
        return kv, np.exp(-k2 / (4 * alpha ** 2)) / k2

    def compute(self, st):
        """accusim/forces.py:359-388."""
        if st.dim != 3 or not st.periodic:
            raise ValueError("Ewald needs a 3D periodic box")
        q = st.charges
        f = np.zeros_like(st.pos)
        if not np.any(q):
            return f, 0.0
        if abs(q.sum()) > 1e-9 * np.sum(np.abs(q)):
            raise ValueError("Ewald summation here requires a charge-neutral system")
        box = st.box
        rcut = self.rcut or 0.5 * float(np.min(box))
        a = self.alpha or 4.0 / rcut
        d, r2 = _pairs(st)
        np.fill_diagonal(r2, np.inf)
        r = np.sqrt(r2)
        qq = q[:, None] * q[None, :]
        inside = r < rcut
        erfc_r = np.where(inside, erfc(a * np.where(inside, r, 0)), 0.0)
        U_real = 0.5 * float(np.sum(np.where(inside, qq * erfc_r / r, 0)))
        coef = np.where(inside, qq * (erfc_r / r + 2 * a / np.sqrt(np.pi) * np.exp(-(a * r) ** 2)) / r2, 0)
        f -= np.einsum("ij,ijk->ik", coef, d)
        kv, w = self.kvectors(box, a)
        V = float(np.prod(box))
        phase = st.pos @ kv.T
        S = (q[:, None] * np.exp(1j * phase)).sum(0)
        U_rec = 2 * np.pi / V * float(np.sum(w * np.abs(S) ** 2))
        im = np.imag(np.conj(S)[None, :] * np.exp(1j * phase))
        f += 4 * np.pi / V * q[:, None] * ((w[None, :] * im) @ kv)
        U_self = -a / np.sqrt(np.pi) * float(np.sum(q ** 2))
        return self.k * f, self.k * (U_real + U_rec + U_self)


def apply_boundaries(st: State):
    """Periodic wrap `pos %= box`: accusim/system.py:124-129 (walls: 130-140)."""
    if st.box is None:
        return
    if st.periodic:
        st.pos %= st.box
        return
    for _ in range(4):
        low = st.pos < 0
        high = st.pos > st.box
        if not (low.any() or high.any()):
            break
        st.pos = np.where(low, -st.pos, st.pos)
        st.pos = np.where(high, 2 * st.box - st.pos, st.pos)
        hit = low | high
        st.vel = np.where(hit, -st.vel, st.vel)


def potential(st, forces):
    """accusim/simulation.py:57-65."""
    f = np.zeros_like(st.pos)
    u = 0.0
    for force in forces:
        fi, ui = force.compute(st)
        f += fi
        u += ui
    return f, u


def kinetic_energy(st):        # accusim/system.py:106-107
    return 0.5 * float(np.sum(st.masses[:, None] * st.vel ** 2))


def momentum(st):              # accusim/system.py:109-110
    return np.sum(st.masses[:, None] * st.vel, axis=0)


def angular_momentum(st):      # accusim/system.py:112-114
    L = np.cross(st.pos, st.masses[:, None] * st.vel)
    return np.atleast_1d(np.sum(L, axis=0))


class LangevinBAOAB:
    """BAOAB Langevin step: accusim/integrators.py:50-71. `normal(shape)` supplies the standard normal
    draws (the reference uses `sim.rng.normal`)."""

    def __init__(self, T, gamma, normal):
        self.T, self.gamma, self.normal = float(T), float(gamma), normal

    def step(self, run, dt):
        st = run.st
        st.vel += 0.5 * dt * run.acc
        st.pos += 0.5 * dt * st.vel
        c1 = np.exp(-self.gamma * dt)
        sig = np.sqrt((1 - c1 ** 2) * K_B * self.T / st.masses)[:, None]
        st.vel = c1 * st.vel + sig * self.normal(st.vel.shape)
        st.pos += 0.5 * dt * st.vel
        apply_boundaries(st)
        run.update_forces()
        st.vel += 0.5 * dt * run.acc


class NoseHooverMTK:
    """Nose-Hoover with the Trotter half-steps of accusim/integrators.py:74-116 (thermostat mass
    Q = N_f kT tau^2, N_f = dim (n - 1)); bath energy Q xi^2 / 2 + N_f kT eta."""

    def __init__(self, T, tau):
        self.T, self.tau = float(T), float(tau)
        self.xi, self.eta, self.Q = 0.0, 0.0, None

    @staticmethod
    def dof(st):
        return st.dim * max(st.n - 1, 1)

    def half(self, st, dt):
        kT, nf = K_B * self.T, self.dof(st)
        if self.Q is None:
            self.Q = nf * kT * self.tau ** 2
        k2 = float(np.sum(st.masses[:, None] * st.vel ** 2))
        self.xi += 0.25 * dt * (k2 - nf * kT) / self.Q
        scale = np.exp(-0.5 * dt * self.xi)
        st.vel *= scale
        self.eta += 0.5 * dt * self.xi
        self.xi += 0.25 * dt * (k2 * scale ** 2 - nf * kT) / self.Q

    def step(self, run, dt):
        st = run.st
        self.half(st, dt)
        st.vel += 0.5 * dt * run.acc
        st.pos += dt * st.vel
        apply_boundaries(st)
        run.update_forces()
        st.vel += 0.5 * dt * run.acc
        self.half(st, dt)

    def bath_energy(self, st):
        if self.Q is None:
            return 0.0
        return 0.5 * self.Q * self.xi ** 2 + self.dof(st) * K_B * self.T * self.eta


class Run:
    """Simulation.run with per-step records: accusim/simulation.py:95-112, record fields of
    accusim/simulation.py:76-93. The integrator is VelocityVerlet (accusim/integrators.py:25-31) unless an
    object with `step(run, dt)` (LangevinBAOAB, NoseHooverMTK) is given."""

    def __init__(self, st, forces, dt, integrator=None):
        self.st, self.forces, self.dt = st, forces, float(dt)
        self.integrator = integrator
        self.time = 0.0
        self.t, self.kinetic, self.potential, self.momentum, self.angular_momentum = [], [], [], [], []
        self.bath = []
        self.update_forces()

    def update_forces(self):
        """accusim/simulation.py:67-70."""
        self.force, self.pe = potential(self.st, self.forces)
        m = self.st.masses
        self.acc = self.force / m[:, None] if len(m) else self.force

    def record(self):
        st = self.st
        self.t.append(self.time)
        self.kinetic.append(kinetic_energy(st))
        self.potential.append(self.pe)
        self.momentum.append(momentum(st))
        self.angular_momentum.append(angular_momentum(st))
        bath = getattr(self.integrator, "bath_energy", None)
        self.bath.append(bath(st) if bath else 0.0)

    def step(self):
        """accusim/integrators.py:25-31."""
        if self.integrator is not None:
            self.integrator.step(self, self.dt)
            return
        st, dt = self.st, self.dt
        st.vel += 0.5 * dt * self.acc
        st.pos += dt * st.vel
        apply_boundaries(st)
        self.update_forces()
        st.vel += 0.5 * dt * self.acc

    def run(self, steps, record_every=1):
        if not self.t:
            self.record()
        for k in range(1, steps + 1):
            self.step()
            self.time += self.dt
            if k % record_every == 0 or k == steps:
                self.record()
        return self

    @property
    def total_energy(self):
        return np.array(self.kinetic) + np.array(self.potential)


def energy_drift(E, kinetic, potential):
    """Report metric max|E-E0| / max(|E0|, max|KE|, max|PE|): accusim/accuracy.py:70-76."""
    E = np.asarray(E)
    scale = max(abs(E[0]), np.max(np.abs(kinetic)), np.max(np.abs(potential)), 1e-300)
    return float(np.max(np.abs(E - E[0])) / scale)


def momentum_drift(P, masses, vel):
    """Report metric max|P-P0| / sum m|v|: accusim/accuracy.py:86-91."""
    P = np.asarray(P)
    pscale = max(float(np.sum(masses[:, None] * np.abs(vel))), 1e-300)
    return float(np.max(np.linalg.norm(P - P[0], axis=1)) / pscale)


def richardson(finals, n, order=2):
    """Timestep-error estimate from finals at dt, dt/2, dt/4: accusim/accuracy.py:191-221.
    Returns (status, value, p)."""
    size = max(float(np.ptp(finals[2])), 1e-300)
    roundoff = 1e-13 * np.sqrt(n * 4)
    e1 = float(np.sqrt(np.mean((finals[0] - finals[1]) ** 2))) / size
    e2 = float(np.sqrt(np.mean((finals[1] - finals[2]) ** 2))) / size
    if e1 < 10 * roundoff:
        return "PASS", e1, None
    p = np.log2(e1 / e2)
    est = e1 * 2 ** p / (2 ** p - 1) if p > 0.2 else e1
    if p < 0.5 * order:
        return ("FAIL" if est > 1e-2 else "WARN"), est, p
    return ("PASS" if est <= 1e-6 else "WARN" if est <= 1e-3 else "FAIL"), est, p
