"""Generate the golden vectors the parity tests pin against, by running the reference accusim itself.

Run where the reference is importable: from $ACCUSIM_REF (a checkout of the reference project), else from the
repository's offline install under baseline/_ref (baseline/install_reference.sh), else an installed accusim:
    ACCUSIM_REF=<checkout> python tests/golden/make_golden.py
The .npz files it writes are committed; nothing at test time imports the reference.

Each case restates a reference test or example setup (file:line inside the accusim project):
  lj_mix_{periodic,open}  tests/test_forces.py:64-76   300 Ar + 200 Kr, 4 nm box
  lj_mix_ortho            the same mixture in a periodic 4 x 3 x 5.2 nm box (unequal edges)
  report_argon108         accusim/accuracy.py:60-110, 191-221: the accuracy report of a 60-step VelocityVerlet
                          run of 108 argon atoms, with the dt/2, dt/4 Richardson runs over 0.3 ps
  calibrate_argon108      accusim/advisor.py:51-79: calibrate_dt from dt = 40 fs (halvings) and from dt unset
                          (suggest_dt), 108 argon atoms, 0.4 ps trials, energy tolerance 1e-5
  report_nacl512          the same for a 512-ion NaCl melt (LJ + DSF, 20 steps of 1 fs, Richardson over 10 fs):
                          adds the two-species timescales and the DSF vs Ewald row (accusim/accuracy.py:148-161)
  coulomb_ortho           rock salt 10 x 8 x 12 sites, perturbed, in its box of unequal edges: DSF (dense and
                          cell paths, tests/test_dsf.py:55-61) and Ewald (tests/test_dsf.py:46-52)
  argon864                examples/rahman_argon.py:19-30 geometry at the fcc 6^3 / L=10.229 sigma config
  lj500_skin              tests/test_nose_hoover.py:6-17, 51-60   skin == fresh list along a VV run
  dsf_rocksalt10          tests/test_dsf.py:55-61       DSF dense == cell path
  dsf_exclusions          tests/test_dsf.py:94-102      exclusions
  dsf_skin                tests/test_dsf.py:119-139     Verlet skin == fresh list, rebuild count
  nacl4096                examples/molten_salt.py:22-33 geometry at the 4096-ion / 1.55 g/cm^3 config
  ewald_melt512           tests/test_dsf.py:46-52       Ewald label oracle on a disordered melt
  thermostats108          tests/test_nose_hoover.py:6-17 argon; Langevin BAOAB and Nose-Hoover runs
  analysis_melt1000       accusim/analysis.py:7-24 rdf (all ions, Na only) on a perturbed rock-salt box
  analysis_msd108         accusim/analysis.py:27-43 msd, and io_traj108.npz written by accusim/io.py:13-26
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

_INSTALL = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "baseline",
                        "_ref")
REF = os.environ.get("ACCUSIM_REF") or (_INSTALL if os.path.isdir(os.path.join(_INSTALL, "accusim")) else None)
if REF:
    sys.path.insert(0, REF)
import accusim  # noqa: E402
from accusim import Q, Simulation, System, VelocityVerlet, k_B  # noqa: E402
from accusim.integrators import Langevin, NoseHoover  # noqa: E402
from accusim.forces import DampedShiftedCoulomb, Ewald, LennardJones, cell_list_pairs  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
N_A = 6.02214076e23


def pairset_digest(i, j, n):
    key = np.sort(np.minimum(i, j).astype(np.int64) * n + np.maximum(i, j).astype(np.int64))
    return hashlib.sha256(key.tobytes()).hexdigest(), len(key)


def state_arrays(s):
    return dict(pos=s.pos.copy(), vel=s.vel.copy(), sp=s.sp.astype(np.int32), ids=s.ids.astype(np.int64),
                box=np.zeros(3) if s.box is None else s.box.copy(), has_box=s.box is not None,
                periodic=bool(s.periodic),
                masses=np.array([x.mass for x in s.species]), charges=np.array([x.charge for x in s.species]),
                species=np.array([x.name for x in s.species]))


def save(name, **kw):
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **kw)
    print(f"{name}: {os.path.getsize(path) / 1024:.0f} KiB")


def lj_mix(periodic, box=None, name=None):
    rng = np.random.default_rng(5)
    edges = np.full(3, 4e-9) if box is None else np.asarray(box, float)
    s = System(3, box=Q(4, "nm") if box is None else edges, periodic=periodic)
    s.add_species("Ar", Q(39.948, "u"))
    s.add_species("Kr", Q(83.8, "u"))
    s.add("Ar", rng.uniform(0, 1, (300, 3)) * edges)
    s.add("Kr", rng.uniform(0, 1, (200, 3)) * edges)
    params = {"Ar": (1.65e-21, 3.4e-10), "Kr": (2.3e-21, 3.6e-10)}
    Fd, Ud = LennardJones(params, pairlist_threshold=10 ** 9).compute(s)
    lj = LennardJones(params, pairlist_threshold=2)
    Fl, Ul = lj.compute(s)
    eps_t, sig_t = lj._tables(s)
    smax = float(np.max(np.where(eps_t > 0, sig_t, 0)))
    rl = (lj.cutoff + lj.skin) * smax
    i, j = cell_list_pairs(s, rl)
    save(name or f"lj_mix_{'periodic' if periodic else 'open'}", **state_arrays(s),
         param_names=np.array(["Ar", "Kr"]), param_eps=np.array([1.65e-21, 2.3e-21]),
         param_sig=np.array([3.4e-10, 3.6e-10]), cutoff=2.5, skin=0.3,
         F_dense=Fd, U_dense=Ud, F_list=Fl, U_list=Ul, list_radius=rl,
         pair_i=i.astype(np.int32), pair_j=j.astype(np.int32))


def fcc(n_cells, L):
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) + 0.25
    pts = np.array([b + [i, j, k] for i in range(n_cells) for j in range(n_cells) for k in range(n_cells)
                    for b in base])
    return pts * L / n_cells


def argon864():
    sig, m = 3.4e-10, Q(39.948, "u").value
    L = 10.229 * sig
    s = System(3, box=L, periodic=True)
    s.add_species("Ar", m)
    s.add("Ar", fcc(6, L))
    s.maxwell_boltzmann(94.4, np.random.default_rng(0))
    init = state_arrays(s)
    lj = LennardJones({"Ar": (120 * k_B.value, sig)}, cutoff=2.5)
    sim = Simulation(s, [lj], integrator=VelocityVerlet(), dt=Q(10, "fs"))
    tr = sim.run(steps=60, positions=False)
    F, U = LennardJones({"Ar": (120 * k_B.value, sig)}, cutoff=2.5, skin=0.0).compute(s)
    i, j = cell_list_pairs(s, 2.8 * sig)
    save("argon864", **{k + "0": v for k, v in init.items()}, **state_arrays(s), eps=120 * k_B.value, sig=sig,
         dt=Q(10, "fs").value, steps=60, kinetic=np.array(tr.kinetic), potential=np.array(tr.potential),
         momentum=np.array(tr.momentum), rebuilds=lj.rebuilds, F=F, U=U, acc=sim.acc,
         pair_i=i.astype(np.int32), pair_j=j.astype(np.int32), list_radius=2.8 * sig)


def lj500_skin():
    m = Q(39.948, "u").value
    L = (4 * 5 ** 3 * m / 1374.0) ** (1 / 3)
    s = System(3, box=L, periodic=True)
    s.add_species("Ar", m)
    s.add("Ar", fcc(5, L))
    s.maxwell_boltzmann(300, np.random.default_rng(3))
    init = state_arrays(s)
    lj = LennardJones({"Ar": (120 * k_B.value, 3.4e-10)}, cutoff=2.5)
    sim = Simulation(s, [lj], integrator=VelocityVerlet(), dt=Q(5, "fs"))
    Us = []
    for _ in range(10):
        sim.run(steps=20, positions=False)
        Us.append(lj.compute(s)[1])
    F0, U0 = LennardJones({"Ar": (120 * k_B.value, 3.4e-10)}, cutoff=2.5, skin=0.0).compute(s)
    save("lj500_skin", **{k + "0": v for k, v in init.items()}, **state_arrays(s), eps=120 * k_B.value,
         sig=3.4e-10, dt=Q(5, "fs").value, rebuilds=lj.rebuilds, U_series=np.array(Us), F=F0, U=U0,
         acc=sim.acc)


def rocksalt(n):
    s = System(3, box=float(n), periodic=True)
    s.add_species("Na", 1.0, charge=1.0)
    s.add_species("Cl", 1.0, charge=-1.0)
    g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    odd = g.sum(1) % 2 == 1
    s.add("Na", g[~odd].astype(float))
    s.add("Cl", g[odd].astype(float))
    return s


def dsf_cases():
    s = rocksalt(10)
    rng = np.random.default_rng(3)
    s.pos = (s.pos + rng.normal(0, 0.2, s.pos.shape)) % s.box
    fd, ud = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9).compute(s)
    fc, uc = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1).compute(s)
    save("dsf_rocksalt10", **state_arrays(s), rcut=2.5, alpha=2.0 / 2.5, k=1.0, skin=0.15 * 2.5,
         F_dense=fd, U_dense=ud, F_list=fc, U_list=uc)

    s = rocksalt(8)
    rng = np.random.default_rng(5)
    s.pos = (s.pos + rng.normal(0, 0.2, s.pos.shape)) % s.box
    ex = [(int(s.ids[2 * m]), int(s.ids[2 * m + 1])) for m in range(50)]
    fd, ud = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9, exclude=ex).compute(s)
    fc, uc = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1, exclude=ex).compute(s)
    f0, u0 = DampedShiftedCoulomb(rcut=2.5, k=1.0).compute(s)
    save("dsf_exclusions", **state_arrays(s), rcut=2.5, alpha=2.0 / 2.5, k=1.0, skin=0.15 * 2.5,
         exclude=np.array(ex, dtype=np.int64), F_dense=fd, U_dense=ud, F_list=fc, U_list=uc, F_noex=f0, U_noex=u0)

    n = 8
    s = rocksalt(n)
    rng = np.random.default_rng(5)
    skinned = DampedShiftedCoulomb(rcut=3.9, alpha=0.6, k=1.0, skin=0.6)
    Us, Ps = [], []
    for _ in range(30):
        s.pos = (s.pos + rng.normal(0, 0.05, s.pos.shape)) % s.box
        f1, u1 = skinned.compute(s)
        Us.append(u1)
        Ps.append(s.pos.copy())
    save("dsf_skin", **state_arrays(s), rcut=3.9, alpha=0.6, k=1.0, skin=0.6, U_series=np.array(Us),
         rebuilds=skinned._vl.rebuilds, F=f1, U=u1, pos_series=np.array(Ps, dtype=np.float64)[::6])


def coulomb_ortho():
    s = System(3, box=np.array([10.0, 8.0, 12.0]), periodic=True)
    s.add_species("Na", 1.0, charge=1.0)
    s.add_species("Cl", 1.0, charge=-1.0)
    g = np.stack(np.meshgrid(np.arange(10), np.arange(8), np.arange(12), indexing="ij"), -1).reshape(-1, 3)
    odd = g.sum(1) % 2 == 1
    s.add("Na", g[~odd].astype(float))
    s.add("Cl", g[odd].astype(float))
    rng = np.random.default_rng(11)
    s.pos = (s.pos + rng.normal(0, 0.2, s.pos.shape)) % s.box
    fd, ud = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9).compute(s)
    fc, uc = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1).compute(s)
    Fe, Ue = Ewald(k=1.0).compute(s)
    save("coulomb_ortho", **state_arrays(s), rcut=2.5, alpha=2.0 / 2.5, k=1.0, F_dense=fd, U_dense=ud,
         F_list=fc, U_list=uc, F_ewald=Fe, U_ewald=Ue)


def nacl4096():
    n = 16
    mass_g = n ** 3 / 2 * (22.98977 + 35.453) / N_A
    L = (mass_g / 1.55) ** (1 / 3) * 1e-2
    s = System(3, box=L, periodic=True)
    s.add_species("Na", Q(22.98977, "u"), charge=Q(1, "e"))
    s.add_species("Cl", Q(35.453, "u"), charge=Q(-1, "e"))
    g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    odd = g.sum(1) % 2 == 1
    s.add("Na", (g[~odd] + 0.5) * L / n)
    s.add("Cl", (g[odd] + 0.5) * L / n)
    s.maxwell_boltzmann(1200, rng=np.random.default_rng(0))
    init = state_arrays(s)
    params = {"Na": (0.544e3 / N_A, 2.35e-10), "Cl": (0.418e3 / N_A, 4.40e-10)}
    lj = LennardJones(params, cutoff=2.5)
    dsf = DampedShiftedCoulomb(rcut=12e-10, alpha=Q(0.2, "1/A"))
    sim = Simulation(s, [lj, dsf], integrator=VelocityVerlet(), dt=Q(1, "fs"))
    tr = sim.run(steps=10, positions=False)
    Flj, Ulj = LennardJones(params, cutoff=2.5, skin=0.0).compute(s)
    Fd, Ud = DampedShiftedCoulomb(rcut=12e-10, alpha=Q(0.2, "1/A"), skin=0.0).compute(s)
    i, j = cell_list_pairs(s, 12.32e-10)
    dig_lj, cnt_lj = pairset_digest(i, j, s.n)
    i, j = cell_list_pairs(s, 13.8e-10)
    dig_dsf, cnt_dsf = pairset_digest(i, j, s.n)
    save("nacl4096", **{k + "0": v for k, v in init.items()}, **state_arrays(s),
         param_names=np.array(["Na", "Cl"]), param_eps=np.array([0.544e3 / N_A, 0.418e3 / N_A]),
         param_sig=np.array([2.35e-10, 4.40e-10]), rcut=12e-10, alpha=0.2e10, dsf_skin=1.8e-10,
         dt=Q(1, "fs").value, steps=10, kinetic=np.array(tr.kinetic), potential=np.array(tr.potential),
         F_lj=Flj, U_lj=Ulj, F_dsf=Fd, U_dsf=Ud, acc=sim.acc,
         pairs_lj_sha=dig_lj, pairs_lj_count=cnt_lj, pairs_dsf_sha=dig_dsf, pairs_dsf_count=cnt_dsf,
         rebuilds_lj=lj.rebuilds, rebuilds_dsf=dsf._vl.rebuilds)


def ewald_melt():
    s = rocksalt(8)
    rng = np.random.default_rng(7)
    s.pos = (s.pos + rng.normal(0, 0.25, s.pos.shape)) % s.box
    Fe, Ue = Ewald(k=1.0).compute(s)
    Fd, Ud = DampedShiftedCoulomb(rcut=3.9, alpha=0.6, k=1.0).compute(s)
    save("ewald_melt512", **state_arrays(s), F=Fe, U=Ue, F_dsf=Fd, U_dsf=Ud, dsf_rcut=3.9, dsf_alpha=0.6)


def thermostats108():
    """108 argon atoms (fcc 3^3 at 1374 kg/m^3, 60 K) under Langevin (120 K, 5e12 1/s, seed 11) and
    Nose-Hoover (120 K, 0.2 ps), 40 steps of 5 fs each, records every 10 steps."""
    m = Q(39.948, "u").value
    L = (4 * 27 * m / 1374.0) ** (1 / 3)
    out = {}
    for name in ("lv", "nh"):
        s = System(3, box=L, periodic=True)
        s.add_species("Ar", m)
        s.add("Ar", fcc(3, L))
        s.maxwell_boltzmann(60.0, np.random.default_rng(3))
        if name == "lv":
            out.update({k + "0": v for k, v in state_arrays(s).items()})
        lj = LennardJones({"Ar": (120 * k_B.value, 3.4e-10)}, cutoff=2.5)
        integ = Langevin(120.0, 5e12) if name == "lv" else NoseHoover(120.0, Q(0.2, "ps"))
        sim = Simulation(s, [lj], integrator=integ, dt=Q(5, "fs"), seed=11)
        tr = sim.run(steps=40, record_every=10, positions=False)
        out.update({f"{name}_pos": s.pos.copy(), f"{name}_vel": s.vel.copy(), f"{name}_acc": sim.acc.copy(),
                    f"{name}_kinetic": np.array(tr.kinetic), f"{name}_potential": np.array(tr.potential),
                    f"{name}_bath": np.array(tr.bath)})
        if name == "nh":
            out.update(nh_xi=integ.xi, nh_eta=integ.eta, nh_Q=integ.Q)
    save("thermostats108", **out, eps=120 * k_B.value, sig=3.4e-10, dt=Q(5, "fs").value, steps=40, record_every=10,
         T=120.0, friction=5e12, seed=11, tau=Q(0.2, "ps").value)


def report_argon108():
    m = Q(39.948, "u").value
    L = (4 * 27 * m / 1374.0) ** (1 / 3)
    s = System(3, box=L, periodic=True)
    s.add_species("Ar", m)
    s.add("Ar", fcc(3, L))
    s.maxwell_boltzmann(90.0, np.random.default_rng(8))
    init = state_arrays(s)
    lj = LennardJones({"Ar": (120 * k_B.value, 3.4e-10)}, cutoff=2.5)
    sim = Simulation(s, [lj], integrator=VelocityVerlet(), dt=Q(5, "fs"))
    sim.run(steps=60, record_every=1, positions=False)
    rep = sim.accuracy_report(convergence_duration=Q(0.3, "ps"))
    save("report_argon108", **init, eps=120 * k_B.value, sig=3.4e-10, dt=Q(5, "fs").value, steps=60,
         convergence_duration=Q(0.3, "ps").value,
         names=np.array([c.name for c in rep.checks]), statuses=np.array([c.status for c in rep.checks]),
         values=np.array([np.nan if c.value is None else float(c.value) for c in rep.checks]))


def report_nacl512():
    n = 8
    mass_g = n ** 3 / 2 * (22.98977 + 35.453) / N_A
    L = (mass_g / 1.55) ** (1 / 3) * 1e-2
    s = System(3, box=L, periodic=True)
    s.add_species("Na", Q(22.98977, "u"), charge=Q(1, "e"))
    s.add_species("Cl", Q(35.453, "u"), charge=Q(-1, "e"))
    g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    odd = g.sum(1) % 2 == 1
    s.add("Na", (g[~odd] + 0.5) * L / n)
    s.add("Cl", (g[odd] + 0.5) * L / n)
    s.maxwell_boltzmann(1300, rng=np.random.default_rng(12))
    init = state_arrays(s)
    params = {"Na": (0.544e3 / N_A, 2.35e-10), "Cl": (0.418e3 / N_A, 4.40e-10)}
    lj = LennardJones(params, cutoff=2.5)
    dsf = DampedShiftedCoulomb(rcut=10e-10, alpha=Q(0.2, "1/A"))
    sim = Simulation(s, [lj, dsf], integrator=VelocityVerlet(), dt=Q(1, "fs"))
    sim.run(steps=20, record_every=1, positions=False)
    rep = sim.accuracy_report(convergence_duration=Q(10, "fs"))
    save("report_nacl512", **init, param_names=np.array(["Na", "Cl"]),
         param_eps=np.array([0.544e3 / N_A, 0.418e3 / N_A]), param_sig=np.array([2.35e-10, 4.40e-10]),
         rcut=10e-10, alpha=0.2e10, dt=Q(1, "fs").value, steps=20, convergence_duration=Q(10, "fs").value,
         names=np.array([c.name for c in rep.checks]), statuses=np.array([c.status for c in rep.checks]),
         values=np.array([np.nan if c.value is None else float(c.value) for c in rep.checks]))


def calibrate_argon108():
    from accusim.advisor import calibrate_dt
    m = Q(39.948, "u").value
    L = (4 * 27 * m / 1374.0) ** (1 / 3)
    s = System(3, box=L, periodic=True)
    s.add_species("Ar", m)
    s.add("Ar", fcc(3, L))
    s.maxwell_boltzmann(90.0, np.random.default_rng(21))
    init = state_arrays(s)
    out = {}
    for tag, dt0 in (("from40fs", Q(40, "fs")), ("suggested", None)):
        lj = LennardJones({"Ar": (120 * k_B.value, 3.4e-10)}, cutoff=2.5)
        sim = Simulation(s.copy(), [lj], integrator=VelocityVerlet(), dt=dt0)
        dt, drift = calibrate_dt(sim, Q(0.4, "ps"), energy_tol=1e-5)
        out[f"{tag}_dt"], out[f"{tag}_drift"] = dt, drift
    save("calibrate_argon108", **init, eps=120 * k_B.value, sig=3.4e-10, trial=Q(0.4, "ps").value, tol=1e-5,
         dt0=Q(40, "fs").value, **out)


def analysis_cases():
    from accusim import analysis
    from accusim import io as aio
    # rdf: 1000 ions of rock salt (10^3 sites, a/2 = 2.82 A) displaced by seeded 0.3 A noise
    s = System(3, box=10 * 2.82e-10, periodic=True)
    s.add_species("Na", Q(22.98977, "u").value, charge=1.602176634e-19)
    s.add_species("Cl", Q(35.453, "u").value, charge=-1.602176634e-19)
    g = np.stack(np.meshgrid(*[np.arange(10)] * 3, indexing="ij"), -1).reshape(-1, 3)
    odd = g.sum(1) % 2 == 1
    rng = np.random.default_rng(17)
    s.add("Na", ((g[~odd] + 0.5) * 2.82e-10 + rng.normal(0, 0.3e-10, (int((~odd).sum()), 3))) % s.box)
    s.add("Cl", ((g[odd] + 0.5) * 2.82e-10 + rng.normal(0, 0.3e-10, (int(odd.sum()), 3))) % s.box)
    rmax = 0.45 * 10 * 2.82e-10
    r_all, g_all = analysis.rdf(s, rmax, bins=120)
    r_na, g_na = analysis.rdf(s, rmax, bins=60, species="Na")
    save("analysis_melt1000", **state_arrays(s), rmax=rmax, r_all=r_all, g_all=g_all, r_na=r_na, g_na=g_na)
    # msd and io: 108 argon atoms, positions recorded every step for 20 steps of 10 fs
    m = Q(39.948, "u").value
    L = (4 * 27 * m / 1374.0) ** (1 / 3)
    s = System(3, box=L, periodic=True)
    s.add_species("Ar", m)
    s.add("Ar", fcc(3, L))
    s.maxwell_boltzmann(300.0, np.random.default_rng(8))
    sim = Simulation(s, [LennardJones({"Ar": (120 * k_B.value, 3.4e-10)}, cutoff=2.5)], integrator=VelocityVerlet(),
                     dt=Q(10, "fs"))
    tr = sim.run(steps=20, record_every=1, positions=True)
    t, msd = analysis.msd(tr, box=s.box)
    save("analysis_msd108", t_frames=np.array(tr.t), frames=np.array(tr.positions), box=s.box.copy(), t=t, msd=msd)
    aio.save(tr, s, os.path.join(OUT, "io_traj108.npz"))
    print(f"io_traj108: {os.path.getsize(os.path.join(OUT, 'io_traj108.npz')) / 1024:.0f} KiB")


CASES = {
    "lj_mix": lambda: (lj_mix(True), lj_mix(False)),
    "lj_mix_ortho": lambda: lj_mix(True, box=(4e-9, 3e-9, 5.2e-9), name="lj_mix_ortho"),
    "coulomb_ortho": coulomb_ortho,
    "report_argon108": report_argon108,
    "report_nacl512": report_nacl512,
    "calibrate_argon108": calibrate_argon108,
}


if __name__ == "__main__":
    print("reference accusim", accusim.__version__, "from", os.path.dirname(accusim.__file__))
    if len(sys.argv) > 1:   # named cases only: python make_golden.py lj_mix_ortho
        for name in sys.argv[1:]:
            CASES[name]()
        sys.exit(0)
    lj_mix(True)
    lj_mix(False)
    CASES["lj_mix_ortho"]()
    coulomb_ortho()
    argon864()
    lj500_skin()
    dsf_cases()
    nacl4096()
    ewald_melt()
    thermostats108()
    report_argon108()
    report_nacl512()
    calibrate_argon108()
    analysis_cases()
