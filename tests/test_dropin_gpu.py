"""Parity of the FP64 drop-in plug-ins (C ABI kernels) with the reference: golden vectors generated by the
reference itself and the CPU oracle. Tolerances: pair sets bit-exact (ties within 1 ulp of rc^2 reported
and allowed); forces max|dF| <= 1e-12 max|F_ref|, energies |dU| <= 1e-12 |U_ref| (the norm of the
reference's own skin tests, tests/test_nose_hoover.py:45-46)."""
import hashlib

import numpy as np
import pytest

from oracle import accusim_port as port
from tests._helpers import pair_keys, rel_max

pytestmark = pytest.mark.gpu

TOL = 1e-12


def product_system(g, suffix=""):
    from accusim import System
    box = g["box" + suffix] if bool(g["has_box" + suffix]) else None
    s = System(3, box=box, periodic=bool(g["periodic" + suffix]))
    for name, m, q in zip(g["species" + suffix], g["masses" + suffix], g["charges" + suffix]):
        s.add_species(str(name), float(m), charge=float(q))
    s.pos = g["pos" + suffix].copy()
    s.vel = g["vel" + suffix].copy()
    s.sp = g["sp" + suffix].astype(int)
    s.ids = g["ids" + suffix].astype(int)
    s._next_id = int(s.ids.max()) + 1
    s.eint = np.zeros(s.n)
    return s


def _ties(s, keys_a, keys_b, rc):
    """Pairs in exactly one set must be r^2 ties with rc^2 (within 4 ulp)."""
    diff = np.setxor1d(keys_a, keys_b)
    for key in diff:
        i, j = divmod(int(key), s.n)
        d = s.pos[j] - s.pos[i]
        if s.periodic:
            d -= s.box * np.round(d / s.box)
        r2 = float(d @ d)
        assert abs(r2 - rc ** 2) <= 4 * np.spacing(rc ** 2), f"pair {i},{j} differs and is not a tie"
    return len(diff)


@pytest.mark.parametrize("kind", ["periodic", "open", "ortho"])
def test_pair_set_matches_reference_lj_mix(golden, kind):
    from devinproj_b200 import cell_list_pairs
    g = golden(f"lj_mix_{kind}")
    s = product_system(g)
    i, j = cell_list_pairs(s, float(g["list_radius"]))
    assert np.all(i < j)
    ties = _ties(s, pair_keys(i, j, s.n), pair_keys(g["pair_i"], g["pair_j"], s.n), float(g["list_radius"]))
    assert ties == 0


def test_pair_set_matches_reference_argon864(golden):
    from devinproj_b200 import cell_list_pairs
    g = golden("argon864")
    s = product_system(g)
    i, j = cell_list_pairs(s, float(g["list_radius"]))
    assert _ties(s, pair_keys(i, j, s.n), pair_keys(g["pair_i"], g["pair_j"], s.n), float(g["list_radius"])) == 0


def test_pair_set_digest_nacl4096(golden):
    from devinproj_b200 import cell_list_pairs
    g = golden("nacl4096")
    s = product_system(g)
    i, j = cell_list_pairs(s, 12.32e-10)
    key = pair_keys(i, j, s.n)
    assert len(key) == int(g["pairs_lj_count"])
    assert hashlib.sha256(key.tobytes()).hexdigest() == str(g["pairs_lj_sha"])
    i, j = cell_list_pairs(s, 13.8e-10)
    key = pair_keys(i, j, s.n)
    assert len(key) == int(g["pairs_dsf_count"])
    assert hashlib.sha256(key.tobytes()).hexdigest() == str(g["pairs_dsf_sha"])


@pytest.mark.parametrize("kind", ["periodic", "open", "ortho"])
def test_lj_fp64_matches_reference(golden, kind):
    from devinproj_b200 import LennardJones
    g = golden(f"lj_mix_{kind}")
    s = product_system(g)
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    Fd, Ud = LennardJones(params, pairlist_threshold=10 ** 9).compute(s)
    Fl, Ul = LennardJones(params, pairlist_threshold=2).compute(s)
    assert rel_max(Fd, g["F_dense"]) <= TOL and abs(Ud - g["U_dense"]) <= TOL * abs(g["U_dense"])
    assert rel_max(Fl, g["F_list"]) <= TOL and abs(Ul - g["U_list"]) <= TOL * abs(g["U_list"])


def test_lj_verlet_skin_matches_reference_along_trajectory(golden):
    """Skin list == fresh list along a VV run, and the rebuild count equals the reference's
    (tests/test_nose_hoover.py:51-60)."""
    from accusim import Simulation
    from devinproj_b200 import LennardJones, VelocityVerlet
    g = golden("lj500_skin")
    s = product_system(g, "0")
    eps, sig = float(g["eps"]), float(g["sig"])
    lj = LennardJones({"Ar": (eps, sig)}, cutoff=2.5)
    fresh = LennardJones({"Ar": (eps, sig)}, cutoff=2.5, skin=0.0)
    sim = Simulation(s, [lj], integrator=VelocityVerlet(), dt=float(g["dt"]))
    Us = []
    for _ in range(10):
        sim.run(steps=20, positions=False)
        f1, u1 = lj.compute(s)
        f0, u0 = fresh.compute(s)
        assert np.max(np.abs(f1 - f0)) <= TOL * np.max(np.abs(f0))
        assert abs(u1 - u0) <= TOL * abs(u0)
        Us.append(u1)
    assert lj.rebuilds == int(g["rebuilds"])
    # chaotic growth of 1e-16 differences over 200 steps stays far below this
    assert np.max(np.abs(np.array(Us) - g["U_series"])) <= 1e-8 * np.max(np.abs(g["U_series"]))


def test_velocity_verlet_matches_reference_trajectory(golden):
    """60 VV steps of the 864-atom argon case through Simulation.run with the drop-ins."""
    from accusim import Simulation
    from devinproj_b200 import LennardJones, VelocityVerlet
    g = golden("argon864")
    s = product_system(g, "0")
    lj = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    sim = Simulation(s, [lj], integrator=VelocityVerlet(), dt=float(g["dt"]))
    tr = sim.run(steps=int(g["steps"]), positions=False)
    assert rel_max(np.array(tr.kinetic), g["kinetic"]) <= 1e-9
    assert rel_max(np.array(tr.potential), g["potential"]) <= 1e-9
    d = s.pos - g["pos"]
    d -= s.box * np.round(d / s.box)
    assert np.max(np.abs(d)) <= 1e-9 * s.box[0]
    assert lj.rebuilds == int(g["rebuilds"])
    # forces at the final state, fresh list, against the reference's
    F, U = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5, skin=0.0).compute(s)
    Fo, Uo = port.LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5, skin=0.0).compute(
        port.State(s.pos, s.vel, s.sp, s.ids, s.box, True, [("Ar", float(g["masses"][0]), 0.0)]))
    assert rel_max(F, Fo) <= TOL and abs(U - Uo) <= TOL * abs(Uo)


def test_velocity_verlet_step_is_bit_identical_given_forces():
    """With the same accelerations the device kick/drift/wrap is the reference's IEEE sequence exactly."""
    import torch

    from devinproj_b200 import _lib
    from devinproj_b200.device import stream_handle, to_dev
    rng = np.random.default_rng(11)
    box = np.array([3.1, 2.7, 4.4])
    pos = rng.uniform(0, 1, (1000, 3)) * box
    vel = rng.normal(size=(1000, 3))
    acc = rng.normal(size=(1000, 3)) * 1e3
    dt = 1.7e-3
    ref_v = vel + 0.5 * dt * acc
    ref_x = pos + dt * ref_v
    ref_x %= box
    L = _lib.lib()
    x, v, a = to_dev(pos), to_dev(vel), to_dev(acc)
    _lib.check(L.acs_vv_kick(v.data_ptr(), a.data_ptr(), 1000, 0.5 * dt, stream_handle()))
    barr, bp = _lib.dbl3(box)
    _lib.check(L.acs_vv_drift_wrap(x.data_ptr(), v.data_ptr(), 1000, dt, bp, 1, stream_handle()))
    torch.cuda.synchronize()
    assert np.array_equal(v.cpu().numpy(), ref_v)
    assert np.array_equal(x.cpu().numpy(), ref_x)


def test_dsf_fp64_matches_reference(golden):
    from devinproj_b200 import DampedShiftedCoulomb
    g = golden("dsf_rocksalt10")
    s = product_system(g)
    fd, ud = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9).compute(s)
    fc, uc = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1).compute(s)
    assert rel_max(fd, g["F_dense"]) <= TOL and abs(ud - g["U_dense"]) <= TOL * abs(g["U_dense"])
    assert rel_max(fc, g["F_list"]) <= TOL and abs(uc - g["U_list"]) <= TOL * abs(g["U_list"])


def test_dsf_fp64_matches_reference_in_orthorhombic_box(golden):
    from devinproj_b200 import DampedShiftedCoulomb
    g = golden("coulomb_ortho")
    s = product_system(g)
    fd, ud = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9).compute(s)
    fc, uc = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1).compute(s)
    assert rel_max(fd, g["F_dense"]) <= TOL and abs(ud - g["U_dense"]) <= TOL * abs(g["U_dense"])
    assert rel_max(fc, g["F_list"]) <= TOL and abs(uc - g["U_list"]) <= TOL * abs(g["U_list"])


def test_dsf_exclusions_match_reference(golden):
    from devinproj_b200 import DampedShiftedCoulomb
    g = golden("dsf_exclusions")
    s = product_system(g)
    ex = [tuple(map(int, p)) for p in g["exclude"]]
    fd, ud = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9, exclude=ex).compute(s)
    fc, uc = DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1, exclude=ex).compute(s)
    f0, u0 = DampedShiftedCoulomb(rcut=2.5, k=1.0).compute(s)
    assert rel_max(fd, g["F_dense"]) <= TOL and abs(ud - g["U_dense"]) <= TOL * abs(g["U_dense"])
    assert rel_max(fc, g["F_list"]) <= TOL and abs(uc - g["U_list"]) <= TOL * abs(g["U_list"])
    assert rel_max(f0, g["F_noex"]) <= TOL and abs(u0 - g["U_noex"]) <= TOL * abs(g["U_noex"])


def test_dsf_verlet_skin_matches_reference_rebuilds(golden):
    """tests/test_dsf.py:119-139: 30 perturbations regenerated from the same seed."""
    from accusim import System
    from devinproj_b200 import DampedShiftedCoulomb
    g = golden("dsf_skin")
    n = 8
    s = System(3, box=float(n), periodic=True)
    s.add_species("Na", 1.0, charge=1.0)
    s.add_species("Cl", 1.0, charge=-1.0)
    gr = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3).astype(float)
    odd = gr.sum(1) % 2 == 1
    s.add("Na", gr[~odd])
    s.add("Cl", gr[odd])
    rng = np.random.default_rng(5)
    skinned = DampedShiftedCoulomb(rcut=3.9, alpha=0.6, k=1.0, skin=0.6)
    Us = []
    for _ in range(30):
        s.pos = (s.pos + rng.normal(0, 0.05, s.pos.shape)) % s.box
        f1, u1 = skinned.compute(s)
        f0, u0 = DampedShiftedCoulomb(rcut=3.9, alpha=0.6, k=1.0, skin=0.0).compute(s)
        assert np.max(np.abs(f1 - f0)) <= TOL * np.max(np.abs(f0))
        assert abs(u1 - u0) <= TOL * abs(u0)
        Us.append(u1)
    assert skinned._vl.rebuilds == int(g["rebuilds"])
    assert np.max(np.abs(np.array(Us) - g["U_series"])) <= TOL * np.max(np.abs(g["U_series"]))
    assert rel_max(f1, g["F"]) <= TOL


def test_nacl4096_lj_plus_dsf_matches_reference(golden):
    from accusim import Simulation
    from devinproj_b200 import DampedShiftedCoulomb, LennardJones, VelocityVerlet
    g = golden("nacl4096")
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    s = product_system(g)
    F, U = LennardJones(params, cutoff=2.5, skin=0.0).compute(s)
    assert rel_max(F, g["F_lj"]) <= TOL and abs(U - g["U_lj"]) <= TOL * abs(g["U_lj"])
    F, U = DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]), skin=0.0).compute(s)
    assert rel_max(F, g["F_dsf"]) <= TOL and abs(U - g["U_dsf"]) <= TOL * abs(g["U_dsf"])
    # the 10-step trajectory from the initial state
    s = product_system(g, "0")
    lj = LennardJones(params, cutoff=2.5)
    dsf = DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]))
    sim = Simulation(s, [lj, dsf], integrator=VelocityVerlet(), dt=float(g["dt"]))
    tr = sim.run(steps=int(g["steps"]), positions=False)
    assert rel_max(np.array(tr.kinetic), g["kinetic"]) <= 1e-11
    assert rel_max(np.array(tr.potential), g["potential"]) <= 1e-11
    assert lj.rebuilds == int(g["rebuilds_lj"]) and dsf._vl.rebuilds == int(g["rebuilds_dsf"])


def test_forces_are_negative_gradient_and_newton3():
    """tests/test_forces.py:30-52 on the GPU plug-ins: central differences of U and sum F = 0."""
    from accusim import System
    from devinproj_b200 import DampedShiftedCoulomb, LennardJones
    rng = np.random.default_rng(0)
    for periodic in (False, True):
        s = System(3, box=2e-9 if periodic else None, periodic=periodic)
        s.add_species("A", 40 * 1.66053906660e-27, charge=1.602176634e-19)
        s.add_species("B", 20 * 1.66053906660e-27, charge=-1.602176634e-19)
        pts = rng.uniform(0.2e-9, 1.8e-9, size=(6, 3))
        s.add("A", pts[:3])
        s.add("B", pts[3:])
        for f in (LennardJones({"A": (1.0e3 / 6.022e23, 3.4e-10), "B": (0.5e3 / 6.022e23, 2.8e-10)}, cutoff=5),
                  DampedShiftedCoulomb(rcut=0.9e-9)):
            F, _ = f.compute(s)
            assert np.allclose(F.sum(axis=0), 0, atol=1e-10 * np.max(np.abs(F)))
            h = 1e-15
            for i in range(s.n):
                for k in range(3):
                    s.pos[i, k] += h
                    up = f.compute(s)[1]
                    s.pos[i, k] -= 2 * h
                    down = f.compute(s)[1]
                    s.pos[i, k] += h
                    assert -(up - down) / (2 * h) == pytest.approx(F[i, k], rel=1e-4,
                                                                   abs=1e-6 * np.max(np.abs(F)) + 1e-300)


def test_lj_minimum_and_small_systems():
    from accusim import System
    from devinproj_b200 import DampedShiftedCoulomb, LennardJones
    s = System(3)
    s.add_species("Ar", 6.6e-26)
    sigma = 3.4e-10
    s.add("Ar", [[0, 0, 0], [2 ** (1 / 6) * sigma, 0, 0]])
    F, _ = LennardJones({"Ar": (1e-21, sigma)}, cutoff=10).compute(s)
    assert np.allclose(F, 0, atol=1e-20)
    one = System(3)
    one.add_species("Ar", 6.6e-26, charge=1.0)
    one.add("Ar", [[0, 0, 0]])
    F, U = LennardJones({"Ar": (1e-21, sigma)}).compute(one)
    assert F.shape == (1, 3) and U == 0.0
    F, U = DampedShiftedCoulomb(rcut=1.0, alpha=0.5, k=1.0).compute(one)
    assert np.all(F == 0)
    c, erc, _ = port.DampedShiftedCoulomb(rcut=1.0, alpha=0.5, k=1.0).constants()
    assert U == pytest.approx(-(erc / 2 + 0.5 / np.sqrt(np.pi)), rel=1e-14)


def _rocksalt(n):
    """Unit-charge rock salt on the integer grid, unit masses and box n (tests/test_dsf.py:7-15)."""
    from accusim import System
    s = System(3, box=float(n), periodic=True)
    s.add_species("Na", 1.0, charge=1.0)
    s.add_species("Cl", 1.0, charge=-1.0)
    g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    odd = g.sum(1) % 2 == 1
    s.add("Na", g[~odd].astype(float))
    s.add("Cl", g[odd].astype(float))
    return s


def test_dsf_known_answers():
    """The GPU DSF plug-in against the reference's own DSF checks (tests/test_dsf.py:18-52): the Madelung
    energy of rock salt within 2e-3 at rc 3.9, alpha 0.6; forces are the energy's gradient and sum to
    zero; a pair just inside the cutoff feels no force and its energy is the self term; on a disordered
    melt the energy is within 3% of Ewald's (the device Ewald, itself pinned to the reference)."""
    from accusim import System
    from devinproj_b200 import DampedShiftedCoulomb
    from devinproj_b200.ewald import Ewald
    s = _rocksalt(8)
    _, U = DampedShiftedCoulomb(rcut=3.9, alpha=0.6, k=1.0).compute(s)
    assert abs(-2 * U / s.n / 1.747564594633 - 1) < 2e-3

    s = _rocksalt(4)
    rng = np.random.default_rng(1)
    s.pos += rng.normal(0, 0.1, s.pos.shape)
    dsf = DampedShiftedCoulomb(rcut=1.9, k=1.0)
    f, _ = dsf.compute(s)
    h = 1e-6
    for i, ax in [(0, 0), (5, 1), (17, 2)]:
        s.pos[i, ax] += h
        _, up = dsf.compute(s)
        s.pos[i, ax] -= 2 * h
        _, um = dsf.compute(s)
        s.pos[i, ax] += h
        assert abs(-(up - um) / (2 * h) - f[i, ax]) < 1e-6 * max(1, abs(f[i, ax]))
    assert np.allclose(f.sum(0), 0, atol=1e-10)

    two = System(3)
    two.add_species("A", 1.0, charge=1.0)
    two.add("A", [[0, 0, 0], [1.9 - 1e-9, 0, 0]])
    f2, u2 = dsf.compute(two)
    _, erc, _ = port.DampedShiftedCoulomb(rcut=1.9, alpha=dsf.alpha, k=1.0).constants()
    self_term = 2 * (erc / 3.8 + dsf.alpha / np.sqrt(np.pi))
    assert abs(f2[0, 0]) < 1e-7 and abs(u2 + self_term) < 1e-7

    s = _rocksalt(4)
    rng = np.random.default_rng(2)
    s.pos = (s.pos + rng.normal(0, 0.25, s.pos.shape)) % s.box
    _, ue = Ewald(k=1.0).compute(s)
    _, ud = DampedShiftedCoulomb(rcut=1.99, alpha=0.9, k=1.0).compute(s)
    assert abs(ud / ue - 1) < 3e-2


def test_list_capacity_overflow_regrows():
    """A dense clump far above the capacity estimate: the build reports overflow and is redone bigger."""
    from accusim import System
    from devinproj_b200.forces import DeviceNeighborList
    from devinproj_b200.device import to_dev
    rng = np.random.default_rng(2)
    s = System(3, box=10.0, periodic=True)
    s.add_species("A", 1.0)
    s.add("A", np.concatenate([rng.uniform(0, 10, (2000, 3)), rng.uniform(4.5, 5.5, (600, 3))]))
    nl = DeviceNeighborList()
    nl.build(s, to_dev(s.pos), 1.0)
    i, j = nl.pairs(s.n)
    st = port.State(s.pos, s.vel, s.sp, s.ids, s.box, True, [("A", 1.0, 0.0)])
    oi, oj = port.cell_list_pairs(st, 1.0)
    assert np.array_equal(pair_keys(i, j, s.n), pair_keys(oi, oj, s.n))
    assert nl.maxnb >= int(nl.nnb.max().item())


@pytest.mark.parametrize("kind", ["lv", "nh"])
def test_dropin_thermostats_match_reference(golden, kind):
    """The Langevin (BAOAB, normal draws from `sim.rng` as the reference takes them) and Nose-Hoover
    plug-ins inside `Simulation.run`: 40 steps of 108 argon atoms against the reference's run. The device
    FP64 forces differ from the reference's at round-off (summation order), so the trajectories agree to
    the VelocityVerlet trajectory test's 1e-9, not bitwise; the report gains its thermostat rows."""
    from accusim import Simulation
    from devinproj_b200 import Langevin, LennardJones, NoseHoover
    g = golden("thermostats108")
    s = product_system(g, "0")
    lj = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    integ = Langevin(float(g["T"]), float(g["friction"])) if kind == "lv" else NoseHoover(float(g["T"]), float(g["tau"]))
    sim = Simulation(s, [lj], integrator=integ, dt=float(g["dt"]), seed=int(g["seed"]))
    tr = sim.run(steps=int(g["steps"]), record_every=int(g["record_every"]), positions=False)
    d = s.pos - g[f"{kind}_pos"]
    d -= s.box * np.round(d / s.box)
    assert np.max(np.abs(d)) <= 1e-9 * s.box[0]
    assert rel_max(s.vel, g[f"{kind}_vel"]) <= 1e-9
    assert rel_max(np.array(tr.kinetic), g[f"{kind}_kinetic"]) <= 1e-9
    assert rel_max(np.array(tr.potential), g[f"{kind}_potential"]) <= 1e-9
    if kind == "nh":
        assert rel_max(np.array(tr.bath), g["nh_bath"]) <= 1e-9
        assert abs(integ.xi - g["nh_xi"]) <= 1e-9 * abs(g["nh_xi"]) and integ.Q == g["nh_Q"]
    rows = {c.name for c in sim.accuracy_report().checks}
    assert "thermostat" in rows and (("extended energy" in rows) == (kind == "nh"))


@pytest.mark.parametrize("case", ["report_argon108", "report_nacl512"])
def test_accuracy_report_matches_reference(golden, case):
    """The accuracy report (accusim/accuracy.py:60-182, 191-221) of a short VelocityVerlet run with the dt/2,
    dt/4 Richardson runs, through the plug-ins, against the reference's own report: 108 argon atoms (60 steps)
    and a 512-ion NaCl melt (LJ + DSF, 20 steps: two species' timescales and the DSF vs Ewald row). The same
    rows and grades; values to 1e-6 relative where they are not round-off (the device FP64 forces differ from
    NumPy's at round-off and the runs are short)."""
    from accusim import Simulation
    from devinproj_b200 import DampedShiftedCoulomb, LennardJones, VelocityVerlet
    g = golden(case)
    s = product_system(g)
    if case == "report_argon108":
        forces = [LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)]
    else:
        params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
        forces = [LennardJones(params, cutoff=2.5), DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]))]
    sim = Simulation(s, forces, integrator=VelocityVerlet(), dt=float(g["dt"]))
    sim.run(steps=int(g["steps"]), record_every=1, positions=False)
    rep = sim.accuracy_report(convergence_duration=float(g["convergence_duration"]))
    assert [c.name for c in rep.checks] == [str(x) for x in g["names"]]
    assert [c.status for c in rep.checks] == [str(x) for x in g["statuses"]]
    for c, v in zip(rep.checks, g["values"]):
        if np.isnan(v):
            assert c.value is None, c.name
        elif c.name == "momentum":        # round-off of a conserved sum: both far below the PASS grade
            assert c.value <= 1e-12 and v <= 1e-12
        elif v == 0.0:
            assert c.value == 0.0, c.name
        else:
            assert abs(c.value - v) <= 1e-6 * abs(v), (c.name, c.value, v)
    # accusim/advisor.py:51-55 on the same end-of-run state: the shortest timescale / 100
    from accusim import suggest_dt
    ratio = float(g["values"][list(g["names"]).index("timestep vs physics")])
    assert suggest_dt(sim) == pytest.approx(float(g["dt"]) / ratio / 100, rel=1e-6)


def test_langevin_o_step_is_bit_identical():
    """Given the same velocities, per-atom sigma and normal draws, acs_langevin_ou computes the reference's
    c1 * v + sig * noise exactly (accusim/integrators.py:66-67)."""
    import torch

    from devinproj_b200 import _lib
    from devinproj_b200.device import stream_handle, to_dev
    rng = np.random.default_rng(5)
    n = 1000
    vel = rng.normal(size=(n, 3)) * 300.0
    noise = rng.normal(size=(n, 3))
    masses = rng.choice([6.6e-26, 1.4e-25], n)
    c1 = np.exp(-5e12 * 5e-15)
    sig = np.sqrt((1 - c1 ** 2) * 1.380649e-23 * 120.0 / masses)
    ref = c1 * vel + sig[:, None] * noise
    L = _lib.lib()
    v, z, sg = to_dev(vel), to_dev(noise), to_dev(sig)   # held: a freed temporary's memory is handed out again
    _lib.check(L.acs_langevin_ou(v.data_ptr(), z.data_ptr(), sg.data_ptr(), n, float(c1), stream_handle()))
    torch.cuda.synchronize()
    assert np.array_equal(v.cpu().numpy(), ref)
