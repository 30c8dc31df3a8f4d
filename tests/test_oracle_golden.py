"""Pin the CPU oracle (NumPy restatement) against golden vectors produced by the reference itself,
and against the reference's own known answers. CPU only."""
import hashlib

import numpy as np
import pytest

from oracle import accusim_port as port
from tests._helpers import oracle_state, pair_keys, rel_max


@pytest.mark.parametrize("kind", ["periodic", "open", "ortho"])
def test_oracle_lj_mix_matches_reference(golden, kind):
    g = golden(f"lj_mix_{kind}")
    st = oracle_state(g)
    params = {str(n): (float(e), float(s)) for n, e, s in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    Fd, Ud = port.LennardJones(params, pairlist_threshold=10 ** 9).compute(st)
    Fl, Ul = port.LennardJones(params, pairlist_threshold=2).compute(st)
    # same expressions in the same order: bit-identical to the reference
    assert np.array_equal(Fd, g["F_dense"]) and Ud == g["U_dense"]
    assert np.array_equal(Fl, g["F_list"]) and Ul == g["U_list"]
    i, j = port.cell_list_pairs(st, float(g["list_radius"]))
    assert np.array_equal(pair_keys(i, j, st.n), pair_keys(g["pair_i"], g["pair_j"], st.n))


def test_oracle_argon864_trajectory_matches_reference(golden):
    g = golden("argon864")
    st = oracle_state(g, "0")
    lj = port.LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    run = port.Run(st, [lj], float(g["dt"])).run(int(g["steps"]))
    assert np.array_equal(st.pos, g["pos"]) and np.array_equal(st.vel, g["vel"])
    assert np.array_equal(np.array(run.kinetic), g["kinetic"])
    assert np.array_equal(np.array(run.potential), g["potential"])
    assert lj.rebuilds == int(g["rebuilds"])
    F, U = port.LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5, skin=0.0).compute(st)
    assert np.array_equal(F, g["F"]) and U == g["U"]
    i, j = port.cell_list_pairs(st, float(g["list_radius"]))
    assert np.array_equal(pair_keys(i, j, st.n), pair_keys(g["pair_i"], g["pair_j"], st.n))


def test_oracle_lj_skin_rebuilds_match_reference(golden):
    g = golden("lj500_skin")
    st = oracle_state(g, "0")
    lj = port.LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    run = port.Run(st, [lj], float(g["dt"]))
    Us = []
    for _ in range(10):
        run.run(20)
        Us.append(lj.compute(st)[1])
    assert lj.rebuilds == int(g["rebuilds"])
    assert np.array_equal(np.array(Us), g["U_series"])
    assert np.array_equal(st.pos, g["pos"])


def test_oracle_dsf_matches_reference(golden):
    g = golden("dsf_rocksalt10")
    st = oracle_state(g)
    fd, ud = port.DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9).compute(st)
    fc, uc = port.DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1).compute(st)
    assert np.array_equal(fd, g["F_dense"]) and ud == g["U_dense"]
    assert np.array_equal(fc, g["F_list"]) and uc == g["U_list"]


def test_oracle_coulomb_in_orthorhombic_box_matches_reference(golden):
    """DSF (dense and cell paths) and Ewald in a periodic box of unequal edges, as the reference computes them."""
    g = golden("coulomb_ortho")
    st = oracle_state(g)
    fd, ud = port.DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9).compute(st)
    fc, uc = port.DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1).compute(st)
    assert np.array_equal(fd, g["F_dense"]) and ud == g["U_dense"]
    assert np.array_equal(fc, g["F_list"]) and uc == g["U_list"]
    F, U = port.Ewald(k=1.0).compute(st)
    assert rel_max(F, g["F_ewald"]) < 1e-12 and abs(U - g["U_ewald"]) <= 1e-12 * abs(g["U_ewald"])


def test_oracle_dsf_exclusions_match_reference(golden):
    g = golden("dsf_exclusions")
    st = oracle_state(g)
    ex = [tuple(map(int, p)) for p in g["exclude"]]
    fd, ud = port.DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=10 ** 9, exclude=ex).compute(st)
    fc, uc = port.DampedShiftedCoulomb(rcut=2.5, k=1.0, pairlist_threshold=1, exclude=ex).compute(st)
    assert np.array_equal(fd, g["F_dense"]) and ud == g["U_dense"]
    assert np.array_equal(fc, g["F_list"]) and uc == g["U_list"]


def test_oracle_nacl4096_matches_reference(golden):
    g = golden("nacl4096")
    st = oracle_state(g)
    params = {str(n): (float(e), float(s)) for n, e, s in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    F, U = port.LennardJones(params, cutoff=2.5, skin=0.0).compute(st)
    assert rel_max(F, g["F_lj"]) < 1e-13 and abs(U - g["U_lj"]) <= 1e-13 * abs(g["U_lj"])
    F, U = port.DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]), skin=0.0).compute(st)
    assert rel_max(F, g["F_dsf"]) < 1e-13 and abs(U - g["U_dsf"]) <= 1e-13 * abs(g["U_dsf"])
    i, j = port.cell_list_pairs(st, 12.32e-10)
    key = pair_keys(i, j, st.n)
    assert len(key) == int(g["pairs_lj_count"])
    assert hashlib.sha256(key.tobytes()).hexdigest() == str(g["pairs_lj_sha"])


def test_oracle_ewald_matches_reference(golden):
    g = golden("ewald_melt512")
    st = oracle_state(g)
    F, U = port.Ewald(k=1.0).compute(st)
    assert rel_max(F, g["F"]) < 1e-12 and abs(U - g["U"]) <= 1e-12 * abs(g["U"])


def _rocksalt(n, cells=1.0):
    g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    odd = g.sum(1) % 2 == 1
    pos = np.concatenate([g[~odd], g[odd]]).astype(float) * cells
    sp = np.concatenate([np.zeros((~odd).sum(), int), np.ones(odd.sum(), int)])
    return port.State(pos, np.zeros_like(pos), sp, np.arange(len(pos)), np.full(3, n * cells), True,
                      [("Na", 1.0, 1.0), ("Cl", 1.0, -1.0)])


def test_oracle_known_answer_madelung():
    """Known answers: Ewald Madelung 1.747564594633 (tests/test_forces.py:90-97) and the DSF
    approximation within 2e-3 (tests/test_dsf.py:18-21)."""
    st = _rocksalt(2)
    _, U = port.Ewald(k=1.0).compute(st)
    assert -U / (st.n / 2) == pytest.approx(1.747564594633, rel=1e-7)
    st = _rocksalt(8)
    _, U = port.DampedShiftedCoulomb(rcut=3.9, alpha=0.6, k=1.0).compute(st)
    assert abs(-2 * U / st.n / 1.747564594633 - 1) < 2e-3


def test_oracle_known_answer_lj_minimum():
    """LJ force vanishes at 2^(1/6) sigma: tests/test_forces.py:55-61."""
    sigma = 3.4e-10
    pos = np.array([[0, 0, 0], [2 ** (1 / 6) * sigma, 0, 0]], float)
    st = port.State(pos, np.zeros_like(pos), np.zeros(2, int), np.arange(2), None, False, [("Ar", 6.6e-26, 0.0)])
    F, _ = port.LennardJones({"Ar": (1e-21, sigma)}, cutoff=10).compute(st)
    assert np.allclose(F, 0, atol=1e-20)


@pytest.mark.parametrize("kind", ["lv", "nh"])
def test_oracle_thermostats_match_reference(golden, kind):
    """Langevin BAOAB (the reference's draws: default_rng(seed).normal) and Nose-Hoover on 108 argon atoms,
    40 steps: bit-identical to the reference's run."""
    g = golden("thermostats108")
    st = oracle_state(g, "0")
    lj = port.LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    if kind == "lv":
        rng = np.random.default_rng(int(g["seed"]))
        integ = port.LangevinBAOAB(float(g["T"]), float(g["friction"]), lambda shape: rng.normal(size=shape))
    else:
        integ = port.NoseHooverMTK(float(g["T"]), float(g["tau"]))
    run = port.Run(st, [lj], float(g["dt"]), integrator=integ).run(int(g["steps"]), int(g["record_every"]))
    assert np.array_equal(st.pos, g[f"{kind}_pos"]) and np.array_equal(st.vel, g[f"{kind}_vel"])
    assert np.array_equal(np.array(run.kinetic), g[f"{kind}_kinetic"])
    assert np.array_equal(np.array(run.potential), g[f"{kind}_potential"])
    assert np.array_equal(np.array(run.bath), g[f"{kind}_bath"])
    if kind == "nh":
        assert integ.xi == g["nh_xi"] and integ.eta == g["nh_eta"] and integ.Q == g["nh_Q"]


def test_philox_known_answers():
    """The oracle's Philox4x32-10 (the engine's Langevin draws) reproduces the published known-answer vectors
    of the algorithm (Random123 distribution, kat_vectors: philox4x32, 10 rounds)."""
    from oracle.philox import normals, philox4x32_10
    cases = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
             ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
             ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
              (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, out in cases:
        assert tuple(int(v) for v in philox4x32_10(np.array([ctr], np.uint64), key)[0]) == out
    z = normals(3, np.arange(200000), 0, 12345)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01
