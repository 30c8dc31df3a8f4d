"""The engine's own neighbour lists (the ones behind the FP32c step) as pair sets, against the reference's pair
search at the list radius (accusim/forces.py:279-321 cell_list_pairs, on the positions of the last rebuild,
which the lists were built from; accusim/forces.py:86-98 VerletList.pairs rebuilds at rc + skin).

Every list entry is decoded back to a pair of caller indices (acs_engine_dump_lists). Checked: no entry names
a foreign or the same atom, every pair is listed in both directions exactly once, and the set of unordered pairs
equals the reference's. A pair may differ only if it is an r^2 tie with the list radius (within 1e-12
relative: the engine filters in Angstrom, the reference in metres); ties are counted and reported (none occur
on these fixtures). DSF-excluded pairs stay listed with the exclusion flag set, exactly on the excluded pairs."""
import hashlib

import numpy as np
import pytest

from oracle import accusim_port as port
from tests._helpers import pair_keys

pytestmark = pytest.mark.gpu

TIE = 1e-12


def engine_pairs(eng, r=None):
    """(unordered pair keys i*n+j with i<j, sorted; excluded keys; build positions SI) of the engine's lists,
    after the structural checks (foreign entries, self pairs, both directions, duplicates)."""
    from devinproj_b200.engine import LEN
    keys, pos = eng.list_entries()
    keys = keys.cpu().numpy()
    n = int(eng.offsets[-1])
    assert np.all(keys >= 0), "a list entry names no atom of its own replica"
    ex = (keys & 1).astype(bool)
    d = keys >> 1
    i, j = d // n, d % n
    assert not np.any(i == j), "self pair in a list"
    fwd = np.sort(i[i < j] * n + j[i < j])
    bwd = np.sort(j[i > j] * n + i[i > j])
    assert len(fwd) == len(bwd) and np.array_equal(fwd, bwd), "a pair is not listed in both directions"
    assert np.all(np.diff(fwd) > 0), "a pair is listed twice"
    exk = np.unique(np.minimum(i[ex], j[ex]) * n + np.maximum(i[ex], j[ex]))
    return fwd, exk, pos.cpu().numpy() * LEN


def compare_sets(got, ref, pos, box, rl, label):
    """Pairs in exactly one of the two sets must be r^2 ties with rl^2; returns the number of ties."""
    diff = np.setxor1d(got, ref)
    n = len(pos)
    for key in diff:
        a, b = divmod(int(key), n)
        dd = pos[b] - pos[a]
        dd -= box * np.round(dd / box)
        r2 = float(dd @ dd)
        assert abs(r2 - rl * rl) <= TIE * rl * rl, f"{label}: pair {a},{b} (r/rl = {np.sqrt(r2) / rl:.9f}) differs"
    print(f"{label}: {len(got)} pairs, {len(diff)} r^2 ties with the list radius")
    return len(diff)


def _system(g, suffix=""):
    from tests.test_dropin_gpu import product_system
    return product_system(g, suffix)


@pytest.mark.parametrize("tpa", [1, 32])
def test_engine_lists_equal_reference_pairs_argon864(golden, tpa):
    from devinproj_b200.engine import start_engine
    from devinproj_b200 import LennardJones
    g = golden("argon864")
    s = _system(g)
    lj = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    eng, rlist, _ = start_engine([s], [lj], [float(g["dt"])], tpa=tpa)
    got, _, pos = engine_pairs(eng)
    assert np.max(np.abs(pos - s.pos)) <= 1e-15 * s.box[0]   # built from the golden positions (in Angstrom)
    ref = pair_keys(g["pair_i"], g["pair_j"], s.n)
    assert compare_sets(got, ref, pos, s.box, rlist, f"argon864 tpa {tpa}") == 0


@pytest.mark.parametrize("kind", ["periodic", "ortho"])
def test_engine_lists_equal_reference_pairs_lj_mixture(golden, kind):
    from devinproj_b200.engine import start_engine
    from devinproj_b200 import LennardJones
    g = golden(f"lj_mix_{kind}")
    s = _system(g)
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    eng, rlist, _ = start_engine([s], [LennardJones(params, cutoff=2.5)], [1e-15])
    got, _, pos = engine_pairs(eng)
    ref = pair_keys(g["pair_i"], g["pair_j"], s.n)
    assert compare_sets(got, ref, pos, s.box, rlist, f"lj_mix_{kind}") == 0


def test_engine_lists_match_reference_digest_nacl4096(golden):
    """The 4096-ion NaCl lists (one list at the DSF list radius 13.8 A = rc + skin, the larger of the two
    forces') hash to the reference's own pair set at 13.8 A; restricted to 12.32 A (the LJ list radius) the
    listed pairs hash to the reference's LJ pair set."""
    from devinproj_b200 import DampedShiftedCoulomb, LennardJones
    from devinproj_b200.engine import start_engine
    g = golden("nacl4096")
    s = _system(g)
    params = {str(n): (float(e), float(sg)) for n, e, sg in zip(g["param_names"], g["param_eps"], g["param_sig"])}
    forces = [LennardJones(params, cutoff=2.5), DampedShiftedCoulomb(rcut=float(g["rcut"]), alpha=float(g["alpha"]))]
    for tpa in (1, 16):
        eng, rlist, _ = start_engine([s], forces, [float(g["dt"])], tpa=tpa)
        assert rlist == pytest.approx(13.8e-10, rel=1e-12)
        got, exk, pos = engine_pairs(eng)
        assert len(exk) == 0 and np.max(np.abs(pos - s.pos)) <= 1e-15 * s.box[0]
        assert len(got) == int(g["pairs_dsf_count"])
        assert hashlib.sha256(got.tobytes()).hexdigest() == str(g["pairs_dsf_sha"]), tpa
        i, j = divmod(got, s.n)
        dd = s.pos[j] - s.pos[i]
        dd -= s.box * np.round(dd / s.box)
        inner = got[np.einsum("ij,ij->i", dd, dd) < (12.32e-10) ** 2]
        assert len(inner) == int(g["pairs_lj_count"])
        assert hashlib.sha256(inner.tobytes()).hexdigest() == str(g["pairs_lj_sha"]), tpa


def test_engine_lists_after_rebuilds_equal_fresh_pair_search():
    """Lists rebuilt inside graph-captured runs (hot argon, ~1 rebuild per few steps): after each of several
    blocks, the engine's pair set equals the oracle's cell_list_pairs (the reference's algorithm, pinned
    bit-exact to it) on the positions of the last rebuild, at the list radius."""
    from devinproj_b200 import configs
    from devinproj_b200.engine import start_engine
    s, forces, dt = configs.argon864(seed=3)
    s.maxwell_boltzmann(300.0, np.random.default_rng(3))
    for tpa in (1, 32):
        eng, rlist, _ = start_engine([s.copy()], forces, [dt], tpa=tpa)
        rb0 = eng.status().rebuilds
        for block in range(4):
            eng.run(37, 0, True)
            eng.check("run")
            got, _, pos = engine_pairs(eng)
            st = port.State(pos, np.zeros_like(pos), s.sp.copy(), s.ids.copy(), s.box.copy(), True,
                            [("Ar", configs.AR_MASS, 0.0)])
            ref = pair_keys(*port.cell_list_pairs(st, rlist), s.n)
            assert compare_sets(got, ref, pos, s.box, rlist, f"hot argon tpa {tpa} block {block}") == 0
        assert eng.status().rebuilds - rb0 >= 8


def test_engine_lists_flag_exactly_the_dsf_exclusions():
    """With DSF exclusions the listed pair set is unchanged (the LJ term still needs those pairs) and the
    exclusion flag sits exactly on the excluded pairs that lie inside the list radius."""
    from devinproj_b200 import DampedShiftedCoulomb, LennardJones, configs
    from devinproj_b200.engine import start_engine
    s, forces, dt = configs.nacl4096(seed=1)
    rng = np.random.default_rng(4)
    ex = set()
    while len(ex) < 300:
        a, b = (int(x) for x in rng.integers(0, s.n, 2))
        if a != b:
            ex.add((min(a, b), max(a, b)))
    dsf = DampedShiftedCoulomb(rcut=forces[1].rcut, alpha=forces[1].alpha, exclude=sorted(ex))
    eng, rlist, _ = start_engine([s], [forces[0], dsf], [dt])
    got, exk, pos = engine_pairs(eng)
    eng0, _, _ = start_engine([s], forces, [dt])
    got0, exk0, _ = engine_pairs(eng0)
    assert np.array_equal(got, got0) and len(exk0) == 0
    n = s.n
    want = np.array(sorted(a * n + b for a, b in ex))
    assert np.array_equal(exk, np.intersect1d(want, got))
    assert len(exk) > 0


@pytest.mark.parametrize("tpa", [1, 32])
def test_engine_lists_with_row_major_cell_order(golden, tpa):
    """The slot order of the cells (Morton by default; row-major with cell_order 0) changes only where atoms sit in
    memory: with row-major order too the lists hold the reference's pair set on the golden argon system and, after
    rebuilds inside graph runs, the oracle's pair set on the positions of the last rebuild; the forces match the
    FP64 oracle."""
    from devinproj_b200 import LennardJones, configs
    from devinproj_b200.engine import ACC, start_engine
    g = golden("argon864")
    s = _system(g)
    lj = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    eng, rlist, _ = start_engine([s], [lj], [float(g["dt"])], tpa=tpa, cell_order=0)
    got, _, pos = engine_pairs(eng)
    assert compare_sets(got, pair_keys(g["pair_i"], g["pair_j"], s.n), pos, s.box, rlist, f"row-major tpa {tpa}") == 0
    h, forces, dt = configs.argon864(seed=3)
    h.maxwell_boltzmann(300.0, np.random.default_rng(3))
    eng, rlist, _ = start_engine([h], forces, [dt], tpa=tpa, cell_order=0)
    rb0 = eng.status().rebuilds
    for block in range(3):
        eng.run(41, 0, True)
        eng.check("run")
        got, _, pos = engine_pairs(eng)
        st = port.State(pos, np.zeros_like(pos), h.sp.copy(), h.ids.copy(), h.box.copy(), True,
                        [("Ar", configs.AR_MASS, 0.0)])
        ref = pair_keys(*port.cell_list_pairs(st, rlist), h.n)
        assert compare_sets(got, ref, pos, h.box, rlist, f"row-major hot argon tpa {tpa} block {block}") == 0
    assert eng.status().rebuilds - rb0 >= 6
    p, v, a = eng.get_state()
    from devinproj_b200.engine import LEN
    st = port.State(p.cpu().numpy() * LEN, np.zeros((h.n, 3)), h.sp.copy(), h.ids.copy(), h.box.copy(), True,
                    [("Ar", configs.AR_MASS, 0.0)])
    Fo, _ = port.LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5, skin=0.0).compute(st)
    F = a.cpu().numpy() * ACC * configs.AR_MASS
    assert float(np.sqrt(np.mean(np.sum((F - Fo) ** 2, 1)) / np.mean(np.sum(Fo ** 2, 1)))) <= 1e-5


@pytest.mark.parametrize("tpa", [1, 32])
def test_engine_lists_with_a_one_cell_axis(tpa):
    """A box with a one-cell axis (29.7 x 20.1 x 6.4 sigma: 6.4 sigma is under three list radii, so that axis has
    one cell and the pair test wraps it), in one engine with a replica that has >= 3 cells per axis: the lists of
    both equal the oracle's pair search at the list radius on the positions of the last rebuild, at the start and
    after rebuilds inside graph runs."""
    from accusim import System
    from devinproj_b200 import LennardJones, configs
    from devinproj_b200.engine import LEN, start_engine
    rng = np.random.default_rng(7)
    a = 1.06 * configs.AR_SIGMA
    systems = []
    for n in (np.array([28, 19, 6]), np.array([12, 12, 12])):
        s = System(3, box=n * a, periodic=True)
        s.add_species("Ar", configs.AR_MASS)
        g = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), -1).reshape(-1, 3)
        s.add("Ar", ((g + 0.5) * a + rng.normal(0, 0.05 * configs.AR_SIGMA, g.shape)) % s.box)
        s.maxwell_boltzmann(300.0, rng)
        systems.append(s)
    lj = LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5)
    eng, rlist, _ = start_engine([x.copy() for x in systems], [lj], [5e-15, 5e-15], tpa=tpa)
    assert 6 * a < 3 * rlist < 12 * a
    rb0 = eng.status().rebuilds
    for block in range(4):
        if block:
            eng.run(29, 0, True)
            eng.check("run")
        keys, pos = eng.list_entries()
        keys = keys.cpu().numpy()
        pos = pos.cpu().numpy() * LEN
        n_all = int(eng.offsets[-1])
        ex = keys >> 1
        i, j = ex // n_all, ex % n_all
        assert np.all(keys >= 0) and not np.any(i == j)
        for r, s in enumerate(systems):
            o0, o1 = int(eng.offsets[r]), int(eng.offsets[r + 1])
            sel = (i >= o0) & (i < o1) & (i < j)
            assert np.all((j[sel] >= o0) & (j[sel] < o1)), "an entry names another replica's atom"
            got = np.sort((i[sel] - o0) * s.n + (j[sel] - o0))
            back = (j >= o0) & (j < o1) & (i > j)
            assert np.array_equal(got, np.sort((j[back] - o0) * s.n + (i[back] - o0))), "not listed both ways"
            p = pos[o0:o1]
            st = port.State(p, np.zeros_like(p), s.sp.copy(), s.ids.copy(), s.box.copy(), True,
                            [("Ar", configs.AR_MASS, 0.0)])
            ref = pair_keys(*port.cell_list_pairs(st, rlist), s.n)
            assert compare_sets(got, ref, p, s.box, rlist, f"replica {r} tpa {tpa} block {block}") == 0
    assert eng.status().rebuilds - rb0 >= 4


@pytest.mark.parametrize("cell_scale", [1.25, 1.5])
@pytest.mark.parametrize("tpa", [1, 32])
def test_engine_lists_with_wider_cells(golden, tpa, cell_scale):
    """Cells wider than the list radius (the autotuner's cell-edge candidates) change only which candidates a warp
    screens: on the golden argon system (whose 3 cells per axis then collapse to one, so every axis wraps) the lists
    hold the reference's pair set, and on a hot 4000-atom fluid (5 cells per axis at edge 1, 4 or 3 when wider) they
    hold the oracle's pair set on the positions of the last rebuild, at the start and after rebuilds inside graph
    runs; the final forces match the FP64 oracle."""
    from devinproj_b200 import LennardJones, configs
    from devinproj_b200.engine import ACC, LEN, start_engine
    g = golden("argon864")
    s = _system(g)
    lj = LennardJones({"Ar": (float(g["eps"]), float(g["sig"]))}, cutoff=2.5)
    eng, rlist, _ = start_engine([s], [lj], [float(g["dt"])], tpa=tpa, cell_scale=cell_scale)
    got, _, pos = engine_pairs(eng)
    ref = pair_keys(g["pair_i"], g["pair_j"], s.n)
    assert compare_sets(got, ref, pos, s.box, rlist, f"argon864 cells x{cell_scale} tpa {tpa}") == 0
    h, lj = configs.lj_fluid(10, seed=5)
    h.maxwell_boltzmann(300.0, np.random.default_rng(5))
    eng, rlist, _ = start_engine([h], [lj], [1e-14], tpa=tpa, cell_scale=cell_scale)
    assert 3 <= int(h.box[0] // (rlist * cell_scale)) < int(h.box[0] // rlist) == 5
    rb0 = eng.status().rebuilds
    for block in range(3):
        if block:
            eng.run(31, 0, True)
            eng.check("run")
        got, _, pos = engine_pairs(eng)
        st = port.State(pos, np.zeros_like(pos), h.sp.copy(), h.ids.copy(), h.box.copy(), True,
                        [("Ar", configs.AR_MASS, 0.0)])
        ref = pair_keys(*port.cell_list_pairs(st, rlist), h.n)
        assert compare_sets(got, ref, pos, h.box, rlist, f"4000-atom cells x{cell_scale} tpa {tpa} block {block}") == 0
    assert eng.status().rebuilds - rb0 >= 4
    p, v, a = eng.get_state()
    st = port.State(p.cpu().numpy() * LEN, np.zeros((h.n, 3)), h.sp.copy(), h.ids.copy(), h.box.copy(), True,
                    [("Ar", configs.AR_MASS, 0.0)])
    Fo, _ = port.LennardJones({"Ar": (configs.AR_EPS, configs.AR_SIGMA)}, cutoff=2.5, skin=0.0).compute(st)
    F = a.cpu().numpy() * ACC * configs.AR_MASS
    assert float(np.sqrt(np.mean(np.sum((F - Fo) ** 2, 1)) / np.mean(np.sum(Fo ** 2, 1)))) <= 1e-5

