"""Host logic of the launch-shape autotuner (no GPU): workload signatures, the candidate set, the JSON cache,
and that a cached workload is answered from the cache without building an engine."""
import json

import pytest

from devinproj_b200 import autotune, configs


def test_signature_buckets_and_distinguishes_workloads():
    s1, _ = configs.lj_fluid(4, seed=0)
    s2, _ = configs.lj_fluid(4, seed=1)            # same shape, other velocities: same bucket
    s3, _ = configs.lj_fluid(5, seed=0)            # more atoms: another bucket
    rl = 2.8 * 3.4e-10
    assert autotune.signature([s1], rl) == autotune.signature([s2], rl)
    assert autotune.signature([s1], rl) != autotune.signature([s3], rl)
    assert autotune.signature([s1], rl) != autotune.signature([s1, s2], rl)     # replica count is part of it
    assert autotune.signature([s1], rl) != autotune.signature([s1], 2 * rl)     # so is the list density
    assert autotune.signature([s1], rl).startswith("n260.0_r1_")     # 256 atoms, bucketed to 2 significant digits
    # the force terms and the GPU model are part of it
    from devinproj_b200 import DampedShiftedCoulomb, LennardJones
    lj = LennardJones({"Ar": (1.6e-21, 3.4e-10)})
    dsf = DampedShiftedCoulomb(rcut=1e-9)
    dsfx = DampedShiftedCoulomb(rcut=1e-9, exclude=[(0, 1)])
    keys = {autotune.signature([s1], rl, ff, device="B200") for ff in ([lj], [lj, dsf], [lj, dsfx], [dsf])}
    assert len(keys) == 4
    assert autotune.signature([s1], rl, [lj], device="B200") != autotune.signature([s1], rl, [lj], device="H100")
    assert autotune.signature([s1], rl, [lj], device="B200").endswith("_fflj_B200")


def test_candidates():
    # threads per atom: at least two list entries per lane, powers of two up to 32; step grids of one thread
    # per slot or 4 or 8 looping blocks per SM
    g = (0, 4, 8)
    assert autotune.candidates(1000, 200) == [(t, k) for t in (1, 2, 4, 8, 16, 32) for k in g]
    assert autotune.candidates(1000, 78) == [(t, k) for t in (1, 2, 4, 8, 16, 32) for k in g]
    assert autotune.candidates(1000, 40) == [(t, k) for t in (1, 2, 4, 8, 16) for k in g]
    assert autotune.candidates(1000, 1) == [(1, k) for k in g]
    # above two million atoms only 1, 2 or 4 threads per atom
    assert autotune.candidates(3_000_000, 200) == [(t, k) for t in (1, 2, 4) for k in g]
    # cell edges searched after the pair: the narrowest complete stencil first
    assert autotune.CELL_SCALES[0] == 1.0 and all(c > 1.0 for c in autotune.CELL_SCALES[1:])


def test_tune_searches_cell_edges_for_the_best_shape(tmp_path, monkeypatch):
    """The search order without a GPU: every (threads per atom, grid) pair at cell edge 1, then the wider cell
    edges for the fastest pair; the fastest of all is returned and cached with every timing."""
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "autotune.json"))
    s, lj = configs.lj_fluid(4, seed=0)
    fake_ms = {}

    class FakeEngine:
        def __init__(self, tpa, gm, cs):
            self.ms = 1.0 + 0.1 * tpa + 0.01 * gm - (0.3 if cs == 1.25 else 0.0)
            fake_ms[(tpa, gm, cs)] = self.ms

        def run(self, *a):
            pass

        def run_timed(self, steps, every):
            return 0.0, 0.0, self.ms * steps

        def check(self, where):
            pass

    import devinproj_b200.engine as engine

    def fake_start(systems, forces, dts, tpa=None, grid_mult=0, cell_scale=1.0, **k):
        return FakeEngine(tpa, grid_mult, cell_scale), None, None

    monkeypatch.setattr(engine, "start_engine", fake_start)
    assert autotune.tune([s], [lj], [1e-15]) == (1, 0, 1.25)
    narrow = {(t, g) for t, g, c in fake_ms if c == 1.0}
    wide = {(t, g, c) for t, g, c in fake_ms if c != 1.0}
    assert len(narrow) == len(fake_ms) - len(wide) > 1          # every pair timed at the narrowest cells
    assert wide == {(1, 0, c) for c in autotune.CELL_SCALES[1:]}  # wider cells only for the fastest pair
    (entry,) = autotune._load().values()
    assert entry["best"] == [1, 0, 1.25] and len(entry["ms_per_step"]) == len(fake_ms)
    assert entry["ms_per_step"]["1,0,1.25"] == min(entry["ms_per_step"].values())


def test_cache_round_trip_and_cached_answer(tmp_path, monkeypatch):
    cache = tmp_path / "sub" / "autotune.json"
    monkeypatch.setattr(autotune, "CACHE", str(cache))
    assert autotune._load() == {}                                   # missing file: empty
    s, lj = configs.lj_fluid(4, seed=0)
    from devinproj_b200.engine import forcefield_from
    _, rlist, _ = forcefield_from([lj], s.species)
    key = autotune.signature([s], rlist, [lj])
    autotune._store({key: {"best": [2, 0], "ms_per_step": {"1,0": 0.2, "2,0": 0.1}}})
    assert json.loads(cache.read_text())[key]["best"] == [2, 0]
    assert autotune._best({"best": [2, 4, 1.5]}) == (2, 4, 1.5)
    assert not (tmp_path / "sub" / "autotune.json.tmp").exists()    # written through a rename

    def no_engine(*a, **k):
        raise AssertionError("a cached workload must not build an engine")

    import devinproj_b200.engine as engine
    monkeypatch.setattr(engine, "start_engine", no_engine)
    assert autotune.tune([s], [lj], [1e-15]) == (2, 0, 1.0)     # an entry tuned before cell edges: edge 1
    cache.write_text("{ not json")
    assert autotune._load() == {}                                   # unreadable cache: empty, not an error


@pytest.mark.gpu
def test_tune_picks_a_measured_candidate(tmp_path, monkeypatch):
    """On the GPU: the tuner times every candidate and stores the fastest one under the workload's key."""
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "autotune.json"))
    s, lj = configs.lj_fluid(4, seed=0)
    best = autotune.tune([s], [lj], [0.005 * configs.AR_TAU], steps=5)
    db = autotune._load()
    (entry,) = db.values()
    assert tuple(entry["best"]) == best
    times = entry["ms_per_step"]
    label = f"{best[0]},{best[1]},{best[2]:g}"
    assert label in times and times[label] == min(times.values())
    wide = [k for k in times if not k.endswith(",1")]           # the wider cell edges, for one pair
    assert len(wide) == len(autotune.CELL_SCALES) - 1 and len({k.rsplit(",", 1)[0] for k in wide}) == 1
