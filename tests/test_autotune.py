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
    assert not (tmp_path / "sub" / "autotune.json.tmp").exists()    # written through a rename

    def no_engine(*a, **k):
        raise AssertionError("a cached workload must not build an engine")

    import devinproj_b200.engine as engine
    monkeypatch.setattr(engine, "start_engine", no_engine)
    assert autotune.tune([s], [lj], [1e-15]) == (2, 0)
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
    assert f"{best[0]},{best[1]}" in times and times[f"{best[0]},{best[1]}"] == min(times.values())
