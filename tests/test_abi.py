"""The C-ABI library loads without a GPU and exports every entry point include/*.h declares; host-only
entry points (grid set-up, workspace queries, status strings) behave as documented. CPU only."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from devinproj_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(acs_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 15
    L = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_abi_version_and_status_strings():
    L = _lib.lib()
    assert L.acs_abi_version() == 1
    assert _lib.status_string(0) == "ok"
    assert "capacity exceeded" in _lib.status_string(_lib.ACS_ERR_LIST_OVERFLOW)
    with pytest.raises(_lib.ListOverflow):
        _lib.check(_lib.ACS_ERR_LIST_OVERFLOW, "x")


@pytest.mark.parametrize("L_sigma,rc_sigma,expect", [(10.229, 2.8, 3), (107.53, 2.8, 38), (6.72, 2.8, 1),
                                                     (9.0, 3.0, 3), (8.99, 3.0, 1)])
def test_grid_setup_matches_reference_binning(L_sigma, rc_sigma, expect):
    """ncell = floor(box / rc), collapsed to 1 below 3 in periodic boxes (accusim/forces.py:287-289)."""
    g = _lib.AcsGrid()
    box = np.full(3, L_sigma * 3.4e-10)
    st = _lib.lib().acs_grid_setup(C.byref(g), box.ctypes.data, 1, None, None, rc_sigma * 3.4e-10)
    assert st == 0
    ref = max(int(box[0] // (rc_sigma * 3.4e-10)), 1)
    ref = 1 if ref < 3 else ref
    assert list(g.ncell) == [ref] * 3 == [expect] * 3
    assert _lib.lib().acs_nlist_work_bytes(1000, C.byref(g)) > 4 * 1000


def test_grid_setup_open_system_and_bad_args():
    g = _lib.AcsGrid()
    lo = np.array([0.0, -1.0, 2.0])
    hi = np.array([10.0, 1.0, 2.0])
    assert _lib.lib().acs_grid_setup(C.byref(g), None, 0, lo.ctypes.data, hi.ctypes.data, 1.5) == 0
    assert list(g.ncell) == [6, 1, 1] and g.periodic == 0 and g.span[2] == 1.5
    assert _lib.lib().acs_grid_setup(C.byref(g), None, 0, None, None, 1.5) == _lib.ACS_ERR_ARG
    assert _lib.lib().acs_grid_setup(C.byref(g), lo.ctypes.data, 1, None, None, 0.0) == _lib.ACS_ERR_ARG


def _engine_config(n=864, box_sigma=10.229, tpa=1, maxnb=96, thermo=None):
    from devinproj_b200 import engine as E
    reps = (E.Replica * 1)()
    reps[0].n = n
    for d in range(3):
        reps[0].box[d] = box_sigma * 3.4
    reps[0].dt = 0.02
    reps[0].rlist = 2.8 * 3.4
    reps[0].half_skin = 0.15 * 3.4
    ff = E.ForceField()
    ff.n_species, ff.lj = 1, 1
    ff.mass[0] = 39.948
    ff.lj_eps[0], ff.lj_sig[0], ff.lj_cutoff = 0.998, 3.4, 2.5
    cfg = E.EngineConfig(1, maxnb, 16, 0, tpa, 0, reps, ff, thermo if thermo is not None else E.Thermostat())
    return cfg, reps


def test_engine_config_validation_is_host_side():
    """acs_engine_bytes sizes the engine's device block on the host: it is positive for valid configurations
    and 0 for invalid ones (threads per atom, box, thermostat parameters); a list radius of half the box or more
    is valid (such a replica rebuilds its lists every step)."""
    from devinproj_b200 import engine as E
    from devinproj_b200.engine import ENGINE_SIGNATURES
    L = _lib.lib()
    res, args = ENGINE_SIGNATURES["acs_engine_bytes"]
    L.acs_engine_bytes.restype, L.acs_engine_bytes.argtypes = res, args
    cfg, keep = _engine_config()
    ok = L.acs_engine_bytes(C.byref(cfg))
    assert ok > 864 * 96 * 4
    for tpa in (2, 4, 8, 16, 32):
        c2, k2 = _engine_config(tpa=tpa)
        assert L.acs_engine_bytes(C.byref(c2)) > 0
    bad = [_engine_config(tpa=3), _engine_config(box_sigma=0.0),
           _engine_config(thermo=E.Thermostat(3, 0, 1.0, 1.0, 0, 0.0)),
           _engine_config(thermo=E.Thermostat(1, 0, 1.0, -1.0, 0, 0.0)),
           _engine_config(thermo=E.Thermostat(2, 0, 1.0, 0.0, 0, 0.0))]
    for c3, k3 in bad:
        assert L.acs_engine_bytes(C.byref(c3)) == 0
    small, ks = _engine_config(box_sigma=5.0)
    assert L.acs_engine_bytes(C.byref(small)) > 0
    good = [E.Thermostat(1, 0, 0.997, 0.05, 7, 0.0), E.Thermostat(2, 0, 0.997, 0.0, 0, 2.0)]
    for th in good:
        c4, k4 = _engine_config(thermo=th)
        assert L.acs_engine_bytes(C.byref(c4)) >= ok
    # the list build's cell edge: 0 (one list radius) or 1..8 list radii; wider cells need fewer cell slots
    for cs, valid in ((0.0, True), (1.0, True), (1.5, True), (8.0, True), (0.99, False), (0.5, False),
                      (8.5, False), (float("nan"), False), (-1.0, False)):
        c5, k5 = _engine_config()
        c5.cell_scale = cs
        assert (L.acs_engine_bytes(C.byref(c5)) > 0) == valid, cs
    c5, k5 = _engine_config(box_sigma=40.0)
    c6, k6 = _engine_config(box_sigma=40.0)
    c6.cell_scale = 1.5
    assert 0 < L.acs_engine_bytes(C.byref(c6)) < L.acs_engine_bytes(C.byref(c5))   # 9^3 cells instead of 14^3


def test_engine_dsf_exclusion_tables():
    """DSF exclusions: the engine's CSR table by atom index (ids mapped through system.ids, both directions,
    pairs with an unknown id dropped) and its host-side validation in acs_engine_bytes."""
    from accusim import System

    from devinproj_b200 import DampedShiftedCoulomb
    from devinproj_b200 import engine as E
    from devinproj_b200.engine import ENGINE_SIGNATURES, dsf_exclusions
    s = System(3, box=20.0, periodic=True)
    s.add_species("Na", 1.0, charge=1.0)
    s.add("Na", np.random.default_rng(0).uniform(0, 20, (6, 3)))
    s.ids = np.array([10, 11, 12, 13, 14, 15])
    f = DampedShiftedCoulomb(rcut=3.0, exclude=[(10, 12), (15, 11), (12, 13), (99, 10)])
    ex_start, ex_ids = dsf_exclusions([f], [s])
    got = {a: sorted(ex_ids[ex_start[a]:ex_start[a + 1]].tolist()) for a in range(6)}
    assert got == {0: [2], 1: [5], 2: [0, 3], 3: [2], 4: [], 5: [1]}
    assert dsf_exclusions([DampedShiftedCoulomb(rcut=3.0)], [s]) is None
    s2 = s.copy()
    s2.ids = np.array([10, 11, 12, 13, 15, 14])
    with pytest.raises(ValueError):
        dsf_exclusions([f], [s, s2])

    L = _lib.lib()
    res, args = ENGINE_SIGNATURES["acs_engine_bytes"]
    L.acs_engine_bytes.restype, L.acs_engine_bytes.argtypes = res, args
    base, keep = _engine_config()
    n0 = L.acs_engine_bytes(C.byref(base))
    cfg, keep = _engine_config()
    cfg.ex_start = ex_start.ctypes.data_as(C.POINTER(C.c_int32))
    cfg.ex_ids = ex_ids.ctypes.data_as(C.POINTER(C.c_int32))
    cfg.n_ex_ids = 6
    assert L.acs_engine_bytes(C.byref(cfg)) >= n0 > 0
    for start in (np.array([1, 1, 2, 4, 5, 5, 6], np.int32), np.array([0, 2, 1, 4, 5, 5, 6], np.int32)):
        bad, keep2 = _engine_config()
        bad.ex_start = start.ctypes.data_as(C.POINTER(C.c_int32))
        bad.ex_ids = ex_ids.ctypes.data_as(C.POINTER(C.c_int32))
        bad.n_ex_ids = 6
        assert L.acs_engine_bytes(C.byref(bad)) == 0
    nul, keep3 = _engine_config()
    nul.n_ex_ids = 6
    assert L.acs_engine_bytes(C.byref(nul)) == 0


def test_rdf_workspace_query():
    g = _lib.AcsGrid()
    box = np.full(3, 30.0)
    assert _lib.lib().acs_grid_setup(C.byref(g), box.ctypes.data, 1, None, None, 14.0) == 0
    assert _lib.lib().acs_rdf_work_bytes(1000, C.byref(g)) == _lib.lib().acs_nlist_work_bytes(1000, C.byref(g)) > 0


def test_engine_erfc_approximation_bound():
    """The FP32 DSF term's erfc (Abramowitz & Stegun 7.1.26, as written in csrc/engine.cu) against scipy's:
    within the method's published 1.5e-7 in FP64, and within 7e-7 when evaluated in FP32 as the kernel does."""
    from scipy.special import erfc
    src = open(os.path.join(os.path.dirname(__file__), "..", "devinproj_b200", "csrc", "engine.cu")).read()
    body = src[src.index("float erfc_as(float x, float e)"):]
    body = body[:body.index("\n}")]
    c = [float(v) for v in re.findall(r"(-?\d+\.\d+)f", body) if float(v) != 1.0]   # p, then a5 .. a1 (Horner)
    p, a5, a4, a3, a2, a1 = c
    x = np.linspace(0.0, 4.0, 400001)
    t = 1.0 / (1.0 + p * x)
    approx = t * (a1 + t * (a2 + t * (a3 + t * (a4 + t * a5)))) * np.exp(-x * x)
    assert np.max(np.abs(approx - erfc(x))) <= 1.5e-7
    f = np.float32
    xf = x.astype(f)
    tf = f(1) / (f(1) + f(p) * xf)
    qf = tf * (f(a1) + tf * (f(a2) + tf * (f(a3) + tf * (f(a4) + tf * f(a5)))))
    assert np.max(np.abs((qf * np.exp(-(xf * xf))).astype(np.float64) - erfc(x))) <= 7e-7
    # the host copy behind the DSF shift constants (erfc(alpha rc)) carries the same coefficients, so the
    # engine's shifted DSF term vanishes at rc under the approximation it evaluates
    host = src[src.index("double erfc_as_host(double x)"):]
    host = host[:host.index("\n}")]
    ch = [float(v) for v in re.findall(r"(-?\d+\.\d+)", host) if float(v) != 1.0]
    assert ch == [p, a5, a4, a3, a2, a1]


def test_default_threads_per_atom_follow_measured_optima():
    """The size heuristic for threads per atom (host only) picks the B200 optima measured for these systems:
    few cells -> a warp per atom (16 for the long DSF lists of NaCl), otherwise 1-4 threads per atom."""
    from devinproj_b200.engine import default_tpa
    assert default_tpa(864, 78, 27) == 32            # argon 864, 3^3 cells
    assert default_tpa(4000, 78, 216) == 32          # LJ fcc 10^3
    assert default_tpa(4096, 370, 27) == 16          # NaCl 4096, LJ + DSF
    assert default_tpa(16384, 78, 729) == 4          # LJ fcc 16^3
    assert default_tpa(32000, 78, 1331) == 4         # LJ fcc 20^3 (2 and 4 measured alike)
    assert default_tpa(108000, 78, 4913) == 1        # LJ fcc 30^3
    assert default_tpa(1048576, 78, 54872) == 1      # the 1M-atom fluid
