"""acs_lj_fp64_noalloc: the LJ force entry point for callers that cannot allocate device memory (an external
memory pool owns the GPU, allocation is forbidden once the run has started, or the host hands the plug-in
only its input and output buffers). It keeps its reduction scratch in a fixed array inside the library, so
it takes no work buffer. Checked here through the C ABI against acs_lj_fp64 on the same inputs, on two
calls in a row, with the drop-in tolerance (max|dF| <= 1e-12 max|F|, |dU| <= 1e-12 |U|); and its size limit
is checked without launching anything.

This file is collected last on purpose (the name sorts after the other test files)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12
MAX_ATOMS = 2_097_152


def _call_both(s, lj, use_list):
    import torch

    from devinproj_b200 import _lib
    from devinproj_b200.device import stream_handle, to_dev
    from devinproj_b200.forces import DeviceNeighborList
    L = _lib.lib()
    n = s.n
    pos = to_dev(s.pos)
    sp = to_dev(s.sp, torch.int32)
    eps, sig = lj._tables(s)
    eps = np.ascontiguousarray(eps)
    sig = np.ascontiguousarray(sig)
    nl = None
    if use_list:
        rc, skin = lj.list_radius(s)
        nl = DeviceNeighborList().build(s, pos, rc + skin)
    box = np.ascontiguousarray(s.box, dtype=np.float64)
    args = (pos.data_ptr(), sp.data_ptr(), n, box.ctypes.data, 1, nl.nbr.data_ptr() if nl else None,
            nl.nnb.data_ptr() if nl else None, nl.maxnb if nl else 0, len(s.species), eps.ctypes.data,
            sig.ctypes.data, float(lj.cutoff))
    F_ref = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    E_ref = torch.zeros(1, dtype=torch.float64, device="cuda")
    ws = torch.empty(L.acs_force_work_bytes(n), dtype=torch.uint8, device="cuda")
    assert L.acs_lj_fp64(*args, F_ref.data_ptr(), E_ref.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle()) == 0
    F = torch.full((n, 3), float("nan"), dtype=torch.float64, device="cuda")
    E = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    assert L.acs_lj_fp64_noalloc(*args, F.data_ptr(), E.data_ptr(), stream_handle()) == 0
    torch.cuda.synchronize()
    return F_ref.cpu().numpy(), float(E_ref.item()), F.cpu().numpy(), float(E.item())


def test_noalloc_matches_workspace_entry_point_on_two_calls_in_a_row():
    from devinproj_b200 import configs
    # call 1: the 864-atom argon case, perturbed, through its neighbour list
    s, forces, _ = configs.argon864(seed=0)
    s.pos = (s.pos + np.random.default_rng(1).normal(0, 0.05 * configs.AR_SIGMA, s.pos.shape)) % s.box
    F_ref, U_ref, F, U = _call_both(s, forces[0], use_list=True)
    assert np.max(np.abs(F - F_ref)) <= TOL * np.max(np.abs(F_ref))
    assert abs(U - U_ref) <= TOL * abs(U_ref)
    # call 2, straight after: a different, larger system on the dense path; the shared scratch from call 1
    # must not leak into it
    s2, lj2 = configs.lj_fluid(7, seed=3)
    F_ref, U_ref, F, U = _call_both(s2, lj2, use_list=False)
    assert np.max(np.abs(F - F_ref)) <= TOL * np.max(np.abs(F_ref))
    assert abs(U - U_ref) <= TOL * abs(U_ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from devinproj_b200 import _lib
    L = _lib.lib()
    eps = np.ones(1)
    sig = np.ones(1)
    st = L.acs_lj_fp64_noalloc(None, None, MAX_ATOMS + 1, None, 1, None, None, 0, 1, eps.ctypes.data,
                               sig.ctypes.data, 2.5, None, None, None)
    assert st == _lib.ACS_ERR_UNSUPPORTED
    assert "unsupported" in _lib.status_string(st)
