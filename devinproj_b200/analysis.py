"""`rdf` (accusim/analysis.py:7-24) with the pair-distance histogram on the GPU.

acs_rdf_hist counts pair distances over a cell list at radius rmax with the reference's FP64 minimum image and
NumPy's uniform-bin histogram rule, so its counts equal the reference's O(n^2) NumPy histogram while needing
O(n) memory; the ideal-gas normalisation is the reference's NumPy expression. accusim's own `msd` and trajectory
files (accusim/analysis.py:27-43, accusim/io.py) work unchanged on `GpuSimulation` trajectories, which are
accusim `Trajectory` objects.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import Workspace, require_cuda, stream_handle, to_dev

_ws = Workspace()


def rdf(system, rmax, bins=100, species=None):
    """Radial distribution function g(r) in a periodic 3-D box (minimum image). Returns (r, g)."""
    s = system
    if not s.periodic or s.box is None:
        raise ValueError("rdf needs a periodic box (for normalisation)")
    if rmax > 0.5 * np.min(np.broadcast_to(s.box, (s.dim,))):
        raise ValueError("rmax must be at most half the box")
    if s.dim != 3:
        raise ValueError("accusim_b200 rdf handles 3-dimensional systems")
    require_cuda()
    L = _lib.lib()
    sp_index = -1 if species is None else s.species_index(species)
    n = s.n if species is None else int(np.count_nonzero(s.sp == sp_index))
    g = _lib.AcsGrid()
    boxarr = np.ascontiguousarray(np.broadcast_to(s.box, (3,)), dtype=np.float64)
    _lib.check(L.acs_grid_setup(C.byref(g), boxarr.ctypes.data, 1, None, None, float(rmax)), "acs_grid_setup")
    pos_d = to_dev(np.asarray(s.pos, dtype=np.float64))
    sp_d = to_dev(np.asarray(s.sp), torch.int32)
    hist_d = torch.zeros(bins, dtype=torch.int64, device="cuda")
    ws = _ws.get(L.acs_rdf_work_bytes(s.n, C.byref(g)))
    _lib.check(L.acs_rdf_hist(pos_d.data_ptr(), sp_d.data_ptr(), s.n, C.byref(g), sp_index, int(bins), float(rmax),
                              hist_d.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle()), "acs_rdf_hist")
    hist = hist_d.cpu().numpy()
    edges = np.linspace(0, rmax, bins + 1)
    V = float(np.prod(np.broadcast_to(s.box, (s.dim,))))
    shell = 4 / 3 * np.pi * (edges[1:] ** 3 - edges[:-1] ** 3)
    ideal = shell * n * (n - 1) / 2 / V
    return 0.5 * (edges[1:] + edges[:-1]), hist / ideal
