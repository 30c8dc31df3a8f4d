"""GPU drop-ins for accusim's short-range forces: `LennardJones`, `DampedShiftedCoulomb` and the `VerletList` they
share (accusim/forces.py:78-175, :391-452).

The classes subclass accusim's own: constructor arguments, attributes (`params`, `cutoff`, `skin`,
`pairlist_threshold`, `rcut`, `alpha`, `k`, `exclude`, `rebuilds`, `_vl.rebuilds`) and the Lorentz-Berthelot
`_tables` are inherited, so accusim code that reads them or checks `isinstance` against the reference classes
sees the same objects. `compute(system) -> (F[n, 3] float64 N, U float J)` keeps the reference contract; the
pair search and the pair loops run as FP64 CUDA kernels in libaccusim_b200.so. On a `GpuSystem` the device
copy of the positions is used directly.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._accusim import forces as _af
from .device import DevStatus, Workspace, require_cuda, stream_handle, to_dev
from .state import is_gpu_system


def _check_system(s):
    if s.dim != 3:
        raise ValueError("accusim_b200 GPU forces handle 3-dimensional systems")


def _box_args(s):
    if s.box is None:
        return None, None, 0
    arr, p = _lib.dbl3(s.box)
    return arr, p, 1 if s.periodic else 0


class DeviceNeighborList:
    """Full (both-direction) neighbour list on the device, warp-interleaved (include/accusim_b200.h)."""

    def __init__(self):
        self.nbr = None
        self.nnb = None
        self.maxnb = 0
        self.ws = Workspace()
        self.status = None

    def _capacity(self, s, R, lo=None, hi=None):
        if s.box is not None:
            vol = float(np.prod(s.box))
        else:
            ext = np.maximum(hi - lo, R)
            vol = float(np.prod(ext))
        expected = s.n / max(vol, 1e-300) * 4.0 / 3.0 * math.pi * R ** 3
        return int(min(max(expected * 1.35 + 24, 16), s.n - 1 if s.n > 1 else 1) + 7) // 8 * 8

    def build(self, s, pos_d, R):
        """All j != i with minimum-image |d|^2 < R**2 (cell binning of accusim/forces.py:279-321)."""
        L = _lib.lib()
        n = s.n
        g = _lib.AcsGrid()
        boxarr, boxp, periodic = _box_args(s)
        lo = hi = None
        if s.box is None:   # open box: the grid spans the particles' extent
            ext = torch.stack([pos_d.min(dim=0).values, pos_d.max(dim=0).values]).cpu().numpy()
            lo, hi = np.ascontiguousarray(ext[0]), np.ascontiguousarray(ext[1])
            lop, hip = lo.ctypes.data, hi.ctypes.data
        else:
            lop = hip = None
        _lib.check(L.acs_grid_setup(C.byref(g), boxp, periodic, lop, hip, float(R)), "acs_grid_setup")
        g.rc2 = R ** 2
        wbytes = L.acs_nlist_work_bytes(n, C.byref(g))
        if self.status is None:
            self.status = DevStatus()
        maxnb = max(self.maxnb, self._capacity(s, R, lo, hi))
        for _ in range(4):
            npad = (n + 31) // 32 * 32
            if self.nbr is None or self.nbr.numel() < npad * maxnb:
                self.nbr = torch.empty(npad * maxnb, dtype=torch.int32, device="cuda")
            if self.nnb is None or self.nnb.numel() < n:
                self.nnb = torch.empty(n, dtype=torch.int32, device="cuda")
            ws = self.ws.get(wbytes)
            self.status.clear()
            _lib.check(L.acs_nlist_build(pos_d.data_ptr(), n, C.byref(g), maxnb, self.nbr.data_ptr(),
                                         self.nnb.data_ptr(), ws.data_ptr(), ws.numel(), self.status.ptr,
                                         stream_handle()), "acs_nlist_build")
            st = self.status.read()
            if st[0] & _lib.FLAG_OVERFLOW:
                maxnb = (int(st[1]) + 8 + 7) // 8 * 8
                continue
            self.maxnb = maxnb
            return self
        raise _lib.ListOverflow(_lib.ACS_ERR_LIST_OVERFLOW, "acs_nlist_build")

    def pairs(self, n):
        """Unique pairs (i < j) as host int64 arrays."""
        L = _lib.lib()
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        cap = int(self.nnb[:n].sum().item()) // 2 + 1
        pi = torch.empty(cap, dtype=torch.int32, device="cuda")
        pj = torch.empty(cap, dtype=torch.int32, device="cuda")
        _lib.check(L.acs_nlist_pairs(self.nbr.data_ptr(), self.nnb.data_ptr(), n, self.maxnb, pi.data_ptr(),
                                     pj.data_ptr(), cap, cnt.data_ptr(), stream_handle()), "acs_nlist_pairs")
        m = int(cnt.item())
        if m > cap:
            raise RuntimeError("pair count exceeds capacity")
        return pi[:m].cpu().numpy().astype(np.int64), pj[:m].cpu().numpy().astype(np.int64)


class VerletList:
    """Cell-list pairs within rc + skin, reused until some particle has moved skin/2 or more; rebuilt when
    ids, box or rc change (accusim/forces.py:78-98). The list, reference positions and the displacement
    test live on the device."""

    def __init__(self):
        self._state = None
        self.rebuilds = 0
        self._flag = None

    def _same_ids(self, s, st):
        """ids unchanged since the last build (a GpuSystem whose ids were not touched needs no comparison)."""
        if is_gpu_system(s) and st["ids_version"] == (id(s), s.ids_version()):
            return True
        ids = s.ids
        return st["ids"].shape == ids.shape and np.array_equal(st["ids"], ids)

    def pairs(self, s, pos_d, rc, skin) -> DeviceNeighborList:
        st = self._state
        if st is not None and self._same_ids(s, st) and np.array_equal(st["box"], s.box) and st["rc"] == rc \
                and skin > 0:
            if self._flag is None:
                self._flag = torch.zeros(1, dtype=torch.int32, device="cuda")
            boxarr, boxp, periodic = _box_args(s)
            _lib.check(_lib.lib().acs_nlist_displacement(pos_d.data_ptr(), st["pos0"].data_ptr(), s.n, boxp,
                                                         periodic, (0.5 * skin) ** 2, self._flag.data_ptr(),
                                                         stream_handle()), "acs_nlist_displacement")
            if int(self._flag.item()) == 0:
                return st["list"]
        nl = st["list"] if st is not None else DeviceNeighborList()
        nl.build(s, pos_d, rc + skin)
        ids = s.ids.copy()
        self._state = dict(list=nl, pos0=pos_d.clone(), ids=ids, box=None if s.box is None else s.box.copy(), rc=rc,
                           ids_version=(id(s), s.ids_version()) if is_gpu_system(s) else None)
        self.rebuilds += 1
        return nl


class _Scratch:
    def __init__(self):
        self.ws = Workspace()
        self.energy = None

    def energy_buf(self):
        if self.energy is None:
            self.energy = torch.zeros(1, dtype=torch.float64, device="cuda")
        return self.energy


class LennardJones(_af.LennardJones):
    """accusim's 12-6 Lennard-Jones (Lorentz-Berthelot mixing, energy shifted to zero at cutoff*sigma_ij) with
    its pair search and pair loop on the GPU: the Verlet list for n >= pairlist_threshold, the dense all-pairs
    kernel below."""

    def __init__(self, params: dict, cutoff: float = 2.5, pairlist_threshold: int = 400, skin: float = 0.3):
        super().__init__(params, cutoff=cutoff, pairlist_threshold=pairlist_threshold, skin=skin)
        self._vl = VerletList()
        self._scr = _Scratch()

    def list_radius(self, s):
        eps_t, sig_t = self._tables(s)
        smax = float(np.max(np.where(eps_t > 0, sig_t, 0)))
        return self.cutoff * smax, self.skin * smax

    def compute_device(self, s, pos_d, sp_d):
        """Forces as a device tensor (n, 3) and the energy as a device scalar."""
        n = s.n
        eps_t, sig_t = self._tables(s)
        F = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        E = self._scr.energy_buf()
        if n < 2 or not np.any(eps_t > 0):
            F.zero_()
            E.zero_()
            return F, E
        nl = None
        if n >= self.pairlist_threshold:
            rc, skin = self.list_radius(s)
            nl = self._vl.pairs(s, pos_d, rc, skin)
        L = _lib.lib()
        ws = self._scr.ws.get(L.acs_force_work_bytes(n))
        boxarr, boxp, periodic = _box_args(s)
        eps_c = np.ascontiguousarray(eps_t, dtype=np.float64)
        sig_c = np.ascontiguousarray(sig_t, dtype=np.float64)
        _lib.check(L.acs_lj_fp64(pos_d.data_ptr(), sp_d.data_ptr(), n, boxp, periodic,
                                 nl.nbr.data_ptr() if nl else None, nl.nnb.data_ptr() if nl else None,
                                 nl.maxnb if nl else 0, len(s.species), eps_c.ctypes.data, sig_c.ctypes.data,
                                 float(self.cutoff), F.data_ptr(), E.data_ptr(), ws.data_ptr(), ws.numel(),
                                 stream_handle()), "acs_lj_fp64")
        return F, E

    def compute(self, s):
        if s.n < 2:
            return np.zeros((s.n, s.dim)), 0.0
        _check_system(s)
        require_cuda()
        F, E = self.compute_device(s, *_device_positions(s))
        return F.cpu().numpy(), float(E.item())


class DampedShiftedCoulomb(_af.DampedShiftedCoulomb):
    """accusim's damped shifted force electrostatics (Fennell & Gezelter 2006; `exclude` id pairs, skin 0.15
    rcut by default) with its pair search and pair loop on the GPU."""

    def __init__(self, rcut, alpha=None, k=None, pairlist_threshold=400, exclude=(), skin=None):
        kw = {} if k is None else {"k": k}
        super().__init__(rcut, alpha=alpha, pairlist_threshold=pairlist_threshold, exclude=exclude, skin=skin, **kw)
        self._vl = VerletList()
        self._scr = _Scratch()

    def _exclusion_csr(self, s):
        """Excluded pairs as a CSR table by atom index, both directions (device int32), or (None, None). Cached
        for a GpuSystem whose ids were not touched since."""
        if not self.exclude:
            return None, None
        key = (id(s), s.ids_version(), len(self.exclude)) if is_gpu_system(s) else None
        cached = getattr(self, "_ex_cache", None)
        if key is not None and cached is not None and cached[0] == key:
            return cached[1]
        out = self._exclusion_table(s)
        if key is not None:
            self._ex_cache = (key, out)
        return out

    def _exclusion_table(self, s):
        where = {int(pid): k for k, pid in enumerate(s.ids)}
        ex = [(where[a], where[b]) for a, b in self.exclude if a in where and b in where]
        if not ex:
            return None, None
        ex = np.array(ex, dtype=np.int64)
        src = np.concatenate([ex[:, 0], ex[:, 1]])
        dst = np.concatenate([ex[:, 1], ex[:, 0]])
        order = np.lexsort((dst, src))
        src, dst = src[order], dst[order]
        start = np.zeros(s.n + 1, dtype=np.int32)
        np.add.at(start, src + 1, 1)
        start = np.cumsum(start).astype(np.int32)
        return to_dev(start), to_dev(dst.astype(np.int32))

    def compute_device(self, s, pos_d):
        """Forces as a device tensor (n, 3) and the energy as a device scalar."""
        n = s.n
        F = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        E = self._scr.energy_buf()
        if is_gpu_system(s):
            q_d, charged = s.device_charges()
        else:
            q = np.asarray(s.charges, dtype=np.float64)
            q_d, charged = to_dev(q), bool(np.any(q))
        if not charged:
            F.zero_()
            E.zero_()
            return F, E
        nl = None
        if n >= self.pairlist_threshold:
            nl = self._vl.pairs(s, pos_d, self.rcut, self.skin)
        exs, exi = self._exclusion_csr(s)
        L = _lib.lib()
        ws = self._scr.ws.get(L.acs_force_work_bytes(n))
        boxarr, boxp, periodic = _box_args(s)
        _lib.check(L.acs_dsf_fp64(pos_d.data_ptr(), q_d.data_ptr(), n, boxp, periodic,
                                  nl.nbr.data_ptr() if nl else None, nl.nnb.data_ptr() if nl else None,
                                  nl.maxnb if nl else 0, exs.data_ptr() if exs is not None else None,
                                  exi.data_ptr() if exi is not None else None, float(self.alpha), float(self.rcut),
                                  float(self.k), F.data_ptr(), E.data_ptr(), ws.data_ptr(), ws.numel(),
                                  stream_handle()), "acs_dsf_fp64")
        return F, E

    def compute(self, s):
        q = s.charges
        if not np.any(q):
            return np.zeros((s.n, s.dim)), 0.0
        _check_system(s)
        require_cuda()
        F, E = self.compute_device(s, _device_positions(s)[0])
        return F.cpu().numpy(), float(E.item())


def _device_positions(s):
    """(positions, species) of a system as device tensors: a GpuSystem's resident copy, else one upload."""
    if is_gpu_system(s):
        return s.device_state()[0], s.device_species()
    return to_dev(np.asarray(s.pos, dtype=np.float64)), to_dev(np.asarray(s.sp), torch.int32)


def cell_list_pairs(s, rc):
    """All pairs (i < j) closer than rc, found on the device (accusim/forces.py:279-321)."""
    _check_system(s)
    require_cuda()
    nl = DeviceNeighborList().build(s, _device_positions(s)[0], rc)
    i, j = nl.pairs(s.n)
    order = np.lexsort((j, i))
    return i[order], j[order]
