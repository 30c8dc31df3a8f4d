"""GPU drop-ins for accusim's short-range forces: `LennardJones`, `DampedShiftedCoulomb` and the
`VerletList` they share (accusim/forces.py:78-175, :391-452).

Same constructor arguments, attributes and `compute(system) -> (F[n, 3] float64 N, U float J)` contract as
the reference; the pair search and pair loops run as FP64 CUDA kernels in libaccusim_b200.so. Systems
may be this package's `System` or the reference's; only `pos`, `sp`, `ids`, `box`, `periodic`,
`species` and `n` are read.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from .device import DevStatus, Workspace, require_cuda, stream_handle, to_dev
from .system import species_arrays
from .units import k_e, si


class Force:
    """Plug-in base with the reference's class flags (accusim/forces.py:15-21)."""

    conservative = True
    external = False
    central = True

    def compute(self, system):
        raise NotImplementedError


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

    def _capacity(self, s, pos_d, R):
        if s.box is not None:
            vol = float(np.prod(s.box))
        else:
            ext = np.maximum(np.ptp(s.pos, axis=0), R)
            vol = float(np.prod(ext))
        expected = s.n / max(vol, 1e-300) * 4.0 / 3.0 * math.pi * R ** 3
        return int(min(max(expected * 1.35 + 24, 16), s.n - 1 if s.n > 1 else 1) + 7) // 8 * 8

    def build(self, s, pos_d, R):
        """All j != i with minimum-image |d|^2 < R**2 (cell binning of accusim/forces.py:279-321)."""
        L = _lib.lib()
        n = s.n
        g = _lib.AcsGrid()
        boxarr, boxp, periodic = _box_args(s)
        if s.box is None:
            lo = np.ascontiguousarray(s.pos.min(axis=0), dtype=np.float64)
            hi = np.ascontiguousarray(s.pos.max(axis=0), dtype=np.float64)
            lop, hip = lo.ctypes.data, hi.ctypes.data
        else:
            lop = hip = None
        _lib.check(L.acs_grid_setup(C.byref(g), boxp, periodic, lop, hip, float(R)), "acs_grid_setup")
        g.rc2 = R ** 2
        wbytes = L.acs_nlist_work_bytes(n, C.byref(g))
        if self.status is None:
            self.status = DevStatus()
        maxnb = max(self.maxnb, self._capacity(s, pos_d, R))
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

    def pairs(self, s, pos_d, rc, skin) -> DeviceNeighborList:
        st = self._state
        if st is not None and st["ids"].shape == s.ids.shape and np.array_equal(st["ids"], s.ids) \
                and np.array_equal(st["box"], s.box) and st["rc"] == rc and skin > 0:
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
        self._state = dict(list=nl, pos0=pos_d.clone(), ids=s.ids.copy(),
                           box=None if s.box is None else s.box.copy(), rc=rc)
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


class LennardJones(Force):
    """12-6 Lennard-Jones with Lorentz-Berthelot mixing, truncated at cutoff*sigma_ij with the energy
    shifted to zero there (accusim/forces.py:101-175). params: {species: (epsilon J, sigma m)}; species
    not listed do not interact. `cutoff`, `skin` in units of sigma; N >= pairlist_threshold uses the
    Verlet list, smaller systems the dense all-pairs kernel."""

    def __init__(self, params: dict, cutoff: float = 2.5, pairlist_threshold: int = 400, skin: float = 0.3):
        self.params = {k: (si(e, "J"), si(sg, "m")) for k, (e, sg) in params.items()}
        self.cutoff = cutoff
        self.pairlist_threshold = pairlist_threshold
        self.skin = skin
        self._vl = VerletList()
        self._scr = _Scratch()

    @property
    def rebuilds(self):
        return self._vl.rebuilds

    def _tables(self, s):
        """Lorentz-Berthelot tables (accusim/forces.py:144-155)."""
        k = len(s.species)
        eps = np.zeros((k, k))
        sig = np.ones((k, k))
        for a, A in enumerate(s.species):
            for b, B in enumerate(s.species):
                if A.name in self.params and B.name in self.params:
                    ea, sa = self.params[A.name]
                    eb, sb = self.params[B.name]
                    eps[a, b] = np.sqrt(ea * eb)
                    sig[a, b] = 0.5 * (sa + sb)
        return eps, sig

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
            return np.zeros_like(s.pos), 0.0
        _check_system(s)
        require_cuda()
        F, E = self.compute_device(s, to_dev(s.pos), to_dev(s.sp, torch.int32))
        return F.cpu().numpy(), float(E.item())


class DampedShiftedCoulomb(Force):
    """Damped shifted force electrostatics (Fennell & Gezelter 2006): pair potential erfc(a r)/r shifted
    so energy and force vanish at rcut, plus the self term (accusim/forces.py:391-452). `exclude` lists id
    pairs with no interaction; `skin` defaults to 0.15 rcut."""

    def __init__(self, rcut, alpha=None, k=k_e, pairlist_threshold=400, exclude=(), skin=None):
        self.pairlist_threshold = pairlist_threshold
        self.exclude = [tuple(p) for p in exclude]
        self.k = si(k, "J*m/C^2")
        self.rcut = si(rcut, "m")
        self.alpha = 2.0 / self.rcut if alpha is None else si(alpha, "1/m")
        self.skin = 0.15 * self.rcut if skin is None else si(skin, "m")
        self._vl = VerletList()
        self._scr = _Scratch()

    @property
    def rebuilds(self):
        return self._vl.rebuilds

    def _exclusion_csr(self, s):
        if not self.exclude:
            return None, None
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

    def compute_device(self, s, pos_d, q_d=None):
        n = s.n
        F = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        E = self._scr.energy_buf()
        q = s.charges
        if not np.any(q):
            F.zero_()
            E.zero_()
            return F, E
        if q_d is None or q_d.dtype != torch.float64:
            q_d = to_dev(q.astype(np.float64))
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
            return np.zeros_like(s.pos), 0.0
        _check_system(s)
        require_cuda()
        F, E = self.compute_device(s, to_dev(s.pos))
        return F.cpu().numpy(), float(E.item())


def cell_list_pairs(s, rc):
    """All pairs (i < j) closer than rc, found on the device (accusim/forces.py:279-321)."""
    _check_system(s)
    require_cuda()
    nl = DeviceNeighborList().build(s, to_dev(s.pos), rc)
    i, j = nl.pairs(s.n)
    order = np.lexsort((j, i))
    return i[order], j[order]
