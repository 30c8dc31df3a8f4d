"""Ewald summation on the device, with the interface of accusim's `Ewald` (accusim/forces.py:333-388).

Exact periodic electrostatics for a neutral 3-D periodic system: real-space erfc sum over minimum-image
pairs inside rcut, reciprocal sum over the k-vectors |n| <= kmax (built on the host exactly as the
reference builds them), self term. Defaults: rcut = L_min / 2, alpha = 4 / rcut, kmax = 12. FP64.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import Workspace, require_cuda, stream_handle, to_dev
from .forces import Force
from .units import k_e, si

_lib.SIGNATURES.update({
    "acs_ewald_work_bytes": (_lib.SZ, [_lib.I64, _lib.I32]),
    "acs_ewald_fp64": (_lib.C.c_int, [_lib.P] * 4 + [_lib.P, _lib.P, _lib.I32, _lib.DBL, _lib.DBL, _lib.DBL, _lib.P,
                                                    _lib.P, _lib.P, _lib.SZ, _lib.P]),
    "acs_umma_gemm_test": (_lib.C.c_int, [_lib.P, _lib.P, _lib.P, _lib.I32, _lib.I32, _lib.P, _lib.P]),
})
# acs_ewald_fp64(pos, q, n, box3, kvec, kw, K, alpha, rcut, k, force, energy3, work, bytes, stream)
_lib.SIGNATURES["acs_ewald_fp64"] = (_lib.C.c_int, [_lib.P, _lib.P, _lib.I64, _lib.P, _lib.P, _lib.P, _lib.I32,
                                                    _lib.DBL, _lib.DBL, _lib.DBL, _lib.P, _lib.P, _lib.P, _lib.SZ,
                                                    _lib.P])


def _bind():
    L = _lib.lib()
    for name in ("acs_ewald_work_bytes", "acs_ewald_fp64", "acs_umma_gemm_test"):
        res, args = _lib.SIGNATURES[name]
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args
    return L


class Ewald(Force):
    """Exact periodic electrostatics by Ewald summation (3D orthorhombic box, neutral system)."""

    def __init__(self, k=k_e, alpha=None, rcut=None, kmax=12):
        self.k = si(k, "J*m/C^2")
        self.alpha = None if alpha is None else si(alpha, "1/m")
        self.rcut = None if rcut is None else si(rcut, "m")
        self.kmax = kmax
        self._kcache = None
        self._ws = Workspace()

    def _kvectors(self, box, alpha):
        """accusim/forces.py:347-357: |n| <= kmax sphere without n = 0, k = 2 pi n / box,
        w = exp(-k^2 / (4 alpha^2)) / k^2."""
        key = (tuple(box), alpha, self.kmax)
        if self._kcache is None or self._kcache[0] != key:
            n = np.arange(-self.kmax, self.kmax + 1)
            N = np.stack(np.meshgrid(n, n, n, indexing="ij"), -1).reshape(-1, 3)
            N = N[np.sum(N ** 2, axis=1) <= self.kmax ** 2]
            N = N[np.any(N != 0, axis=1)]
            kv = 2 * np.pi * N / box
            k2 = np.sum(kv ** 2, axis=1)
            w = np.exp(-k2 / (4 * alpha ** 2)) / k2
            self._kcache = (key, to_dev(np.ascontiguousarray(kv)), to_dev(np.ascontiguousarray(w)), len(w))
        return self._kcache[1], self._kcache[2], self._kcache[3]

    def compute_device(self, s, pos_d, q):
        if s.dim != 3 or not s.periodic:
            raise ValueError("Ewald needs a 3D periodic box")
        if abs(q.sum()) > 1e-9 * np.sum(np.abs(q)):
            raise ValueError("Ewald summation here requires a charge-neutral system")
        L = _bind()
        box = np.ascontiguousarray(s.box, dtype=np.float64)
        rcut = self.rcut or 0.5 * float(np.min(box))
        a = self.alpha or 4.0 / rcut
        kv, w, K = self._kvectors(box, a)
        n = s.n
        F = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        e3 = torch.zeros(3, dtype=torch.float64, device="cuda")
        ws = self._ws.get(L.acs_ewald_work_bytes(n, K))
        q_d = to_dev(q.astype(np.float64))   # held until the launch: a freed tensor's memory is handed out again
        _lib.check(L.acs_ewald_fp64(pos_d.data_ptr(), q_d.data_ptr(), n, box.ctypes.data,
                                    kv.data_ptr(), w.data_ptr(), K, float(a), float(rcut), float(self.k), F.data_ptr(),
                                    e3.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle()), "acs_ewald_fp64")
        e = e3.cpu().numpy()
        V = float(np.prod(box))
        U = self.k * (e[0] + 2 * np.pi / V * e[1] - a / np.sqrt(np.pi) * float(np.sum(q ** 2)))
        return F, U

    def compute(self, s):
        q = s.charges
        if s.dim != 3 or not s.periodic:
            raise ValueError("Ewald needs a 3D periodic box")
        if not np.any(q):
            return np.zeros_like(s.pos), 0.0
        if abs(q.sum()) > 1e-9 * np.sum(np.abs(q)):   # the reference's order: checked before any work
            raise ValueError("Ewald summation here requires a charge-neutral system")
        require_cuda()
        F, U = self.compute_device(s, to_dev(s.pos), q)
        return F.cpu().numpy(), float(U)
