"""accusim's `Ewald` (accusim/forces.py:333-388) evaluated on the device.

Exact periodic electrostatics for a neutral 3-D periodic system: real-space erfc sum over minimum-image pairs
inside rcut, reciprocal sum over the k-vectors |n| <= kmax, self term, in FP64. The class subclasses accusim's:
the constructor, the defaults (rcut = L_min / 2, alpha = 4 / rcut, kmax = 12) and the k-vector set and weights
(`_kvectors`) are accusim's own; the real-space and reciprocal sums run as CUDA kernels.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._accusim import forces as _af
from .device import Workspace, require_cuda, stream_handle, to_dev

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


class Ewald(_af.Ewald):
    """Exact periodic electrostatics by Ewald summation (3D orthorhombic box, neutral system), on the GPU."""

    def _device_kvectors(self, box, alpha):
        """accusim's k-vectors and weights for this box and alpha, as device tensors (cached)."""
        kv, w = self._kvectors(box, alpha)
        key = (tuple(box), alpha, self.kmax)
        cached = getattr(self, "_dev_k", None)
        if cached is None or cached[0] != key:
            cached = (key, to_dev(np.ascontiguousarray(kv, dtype=np.float64)),
                      to_dev(np.ascontiguousarray(w, dtype=np.float64)), len(w))
            self._dev_k = cached
        return cached[1], cached[2], cached[3]

    def compute_device(self, s, pos_d, q):
        if s.dim != 3 or not s.periodic:
            raise ValueError("Ewald needs a 3D periodic box")
        if abs(q.sum()) > 1e-9 * np.sum(np.abs(q)):
            raise ValueError("Ewald summation here requires a charge-neutral system")
        L = _bind()
        box = np.ascontiguousarray(s.box, dtype=np.float64)
        rcut = self.rcut or 0.5 * float(np.min(box))
        a = self.alpha or 4.0 / rcut
        kv, w, K = self._device_kvectors(box, a)
        n = s.n
        F = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        e3 = torch.zeros(3, dtype=torch.float64, device="cuda")
        if getattr(self, "_ws", None) is None:
            self._ws = Workspace()
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
        F, U = self.compute_device(s, to_dev(np.asarray(s.pos, dtype=np.float64)), q)
        return F.cpu().numpy(), float(U)
