"""Device plumbing: PyTorch owns device memory and streams; kernels come from libaccusim_b200.so."""
from __future__ import annotations

import numpy as np
import torch

from . import _lib


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("accusim_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
    _lib.lib()
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def to_dev(a, dtype=None) -> torch.Tensor:
    """Host array -> contiguous device tensor (one H2D copy)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to("cuda", non_blocking=False)


class Workspace:
    """Grow-only scratch buffer handed to the C ABI as (pointer, bytes)."""

    def __init__(self):
        self.buf = None

    def get(self, nbytes: int) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(nbytes + (nbytes >> 3), dtype=torch.uint8, device="cuda")
        return self.buf


class DevStatus:
    """The acs_dev_status block (8 int32 words) in device memory."""

    def __init__(self):
        self.t = torch.zeros(_lib.STATUS_WORDS, dtype=torch.int32, device="cuda")

    def clear(self):
        self.t.zero_()
        self.t[3] = -1

    def read(self) -> np.ndarray:
        return self.t.cpu().numpy()

    @property
    def ptr(self):
        return self.t.data_ptr()
