"""Counter-based normal draws for the engine's Langevin thermostat (test infrastructure: the oracle).

Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw ("Parallel random numbers: as easy as 1, 2,
3", SC 2011): a 4 x 32-bit counter and a 2 x 32-bit key, ten rounds of two 32 x 32 -> 64-bit products
with the multipliers 0xD2511F53 and 0xCD9E8D57, the key bumped by the Weyl constants 0x9E3779B9 and
0xBB67AE85 between rounds. Standard normals come from the Box-Muller transform of u = (x + 1/2) 2^-32.
The engine (csrc/engine.cu) uses counter (O-step index lo, hi, atom id, replica) and key (seed lo, hi).
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr, key):
    """ctr: (..., 4) uint32, key: (2,) integers -> (..., 4) uint32."""
    c = [np.asarray(ctr, np.uint64)[..., q] for q in range(4)]
    k0, k1 = int(key[0]) & 0xFFFFFFFF, int(key[1]) & 0xFFFFFFFF
    for r in range(10):
        if r:
            k0, k1 = (k0 + W0) & 0xFFFFFFFF, (k1 + W1) & 0xFFFFFFFF
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c = [hi1 ^ c[1] ^ np.uint64(k0), lo1, hi0 ^ c[3] ^ np.uint64(k1), lo0]
    return np.stack(c, -1).astype(np.uint32)


def normals(step, ids, replica, seed):
    """(n, 3) standard normals for O-step `step` of atoms `ids` of `replica` (engine's draw)."""
    ids = np.asarray(ids, np.uint64)
    ctr = np.zeros(ids.shape + (4,), np.uint64)
    ctr[..., 0] = int(step) & 0xFFFFFFFF
    ctr[..., 1] = (int(step) >> 32) & 0xFFFFFFFF
    ctr[..., 2] = ids
    ctr[..., 3] = int(replica)
    x = philox4x32_10(ctr, (int(seed) & 0xFFFFFFFF, (int(seed) >> 32) & 0xFFFFFFFF)).astype(np.float64)
    u = (x + 0.5) * 2.0 ** -32
    r1 = np.sqrt(-2.0 * np.log(u[..., 0]))
    r2 = np.sqrt(-2.0 * np.log(u[..., 2]))
    t1, t2 = np.pi * (2.0 * u[..., 1]), np.pi * (2.0 * u[..., 3])
    return np.stack([r1 * np.cos(t1), r1 * np.sin(t1), r2 * np.cos(t2)], -1)
