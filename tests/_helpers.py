"""Shared test helpers: turn a golden fixture into oracle or product state."""
import numpy as np

from oracle import accusim_port as port


def oracle_state(g, suffix=""):
    box = g["box" + suffix] if bool(g["has_box" + suffix]) else None
    species = [(str(n), float(m), float(q)) for n, m, q in
               zip(g["species" + suffix], g["masses" + suffix], g["charges" + suffix])]
    return port.State(g["pos" + suffix].copy(), g["vel" + suffix].copy(), g["sp" + suffix].astype(int),
                      g["ids" + suffix].astype(int), None if box is None else box.copy(),
                      bool(g["periodic" + suffix]), species)


def pair_keys(i, j, n):
    i = np.asarray(i, dtype=np.int64)
    j = np.asarray(j, dtype=np.int64)
    return np.sort(np.minimum(i, j) * n + np.maximum(i, j))


def rel_max(a, b):
    """max|a-b| / max|b|: the norm the reference's own skin tests use."""
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
