"""The pair-kernel error floor used to assess the learned correction (CPU, FP64): on a synthetic residual
that is exactly pair-additive within R, the fit recovers it; a residual from beyond R is not recovered."""
import numpy as np

from devinproj_b200.learned import pair_kernel_bound


def _dataset(kernel, n=96, L=12e-10, snaps=6, seed=0):
    rng = np.random.default_rng(seed)
    sp = np.arange(n) % 2
    q = np.where(sp == 0, 1.0, -1.0)
    pos, res, dsf = [], [], []
    for _ in range(snaps):
        p = rng.uniform(0, L, (n, 3))
        d = p[None, :, :] - p[:, None, :]
        d -= L * np.round(d / L)
        r = np.linalg.norm(d, axis=-1)
        np.fill_diagonal(r, np.inf)
        f = (q[:, None] * q[None, :] * kernel(r) / r)[:, :, None] * d
        pos.append(p)
        res.append(f.sum(1))
        dsf.append(rng.normal(0, 1.0, (n, 3)) * np.sqrt(np.mean(np.sum(res[-1] ** 2, 1)) / 3))
    return dict(pos=np.array(pos), sp=sp, box=np.array([L, L, L]), residual=np.array(res), dsf=np.array(dsf),
                species=[("A", 1.0, 1.0), ("B", 1.0, -1.0)])


def test_pair_additive_residual_is_recovered():
    R = 5e-10
    kernel = lambda r: np.where(r < R, np.exp(-(r - 2.5e-10) ** 2 / (0.5e-10) ** 2), 0.0)  # noqa: E731
    d = _dataset(kernel)
    e0, e1 = pair_kernel_bound(d, range(4), range(4, 6), R, spacing=0.05e-10, device="cpu")
    assert e1 < 0.05 * e0


def test_residual_from_beyond_the_radius_is_not_recovered():
    kernel = lambda r: np.where((r > 4e-10) & (r < 5.5e-10), 1.0, 0.0)  # noqa: E731
    d = _dataset(kernel)
    e0, e1 = pair_kernel_bound(d, range(4), range(4, 6), 3e-10, spacing=0.1e-10, device="cpu")
    assert e1 > 0.5 * e0
