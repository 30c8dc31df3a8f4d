"""Learned DSF->Ewald force correction (no counterpart in the reference).

Damped shifted force electrostatics (accusim/forces.py:391-452) truncates the Coulomb sum at rc; exact
periodic electrostatics is Ewald (accusim/forces.py:333-388). This module learns the residual
F_Ewald - F_DSF per ion from its local environment and adds it to DSF:

* descriptors: for each ion, 32 Gaussian radial channels per neighbour species within 10 A -> 64
  invariant features D and 64 vector features V (sums of g_k(r) fc(r) r_hat);
* network: an MLP 80 -> 64 -> 64 -> 64 (SiLU) on the standardised invariants, BF16 weights, FP32
  accumulation, run by hand-written tcgen05 tensor-core kernels (forward and backward);
* prediction: F_i = scale * sum_c C_c(D_i) V_c(i), rotation-equivariant by construction;
* training: Adam on labels from the device Ewald (parity-checked against the reference's Ewald) minus
  FP64 DSF, on snapshots of a NaCl melt;
* validation: the corrected forces are checked against Ewald; if they are not better than plain DSF the
  correction is switched off (fallback to plain DSF).
"""
from __future__ import annotations

import math
import os

import numpy as np
import torch

from . import _lib
from .device import DevStatus, stream_handle, to_dev
from .engine import LEN
from .forces import DeviceNeighborList

P = _lib.P
_lib.SIGNATURES.update({
    "acs_descriptors": (_lib.C.c_int, [P, P, _lib.I64, P, _lib.C.c_int, P, P, _lib.I32, P, P, P, P, P, P]),
    "acs_mlp_grad_bytes": (_lib.SZ, [_lib.I64]),
    "acs_mlp_param_count": (_lib.I32, []),
    "acs_mlp_forward": (_lib.C.c_int, [P, P, _lib.I64, P, P, P, _lib.C.c_float, P, P, P]),
    "acs_mlp_train_step": (_lib.C.c_int, [P, P, P, _lib.I64, P, P, P, P, P, P, _lib.C.c_float, _lib.I32,
                                          _lib.C.c_float, P, _lib.SZ, P, P, P, P]),
})

N_IN, N_H, N_OUT, N_PARAM = 80, 64, 64, 3 * 64 * 80
RC_DESC = 10.0      # A
R0_DESC = 1.8       # A, first Gaussian centre
N_RBF = 32


def _bind():
    L = _lib.lib()
    for name in ("acs_descriptors", "acs_mlp_grad_bytes", "acs_mlp_param_count", "acs_mlp_forward",
                 "acs_mlp_train_step"):
        res, args = _lib.SIGNATURES[name]
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args
    return L


def rbf_params(rc=RC_DESC, r0=R0_DESC):
    dmu = (rc - r0) / (N_RBF - 1)
    s = dmu
    return dict(r0=r0, dmu=dmu, s=s, rc=rc)


class DescriptorBuilder:
    """Descriptors of a periodic two-species system on the device (engine length unit: A)."""

    def __init__(self, rc=RC_DESC, r0=R0_DESC):
        self.p = rbf_params(rc, r0)
        # host array: the C entry point reads these six numbers on the host
        self.params6 = np.ascontiguousarray([self.p["r0"], self.p["dmu"], 1.0 / (2 * self.p["s"] ** 2), self.p["rc"], 0, 0],
                                            dtype=np.float32)
        self.mean = torch.zeros(64, dtype=torch.float32, device="cuda")
        self.inv_std = torch.ones(64, dtype=torch.float32, device="cuda")
        self.nl = DeviceNeighborList()

    def set_stats(self, mean, std):
        self.mean = to_dev(np.asarray(mean, np.float32))
        self.inv_std = to_dev(1.0 / np.maximum(np.asarray(std, np.float32), 1e-6))

    def compute(self, s):
        """X (n x 80 BF16, standardised) and V (n x 64 x 3 FP32) for a system in SI (converted to A here)."""
        L = _bind()
        n = s.n
        view = _AView(s)
        pos_d = to_dev(view.pos)
        self.nl.build(view, pos_d, self.p["rc"])
        X = torch.empty((n, N_IN), dtype=torch.bfloat16, device="cuda")
        V = torch.empty((n, 64, 3), dtype=torch.float32, device="cuda")
        sp = to_dev(s.sp, torch.int32)
        box = np.ascontiguousarray(view.box, dtype=np.float64)
        _lib.check(L.acs_descriptors(pos_d.data_ptr(), sp.data_ptr(), n, box.ctypes.data, 1, self.nl.nbr.data_ptr(),
                                     self.nl.nnb.data_ptr(), self.nl.maxnb, self.params6.ctypes.data, self.mean.data_ptr(),
                                     self.inv_std.data_ptr(), X.data_ptr(), V.data_ptr(), stream_handle()),
                   "acs_descriptors")
        return X, V


class _AView:
    """A periodic system's geometry in A (what the neighbour list and descriptors work in)."""

    def __init__(self, s):
        self.pos = np.ascontiguousarray(s.pos / LEN)
        self.box = np.asarray(s.box) / LEN
        self.periodic = True
        self.n = s.n
        self.dim = 3
        self.ids = s.ids


class MLP:
    """Parameters (FP32 master + BF16 operand copies), Adam state and the tensor-core kernels."""

    def __init__(self, seed=0):
        L = _bind()
        assert L.acs_mlp_param_count() == N_PARAM
        rng = np.random.default_rng(seed)
        th = np.zeros((3, 64, 80), np.float32)
        th[0][:, :66] = rng.normal(0, 1 / math.sqrt(66), (64, 66))
        th[1][:, :64] = rng.normal(0, 1 / math.sqrt(64), (64, 64))
        th[2][:, :64] = rng.normal(0, 0.1 / math.sqrt(64), (64, 64))
        self.set_params(th.reshape(-1))
        self.step = 0
        self.status = DevStatus()
        self._gpart = None
        self._loss = None

    def set_params(self, theta):
        th = np.asarray(theta, np.float32).reshape(3, 64, 80)
        self.theta = to_dev(th.reshape(-1).copy())
        self.m = torch.zeros(N_PARAM, dtype=torch.float32, device="cuda")
        self.v = torch.zeros(N_PARAM, dtype=torch.float32, device="cuda")
        bf = lambda a: to_dev(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16)  # noqa: E731
        self.W1 = bf(th[0])
        self.W2 = bf(th[1][:, :64])
        self.W3 = bf(th[2][:, :64])
        self.W2T = bf(th[1][:, :64].T)
        self.W3T = bf(th[2][:, :64].T)
        self.b2 = to_dev(np.ascontiguousarray(th[1][:, 64], np.float32))
        self.b3 = to_dev(np.ascontiguousarray(th[2][:, 64], np.float32))
        self._w5 = (_lib.C.c_void_p * 5)(*[w.data_ptr() for w in (self.W1, self.W2, self.W3, self.W2T, self.W3T)])

    def params(self):
        return self.theta.cpu().numpy()

    def forward(self, X, V, out_scale=1.0, out=None):
        L = _bind()
        n = X.shape[0]
        F = out if out is not None else torch.empty((n, 3), dtype=torch.float32, device="cuda")
        _lib.check(L.acs_mlp_forward(X.data_ptr(), V.data_ptr(), n, self._w5, self.b2.data_ptr(), self.b3.data_ptr(),
                                     float(out_scale), F.data_ptr(), self.status.ptr, stream_handle()), "acs_mlp_forward")
        return F

    def _bufs(self, n):
        L = _bind()
        need = L.acs_mlp_grad_bytes(n)
        if self._gpart is None or self._gpart.numel() * 4 < need:
            self._gpart = torch.empty(need // 4 + 64, dtype=torch.float32, device="cuda")
            self._loss = torch.empty((n + 127) // 128 * 4 + 4, dtype=torch.float32, device="cuda")
        return need

    def train_step(self, X, V, Y, lr, weight_decay=0.0, grad_out=None):
        """One Adam step on the batch; returns the batch loss as a device scalar."""
        L = _bind()
        n = X.shape[0]
        need = self._bufs(n)
        self.step += 1
        _lib.check(L.acs_mlp_train_step(X.data_ptr(), V.data_ptr(), Y.data_ptr(), n, self._w5, self.b2.data_ptr(),
                                        self.b3.data_ptr(), self.theta.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                                        float(lr), self.step, float(weight_decay), self._gpart.data_ptr(), need,
                                        self._loss.data_ptr(), grad_out.data_ptr() if grad_out is not None else None,
                                        self.status.ptr, stream_handle()), "acs_mlp_train_step")
        return self._loss[: (n + 127) // 128 * 4].sum()

    def gradient(self, X, V, Y):
        """(loss, gradient) of the batch without changing the parameters (lr = 0)."""
        g = torch.empty(N_PARAM, dtype=torch.float32, device="cuda")
        step0 = self.step
        m0, v0 = self.m.clone(), self.v.clone()
        loss = self.train_step(X, V, Y, 0.0, grad_out=g)
        self.step = step0
        self.m, self.v = m0, v0
        return float(loss.item()), g.cpu().numpy()

    def check(self):
        st = self.status.read()
        if st[0] & _lib.FLAG_TIMEOUT:
            raise _lib.AcsError(_lib.ACS_ERR_TIMEOUT, "tensor-core MLP")


def force_units():
    """SI force -> engine force unit (kJ/mol/A)."""
    from .engine import ENERGY
    return LEN / ENERGY


def rms_rel(F, Fref):
    F = np.asarray(F, float)
    Fref = np.asarray(Fref, float)
    return float(np.sqrt(np.mean(np.sum((F - Fref) ** 2, 1)) / np.mean(np.sum(Fref ** 2, 1))))


def generate_dataset(n_snapshots, seed=0, n_sites=20, T=1300.0, melt_T=4000.0, melt_steps=2000, equil_steps=2000,
                     interval=20, rcut=10e-10, alpha=0.2e10, verbose=False):
    """Snapshots of a NaCl melt (LJ + DSF, FP32-compensated engine) with labels F_Ewald - F_DSF (SI, FP64,
    device Ewald with the reference's default parameters). As the reference's molten-salt example does
    (examples/molten_salt.py:38-44): Langevin melting at `melt_T`, Langevin cooling to T (friction 5/ps),
    then NVE sampling every `interval` steps. Returns a dict of host arrays."""
    from . import configs
    from .engine import GpuSimulation
    from .ewald import Ewald
    from .integrators import Langevin
    s, forces = configs.nacl_melt(n_sites, T=melt_T, rcut=rcut, alpha=alpha, seed=seed)
    dt = 1e-15
    for temp, steps in ((melt_T, melt_steps), (T, equil_steps)):
        GpuSimulation(s, forces, integrator=Langevin(temp, 5e12), dt=dt, seed=seed).run(
            steps=steps, record_every=steps, positions=False)
    sim = GpuSimulation(s, forces, dt=dt)
    ew = Ewald(k=forces[1].k)
    dsf = forces[1]
    pos, sp, res, fd = [], [], [], []
    for k in range(n_snapshots):
        sim.run(steps=interval, record_every=interval, positions=False)
        Fe, _ = ew.compute(s)
        Fd, _ = dsf.compute(s)
        pos.append(s.pos.copy())
        res.append(Fe - Fd)
        fd.append(Fd)
        if verbose and k % 100 == 0:
            print(f"snapshot {k}: T = {s.temperature():.0f} K, DSF vs Ewald RMS rel err {rms_rel(Fd, Fe):.3f}",
                  flush=True)
    return dict(pos=np.array(pos), sp=s.sp.copy(), box=s.box.copy(), residual=np.array(res), dsf=np.array(fd),
                species=[(x.name, x.mass, x.charge) for x in s.species], T=T)


def pair_kernel_bound(data, train_idx, test_idx, R, spacing=0.25e-10, device="cuda", chunk=512):
    """How far any correction built from pair terms within R can go: fit the residual F_Ewald - F_DSF as
    sum_{j: r_ij < R} q_i q_j h_t(r_ij) r_hat_ij, with one free radial function h_t per species pair
    (piecewise linear on a `spacing` grid), by least squares over the train snapshots. Every pair-additive
    electrostatic correction of range R, DSF's own kernel included, is one such function, so the fitted
    error is a floor for them; the learned network sees the same 10 A neighbourhood through its descriptors.
    Returns (mean RMS relative error of plain DSF, of the fitted correction) against Ewald on test
    snapshots. Analysis only (torch FP64), not part of the step path."""
    f64 = torch.float64
    box = torch.as_tensor(np.asarray(data["box"], float), dtype=f64, device=device)
    sp = torch.as_tensor(np.asarray(data["sp"]), dtype=torch.long, device=device)
    qs = np.array([c for (_, _, c) in data["species"]], float)
    q = torch.as_tensor(qs / np.max(np.abs(qs)), dtype=f64, device=device)[sp]
    nb = int(math.ceil(R / spacing)) + 1
    nf = 3 * nb

    def feats(k):
        pos = torch.as_tensor(data["pos"][k], dtype=f64, device=device)
        n = pos.shape[0]
        phi = torch.zeros((n, nf, 3), dtype=f64, device=device)
        for i0 in range(0, n, chunk):
            d = pos[None, :, :] - pos[i0:i0 + chunk, None, :]
            d -= box * torch.round(d / box)
            r = torch.linalg.norm(d, dim=-1)
            ii, jj = torch.nonzero((r < R) & (r > 0), as_tuple=True)
            rr = r[ii, jj]
            vec = (q[i0 + ii] * q[jj] / rr)[:, None] * d[ii, jj]
            x = rr / spacing
            b0 = torch.floor(x)
            w1 = (x - b0)[:, None]
            col = (sp[i0 + ii] + sp[jj]) * nb + b0.long()
            rows = i0 + ii
            phi.index_put_((rows, col), (1.0 - w1) * vec, accumulate=True)
            phi.index_put_((rows, col + 1), w1 * vec, accumulate=True)
        return phi

    G = torch.zeros((nf, nf), dtype=f64, device=device)
    h = torch.zeros(nf, dtype=f64, device=device)
    for k in train_idx:
        phi = feats(k)
        y = torch.as_tensor(data["residual"][k], dtype=f64, device=device)
        A = phi.permute(0, 2, 1).reshape(-1, nf)
        G += A.T @ A
        h += A.T @ y.reshape(-1)
    ridge = 1e-9 * torch.trace(G) / nf
    w = torch.linalg.solve(G + ridge * torch.eye(nf, dtype=f64, device=device), h)
    e0, e1 = [], []
    for k in test_idx:
        pred = torch.einsum("nfc,f->nc", feats(k), w).cpu().numpy()
        Fe = data["dsf"][k] + data["residual"][k]
        e0.append(rms_rel(data["dsf"][k], Fe))
        e1.append(rms_rel(data["dsf"][k] + pred, Fe))
    return float(np.mean(e0)), float(np.mean(e1))


class LearnedCorrection:
    """DSF + learned residual: fit on a dataset, predict corrections, check against Ewald."""

    def __init__(self, seed=0):
        self.desc = DescriptorBuilder()
        self.mlp = MLP(seed)
        self.scale = 1.0          # engine force units per network output unit
        self.enabled = True

    def _system(self, data, k):
        from ._accusim import system as _asys
        s = _asys.System(3, box=data["box"], periodic=True)
        for name, m, q in data["species"]:
            s.add_species(name, m, charge=q)
        s.pos = data["pos"][k]
        s.vel = np.zeros_like(s.pos)
        s.sp = data["sp"]
        s.ids = np.arange(len(s.sp))
        s.eint = np.zeros(len(s.sp))
        return s

    def featurize(self, data, idx):
        """Device tensors X, V, Y (Y = residual / scale, engine units) for snapshots idx."""
        Xs, Vs, Ys = [], [], []
        fu = force_units()
        for k in idx:
            X, V = self.desc.compute(self._system(data, k))
            Xs.append(X)
            Vs.append(V)
            Ys.append(to_dev((data["residual"][k] * fu / self.scale).astype(np.float32)))
        return torch.cat(Xs), torch.cat(Vs), torch.cat(Ys)

    def fit_stats(self, data, idx):
        """Feature standardisation and output scale from a few snapshots."""
        self.desc.set_stats(np.zeros(64), np.ones(64))
        feats = []
        for k in idx:
            X, _ = self.desc.compute(self._system(data, k))
            feats.append(X[:, :64].float().cpu().numpy())
        f = np.concatenate(feats)
        self.desc.set_stats(f.mean(0), f.std(0))
        fu = force_units()
        self.scale = float(np.sqrt(np.mean(np.sum((data["residual"][idx] * fu) ** 2, -1))))

    def train(self, data, train_idx, epochs=20, batch_tiles=64, lr=2e-3, weight_decay=0.0, seed=0, verbose=False):
        self.fit_stats(data, train_idx[: min(len(train_idx), 8)])
        X, V, Y = self.featurize(data, train_idx)
        n = X.shape[0]
        bs = batch_tiles * 128
        g = torch.Generator(device="cuda").manual_seed(seed)
        history = []
        nsteps = epochs * max(1, n // bs)
        k = 0
        for ep in range(epochs):
            perm = torch.randperm(n, device="cuda", generator=g)
            tot = torch.zeros((), dtype=torch.float32, device="cuda")
            nb = 0
            for b0 in range(0, n - bs + 1, bs):
                sel = perm[b0:b0 + bs]
                lr_k = lr * 0.5 * (1 + math.cos(math.pi * k / max(nsteps, 1)))
                tot += self.mlp.train_step(X[sel], V[sel], Y[sel], lr_k, weight_decay)
                nb += 1
                k += 1
            history.append(float((tot / max(nb, 1)).item()))
            if verbose:
                print(f"epoch {ep}: train loss {history[-1]:.4f}", flush=True)
        self.mlp.check()
        return history

    def predict(self, s):
        """Correction forces (SI, n x 3) for a system."""
        X, V = self.desc.compute(s)
        F = self.mlp.forward(X, V, out_scale=self.scale)
        return F.cpu().numpy().astype(np.float64) / force_units()

    def errors(self, data, idx):
        """(plain DSF, corrected) RMS relative force error against Ewald over snapshots idx."""
        e0, e1 = [], []
        for k in idx:
            s = self._system(data, k)
            Fe = data["dsf"][k] + data["residual"][k]
            Fd = data["dsf"][k]
            Fc = Fd + self.predict(s)
            e0.append(rms_rel(Fd, Fe))
            e1.append(rms_rel(Fc, Fe))
        return float(np.mean(e0)), float(np.mean(e1))

    def validate(self, s, dsf_force, ewald_force):
        """Check the corrected forces on one state against Ewald; switch the correction off (fallback to plain
        DSF) unless it improves on DSF by more than 0.1 % relative. Returns (err_dsf, err_corrected, enabled)."""
        e0 = rms_rel(dsf_force, ewald_force)
        e1 = rms_rel(dsf_force + self.predict(s), ewald_force)
        self.enabled = e1 < (1.0 - 1e-3) * e0
        return e0, e1, self.enabled

    def save(self, path):
        np.savez(path, theta=self.mlp.params(), mean=self.desc.mean.cpu().numpy(),
                 inv_std=self.desc.inv_std.cpu().numpy(), scale=self.scale)

    def load(self, path):
        z = np.load(path)
        self.mlp.set_params(z["theta"])
        self.desc.mean = to_dev(z["mean"])
        self.desc.inv_std = to_dev(z["inv_std"])
        self.scale = float(z["scale"])
        return self


if __name__ == "__main__":   # pragma: no cover - manual training run
    import argparse
    ap = argparse.ArgumentParser(description="train the learned DSF->Ewald correction on an 8000-ion NaCl melt")
    ap.add_argument("--snapshots", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--out", default="learned_dsf.npz")
    a = ap.parse_args()
    d = generate_dataset(a.snapshots, verbose=True)
    n_train = int(0.9 * a.snapshots)
    lc = LearnedCorrection()
    lc.train(d, np.arange(n_train), epochs=a.epochs, verbose=True)
    print("held-out errors (DSF, corrected):", lc.errors(d, np.arange(n_train, a.snapshots)))
    lc.save(a.out)
