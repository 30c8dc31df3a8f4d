"""Ewald on the device against the reference's Ewald (golden vectors, Madelung known answer), and the
tcgen05 tensor-core primitive the learned correction is built on. Tolerances: Ewald force max|dF| <=
1e-10 max|F| and energy 1e-10 relative (FP64, different summation order); tensor-core product of
BF16-rounded inputs against an FP32 CUDA-core product: 1e-5 relative (FP32 accumulation order)."""
import numpy as np
import pytest

from tests._helpers import rel_max
from tests.test_dropin_gpu import product_system

pytestmark = pytest.mark.gpu


def test_ewald_matches_reference_in_orthorhombic_box(golden):
    from devinproj_b200.ewald import Ewald
    g = golden("coulomb_ortho")
    s = product_system(g)
    F, U = Ewald(k=1.0).compute(s)
    assert rel_max(F, g["F_ewald"]) <= 1e-10
    assert abs(U - g["U_ewald"]) <= 1e-10 * abs(g["U_ewald"])


def test_ewald_matches_reference_on_disordered_melt(golden):
    from devinproj_b200.ewald import Ewald
    g = golden("ewald_melt512")
    s = product_system(g)
    F, U = Ewald(k=1.0).compute(s)
    assert rel_max(F, g["F"]) <= 1e-10
    assert abs(U - g["U"]) <= 1e-10 * abs(g["U"])


@pytest.mark.parametrize("cells", [1, 2])
def test_ewald_madelung_known_answer(cells):
    """tests/test_forces.py:90-97: NaCl Madelung constant 1.747564594633, forces vanish on the lattice."""
    from accusim import System
    from devinproj_b200.ewald import Ewald
    s = System(3, box=2.0 * cells, periodic=True)
    s.add_species("Na", 1.0, charge=1.0)
    s.add_species("Cl", 1.0, charge=-1.0)
    for x in range(2 * cells):
        for y in range(2 * cells):
            for z in range(2 * cells):
                s.add("Na" if (x + y + z) % 2 == 0 else "Cl", [[x, y, z]])
    F, U = Ewald(k=1.0).compute(s)
    assert -U / (s.n / 2) == pytest.approx(1.747564594633, rel=1e-7)
    assert np.allclose(F, 0, atol=1e-6)


@pytest.mark.parametrize("N,K", [(64, 64), (64, 80), (128, 128), (16, 16), (32, 48)])
def test_tcgen05_gemm_primitive(N, K):
    import torch

    from devinproj_b200 import _lib
    from devinproj_b200.device import stream_handle
    from devinproj_b200.ewald import _bind
    L = _bind()
    g = torch.Generator().manual_seed(N * 1000 + K)
    A = torch.randn(128, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    Ad, Bd = A.cuda(), B.cuda()
    D = torch.full((128, N), float("nan"), dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(L.acs_umma_gemm_test(Ad.data_ptr(), Bd.data_ptr(), D.data_ptr(), N, K, st.data_ptr(), stream_handle()))
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ref = A.float() @ B.float().T
    got = D.cpu()
    assert torch.isfinite(got).all()
    assert (got - ref).abs().max().item() <= 1e-5 * ref.abs().max().item()


def _bf16(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).float().numpy().astype(np.float64)


def test_mlp_forward_and_gradients_match_fp64_oracle():
    """Tensor-core forward and backward against the FP64 NumPy oracle on the same BF16-rounded inputs and
    weights. Tolerance 3e-2 relative (BF16 activations between layers), loss 1e-2."""
    import torch

    from devinproj_b200.device import to_dev
    from devinproj_b200.learned import MLP
    from oracle import mlp_port
    rng = np.random.default_rng(3)
    n = 300                                   # three tiles, the last one partial
    X = rng.normal(size=(n, 80))
    X[:, 64:80] = 0.0
    sp = rng.integers(0, 2, n)
    X[np.arange(n), 64 + sp] = 1.0
    X[:, 79] = 1.0
    X = _bf16(X)
    V = rng.normal(size=(n, 64, 3)) * 0.3
    Y = rng.normal(size=(n, 3))
    mlp = MLP(seed=5)
    th = mlp.params().astype(np.float64).reshape(3, 64, 80)
    th[2][:, :64] *= 10.0                     # larger last layer so every gradient block is exercised
    th[1][:, 64] = rng.normal(size=64) * 0.1
    th[2][:, 64] = rng.normal(size=64) * 0.1
    mlp.set_params(th.reshape(-1))
    thq = th.copy()                           # the weights the tensor cores see (biases b2, b3 stay FP32)
    thq[0] = _bf16(th[0])
    thq[1][:, :64] = _bf16(th[1][:, :64])
    thq[2][:, :64] = _bf16(th[2][:, :64])
    Xd = to_dev(X.astype(np.float32)).to(torch.bfloat16)
    Vd = to_dev(V.astype(np.float32))
    Yd = to_dev(Y.astype(np.float32))
    L_ref, g_ref, F_ref = mlp_port.loss_and_grad(thq.reshape(-1), X, V.astype(np.float32).astype(np.float64),
                                                 Y.astype(np.float32).astype(np.float64))
    F = mlp.forward(Xd, Vd).cpu().numpy()
    assert np.sqrt(np.mean((F - F_ref) ** 2)) <= 2e-2 * np.sqrt(np.mean(F_ref ** 2))
    loss, g = mlp.gradient(Xd, Vd, Yd)
    mlp.check()
    assert loss == pytest.approx(L_ref, rel=1e-2)
    for layer in range(3):
        gl, rl = g.reshape(3, 64, 80)[layer], g_ref.reshape(3, 64, 80)[layer]
        assert np.linalg.norm(gl - rl) <= 3e-2 * np.linalg.norm(rl), layer


def test_descriptors_match_fp64_oracle():
    from devinproj_b200 import configs
    from devinproj_b200.engine import LEN
    from devinproj_b200.learned import DescriptorBuilder
    from oracle import mlp_port
    s, _ = configs.nacl_melt(8, seed=2)
    s.pos = (s.pos + np.random.default_rng(0).normal(0, 0.3e-10, s.pos.shape)) % s.box
    db = DescriptorBuilder()
    X, V = db.compute(s)
    p = db.p
    D_ref, V_ref = mlp_port.descriptors(s.pos / LEN, s.sp, s.box / LEN, p["rc"], p["r0"], p["dmu"], p["s"])
    V = V.cpu().numpy()
    assert np.max(np.abs(V - V_ref)) <= 1e-4 * np.max(np.abs(V_ref))
    X = X.float().cpu().numpy()
    X_ref = mlp_port.inputs(D_ref, s.sp, np.zeros(64), np.ones(64))
    assert np.max(np.abs(X - X_ref)) <= 1e-2 * np.max(np.abs(X_ref))
    assert np.all(X[:, 79] == 1.0) and np.all(X[np.arange(s.n), 64 + s.sp] == 1.0)


def test_engine_descriptors_match_fp64_oracle():
    """The descriptors the engine computes inside its step (FP32 images, shift-coded neighbour list) against
    the FP64 oracle on the same state; same tolerances as the stand-alone kernel."""
    from devinproj_b200 import GpuSimulation, configs
    from devinproj_b200.engine import LEN
    from devinproj_b200.learned import LearnedCorrection
    from oracle import mlp_port
    s, forces = configs.nacl_melt(8, rcut=10e-10, seed=3)
    s.pos = (s.pos + np.random.default_rng(1).normal(0, 0.3e-10, s.pos.shape)) % s.box
    lc = LearnedCorrection(seed=0)
    sim = GpuSimulation(s, forces, dt=1e-15, correction=lc, validate_every=0)
    X = sim.engine._cX[: s.n].float().cpu().numpy()
    V = sim.engine._cV[: s.n].cpu().numpy()
    p = lc.desc.p
    D_ref, V_ref = mlp_port.descriptors(s.pos / LEN, s.sp, s.box / LEN, p["rc"], p["r0"], p["dmu"], p["s"])
    assert np.max(np.abs(V - V_ref)) <= 1e-4 * np.max(np.abs(V_ref))
    X_ref = mlp_port.inputs(D_ref, s.sp, np.zeros(64), np.ones(64))
    assert np.max(np.abs(X - X_ref)) <= 1e-2 * np.max(np.abs(X_ref))
    assert np.all(X[:, 79] == 1.0) and np.all(X[np.arange(s.n), 64 + s.sp] == 1.0)


def test_learned_correction_beats_plain_dsf_on_held_out_melt():
    """Small-scale version of the learned DSF->Ewald correction: 512-ion melt, labels from the device Ewald
    (pinned to the reference above); the corrected forces must be closer to Ewald than plain DSF on
    snapshots not used in training, and validation keeps the correction switched on."""
    from devinproj_b200.learned import LearnedCorrection, generate_dataset
    d = generate_dataset(40, seed=1, n_sites=8, melt_steps=1500, equil_steps=500, interval=25)
    lc = LearnedCorrection(seed=0)
    hist = lc.train(d, np.arange(32), epochs=60, batch_tiles=4, lr=3e-3)
    assert hist[-1] < hist[0]
    e0, e1 = lc.errors(d, np.arange(32, 40))
    print(f"held-out RMS relative force error vs Ewald: DSF {e0:.4f}, DSF + learned {e1:.4f} ({e0 / e1:.2f}x)")
    assert e1 < 0.8 * e0
    s = lc._system(d, 39)
    _, _, on = lc.validate(s, d["dsf"][39], d["dsf"][39] + d["residual"][39])
    assert on


def test_engine_runs_learned_correction_inside_the_step_loop():
    """The correction evaluated inside the engine's graph equals the stand-alone prediction on the same state,
    the Ewald validation runs every `validate_every` steps, and a correction that makes forces worse is
    switched off (fallback to plain DSF)."""
    from devinproj_b200 import GpuSimulation, configs
    from devinproj_b200.engine import ACC
    from devinproj_b200.learned import LearnedCorrection, generate_dataset, rms_rel
    d = generate_dataset(12, seed=4, n_sites=8, melt_steps=800, equil_steps=200, interval=20)
    lc = LearnedCorrection(seed=1)
    lc.train(d, np.arange(10), epochs=30, batch_tiles=4, lr=3e-3)
    s, forces = configs.nacl_melt(8, T=1300.0, rcut=10e-10, seed=4)
    s.pos = d["pos"][11].copy()
    sim = GpuSimulation(s, forces, dt=1e-15, correction=lc, validate_every=50)
    plain = GpuSimulation(s.copy(), forces, dt=1e-15)
    F_corr = lc.predict(s)
    m = s.masses[:, None]
    assert rms_rel(sim.force - plain.force, F_corr) <= 2e-2
    sim.run(steps=120, record_every=10, positions=False)
    assert [v[0] for v in sim.validations] == [50, 100]
    assert len(sim.trajectory.t) == 13
    # an untrained network (large random output) is worse than plain DSF: validation turns it off
    bad = LearnedCorrection(seed=2)
    bad.desc = lc.desc
    bad.scale = 50.0 * lc.scale
    sim2 = GpuSimulation(s.copy(), forces, dt=1e-15, correction=bad, validate_every=20)
    sim2.run(steps=40, record_every=20, positions=False)
    assert sim2.validations[0][3] is False and sim2.correction is None
    assert np.all(np.isfinite(sim2.system.pos))
    del m, ACC
