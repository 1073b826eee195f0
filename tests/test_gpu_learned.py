"""Learned warm start on the GPU: the hand-written forward/backward kernels against the CPU
oracle's gradient, and the trained network's gain over the cold-start block Davidson on
held-out sweep points (r0, eps_env), with the plain dense FP64 solve as the judge."""
import numpy as np
import pytest

from oracle import mlp_oracle as MO
from oracle import wtb_oracle as O
from wantibexos_b200 import synth, wtbgpu

pytestmark = pytest.mark.gpu


def test_gradients_match_cpu_oracle(gpu_ctx):
    net = wtbgpu.Net(gpu_ctx, seed=3)
    p = MO.init_params(5, scale_last=1.0)
    net.set_params(p)
    F, CAR, A = MO.random_problem(256, 2, 11)
    loss, g = net.loss_grad(F, CAR, A, nsamp=2)
    lref, gref = MO.loss_grad(p.astype(np.float64), F, CAR, A, 2, bf16=True)
    # bf16 operands with FP32 accumulation on the GPU vs float64 with the same roundings
    assert abs(loss - lref) <= 2e-3 * abs(lref)
    P = MO.unflatten(g)
    R = MO.unflatten(gref)
    errs = {name: float(np.linalg.norm(P[name] - R[name]) / np.linalg.norm(R[name]))
            for name in ("W1", "b1", "W2", "b2", "W3", "b3")}
    print("gradient relative errors", errs)
    assert max(errs.values()) < 2e-2, errs
    net.close()


def _setup(ctx, r0, eps, n=12):
    m = synth.config_model("c1")
    kpts = O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat)
    ctx.set_model(m)
    ctx.bands(kpts, 2, 2, want_vectors=False)
    ctx.velocity(0.05, want=False)
    c = wtbgpu.coulomb_params("V2DRK", [n, n, 1], 1e-3, [eps, eps, eps], 1.0, 1.0, 0.0, r0)
    ctx.bse_build(c)


def test_trained_network_beats_cold_start(gpu_ctx):
    rng = np.random.default_rng(2024)
    pts = np.column_stack([rng.uniform(10, 60, 40), rng.uniform(1, 5, 40)])
    train, held = pts[:32], pts[32:]
    net = wtbgpu.Net(gpu_ctx, seed=1)
    for r0, eps in train:
        _setup(gpu_ctx, r0, eps)
        gpu_ctx.bse_solve(False, False)
        A = gpu_ctx.bse_eigvecs(1, 32)
        _setup(gpu_ctx, r0, eps)
        net.add_sample(net.glob([0, 0, 0], r0, eps), A)
    for r0, eps in held:
        _setup(gpu_ctx, r0, eps)
        gpu_ctx.bse_solve(False, False)
        A = gpu_ctx.bse_eigvecs(1, 32)
        _setup(gpu_ctx, r0, eps)
        net.add_sample(net.glob([0, 0, 0], r0, eps), A)
    before = net.eval_loss(32, 8)
    hist = net.train(60, batch=8, lr=1e-3, first=0, count=32)
    after = net.eval_loss(32, 8)
    assert hist[-1] < hist[0]
    assert after < 0.7 * before
    cold, warm = [], []
    for r0, eps in held:
        _setup(gpu_ctx, r0, eps)
        W, _, _, it_c, _ = gpu_ctx.bse_davidson(32, nb=40, tol=1e-6, want_act=False)
        X0 = np.zeros((gpu_ctx.N, 40), dtype=np.complex128)
        X0[:, :32] = net.predict(net.glob([0, 0, 0], r0, eps))
        D = np.real(np.diag(gpu_ctx.bse_get_matrix()))
        for j, i in enumerate(np.argsort(D)[:8]):
            X0[i, 32 + j] = 1.0
        W2, _, _, it_w, _ = gpu_ctx.bse_davidson(32, nb=40, tol=1e-6, X0=X0, want_act=False)
        Wd, _ = gpu_ctx.bse_solve(False, False, want_act=False)
        assert np.abs(W - Wd[:32]).max() < 1e-6
        assert np.abs(W2 - Wd[:32]).max() < 1e-6
        cold.append(it_c)
        warm.append(it_w)
    print("davidson iterations cold", cold, "warm", warm)
    assert np.mean(warm) < np.mean(cold)
    net.close()


@pytest.mark.parametrize("M,N,K", [(128, 256, 32), (300, 512, 512), (512, 32, 512), (320, 512, 512),
                                   (1000, 160, 96), (64, 48, 1024)])
def test_tensor_core_gemm_matches_numpy(gpu_ctx, M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    Cg = gpu_ctx.gemm_bf16(A, B)
    ref = MO.bf16_round(A) @ MO.bf16_round(B).T
    assert np.abs(Cg - ref).max() <= 1e-4 * np.abs(ref).max() + 1e-3
