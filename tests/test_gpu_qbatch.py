"""Exciton band structure in one call (the Q loop of bsebnds, bse_kpath-tool.f90:246-435):
every Q of a path through wtbg_bse_q_batch.  Below N = 2048 the one-stage tridiagonalisation of
each Q is replayed from one captured CUDA graph (autotuned mat-vec chunk); from N = 2048 the Q
points run in groups, each Q's build and dense -> band stage leaving its band in a slot and one
persistent bulge-chasing launch reducing the whole group's bands.

Parity: the batch gives exactly what one wtbg_bse_q_eigenvalues call per Q gives (same kernels,
same launch parameters; graph replay or grouped bands), the two-stage group agrees with the
one-stage reduction to 1e-9 eV, and the Q eigenvalues agree with the oracle's dense eigvalsh of
its own Q kernel to 1e-9 eV.  The config-4 size (64 Q, N = 8100) is timed.
"""
import time

import numpy as np
import pytest

from oracle import wtb_oracle as O
from wantibexos_b200 import synth, wtbgpu

pytestmark = pytest.mark.gpu


def _qpath(rlat, npts):
    """Gamma-M-K-Gamma, junction points kept once."""
    nodes = [(0, 0, 0), (0.5, 0, 0), (0.5, 0, 0), (1 / 3, 1 / 3, 0), (1 / 3, 1 / 3, 0), (0, 0, 0)]
    q, _ = O.kpathbse(rlat, nodes, npts)
    keep = [r for r in range(q.shape[0]) if not (r > 0 and r % npts == 0)]
    return q[keep]


def _coul(n, r0, eps):
    return wtbgpu.coulomb_params("V2DRK", [n, n, 1], 1e-3, [eps] * 3, 1.0, 1.0, 0.0, r0)


def test_q_batch_matches_oracle_and_single_calls(gpu_ctx):
    m = synth.config_model("c1")
    n, nv, nc = 6, 2, 2
    kpts = O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat)
    energy, vector, _, _ = O.bands(m, kpts, nv, nc)
    qs = _qpath(m.rlat, 4)[[0, 2, 5, 8]]
    p = O.CoulombParams("V2DRK", 1e-3, [2.5] * 3, 1.0, 1.0, 0.0, 35.0, [n, n, 1], m.rlat)
    kqs = [O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat, q=q[1:]) for q in qs]
    gpu_ctx.set_model(m)
    gpu_ctx.bands(kpts, nv, nc)
    W, ms = gpu_ctx.bse_q_batch(kqs, qs, _coul(n, 35.0, 2.5))
    assert W.shape == (len(qs), n * n * nv * nc) and (ms > 0).all()
    for iq, (q, kq) in enumerate(zip(qs, kqs)):
        eq, vq, _, _ = O.bands(m, kq, nv, nc)
        H = O.bse_matrix_q(p, q, kpts, energy, vector, eq, vq, nv, nc)
        assert np.abs(W[iq] - np.linalg.eigvalsh(H, UPLO="U")).max() < 1e-9, iq
        assert np.array_equal(W[iq], gpu_ctx.bse_q_eigenvalues(kq, q, _coul(n, 35.0, 2.5))), iq


def test_q_batch_graph_equals_eager():
    """N = 1296 (above the autotuner's floor): graph replay and eager launches agree bit for
    bit, and both count the same launches."""
    m = synth.config_model("c4_w16")
    n, nv, nc = 12, 3, 3
    kpts = O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat)
    qs = _qpath(m.rlat, 4)[[1, 3, 4, 6]]
    kqs = [O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat, q=q[1:]) for q in qs]
    res = {}
    for graph in (False, True):
        ctx = wtbgpu.Context(0)
        ctx.set_model(m)
        ctx.bands(kpts, nv, nc)
        ctx.bse_q_batch(kqs[:1], qs[:1], _coul(n, 35.0, 2.5), graph=graph)   # autotune + sizing
        ctx.reset_stats()
        W, _ = ctx.bse_q_batch(kqs, qs, _coul(n, 35.0, 2.5), graph=graph)
        res[graph] = (W, ctx.stats()["launches"])
        ctx.close()
    assert np.array_equal(res[False][0], res[True][0])
    assert res[False][1] == res[True][1]


def test_q_batch_two_stage_group_equals_single_and_one_stage():
    """The two-stage Q group (stage 1 per Q, one bulge-chasing launch for all bands) equals one
    wtbg_bse_q_eigenvalues call per Q bit for bit and the one-stage reduction to 1e-9 eV."""
    m = synth.config_model("c4_w16")
    n, nv, nc = 12, 3, 3
    kpts = O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat)
    qs = _qpath(m.rlat, 4)[[0, 1, 3, 4, 6]]
    kqs = [O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat, q=q[1:]) for q in qs]
    c = _coul(n, 35.0, 2.5)
    ctx = wtbgpu.Context(0)
    ctx.set_model(m)
    ctx.bands(kpts, nv, nc)
    ctx.set_reduction(2)
    W2, ms = ctx.bse_q_batch(kqs, qs, c, graph=False)
    single = [ctx.bse_q_eigenvalues(kq, q, c) for q, kq in zip(qs, kqs)]
    ctx.set_reduction(1)
    W1, _ = ctx.bse_q_batch(kqs, qs, c, graph=False)
    ctx.close()
    assert (ms > 0).all()
    for iq in range(len(qs)):
        assert np.array_equal(W2[iq], single[iq]), iq
    assert np.abs(W2 - W1).max() < 1e-9


def test_q_batch_config4_timing():
    """Config 4 exciton bands: w=16 material, 30x30 mesh, nv=nc=3 (N = 8100), 64 Q on
    Gamma-M-K-Gamma, V2DRK r0=35, eps_env=2.5: all 64 Q in one call (two-stage reduction, the 64
    bands chased in one launch), against one call per Q for the first points."""
    m = synth.config_model("c4_w16")
    n, nv, nc = 30, 3, 3
    kpts = O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat)
    qs = _qpath(m.rlat, 22)
    assert qs.shape[0] == 64
    kqs = [O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat, q=q[1:]) for q in qs]
    c = _coul(n, 35.0, 2.5)
    ctx = wtbgpu.Context(0)
    ctx.set_model(m)
    ctx.bands(kpts, nv, nc)
    ctx.bse_q_batch(kqs[:1], qs[:1], c, graph=False)   # sizing, module loading
    t0 = time.perf_counter()
    W, ms = ctx.bse_q_batch(kqs, qs, c, graph=True)
    wall = time.perf_counter() - t0
    single = [ctx.bse_q_eigenvalues(kqs[i], qs[i], c) for i in (0, 31, 63)]
    for j, i in enumerate((0, 31, 63)):
        assert np.array_equal(W[i], single[j]), i
    assert np.all(np.diff(W, axis=1) >= 0)
    print(f"config-4 Q batch: 64 Q x N=8100 in {wall:.2f} s wall, {ms.sum() / 1e3:.2f} s device, "
          f"{ms.sum() / 64:.1f} ms per Q; lowest exciton {W[:, 0].min():.4f}..{W[:, 0].max():.4f} eV")
    ctx.close()
