"""Exciton vectors at scale: the config-2 model on a 24x24 mesh (N = 9216, two-stage reduction).
The tridiagonal eigenvectors come from inverse iteration with eigenvalues grouped into clusters
closer than 1e-7 ||T|| (re-orthogonalised inside a cluster), then go back through the bulge-chasing
and the panel reflectors.  Checked on the 32 lowest states and 32 states from the middle of the
spectrum: orthonormality max |A^H A - I| and the residual max |H A - A diag(W)| with H the rebuilt
BSE matrix applied in FP64, both bounded and printed."""
import numpy as np
import pytest

from oracle import wtb_oracle as O
from wantibexos_b200 import synth, wtbgpu

pytestmark = pytest.mark.gpu


def test_exciton_vectors_orthonormal_with_small_residual_n9216(gpu_ctx):
    m = synth.config_model("c2")
    n = 24
    kpts = O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat)
    c = wtbgpu.coulomb_params("V2DRK", [n, n, 1], 1e-3, [1, 1, 1], 1.0, 1.0, 0.0, 30.0)
    ctx = gpu_ctx
    ctx.set_reduction(0)
    ctx.set_model(m)
    ctx.bands(kpts, 4, 4, want_vectors=False)
    ctx.velocity(0.03, want=False)
    ctx.bse_build(c)
    W, _ = ctx.bse_solve(False, False)
    N = W.shape[0]
    assert N == 9216
    mid = N // 2
    A_lo = ctx.bse_eigvecs(1, 32)
    A_mid = ctx.bse_eigvecs(mid + 1, mid + 32)
    ctx.bse_build(c)          # the reduction overwrote the matrix
    ctx.set_fast_product(0)   # FP64 product
    hnorm = np.abs(W).max()
    for A, w in ((A_lo, W[:32]), (A_mid, W[mid:mid + 32])):
        G = A.conj().T @ A
        orth = np.abs(G - np.eye(32)).max()
        HA = ctx.bse_apply(A)
        res = np.abs(HA - A * w[None, :]).max() / hnorm
        print(f"N={N}: max|A^H A - I| = {orth:.2e}, max|H A - A W| / max|W| = {res:.2e}")
        assert orth < 1e-9
        assert res < 1e-11
