"""Precision form (config 3): the Fourier sums H(k) of the band stage and the band overlaps of
the BSE kernel as 3-term split-BF16 tensor-core GEMMs with FP32 accumulation; the per-k
diagonalisation, the q -> 0 cell average, the velocities and the BSE tridiagonalisation stay FP64.

Errors are taken against the FP64 form of the same deck, which the parity tests pin to the
oracle: band energies (all k, all nv + nc bands), the lowest 64 exciton energies, and eps2 at
its peaks relative to its maximum. The bars are the FP64-oracle bars of the fast form: 0.5 meV
on exciton energies and 1e-3 on eps2.

WTB_PREC_MESH sets the mesh of the error report on the config-2 model (default 24: N = 9216;
48 is config 3 itself, N = 36864).
"""
import json
import os

import numpy as np
import pytest

from oracle import wtb_oracle as O
from wantibexos_b200 import synth, wtbgpu

pytestmark = pytest.mark.gpu


def _f154(x):
    return np.array([float(f"{v:15.4f}") for v in np.ravel(x)]).reshape(np.shape(x))


def _peak_rel(ref, x):
    pk = np.where((ref[1:-1] > ref[:-2]) & (ref[1:-1] >= ref[2:]))[0] + 1
    if len(pk) == 0:
        pk = np.array([int(np.argmax(ref))])
    return float(np.abs(x[pk] - ref[pk]).max() / np.abs(ref).max())


def _run(ctx, m, n, nv, nc, r0, sme, prec):
    ctx.set_precision(prec)
    ctx.set_model(m)
    kpt = O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat)
    e, _, _, _ = ctx.bands(kpt, nv, nc, want_vectors=False)
    t_bands = ctx.last_ms
    ctx.velocity(sme, want=False)
    coul = wtbgpu.coulomb_params("V2DRK", [n, n, 1], 1e-3, [1.0] * 3, 1.0, 1.0, 0.0, r0)
    ctx.bse_build(coul)
    t_build = ctx.last_ms
    H = ctx.bse_get_matrix() if n * n * nv * nc <= 2304 else None
    W, act = ctx.bse_solve(False, False)
    vcell = abs(np.cross(m.rlat[0], m.rlat[1]) @ m.rlat[2])
    _, eps = ctx.spectrum(_f154(W), _f154(act[:, :6]), [n, n, 1], vcell, 0.0, 6.0, 2001.0, sme, True, 2.0)
    ctx.set_precision(0)
    return dict(e=e, W=W, eps2=eps[:, 1, 0].astype(np.float64), H=H, t_bands=t_bands, t_build=t_build)


def test_precision_form_small(gpu_ctx):
    """config-2 model on a 6x6 mesh (N = 576): matrix, bands and excitons close to FP64."""
    m = synth.config_model("c2")
    ref = _run(gpu_ctx, m, 6, 4, 4, 30.0, 0.03, 0)
    pre = _run(gpu_ctx, m, 6, 4, 4, 30.0, 0.03, 1)
    assert np.abs(pre["e"] - ref["e"]).max() < 2e-4
    assert np.abs(pre["H"] - ref["H"]).max() < 2e-4 * np.abs(ref["H"]).max()
    assert np.abs(pre["W"] - ref["W"]).max() < 5e-4
    assert not np.array_equal(pre["W"], ref["W"])   # the tensor-core path really ran


def test_precision_form_error_report():
    n = int(os.environ.get("WTB_PREC_MESH", "24"))
    m = synth.config_model("c2")
    ctx = wtbgpu.Context(0)
    try:
        ref = _run(ctx, m, n, 4, 4, 30.0, 0.03, 0)
        pre = _run(ctx, m, n, 4, 4, 30.0, 0.03, 1)
    finally:
        ctx.close()
    rep = {
        "mesh": n, "N": n * n * 16,
        "band_max_abs_err_eV": float(np.abs(pre["e"] - ref["e"]).max()),
        "exciton64_max_abs_err_meV": float(np.abs(pre["W"][:64] - ref["W"][:64]).max() * 1e3),
        "eps2_peak_rel_err": _peak_rel(ref["eps2"], pre["eps2"]),
        "eps2_max_rel_err": float(np.abs(pre["eps2"] - ref["eps2"]).max() / np.abs(ref["eps2"]).max()),
        "bands_ms": [ref["t_bands"], pre["t_bands"]], "build_ms": [ref["t_build"], pre["t_build"]],
    }
    print("precision form:", json.dumps(rep))
    assert rep["band_max_abs_err_eV"] < 2e-4
    assert rep["exciton64_max_abs_err_meV"] < 0.5
    assert rep["eps2_peak_rel_err"] < 1e-3
