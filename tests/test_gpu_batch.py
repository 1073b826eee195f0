"""Ragged batch (config 4): the k-mesh bands of four models with w = 8, 16, 24, 40 in one
persistent launch give exactly what separate launches give."""
import time

import numpy as np
import pytest

from oracle import wtb_oracle as O
from wantibexos_b200 import synth, wtbgpu

pytestmark = pytest.mark.gpu

NAMES = ["c4_w8", "c4_w16", "c4_w24", "c4_w40"]


def _setup(meshes):
    models = [synth.config_model(n) for n in NAMES]
    kpts = [O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat) for n, m in zip(meshes, models)]
    nvs = [2, 2, 3, 4]
    return models, kpts, nvs, nvs


def test_bands_batch_equals_single_launches():
    models, kpts, nvs, ncs = _setup([12, 10, 8, 6])
    ctxs = [wtbgpu.Context(0) for _ in models]
    for c, m in zip(ctxs, models):
        c.set_model(m)
    gaps = wtbgpu.bands_batch(ctxs, kpts, nvs, ncs)
    hb = [c.velocity(0.05) for c in ctxs]
    for c, m, k, nv, nc, g, h in zip(ctxs, models, kpts, nvs, ncs, gaps, hb):
        ref = wtbgpu.Context(0)
        ref.set_model(m)
        e, _, _, gap = ref.bands(k, nv, nc, want_vectors=False)
        assert gap == g
        assert np.array_equal(ref.velocity(0.05), h)
        ref.close()
        c.close()


def test_bands_batch_config4_meshes_timing():
    """Config-4 sizes: meshes 60^2, 48^2, 36^2, 24^2 (7776 k-points) in one launch."""
    models, kpts, nvs, ncs = _setup([60, 48, 36, 24])
    ctxs = [wtbgpu.Context(0) for _ in models]
    for c, m in zip(ctxs, models):
        c.set_model(m)
    wtbgpu.bands_batch(ctxs, kpts, nvs, ncs)
    t0 = time.perf_counter()
    wtbgpu.bands_batch(ctxs, kpts, nvs, ncs)
    tb = ctxs[0].last_ms
    ts = 0.0
    for c, k, nv, nc in zip(ctxs, kpts, nvs, ncs):
        c.bands(k, nv, nc, want_vectors=False)
        ts += c.last_ms
    print(f"config-4 bands: one persistent launch {tb:.2f} ms, four launches {ts:.2f} ms")
    assert tb < 1.5 * ts
    for c in ctxs:
        c.close()
