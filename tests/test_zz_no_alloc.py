"""The allocation-free spectrum entry point against the regular one.

wtbg_spectrum_noalloc serves hosts that own all device memory themselves (their own pool
or a fixed arena) or must not call cudaMalloc during a run, because that call can
synchronise the device and fail with out-of-memory part-way through.  It takes device
pointers the caller owns and keeps its scratch in a fixed static device array.  This file
is collected last so that a failure here never hides the other tests; it passes both alone
in a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

from wantibexos_b200 import wtbgpu

pytestmark = pytest.mark.gpu


def inputs(seed, n, ncomp):
    rng = np.random.default_rng(seed)
    E = np.sort(rng.uniform(0.4, 5.5, n))
    F = rng.uniform(0.0, 2.0, (n, ncomp))
    if ncomp == 6:
        F[:, 3:] -= 1.0   # off-diagonal components can be negative
    return E, F


def call_noalloc(lib, E, F, rtype, ngrid, vc, e0, e1, nw, sme, renorm, spinf):
    import torch
    n, ncomp = F.shape
    dE = torch.tensor(E, dtype=torch.float64, device="cuda")
    dF = torch.tensor(np.asfortranarray(F).T.reshape(-1), dtype=torch.float64, device="cuda")  # (n,ncomp) col-major
    dom = torch.empty(nw, dtype=torch.float64, device="cuda")
    deps = torch.empty(nw * 2 * ncomp, dtype=torch.float32, device="cuda")
    rt = np.array(rtype, dtype=np.int32)
    ng = np.array(ngrid, dtype=np.int32)
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.wtbg_spectrum_noalloc(n, ncomp, dE.data_ptr(), dF.data_ptr(), rt.ctypes.data_as(C.POINTER(C.c_int)),
                                   ng.ctypes.data_as(C.POINTER(C.c_int)), vc, e0, e1, float(nw), sme, int(renorm),
                                   spinf, dom.data_ptr(), deps.data_ptr(), C.c_void_p(stream), err, 256)
    torch.cuda.synchronize()
    assert st == 0, err.value
    eps = deps.cpu().numpy().reshape(ncomp, 2, nw).transpose(2, 1, 0)   # -> (nw, 2, ncomp)
    return dom.cpu().numpy(), eps


@pytest.mark.parametrize("ncomp,rtype", [(6, [1, 1, 1, 0, 0, 0]), (5, [1, 1, 1, 1, 1])])
def test_noalloc_matches_regular_entry_twice(ncomp, rtype):
    lib = wtbgpu.load_library()
    ctx = wtbgpu.Context(0)
    ngrid, vc = [12, 12, 1], 567.2
    for call, seed in enumerate((11, 12)):   # two calls in a row share the static scratch
        n = 700 + 37 * call
        E, F = inputs(seed + ncomp, n, ncomp)
        om_ref, eps_ref = ctx.spectrum(E, F, ngrid, vc, 0.0, 6.0, 1501.0, 0.03, True, 2.0, rtype=rtype)
        om, eps = call_noalloc(lib, E, F, rtype, ngrid, vc, 0.0, 6.0, 1501, 0.03, True, 2.0)
        assert np.array_equal(om, om_ref)
        tol = 4 * np.spacing(np.float32(np.abs(eps_ref).max()))
        assert np.abs(eps.astype(np.float64) - eps_ref.astype(np.float64)).max() <= tol
    ctx.close()


def test_noalloc_at_the_scratch_limit():
    """NESPEC = 8192 with 8 components fills the fixed scratch to its end (eta sits last)."""
    lib = wtbgpu.load_library()
    ctx = wtbgpu.Context(0)
    rtype = [1, 1, 1, 0, 0, 0, 1, 1]
    for call, seed in enumerate((21, 22)):
        n = 40 + 3 * call
        E, F = inputs(seed, n, 8)
        F[:, 3:6] -= 1.0
        om_ref, eps_ref = ctx.spectrum(E, F, [6, 6, 1], 321.5, 0.0, 6.0, 8192.0, 0.05, True, 1.0, rtype=rtype)
        om, eps = call_noalloc(lib, E, F, rtype, [6, 6, 1], 321.5, 0.0, 6.0, 8192, 0.05, True, 1.0)
        assert np.array_equal(om, om_ref)
        tol = 4 * np.spacing(np.float32(np.abs(eps_ref).max()))
        assert np.abs(eps.astype(np.float64) - eps_ref.astype(np.float64)).max() <= tol
    ctx.close()


def test_noalloc_rejects_oversize():
    import torch
    lib = wtbgpu.load_library()
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    err = C.create_string_buffer(256)
    rt = np.ones(9, dtype=np.int32)
    ng = np.array([2, 2, 1], dtype=np.int32)
    st = lib.wtbg_spectrum_noalloc(4, 6, d.data_ptr(), d.data_ptr(), rt.ctypes.data_as(C.POINTER(C.c_int)),
                                   ng.ctypes.data_as(C.POINTER(C.c_int)), 1.0, 0.0, 1.0, 9000.0, 0.1, 1, 1.0,
                                   d.data_ptr(), d.data_ptr(), None, err, 256)
    assert st == -8 and b"8192" in err.value
    for nw, ncomp in ((8193.0, 8), (8192.0, 9)):
        st = lib.wtbg_spectrum_noalloc(4, ncomp, d.data_ptr(), d.data_ptr(), rt.ctypes.data_as(C.POINTER(C.c_int)),
                                       ng.ctypes.data_as(C.POINTER(C.c_int)), 1.0, 0.0, 1.0, nw, 0.1, 1, 1.0,
                                       d.data_ptr(), d.data_ptr(), None, err, 256)
        assert st == -8
