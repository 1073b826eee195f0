"""ctypes binding of libwtbgpu.so (the C-ABI declared in include/wtbgpu.h).

This is the Python view of the same entry points a Fortran ISO_C_BINDING interface binds;
tests and the benchmark drive the library through it.  There is no fallback: if the
shared library is missing or no CUDA device is present, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwtbgpu.so")

COULOMB_TYPES = {"V2DK": 1, "V3D": 2, "V3DL": 3, "V2DT": 4, "V2DT2": 5, "V2DOH": 6,
                 "V2DRK": 7, "V1DT": 8, "V0DT": 9}

# every entry point of include/wtbgpu.h
EXPORTS = ["wtbg_create", "wtbg_destroy", "wtbg_error_string", "wtbg_last_error",
           "wtbg_last_device_ms", "wtbg_set_model", "wtbg_bands", "wtbg_velocity",
           "wtbg_sp_table", "wtbg_bse_build", "wtbg_bse_get_matrix", "wtbg_bse_solve",
           "wtbg_bse_eigvecs", "wtbg_spectrum", "wtbg_bse_q_eigenvalues", "wtbg_set_profiling",
           "wtbg_get_stats", "wtbg_reset_stats", "wtbg_spectrum_noalloc", "wtbg_bse_davidson",
           "wtbg_bse_spectrum_fast", "wtbg_set_fast_product", "wtbg_bse_apply", "wtbg_net_create",
           "wtbg_net_destroy", "wtbg_net_num_params", "wtbg_net_get_params", "wtbg_net_set_params",
           "wtbg_net_features", "wtbg_net_add_sample", "wtbg_net_num_samples", "wtbg_net_train",
           "wtbg_net_eval_loss", "wtbg_net_predict", "wtbg_net_loss_grad", "wtbg_gemm_bf16",
           "wtbg_bse_build_q", "wtbg_set_temperature", "wtbg_eigsys", "wtbg_dos",
           "wtbg_bands_batch", "wtbg_bse_q_batch", "wtbg_set_precision", "wtbg_berry", "wtbg_sp_optbz",
           "wtbg_bse_lowest", "wtbg_set_reduction"]


class WtbgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"wtbg status {status}: {message}")
        self.status = status


class Stats(C.Structure):
    _fields_ = [("launches", C.c_longlong), ("hemv_launches", C.c_longlong), ("hemv_ms", C.c_double),
                ("hemv_bytes", C.c_double), ("build_launches", C.c_longlong), ("build_ms", C.c_double),
                ("build_bytes", C.c_double), ("fast_launches", C.c_longlong), ("fast_ms", C.c_double),
                ("fast_bytes", C.c_double), ("dav_fast_iters", C.c_longlong), ("dav_fp64_iters", C.c_longlong),
                ("her2k_launches", C.c_longlong), ("her2k_ms", C.c_double), ("her2k_flops", C.c_double),
                ("tri_ms", C.c_double), ("tdsolve_ms", C.c_double), ("dav_fallbacks", C.c_longlong),
                ("stage1_ms", C.c_double), ("stage2_ms", C.c_double), ("panel_ms", C.c_double),
                ("hemm_ms", C.c_double), ("hemm_flops", C.c_double)]


class Coulomb(C.Structure):
    _fields_ = [("coultype", C.c_int), ("ngrid", C.c_int * 3), ("ktol", C.c_double),
                ("ediel", C.c_double * 3), ("lc", C.c_double), ("ez", C.c_double),
                ("w", C.c_double), ("r0", C.c_double)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libwtbgpu.so and declare the signatures (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built (run python -m wantibexos_b200.build)")
    lib = C.CDLL(path)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    fp = C.POINTER(C.c_float)
    sig = {
        "wtbg_create": (C.c_int, [C.POINTER(P), C.c_int]),
        "wtbg_destroy": (C.c_int, [P]),
        "wtbg_error_string": (C.c_char_p, [C.c_int]),
        "wtbg_last_error": (C.c_char_p, [P]),
        "wtbg_last_device_ms": (C.c_double, [P]),
        "wtbg_set_model": (C.c_int, [P, C.c_int, C.c_int, dp, dp, ip, ip, dp, C.c_double, C.c_double]),
        "wtbg_bands": (C.c_int, [P, C.c_int, dp, C.c_int, C.c_int, dp, dp, ip, dp]),
        "wtbg_velocity": (C.c_int, [P, C.c_double, dp]),
        "wtbg_sp_table": (C.c_int, [P, fp]),
        "wtbg_bse_build": (C.c_int, [P, C.POINTER(Coulomb)]),
        "wtbg_bse_get_matrix": (C.c_int, [P, dp]),
        "wtbg_bse_solve": (C.c_int, [P, C.c_int, C.c_int, dp, dp]),
        "wtbg_bse_eigvecs": (C.c_int, [P, C.c_int, C.c_int, dp]),
        "wtbg_spectrum": (C.c_int, [P, C.c_int, C.c_int, dp, dp, ip, ip, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_int, C.c_double, dp, fp]),
        "wtbg_bse_q_eigenvalues": (C.c_int, [P, C.c_int, dp, dp, C.POINTER(Coulomb), dp]),
        "wtbg_bse_q_batch": (C.c_int, [P, C.c_int, C.c_int, dp, dp, C.POINTER(Coulomb), C.c_int, dp, dp]),
        "wtbg_set_profiling": (C.c_int, [P, C.c_int]),
        "wtbg_get_stats": (C.c_int, [P, C.POINTER(Stats)]),
        "wtbg_reset_stats": (C.c_int, [P]),
        "wtbg_bse_davidson": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, dp, C.c_int, C.c_int,
                                        dp, dp, dp, ip, dp]),
        "wtbg_set_reduction": (C.c_int, [P, C.c_int]),
        "wtbg_bse_lowest": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_double, dp, C.c_int, C.c_int, dp, dp, dp,
                                      ip, dp, ip]),
        "wtbg_bse_spectrum_fast": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, ip, C.c_double,
                                             C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                             dp, fp]),
        "wtbg_set_fast_product": (C.c_int, [P, C.c_int]),
        "wtbg_set_precision": (C.c_int, [P, C.c_int]),
        "wtbg_berry": (C.c_int, [P, C.c_int, dp, C.c_double, C.c_double, dp]),
        "wtbg_sp_optbz": (C.c_int, [P, C.c_int, dp, C.c_int, C.c_int, C.c_double, dp]),
        "wtbg_net_create": (C.c_int, [P, C.POINTER(P), C.c_ulonglong]),
        "wtbg_net_destroy": (C.c_int, [P]),
        "wtbg_net_num_params": (C.c_longlong, []),
        "wtbg_net_get_params": (C.c_int, [P, fp]),
        "wtbg_net_set_params": (C.c_int, [P, fp]),
        "wtbg_net_features": (C.c_int, [P, dp, fp, fp]),
        "wtbg_net_add_sample": (C.c_int, [P, dp, dp]),
        "wtbg_net_num_samples": (C.c_int, [P]),
        "wtbg_net_train": (C.c_int, [P, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, fp]),
        "wtbg_net_eval_loss": (C.c_int, [P, C.c_int, C.c_int, fp]),
        "wtbg_net_predict": (C.c_int, [P, dp, dp]),
        "wtbg_net_loss_grad": (C.c_int, [P, C.c_int, C.c_longlong, fp, fp, fp, fp, fp]),
        "wtbg_bse_apply": (C.c_int, [P, C.c_int, dp, dp]),
        "wtbg_set_temperature": (C.c_int, [P, C.c_int, C.c_double]),
        "wtbg_eigsys": (C.c_int, [P, C.c_int, dp, dp, dp, ip]),
        "wtbg_bands_batch": (C.c_int, [C.POINTER(P), C.c_int, ip, C.POINTER(dp), ip, ip, dp]),
        "wtbg_dos": (C.c_int, [P, C.c_longlong, dp, dp, C.c_int, C.c_longlong, C.c_int, dp, C.c_double, dp]),
        "wtbg_bse_build_q": (C.c_int, [P, C.c_int, dp, dp, C.POINTER(Coulomb)]),
        "wtbg_gemm_bf16": (C.c_int, [P, C.c_int, C.c_int, C.c_int, fp, fp, fp]),
        "wtbg_spectrum_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, ip, ip, C.c_double,
                                            C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                            C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p,
                                            C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _f64(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def coulomb_params(coultype: str, ngrid, ktol, ediel, lc, ez, w, r0) -> Coulomb:
    t = coultype.strip()
    if t not in COULOMB_TYPES:
        raise ValueError("Wrong Coulomb Potential")
    c = Coulomb()
    c.coultype = COULOMB_TYPES[t]
    for i in range(3):
        c.ngrid[i] = int(ngrid[i])
        c.ediel[i] = float(ediel[i])
    c.ktol, c.lc, c.ez, c.w, c.r0 = float(ktol), float(lc), float(ez), float(w), float(r0)
    return c


class Context:
    """One device context (wtbg_create/wtbg_destroy)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self.h = C.c_void_p()
        st = self.lib.wtbg_create(C.byref(self.h), device)
        if st != 0:
            raise WtbgError(st, self.lib.wtbg_error_string(st).decode())
        self.N = 0
        self.nk = 0

    def close(self):
        if self.h:
            self.lib.wtbg_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int):
        if st != 0:
            msg = self.lib.wtbg_last_error(self.h).decode()
            raise WtbgError(st, f"{self.lib.wtbg_error_string(st).decode()}: {msg}")

    @property
    def last_ms(self) -> float:
        return float(self.lib.wtbg_last_device_ms(self.h))

    def set_profiling(self, on: bool) -> None:
        self._check(self.lib.wtbg_set_profiling(self.h, int(bool(on))))

    def stats(self) -> dict:
        s = Stats()
        self._check(self.lib.wtbg_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def reset_stats(self) -> None:
        self._check(self.lib.wtbg_reset_stats(self.h))

    # ---------------------------------------------------------------- stages
    def set_model(self, model) -> None:
        # (nvec, w, w) arrays in Fortran order = hopmatrices(iR, m, n)
        hre = np.asfortranarray(model.hre)
        him = np.asfortranarray(model.him)
        rvec = np.asfortranarray(model.rvec.astype(np.int32))
        deg = np.ascontiguousarray(model.deg.astype(np.int32))
        rlat = _f64(model.rlat)
        self.w = model.w
        self._check(self.lib.wtbg_set_model(self.h, model.w, model.nvec, _dp(hre), _dp(him), _ip(rvec),
                                            _ip(deg), _dp(rlat), float(model.efermi), float(model.scs)))

    def bands(self, kpt: np.ndarray, nv: int, nc: int, want_vectors: bool = True):
        kpt = _f64(kpt)
        nk = kpt.shape[0]
        nb = nv + nc
        eigv = np.zeros((nk, nb), order="F")
        vec = np.zeros((nk, nb, self.w), dtype=np.complex128, order="F") if want_vectors else None
        nocp = np.zeros(nk, dtype=np.int32)
        gap = np.zeros(1)
        vp = vec.ctypes.data_as(C.POINTER(C.c_double)) if vec is not None else None
        self._check(self.lib.wtbg_bands(self.h, nk, _dp(kpt), nv, nc, _dp(eigv), vp, _ip(nocp), _dp(gap)))
        self.nk, self.nv, self.nc = nk, nv, nc
        self.N = nk * nc * nv
        return eigv, vec, nocp, float(gap[0])

    def velocity(self, sme: float, want: bool = True):
        h = np.zeros((self.N, 5), dtype=np.complex128, order="F") if want else None
        hp = h.ctypes.data_as(C.POINTER(C.c_double)) if h is not None else None
        self._check(self.lib.wtbg_velocity(self.h, float(sme), hp))
        return h

    def sp_table(self):
        out = np.zeros((self.N, 15), dtype=np.float32, order="F")
        self._check(self.lib.wtbg_sp_table(self.h, _fp(out)))
        return out

    def bse_build(self, coul: Coulomb) -> None:
        self._check(self.lib.wtbg_bse_build(self.h, C.byref(coul)))

    def bse_get_matrix(self):
        H = np.zeros((self.N, self.N), dtype=np.complex128, order="F")
        self._check(self.lib.wtbg_bse_get_matrix(self.h, H.ctypes.data_as(C.POINTER(C.c_double))))
        return H

    def bse_solve(self, dtfull: bool = False, cpol: bool = False, want_act: bool = True):
        W = np.zeros(self.N)
        act = np.zeros((self.N, 8), order="F") if want_act else None
        self._check(self.lib.wtbg_bse_solve(self.h, int(dtfull), int(cpol), _dp(W), _dp(act)))
        return W, act

    def bse_davidson(self, nev: int, nb: int = 40, largest: bool = False, max_iter: int = 200, tol: float = 1e-6,
                     X0=None, dtfull: bool = False, cpol: bool = False, want_act: bool = True,
                     want_vectors: bool = False, check: bool = True):
        """Block Davidson for the nev lowest (or highest) states; returns (W, act, X, iters, maxres)."""
        W = np.zeros(nev)
        act = np.zeros((nev, 8), order="F") if want_act else None
        X = np.zeros((self.N, nev), dtype=np.complex128, order="F") if want_vectors else None
        x0 = None
        if X0 is not None:
            x0 = np.asfortranarray(np.asarray(X0, dtype=np.complex128))
        it = C.c_int(0)
        mr = C.c_double(0.0)
        st = self.lib.wtbg_bse_davidson(self.h, nev, nb, int(bool(largest)), max_iter, float(tol),
                                        x0.ctypes.data_as(C.POINTER(C.c_double)) if x0 is not None else None,
                                        int(dtfull), int(cpol), _dp(W), _dp(act),
                                        X.ctypes.data_as(C.POINTER(C.c_double)) if X is not None else None,
                                        C.byref(it), C.byref(mr))
        if check or st not in (0, -4):
            self._check(st)
        return W, act, X, it.value, mr.value

    def set_reduction(self, mode: int) -> None:
        """0 automatic, 1 one-stage, 2 two-stage reduction for the dense solves."""
        self._check(self.lib.wtbg_set_reduction(self.h, int(mode)))

    def bse_lowest(self, nev: int, nb: int = 40, max_iter: int = 200, tol: float = 1e-6, X0=None,
                   dtfull: bool = False, cpol: bool = False, want_act: bool = True, want_vectors: bool = False):
        """The nev lowest excitons by block Davidson with the dense FP64 solve as fallback; returns
        (W, act, X, iters, maxres, used_dense)."""
        W = np.zeros(nev)
        act = np.zeros((nev, 8), order="F") if want_act else None
        X = np.zeros((self.N, nev), dtype=np.complex128, order="F") if want_vectors else None
        x0 = None
        if X0 is not None:
            x0 = np.asfortranarray(np.asarray(X0, dtype=np.complex128))
        it = C.c_int(0)
        mr = C.c_double(0.0)
        used = C.c_int(0)
        self._check(self.lib.wtbg_bse_lowest(self.h, nev, nb, max_iter, float(tol),
                                             x0.ctypes.data_as(C.POINTER(C.c_double)) if x0 is not None else None,
                                             int(dtfull), int(cpol), _dp(W), _dp(act),
                                             X.ctypes.data_as(C.POINTER(C.c_double)) if X is not None else None,
                                             C.byref(it), C.byref(mr), C.byref(used)))
        return W, act, X, it.value, mr.value, bool(used.value)

    def bse_spectrum_fast(self, nsteps, e1, emax, ngrid, vcell3d, ebse0, ebsef, numbse, sme, renorm, spinf,
                          dtfull=False, cpol=False):
        """Haydock spectrum; returns (omega (nw,), eps (nw, 2, 8) float32)."""
        nw = int(numbse)
        ng = np.array(ngrid, dtype=np.int32)
        om = np.zeros(nw)
        eps = np.zeros((nw, 2, 8), dtype=np.float32, order="F")
        self._check(self.lib.wtbg_bse_spectrum_fast(self.h, int(nsteps), int(dtfull), int(cpol), float(e1), float(emax),
                                                    _ip(ng), float(vcell3d), float(ebse0), float(ebsef),
                                                    float(numbse), float(sme), int(bool(renorm)), float(spinf),
                                                    _dp(om), _fp(eps)))
        return om, eps

    def eigsys(self, kpt, want_vectors: bool = True):
        """Every band at every k: (eig (nk, w), vec (nk, w, w) or None, nocp (nk,))."""
        k = _f64(kpt)
        nk = k.shape[0]
        e = np.zeros((nk, self.w), order="F")
        v = np.zeros((nk, self.w, self.w), dtype=np.complex128, order="F") if want_vectors else None
        no = np.zeros(nk, dtype=np.int32)
        self._check(self.lib.wtbg_eigsys(self.h, nk, _dp(k), _dp(e),
                                         v.ctypes.data_as(C.POINTER(C.c_double)) if v is not None else None, _ip(no)))
        return e, v, no

    def dos(self, etb, weights, nkpt, en, sme):
        """endos over the energy grid en for each weight column: (nw, ncol)."""
        etb = _f64(etb)
        w = _f64(np.asarray(weights).reshape(etb.shape[0], -1))
        en = _f64(en)
        out = np.zeros((en.shape[0], w.shape[1]), order="F")
        self._check(self.lib.wtbg_dos(self.h, etb.shape[0], _dp(etb), _dp(w), w.shape[1], int(nkpt), en.shape[0],
                                      _dp(en), float(sme), _dp(out)))
        return out

    def set_temperature(self, on: bool, temp: float = 0.0) -> None:
        """Temperature BSE (occupation factors f_v - f_c) for the later stages."""
        self._check(self.lib.wtbg_set_temperature(self.h, int(bool(on)), float(temp)))

    def set_fast_product(self, mode: int) -> None:
        """0: FP64 product; 1: split-BF16 tensor-core product (Davidson, Haydock, bse_apply)."""
        self._check(self.lib.wtbg_set_fast_product(self.h, int(mode)))

    def bse_apply(self, X):
        """Y = H X with the selected product; X (N, m) complex."""
        X = np.asfortranarray(np.asarray(X, dtype=np.complex128).reshape(self.N, -1))
        Y = np.zeros_like(X, order="F")
        self._check(self.lib.wtbg_bse_apply(self.h, X.shape[1], X.ctypes.data_as(C.POINTER(C.c_double)),
                                            Y.ctypes.data_as(C.POINTER(C.c_double))))
        return Y

    def gemm_bf16(self, A, B):
        """C = A B^T on the tensor cores (bf16 inputs, FP32 accumulation)."""
        A = np.ascontiguousarray(A, dtype=np.float32)
        B = np.ascontiguousarray(B, dtype=np.float32)
        M, K = A.shape
        N = B.shape[0]
        Cm = np.zeros((M, N), dtype=np.float32)
        self._check(self.lib.wtbg_gemm_bf16(self.h, M, N, K, _fp(A), _fp(B), _fp(Cm)))
        return Cm

    def bse_eigvecs(self, n0: int, n1: int):
        A = np.zeros((self.N, n1 - n0 + 1), dtype=np.complex128, order="F")
        self._check(self.lib.wtbg_bse_eigvecs(self.h, n0, n1, A.ctypes.data_as(C.POINTER(C.c_double))))
        return A

    def spectrum(self, E, F, ngrid, vcell3d, ebse0, ebsef, numbse, sme, renorm, spinf, rtype=None):
        """optdiel over the photon grid for every column of F (n, ncomp); returns
        (omega (nw,), eps (nw, 2, ncomp) float32)."""
        E = _f64(E)
        F = _f64(F)
        n, ncomp = F.shape
        if rtype is None:
            rtype = [1, 1, 1, 0, 0, 0][:ncomp] if ncomp == 6 else [1] * ncomp
        rt = np.array(rtype, dtype=np.int32)
        nw = int(numbse)
        ng = np.array(ngrid, dtype=np.int32)
        om = np.zeros(nw)
        eps = np.zeros((nw, 2, ncomp), dtype=np.float32, order="F")
        self._check(self.lib.wtbg_spectrum(self.h, n, ncomp, _dp(E), _dp(F), _ip(rt), _ip(ng), float(vcell3d),
                                           float(ebse0), float(ebsef), float(numbse), float(sme),
                                           int(bool(renorm)), float(spinf), _dp(om), _fp(eps)))
        return om, eps

    def berry(self, kpt, gamma=float(np.float32(0.001)), degtol=float(np.float32(0.0001))):
        """Berry curvature (berryct2) at each k: (nk, 6) = Im of b_xx, b_xy, b_xz, b_yy, b_yz, b_zz."""
        k = _f64(kpt)
        out = np.zeros((k.shape[0], 6), order="F")
        self._check(self.lib.wtbg_berry(self.h, k.shape[0], _dp(k), float(gamma), float(degtol), _dp(out)))
        return out

    def sp_optbz(self, kpt, nv, nc, sme):
        """spoptpolbz sums per k: (nk, 5) = x, y, z, sigma+, sigma-."""
        k = _f64(kpt)
        out = np.zeros((k.shape[0], 5), order="F")
        self._check(self.lib.wtbg_sp_optbz(self.h, k.shape[0], _dp(k), int(nv), int(nc), float(sme), _dp(out)))
        return out

    def set_precision(self, mode: int) -> None:
        """0: FP64 form; 1: precision form (Fourier sums and band overlaps as 3-term split-BF16
        tensor-core GEMMs, FP32 accumulation). Discards the context's bands and matrix."""
        self._check(self.lib.wtbg_set_precision(self.h, int(mode)))

    def bse_build_q(self, kptq, q4, coul: Coulomb) -> None:
        kq = _f64(kptq)
        q = np.ascontiguousarray(np.asarray(q4, dtype=np.float64))
        self._check(self.lib.wtbg_bse_build_q(self.h, kq.shape[0], _dp(kq), _dp(q), C.byref(coul)))

    def bse_q_eigenvalues(self, kptq, q4, coul: Coulomb):
        kq = _f64(kptq)
        q = np.ascontiguousarray(np.asarray(q4, dtype=np.float64))
        W = np.zeros(self.N)
        self._check(self.lib.wtbg_bse_q_eigenvalues(self.h, kq.shape[0], _dp(kq), _dp(q), C.byref(coul), _dp(W)))
        return W

    def bse_q_batch(self, kptqs, q4s, coul: Coulomb, graph: bool = True):
        """Eigenvalues of the Q kernel for every Q of a path in one call: kptqs is a list of
        (nk,3) k+Q meshes, q4s (nq,4). Returns (W (nq,N), per-Q device ms)."""
        blocks = [_f64(k) for k in kptqs]
        nq = len(blocks)
        nk = blocks[0].shape[0] if nq else self.nk
        kq = np.ascontiguousarray(np.concatenate([b.ravel(order="F") for b in blocks])) if nq else np.zeros(3)
        q = np.ascontiguousarray(np.asarray(q4s, dtype=np.float64).reshape(nq, 4))
        W = np.zeros((nq, self.N))
        ms = np.zeros(nq)
        self._check(self.lib.wtbg_bse_q_batch(self.h, nk, nq, _dp(kq), _dp(q), C.byref(coul), int(graph),
                                              _dp(W), _dp(ms)))
        return W, ms


def bands_batch(ctxs, kpts, nvs, ncs):
    """One persistent launch for the k-mesh bands of several contexts (models); returns the
    direct gap of each. Afterwards each context is as after its own Context.bands call."""
    P, dp = C.c_void_p, C.POINTER(C.c_double)
    n = len(ctxs)
    arr = (P * n)(*[c.h for c in ctxs])
    ks = [_f64(k) for k in kpts]
    kp = (dp * n)(*[_dp(k) for k in ks])
    nk = np.array([k.shape[0] for k in ks], dtype=np.int32)
    nv = np.array(nvs, dtype=np.int32)
    nc = np.array(ncs, dtype=np.int32)
    gap = np.zeros(n)
    lib = ctxs[0].lib
    ctxs[0]._check(lib.wtbg_bands_batch(arr, n, _ip(nk), kp, _ip(nv), _ip(nc), _dp(gap)))
    for c, k, a, b in zip(ctxs, ks, nvs, ncs):
        c.nk, c.nv, c.nc = k.shape[0], a, b
        c.N = k.shape[0] * a * b
    return gap


class Net:
    """Learned warm start (wtbg_net_*), bound to a Context's device and stream."""

    NS = 32
    NF = 32
    NCAR = 5

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        self.h = C.c_void_p()
        ctx._check(self.lib.wtbg_net_create(ctx.h, C.byref(self.h), C.c_ulonglong(seed)))
        self.nparam = int(self.lib.wtbg_net_num_params())

    def close(self):
        if self.h:
            self.lib.wtbg_net_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def glob(q, r0, eps):
        return np.array([q[0], q[1], q[2], r0, eps], dtype=np.float64)

    def params(self) -> np.ndarray:
        p = np.zeros(self.nparam, dtype=np.float32)
        self.ctx._check(self.lib.wtbg_net_get_params(self.h, _fp(p)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(np.asarray(p, dtype=np.float32))
        assert p.size == self.nparam
        self.ctx._check(self.lib.wtbg_net_set_params(self.h, _fp(p)))

    def features(self, glob):
        N = self.ctx.N
        F = np.zeros((N, self.NF), dtype=np.float32)
        CAR = np.zeros((self.NCAR, N), dtype=np.complex64)
        self.ctx._check(self.lib.wtbg_net_features(self.h, _dp(np.asarray(glob, dtype=np.float64)), _fp(F),
                                                   CAR.ctypes.data_as(C.POINTER(C.c_float))))
        return F, CAR

    def add_sample(self, glob, A) -> None:
        A = np.asfortranarray(np.asarray(A, dtype=np.complex128)[:, :self.NS])
        assert A.shape == (self.ctx.N, self.NS)
        self.ctx._check(self.lib.wtbg_net_add_sample(self.h, _dp(np.asarray(glob, dtype=np.float64)),
                                                     A.ctypes.data_as(C.POINTER(C.c_double))))

    @property
    def num_samples(self) -> int:
        return int(self.lib.wtbg_net_num_samples(self.h))

    def train(self, epochs: int, batch: int = 8, lr: float = 1e-3, first: int = 0, count: int = 0):
        hist = np.zeros(epochs, dtype=np.float32)
        self.ctx._check(self.lib.wtbg_net_train(self.h, epochs, batch, float(lr), first, count, _fp(hist)))
        return hist

    def eval_loss(self, first: int, count: int) -> float:
        v = np.zeros(1, dtype=np.float32)
        self.ctx._check(self.lib.wtbg_net_eval_loss(self.h, first, count, _fp(v)))
        return float(v[0])

    def predict(self, glob):
        X = np.zeros((self.ctx.N, self.NS), dtype=np.complex128, order="F")
        self.ctx._check(self.lib.wtbg_net_predict(self.h, _dp(np.asarray(glob, dtype=np.float64)),
                                                  X.ctypes.data_as(C.POINTER(C.c_double))))
        return X

    def loss_grad(self, F, CAR, A, nsamp: int):
        """F (M, 32) float32, CAR (5, M) complex64, A (32, M) complex64 with M = nsamp * rows."""
        F = np.ascontiguousarray(F, dtype=np.float32)
        CAR = np.ascontiguousarray(CAR, dtype=np.complex64)
        A = np.ascontiguousarray(A, dtype=np.complex64)
        M = F.shape[0]
        loss = np.zeros(1, dtype=np.float32)
        g = np.zeros(self.nparam, dtype=np.float32)
        self.ctx._check(self.lib.wtbg_net_loss_grad(self.h, nsamp, M // nsamp, _fp(F),
                                                    CAR.ctypes.data_as(C.POINTER(C.c_float)),
                                                    A.ctypes.data_as(C.POINTER(C.c_float)), _fp(loss), _fp(g)))
        return float(loss[0]), g
