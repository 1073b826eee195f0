"""CPU oracle: a numpy/scipy restatement of the WanTiBEXOS BSE exciton + optics path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import this module; the product (libwtbgpu.so and its
drivers) never calls it.

Parity status: **parity unpinned**.  The reference is Fortran 90 (ifort + MKL) and no
Fortran compiler is available, and the reference ships no tests, golden outputs or
known-answer vectors for this path.  This restatement follows the reference line by line
(file:line cited per function), reproduces its single-precision literals and its file
round trips, and uses LAPACK ZHEEV from scipy's bundled OpenBLAS with the reference's
minimum workspace LWORK = 2N-1 in place of MKL's ZHEEV.  Its self-checks (analytic
cases, scipy cross-checks, gauge invariances) are in ``tests/``.

Float32 traps reproduced (all from the reference source):
  * ``cmplx(0.0, x)`` without KIND rounds the phase k.R and R_alpha to float32
    (hamiltonian_tb.f90:64-66, optics.f90:39-47) and the broadening in optsp (optics.f90:139).
  * ``pi = acos(-1.)`` is float32 (mhkpack_subs.f90:413 and elsewhere).
  * ``fermimt(i,i) = cmplx(-efermi,0.0)`` rounds E_F to float32 (hamiltonian_tb.f90:383).
  * ``cic = -(0.0904756)*10**(3)`` is a float32 literal (coulomb_pot.f90:6,...).
  * ``gama = 180.90`` (optics.f90:188), ``hc = 19.746E-06`` (diel-pp-subs.f90:54),
    ``1.0/sqrt(2.)`` (bse_solver-tool-diel.f90:376), ``factor = 0.15`` (optics.f90:335),
    ``alpha1 = 1.76`` (coulomb_pot.f90:8) are float32.
  * optsp assigns ``1./esp`` to a REAL, so the velocity is scaled by Re(1/(dE + i eta))
    (optics.f90:114,148).
"""
from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np
import scipy.linalg.lapack as lapack
import scipy.special as sps

F32 = np.float32


def f32(x):
    """Round a double (or array) to float32 and back, as a real(4) temporary does."""
    return np.asarray(x, dtype=np.float64).astype(np.float32).astype(np.float64) \
        if isinstance(x, np.ndarray) else float(np.float32(x))


PI_F32 = float(np.float32(np.arccos(np.float32(-1.0))))
CIC = float(np.float32(-(np.float32(0.0904756) * np.float32(1000))))
GAMA = float(np.float32(180.90))
HC = float(np.float32(19.746e-6))
SQRT2_F32 = float(np.sqrt(np.float32(2.0)))
INV_SQRT2_F32 = float(np.float32(1.0) / np.sqrt(np.float32(2.0)))
RENORM_FACTOR = float(np.float32(0.15))
ALPHA1_V2DK = float(np.float32(1.76))
CFE = float(np.float32(7.297e-3))
LSPD = float(np.float32(299.792e16))
HBAR = float(np.float32(6.582e-16))


# ----------------------------------------------------------------------------- lattice

def prodvec(v1, v2):
    """general_subs.f90 prodvec: cross product v1 x v2."""
    return np.array([v1[1] * v2[2] - v1[2] * v2[1],
                     v1[2] * v2[0] - v1[0] * v2[2],
                     v1[0] * v2[1] - v1[1] * v2[0]])


def recvec(r1, r2, r3):
    """mhkpack_subs.f90:409-432 (reciprocal vectors with float32 pi)."""
    v23, v31, v12 = prodvec(r2, r3), prodvec(r3, r1), prodvec(r1, r2)
    vol = abs(r1[0] * v23[0] + r1[1] * v23[1] + r1[2] * v23[2])
    s = (2.0 * PI_F32) / vol
    return s * v23, s * v31, s * v12


def vcell2d(rlat):
    """general_subs.f90:195-206."""
    vx = prodvec(rlat[0], rlat[1])
    return math.sqrt(vx[0] ** 2 + vx[1] ** 2 + vx[2] ** 2)


def vcell3d(rlat):
    """general_subs.f90:208-221."""
    vx = prodvec(rlat[0], rlat[1])
    return abs(vx[0] * rlat[2, 0] + vx[1] * rlat[2, 1] + vx[2] * rlat[2, 2])


def monkhorst_pack(n1, n2, n3, shift, rlat, q=None):
    """mhkpack_subs.f90:359-407 (and monhkhorst_packq :305-356 when q is given):
    k = b1/n1*i + b2/n2*j + b3/n3*l + kshift (+ q), order i outer, l inner."""
    b1, b2, b3 = recvec(rlat[0], rlat[1], rlat[2])
    ks = b1 * shift[0] + b2 * shift[1] + b3 * shift[2]
    # kshift(c) = blat1(c)*shift(1)+blat2(c)*shift(2)+blat3(c)*shift(3), left to right
    ks = np.array([b1[c] * shift[0] + b2[c] * shift[1] + b3[c] * shift[2] for c in range(3)])
    out = np.zeros((n1 * n2 * n3, 3))
    cnt = 0
    for i in range(n1):
        for j in range(n2):
            for l in range(n3):
                for c in range(3):
                    v = (b1[c] / n1) * i + (b2[c] / n2) * j + (b3[c] / n3) * l + ks[c]
                    if q is not None:
                        v = q[c] + (b1[c] / n1) * i + (b2[c] / n2) * j + (b3[c] / n3) * l + ks[c]
                    out[cnt, c] = v
                cnt += 1
    return out


def rkmesh2d(rk, rlat):
    """mhkpack_subs.f90:28-52."""
    b = recvec(rlat[0], rlat[1], rlat[2])
    vs = [math.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2) / (2 * PI_F32) for v in b]
    return [int(max(1.0, rk * vs[0] + 0.5)), int(max(1.0, rk * vs[1] + 0.5)), 1]


def rkmesh3d(rk, rlat):
    """mhkpack_subs.f90:2-26."""
    b = recvec(rlat[0], rlat[1], rlat[2])
    vs = [math.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2) / (2 * PI_F32) for v in b]
    return [int(max(1.0, rk * v + 0.5)) for v in vs]


def kpathbse(rlat, ks, npts):
    """mhkpack_subs.f90:132-208: (nks/2)*npts points; the fraction (i-1.)/(npts-1.) is float32.
    Returns (kpt (M,4) = [distance, kx, ky, kz], klabels list)."""
    b1, b2, b3 = recvec(rlat[0], rlat[1], rlat[2])
    nks = len(ks)
    ksx = np.array([[ks[i][0] * b1[c] + ks[i][1] * b2[c] + ks[i][2] * b3[c] for c in range(3)]
                    for i in range(nks)])
    half = nks // 2
    kdis = np.zeros(half)
    tot = 0.0
    for i in range(half):
        d = ksx[2 * i + 1] - ksx[2 * i]
        kdis[i] = math.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
        tot += kdis[i]
    kdis = kdis / tot
    out = np.zeros((half * npts, 4))
    labels = [0.0]
    acc = 0.0
    for j in range(half):
        for i in range(npts):
            t = float(np.float32(np.float32(i) / np.float32(npts - 1)))
            row = (j * npts) + i
            out[row, 0] = acc + kdis[j] * t
            for c in range(3):
                out[row, 1 + c] = ksx[2 * j, c] + (ksx[2 * j + 1, c] - ksx[2 * j, c]) * t
        acc += kdis[j]
        labels.append(acc)
    return out, labels


# ----------------------------------------------------------------------------- bands

def _rcart(model):
    """Cartesian R with the reference's evaluation order ((r1*a1c + r2*a2c) + r3*a3c)."""
    r = model.rvec.astype(np.float64)
    L = model.rlat
    return np.stack([(r[:, 0] * L[0, c] + r[:, 1] * L[1, c]) + r[:, 2] * L[2, c]
                     for c in range(3)], axis=1)


def phases(model, k):
    """exp(i * float32(k.R)) per R (hamiltonian_tb.f90:62-68)."""
    R = _rcart(model)
    kr = (k[0] * R[:, 0] + k[1] * R[:, 1]) + k[2] * R[:, 2]
    kr32 = f32(kr)
    return np.cos(kr32) + 1j * np.sin(kr32)


def hk(model, k):
    """H(k) - f32(E_F) (hamiltonian_tb.f90:71-87)."""
    p = phases(model, k)
    H = model.hre + 1j * model.him
    inv = 1.0 / model.deg.astype(np.float64)
    Hk = np.zeros((model.w, model.w), dtype=np.complex128)
    for i in range(model.nvec):
        Hk = Hk + (p[i] * H[i]) * inv[i]
    Hk[np.diag_indices(model.w)] += -f32(model.efermi)
    return Hk


def zheev(a, lower):
    """ZHEEV with the reference's minimum workspace LWORK = 2N-1."""
    n = a.shape[0]
    w, v, info = lapack.zheev(np.asfortranarray(a), compute_v=1, lower=lower,
                              lwork=max(2 * n - 1, 1))
    if info != 0:
        raise RuntimeError(f"ZHEEV info={info}")
    return w, v


def eigsys(model, k):
    """hamiltonian_tb.f90:2-137.  Returns (energias (w,), autovetores (w,w) rows =
    eigenvectors, nocp).  ZHEEV('V','Lower') leaves component 1 of every vector real."""
    w, v = zheev(hk(model, k), lower=1)
    U = v.T.copy()
    nocp = None
    for i in range(model.w):
        if w[i] > 0.0:
            nocp = i
            break
    if nocp is None:
        raise RuntimeError("eigsys: no eigenvalue above E_F (nocp undefined in the reference)")
    w = w.copy()
    w[nocp:] += model.scs
    return w, U, nocp


def bands(model, kpts, nv, nc):
    """bse_solver-tool-diel.f90:257-313: per-k eigsys and band selection.
    Returns eigv (Nk, nc+nv), vector (Nk, nc+nv, w), nocpk (Nk,), egap."""
    nk = kpts.shape[0]
    eigv = np.zeros((nk, nc + nv))
    vec = np.zeros((nk, nc + nv, model.w), dtype=np.complex128)
    nocp = np.zeros(nk, dtype=np.int64)
    egap = 50.0
    for i in range(nk):
        e, U, no = eigsys(model, kpts[i])
        if nv > no or nc > model.w - no:
            raise RuntimeError("quantumnumbers2: band window exceeds occupied/empty states")
        nocp[i] = no
        eigv[i] = e[no - nv:no + nc]
        vec[i] = U[no - nv:no + nc]
        if eigv[i, nv] - eigv[i, nv - 1] <= egap:
            egap = eigv[i, nv] - eigv[i, nv - 1]
    return eigv, vec, nocp, egap


def quantumnumbers2(nk, nc, nv):
    """general_subs.f90:501-567: stt rows (idx, v, c, k), k outer, c middle, v inner
    (1-based band slots v in 1..nv, c in nv+1..nv+nc, k in 1..nk)."""
    stt = np.zeros((nk * nc * nv, 4), dtype=np.int64)
    cnt = 0
    for i in range(nk):
        for c in range(nv + 1, nv + nc + 1):
            for v in range(1, nv + 1):
                stt[cnt] = (cnt + 1, v, c, i + 1)
                cnt += 1
    return stt


def hlm(model, k):
    """optics.f90:1-97: dH/dk_alpha = sum_R i*f32(R_alpha) * exp(i f32(k.R)) * H(R) / deg,
    with the R=0 diagonal zeroed."""
    R = _rcart(model)
    p = phases(model, k)
    H = model.hre + 1j * model.him
    inv = 1.0 / model.deg.astype(np.float64)
    out = []
    for a in range(3):
        acc = np.zeros((model.w, model.w), dtype=np.complex128)
        ra = 1j * f32(R[:, a])
        for i in range(model.nvec):
            Hi = H[i]
            if np.all(model.rvec[i] == 0):
                Hi = Hi.copy()
                Hi[np.diag_indices(model.w)] = 0.0
            acc = acc + ((ra[i] * p[i]) * Hi) * inv[i]
        out.append(acc)
    return out


def optsp_all(model, kpts, eigv, vec, nv, nc, sme):
    """Loop bse_solver-tool-diel.f90:365-396 over optsp (optics.f90:102-156).
    Returns h (N,5): hrx, hry, hrz, hrsp, hrsm."""
    nk = kpts.shape[0]
    N = nk * nc * nv
    h = np.zeros((N, 5), dtype=np.complex128)
    eta = f32(sme)
    idx = 0
    for ik in range(nk):
        hx, hy, hz = hlm(model, kpts[ik])
        for c in range(nv, nv + nc):
            for v in range(nv):
                ec, ev = eigv[ik, c], eigv[ik, v]
                esp = complex(ec - ev, eta)
                factor = (1.0 / esp).real
                vc, vv = vec[ik, c], vec[ik, v]
                hr = [factor * np.sum(vc.conj() * (hm @ vv)) for hm in (hx, hy, hz)]
                h[idx, 0:3] = hr
                h[idx, 3] = (hr[0] + 1j * hr[1]) * INV_SQRT2_F32
                h[idx, 4] = (hr[0] - 1j * hr[1]) * INV_SQRT2_F32
                idx += 1
    return h


def sp_table(kpts, eigv, nocp, h, nv, nc, fdeh=None):
    """vecres (N,15) real(4) rows (bse_solver-tool-diel.f90:379-393) sorted by column 7
    with the stable bubble sort Bubblem (general_subs.f90:405-440). With ``fdeh`` the
    strengths are multiplied by f_v - f_c (bse_solver-tool-diel-temp.f90:416-423)."""
    stt = quantumnumbers2(kpts.shape[0], nc, nv)
    N = stt.shape[0]
    vr = np.zeros((N, 15), dtype=np.float32)
    for i in range(N):
        v, c, k = stt[i, 1] - 1, stt[i, 2] - 1, stt[i, 3] - 1
        hx, hy, hz, hp, hm = h[i]
        s = [(hx * hx.conjugate()).real, (hy * hy.conjugate()).real,
             (hz * hz.conjugate()).real, (hx * hy.conjugate()).real,
             (hx * hz.conjugate()).real, (hy * hz.conjugate()).real,
             (hp * hp.conjugate()).real, (hm * hm.conjugate()).real]
        if fdeh is not None:
            s = [x * fdeh[i] for x in s]
        vr[i] = [kpts[k, 0], kpts[k, 1], kpts[k, 2], nocp[k], nocp[k] - nv + c + 1,
                 nocp[k] - nv + v + 1, eigv[k, c] - eigv[k, v]] + s
    order = np.argsort(vr[:, 6], kind="stable")
    return vr[order]


# ----------------------------------------------------------------------------- Coulomb

class CoulombParams:
    """The Coulomb inputs of matrizelbse: coultype, ktol, ediel(3), lc, ez, w, r0, ngrid, rlat."""

    def __init__(self, coultype, ktol, ediel, lc, ez, w, r0, ngrid, rlat):
        self.coultype = coultype.strip()
        self.ktol = float(ktol)
        self.ediel = [float(x) for x in ediel]
        self.lc, self.ez, self.w, self.r0 = float(lc), float(ez), float(w), float(r0)
        self.ngrid = [int(x) for x in ngrid]
        self.rlat = np.asarray(rlat, dtype=np.float64)


def _modvec(d):
    return np.sqrt(d[..., 0] ** 2 + d[..., 1] ** 2 + d[..., 2] ** 2)


def coulomb(p: CoulombParams, dk):
    """V(k1 - k2) for an array dk (..., 3) of k1-k2 (coulomb_pot.f90:2-432)."""
    dk = np.asarray(dk, dtype=np.float64)
    modk = _modvec(dk)
    nkt = p.ngrid[0] * p.ngrid[1] * p.ngrid[2]
    t = p.coultype
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        if t == "V2DRK":      # coulomb_pot.f90:276-340
            vbz = 1.0 / (nkt * vcell2d(p.rlat))
            epar, et, eb = p.ediel[1], p.ediel[0], p.ediel[2]
            eta = math.sqrt(epar / p.ez)
            kappa = math.sqrt(epar * p.ez)
            pb = (eb - kappa) / (eb + kappa)
            pt = (et - kappa) / (et + kappa)
            aux1 = (1.0 - (pb * pt * np.exp(-2.0 * modk * eta * p.lc))) * kappa
            aux2 = (1.0 - (pt * np.exp(-eta * modk * p.lc))) * (1.0 - (pb * np.exp(-eta * modk * p.lc)))
            aux3 = p.r0 * modk * np.exp(-modk * p.w)
            ew = (aux1 / aux2) + aux3
            v = (vbz * CIC) * np.exp(-modk * p.w) * (1.0 / ew) * (1.0 / modk)
            return np.where(modk < p.ktol, 0.0, v)
        if t == "V2DK":       # coulomb_pot.f90:2-51
            a0 = 0.5 * (np.linalg.norm(p.rlat[0]) + np.linalg.norm(p.rlat[1]))
            vc = vcell2d(p.rlat)
            r0 = ((p.ediel[1] - 1.0) * p.lc) / (p.ediel[0] + p.ediel[2])
            vbz = 1.0 / (nkt * vc)
            g1 = float(p.ngrid[0] * p.ngrid[1])
            auxi = (2.0 * PI_F32 * r0) / (a0 * math.sqrt(g1))
            ed = (p.ediel[0] + p.ediel[2]) / 2.0
            v0 = vbz * (CIC / ed) * (a0 * math.sqrt(g1) / (2.0 * PI_F32)) * \
                (ALPHA1_V2DK + auxi * 1.0 + 0.0 * auxi ** 2)
            v = vbz * (CIC / ed) * (1.0 / (modk * (1 + (r0 * modk))))
            return np.where(modk < p.ktol, v0, v)
        if t in ("V3D", "V3DL"):  # coulomb_pot.f90:55-122
            vbz = 1.0 / (nkt * vcell3d(p.rlat))
            ed = 1.0 if t == "V3D" else p.ediel[1]
            v = vbz * (CIC / ed) * (1.0 / (modk * modk))
            return np.where(modk < p.ktol, 0.0, v)
        if t == "V2DT":       # coulomb_pot.f90:126-183
            vbz = 1.0 / (nkt * vcell3d(p.rlat))
            gz = np.abs(dk[..., 2])
            gpar = np.sqrt(dk[..., 0] * dk[..., 0] + dk[..., 1] * dk[..., 1])
            rc = 0.5 * p.rlat[2, 2]
            c0 = (vbz * CIC) * (-0.5 * rc * rc)
            c1 = (vbz * CIC) * (1.0 / (modk * modk)) * (1.0 - np.cos(gz * rc) - (gz * rc * np.sin(gz * rc)))
            aux1 = gz / gpar
            aux2 = gpar * rc
            aux3 = gz * rc
            c2 = (vbz * CIC) * (1.0 / (modk * modk)) * (1.0 + (np.exp(-aux2) * (aux1 * np.sin(aux3) - np.cos(aux3))))
            return np.where((gpar < p.ktol) & (gz < p.ktol), c0,
                            np.where((gpar < p.ktol) & (gz >= p.ktol), c1, c2))
        if t == "V0DT":       # coulomb_pot.f90:187-228
            vbz = 1.0 / (nkt * vcell3d(p.rlat))
            cr = 0.5 * min(np.linalg.norm(p.rlat[0]), np.linalg.norm(p.rlat[1]), np.linalg.norm(p.rlat[2]))
            v0 = (vbz * CIC) * 0.5 * cr * cr
            v = (vbz * CIC) * (1.0 / (modk * modk)) * (1.0 - np.cos(cr * modk))
            return np.where(modk < p.ktol, v0, v)
        if t == "V2DT2":      # coulomb_pot.f90:233-272
            vbz = 1.0 / (nkt * vcell3d(p.rlat))
            qxy = np.sqrt(dk[..., 0] * dk[..., 0] + dk[..., 1] * dk[..., 1])
            v = (vbz * CIC) * (1.0 / (modk * modk)) * (1.0 - np.exp(-0.5 * qxy * p.lc) * np.cos(0.5 * p.lc * dk[..., 2]))
            return np.where(modk < p.ktol, 0.0, v)
        if t == "V2DOH":      # coulomb_pot.f90:344-377
            vbz = 1.0 / (nkt * vcell2d(p.rlat))
            v = (vbz * CIC) * np.exp(-p.w * modk) * (1.0 / (p.ez * modk))
            return np.where(modk < p.ktol, 0.0, v)
        if t == "V1DT":       # coulomb_pot.f90:381-432
            vbz = 1.0 / (nkt * vcell3d(p.rlat))
            ax = np.abs(dk[..., 0])
            qyz = np.sqrt(dk[..., 1] * dk[..., 1] + dk[..., 2] * dk[..., 2])
            lc = p.lc
            # integralJ0pot (coulomb_pot.f90:437-469): 100-point trapezoid of r*J0(r q)*log r
            n = 100
            r = (np.arange(n) / (n - 1.0)) * lc + f32(1e-4)   # eta = 1E-04 is real(4)
            f = r[None, :] * sps.j0(r[None, :] * np.ravel(qyz)[:, None]) * np.log(r)[None, :]
            hh = r[1] - r[0]
            integ = np.zeros(f.shape[0])
            for i in range(n - 1):
                integ = integ + (hh / 2.0) * (f[:, i] + f[:, i + 1])
            integ = integ.reshape(np.shape(qyz))
            c_a = (vbz * CIC) * integ
            c_b = (vbz * CIC) * ((lc * lc) / 16.0) * (2.0 * math.log(lc) - 1.0)
            c1 = qyz * lc * sps.j1(qyz * lc) * sps.k0(ax * lc)
            c2 = ax * lc * sps.j0(qyz * lc) * sps.k1(ax * lc)
            c_c = (vbz * CIC) * (1.0 + c1 + c2)
            return np.where((ax < p.ktol) & (qyz >= p.ktol), c_a,
                            np.where((ax < p.ktol) & (qyz < p.ktol), c_b, c_c))
    raise ValueError("Wrong Coulomb Potential")


# ----------------------------------------------------------------------------- BSE

def bse_matrix(p: CoulombParams, kpts, eigv, vec, nv, nc, upper_only=True, fdeh=None):
    """matrizelbse over j >= i (bse_subs.f90:2-124, loop bse_solver-tool-diel.f90:431-458).
    Off-diagonal: V(k_i - k_j) * <c_i|c_j> * <v_i|v_j> with <a|b> = sum conj(a) b.
    Diagonal: (E_c - E_v) + V(0).  Returns the N x N matrix with the upper triangle set."""
    nk = kpts.shape[0]
    ncv = nc * nv
    N = nk * ncv
    Uc = vec[:, nv:nv + nc, :].reshape(nk * nc, -1)
    Uv = vec[:, :nv, :].reshape(nk * nv, -1)
    Mc = Uc.conj() @ Uc.T                  # (nk*nc, nk*nc)
    Mv = Uv.conj() @ Uv.T
    V = coulomb(p, kpts[:, None, :] - kpts[None, :, :])   # (nk, nk)
    Mc4 = Mc.reshape(nk, nc, nk, nc)
    Mv4 = Mv.reshape(nk, nv, nk, nv)
    H = (V[:, None, None, :, None, None] * Mc4[:, :, None, :, :, None]) * Mv4[:, None, :, :, None, :]
    H = H.reshape(N, N)
    de = (eigv[:, nv:][:, :, None] - eigv[:, :nv][:, None, :]).reshape(N)
    vdiag = np.repeat(np.diag(V), ncv)
    if fdeh is None:
        H[np.diag_indices(N)] = de + vdiag
    else:
        # matrizelbsetemp (bse_subs_temp.f90:2-126): element (i, j >= i) times f_i, plus dE on i = j
        H[np.diag_indices(N)] = vdiag
        H = H * np.asarray(fdeh)[:, None]
        H[np.diag_indices(N)] += de
    if upper_only:
        H = np.triu(H)
    return H


def bse_matrix_q(p: CoulombParams, q4, kpts, energy, vector, energyq, vectorq, nv, nc, fdeh=None):
    """matrizelbsekq (bse_subs_kpath.f90:1-208) over j >= i: the Q != 0 kernel adds the
    exchange term -V(Q) <c_{k+Q}|v_k> <v_{k'}|c_{k'+Q}> (zero when |Q| == 0, :116)."""
    nk = kpts.shape[0]
    ncv = nc * nv
    N = nk * ncv
    Uc = vectorq[:, nv:nv + nc, :].reshape(nk * nc, -1)
    Uv = vector[:, :nv, :].reshape(nk * nv, -1)
    Mc = (Uc.conj() @ Uc.T).reshape(nk, nc, nk, nc)
    Mv = (Uv.conj() @ Uv.T).reshape(nk, nv, nk, nv)
    V = coulomb(p, kpts[:, None, :] - kpts[None, :, :])
    H = (V[:, None, None, :, None, None] * Mc[:, :, None, :, :, None]) * Mv[:, None, :, :, None, :]
    H = H.reshape(N, N)
    de = (energyq[:, nv:][:, :, None] - energy[:, :nv][:, None, :]).reshape(N)
    if fdeh is None:
        H[np.diag_indices(N)] = de + np.repeat(np.diag(V), ncv)
    else:
        H[np.diag_indices(N)] = np.repeat(np.diag(V), ncv)
    modq = math.sqrt(q4[1] ** 2 + q4[2] ** 2 + q4[3] ** 2)
    if modq != 0.0:
        vq = float(coulomb(p, np.array([q4[1], q4[2], q4[3]])))
        # vcv(i) = sum conj(c_{k+Q}) v_k ; vvc(j) = sum conj(v_k') c_{k'+Q}
        cq = vectorq[:, nv:nv + nc, :]
        vk = vector[:, :nv, :]
        vcv = np.einsum("kcm,kvm->kcv", cq.conj(), vk).reshape(N)
        vvc = np.einsum("kvm,kcm->kcv", vk.conj(), cq).reshape(N)
        H = H - vq * (vcv[:, None] * vvc[None, :])
    if fdeh is not None:
        # matrizelbsekqtemp (bse_subs_temp.f90:128-337): the interaction part times f_i
        H = H * np.asarray(fdeh)[:, None]
        H[np.diag_indices(N)] += de
    return np.triu(H)


def dielbsev(A, h):
    """bse_subs.f90:336-378: act(i) = |sum_j A(j,i) h(j)|^2 (no conjugate on A)."""
    s = A.T @ h
    return (s * s.conj()).real


def dielbsep(A, h1, h2):
    """bse_subs.f90:278-332: act(i) = Re[(sum A h1) * conj(sum A h2)]."""
    s1, s2 = A.T @ h1, A.T @ h2
    return (s1 * s2.conj()).real


def dielbseptemp(A, h1, h2, f):
    """bse_subs_temp.f90:340-395: act(i) = Re[(sum A h1) * conj(sum A h2 f)]."""
    s1, s2 = A.T @ h1, A.T @ (h2 * f)
    return (s1 * s2.conj()).real


def bse_solve(p: CoulombParams, kpts, eigv, vec, h, nv, nc, dtfull, cpol, want_vectors=False, fdeh=None):
    """bse_solver-tool-diel.f90:431-602 (bse_solver-tool-diel-temp.f90:470-620 with ``fdeh``):
    build, ZHEEV('V','U'), oscillator strengths.
    Returns W (N,), act (N, 8) = xx, yy, zz, xy, xz, yz, sp, sm [, A]."""
    H = bse_matrix(p, kpts, eigv, vec, nv, nc, fdeh=fdeh)
    W, A = zheev(H, lower=0)
    N = W.shape[0]
    act = np.zeros((N, 8))
    if fdeh is None:
        sv = lambda a: dielbsev(A, h[:, a])
        sp = lambda a, b: dielbsep(A, h[:, a], h[:, b])
    else:
        sv = lambda a: dielbseptemp(A, h[:, a], h[:, a], fdeh)
        sp = lambda a, b: dielbseptemp(A, h[:, a], h[:, b], fdeh)
    act[:, 0] = sv(0)
    act[:, 1] = sv(1)
    act[:, 2] = sv(2)
    if dtfull:
        act[:, 3] = sp(0, 1)
        act[:, 4] = sp(0, 2)
        act[:, 5] = sp(1, 2)
    if cpol:
        act[:, 6] = sv(3)
        act[:, 7] = sv(4)
    if want_vectors:
        return W, act, A
    return W, act


# ----------------------------------------------------------------------------- spectrum

def fortran_f(x, w=15, d=4):
    """Fw.d output of a value (the value is formatted exactly, as Fortran does)."""
    s = f"{float(x):{w}.{d}f}"
    if len(s) > w:
        return "*" * w
    return s


def roundtrip_f154(x):
    """The value that ``read(*,*)`` gets back from an F15.4 field."""
    return np.array([float(fortran_f(v)) for v in np.ravel(x)]).reshape(np.shape(x))


def avgsme(e):
    """optics.f90:302-324: 10 * (sum_{i>=2} (e_i - e_{i-1})) / n, summed in order."""
    s = 0.0
    for i in range(1, len(e)):
        s = s + e[i] - e[i - 1]
    return 10.0 * (s / float(len(e)))


def optdiel_grid(rtype, vc, ngrid, omegas, e, f, sme):
    """optdiel (optics.f90:160-244) for every photon energy: returns (re, im)."""
    baux = float(np.float32(ngrid[0] * ngrid[1] * ngrid[2])) * vc
    caux = GAMA / (baux * 1.0)
    delta = 1.0 if rtype == 1 else 0.0
    smef = avgsme(e) + sme
    om = np.asarray(omegas)[:, None]
    eaux = ((om - e[None, :]) ** 2) + (smef ** 2)
    raux = f[None, :] * ((e[None, :] - om) / eaux)
    iaux = f[None, :] * (smef / eaux)
    rpart = raux.sum(axis=1)
    ipart = iaux.sum(axis=1)
    return delta + (rpart * caux), ipart * caux


def imagrenorm(e, diel):
    """optics.f90:327-390 on diel (nw, 3) = [omega, re, im] (modified in place)."""
    aux = e[0] - RENORM_FACTOR
    if aux <= 0.0:
        return diel
    nel = diel.shape[0]
    ibegin = 1
    for i in range(1, nel + 1):
        if diel[i - 1, 0] <= aux:
            ibegin = i
        else:
            break
    aux3 = diel[ibegin, 2]          # dielf(ibegin+1, 3)
    diel[:ibegin, 2] = 0.0
    for i in range(ibegin + 1, nel + 1):
        v = diel[i - 1, 2] - aux3
        diel[i - 1, 2] = 0.0 if v < 0.0 else v
    return diel


def omega_grid(ebse0, ebsef, numbse):
    n = int(numbse)
    return np.array([ebse0 + ((ebsef - ebse0) * (j - 1)) / (numbse - 1.0) for j in range(1, n + 1)])


def bsedielraw(systype, rlat, ngrid, E, F, ebse0, ebsef, numbse, sme, renorm):
    """bse_diel-tool.f90:5-245 on the values read back from bse_opt_diel.dat.
    E (N,), F (N,6) in file order xx, yy, zz, xy, xz, yz.
    Returns dict comp -> (nw, 3) array [omega (f64), re (f32), im (f32)]."""
    spinf = 2.0 if systype.strip() == "NP" else 1.0
    vc = vcell3d(rlat)
    om = omega_grid(ebse0, ebsef, numbse)
    out = {}
    for name, col, rtype in (("xx", 0, 1), ("yy", 1, 1), ("zz", 2, 1),
                             ("xy", 3, 0), ("xz", 4, 0), ("yz", 5, 0)):
        re, im = optdiel_grid(rtype, vc, ngrid, om, E, F[:, col], sme)
        d = np.stack([om, re, im], axis=1)
        if renorm:
            imagrenorm(E, d)
        d[:, 1] = f32(spinf * d[:, 1])
        d[:, 2] = f32(spinf * d[:, 2])
        out[name] = d
    return out


def optprop(e1, e2, efoton):
    """diel-pp-subs.f90:1-73: refractive index, extinction, reflectivity, absorption, loss."""
    aux = np.sqrt(e1 * e1 + e2 * e2)
    n = np.sqrt((aux + e1) / 2.0)
    k = np.sqrt((aux - e1) / 2.0)
    R = ((n - 1.0) * (n - 1.0) + k * k) / ((n + 1.0) * (n + 1.0) + k * k)
    a = (SQRT2_F32 * efoton) * (1.0 / HC) * np.sqrt(aux - e1)
    with np.errstate(divide="ignore", invalid="ignore"):
        L = e2 / (e1 * e1 + e2 * e2)
    return n, k, R, a, L


def exclft(sysdim, ngrid, rlat, fosc, enexc):
    """bse_subs.f90:472-530."""
    nkt = float(ngrid[0] * ngrid[1] * ngrid[2])
    s = sysdim.strip()
    with np.errstate(divide="ignore", invalid="ignore"):
        if s == "3D":
            aux1 = (4.0 * CFE) * (enexc * enexc * enexc)
            aux2 = fosc / nkt
            aux3 = 3.0 * (LSPD * LSPD) * (HBAR * HBAR * HBAR)
            return 1.0 / ((aux1 * aux2) / aux3)
        if s == "2D":
            aux1 = nkt * vcell2d(rlat) * HBAR
            aux2 = (8.0 * PI_F32 * CFE * enexc) * fosc
            return aux1 / aux2
        if s == "1D":
            aux2 = (2.0 * PI_F32 * CFE * enexc * enexc) * fosc
            aux1 = nkt * rlat[0, 0] * HBAR * HBAR * LSPD
            return aux1 / aux2
    raise ValueError("Wrong System dimension")


# ----------------------------------------------------------------------------- drivers

KB_F32 = float(np.float32(8.617330350e-5))   # kb of general_subs.f90:575 (a real(4) literal)


def fermidisteh(ec, ev, temp):
    """general_subs.f90:607-635: f_v - f_c, E_F = 0; T = 0 is replaced by 1E-8 (real(4))."""
    t = float(np.float32(1e-8)) if temp == 0.0 else float(temp)
    beta = 1.0 / (KB_F32 * t)
    with np.errstate(over="ignore"):
        fv = 1.0 / (np.exp(np.asarray(ev) * beta) + 1.0)
        fc = 1.0 / (np.exp(np.asarray(ec) * beta) + 1.0)
    return fv - fc


def gapcortemp(st, phavg, temp):
    """general_subs.f90:569-586 (Varshni-like form, doi 10.1063/1.104723)."""
    aux1 = phavg / (2.0 * KB_F32 * temp)
    return -st * phavg * ((1.0 / math.tanh(aux1)) - 1.0)


def gapcortemp2(st, phavg, temp):
    """general_subs.f90:588-605 (Bose-Einstein form)."""
    return -((2.0 * st) / (math.exp(phavg / temp) - 1.0))


def temperature_shift(deck):
    """tcor of bse_solver-tool-diel-temp.f90:263-282 (TA= FA / VE / BE)."""
    ta = deck["ta"].strip()
    if ta == "VE":
        return gapcortemp(deck["st"], deck["phavg"], deck["temp"])
    if ta == "BE":
        return gapcortemp2(deck["st"], deck["phavg"], deck["temp"])
    return 0.0


def fdeh_states(eigc, eigv, nv, nc, temp):
    """f_v - f_c of every basis state in quantumnumbers2 order (k outer, c, v inner)."""
    ec = eigc[:, nv:nv + nc][:, :, None]
    ev = eigv[:, :nv][:, None, :]
    return fermidisteh(np.broadcast_to(ec, (eigc.shape[0], nc, nv)),
                       np.broadcast_to(ev, (eigc.shape[0], nc, nv)), temp).reshape(-1)


def with_scs(model, scs):
    import copy
    m2 = copy.copy(model)
    m2.scs = scs
    return m2


def run_bse(model, deck, want_vectors=False):
    """The numbers of ``bsesolver`` (bse_solver-tool-diel.f90:2-660) for one deck dict, or of
    ``bsesolvertemp`` (bse_solver-tool-diel-temp.f90) when BSET=T."""
    temp = deck.get("bset", False)
    if temp:
        model = with_scs(model, model.scs + temperature_shift(deck))
    ngrid = list(deck["ngrid"])
    if deck["meshtype"].strip() == "RK2D":
        ngrid = rkmesh2d(deck["rk"], model.rlat)
    elif deck["meshtype"].strip() == "RK3D":
        ngrid = rkmesh3d(deck["rk"], model.rlat)
    kpts = monkhorst_pack(ngrid[0], ngrid[1], ngrid[2], deck["mshift"], model.rlat)
    nv, nc = deck["nv"], deck["nc"]
    eigv, vec, nocp, egap = bands(model, kpts, nv, nc)
    h = optsp_all(model, kpts, eigv, vec, nv, nc, deck["cshift"])
    p = CoulombParams(deck["coultype"], deck["ktol"], deck["ediel"], deck["lc"], deck["ez"],
                      deck["w"], deck["r0"], ngrid, model.rlat)
    fdeh = fdeh_states(eigv, eigv, nv, nc, deck["temp"]) if temp else None
    res = bse_solve(p, kpts, eigv, vec, h, nv, nc, deck["dtfull"], deck["cpol"], want_vectors, fdeh=fdeh)
    out = dict(ngrid=ngrid, kpts=kpts, eigv=eigv, vec=vec, nocp=nocp, egap=egap, h=h,
               W=res[0], act=res[1], fdeh=fdeh)
    if want_vectors:
        out["A"] = res[2]
    return out


def run_bsebnds(model, deck, ks, npts):
    """The numbers of ``bsebnds`` (bse_kpath-tool.f90:3-479): exk (N, nQ) and the Q path; of
    ``bsebndstemp`` (bse_kpath-tool-temp.f90) when BSET_BND=T."""
    temp = deck.get("bsetbnd", False)
    if temp:
        model = with_scs(model, model.scs + temperature_shift(deck))
    ngrid = list(deck["ngrid"])
    if deck["meshtype"].strip() == "RK2D":
        ngrid = rkmesh2d(deck["rk"], model.rlat)
    kpts = monkhorst_pack(ngrid[0], ngrid[1], ngrid[2], deck["mshift"], model.rlat)
    nv, nc = deck["nv"], deck["nc"]
    energy, vector, nocpk, _ = bands(model, kpts, nv, nc)
    qpath, labels = kpathbse(model.rlat, ks, npts)
    p = CoulombParams(deck["coultype"], deck["ktol"], deck["ediel"], deck["lc"], deck["ez"],
                      deck["w"], deck["r0"], ngrid, model.rlat)
    exk = []
    for iq in range(qpath.shape[0]):
        q4 = qpath[iq]
        qpt = monkhorst_pack(ngrid[0], ngrid[1], ngrid[2], deck["mshift"], model.rlat, q=q4[1:])
        energyq, vectorq, _, _ = bands(model, qpt, nv, nc)
        fdeh = fdeh_states(energyq, energy, nv, nc, deck["temp"]) if temp else None
        H = bse_matrix_q(p, q4, kpts, energy, vector, energyq, vectorq, nv, nc, fdeh=fdeh)
        w, info = lapack.zheev(np.asfortranarray(H), compute_v=0, lower=0,
                               lwork=max(2 * H.shape[0] - 1, 1))[0::2]
        exk.append(w)
    return np.array(exk).T, qpath, labels


# ----------------------------------------------------------------------------- band and DOS tools

def spin_diag(systype, dft, w):
    """Diagonal of the Sz operator of spinvl (hamiltonian_tb.f90:281-368) / the up-down split of
    spincont (dos_subs.f90:37-100): +1 up, -1 down (all +1 for NP in spinvl)."""
    s = np.ones(w)
    st = systype.strip()
    w2 = w // 2
    if st == "NP":
        return s
    if st == "SP" or (st == "SOC" and dft.strip() == "V"):
        s[w2:] = -1.0
    else:
        s[1::2] = -1.0
    return s


def spinvl(wf, dft, systype):
    return float(np.real(np.vdot(wf, spin_diag(systype, dft, len(wf)) * wf)))


def spincont(wf, dft, systype):
    if systype.strip() == "NP":
        return 0.0, 0.0
    s = spin_diag(systype, dft, len(wf))
    a2 = np.abs(wf) ** 2
    return float(a2[s > 0].sum()), float(a2[s < 0].sum())


def layercont(wf, ow):
    """dos_subs.f90:154-181."""
    return float(np.real(np.sum(wf * np.asarray(ow) * wf.conj())))


def gaussian(de, sme):
    """general_subs.f90:471-487 (pi = acos(-1.) in real(4))."""
    pi = float(np.float32(np.pi))
    norm = 1.0 / (sme * math.sqrt(2.0 * pi))
    return norm * np.exp(-1.0 * (de * de) / (2.0 * sme * sme))


def bandstool(model, ks, npts, orbw=None, dft="V"):
    """bands-kpath-tool.f90: rows (band, k) = real(4) of (distance, E, <Sz>, layer weight)."""
    kp, labels = kpathbse(model.rlat, ks, npts)
    w = model.w
    ow = np.ones(w) if orbw is None else np.asarray(orbw)
    out = np.zeros((w, kp.shape[0], 4), dtype=np.float32)
    for j in range(kp.shape[0]):
        e, U, _ = eigsys(model, kp[j, 1:])
        for i in range(w):
            out[i, j] = [kp[j, 0], e[i], spinvl(U[i], dft, model.systype), layercont(U[i], ow)]
    return out, labels


# berry tools: "double precision,parameter :: gammas= 0.001" and the degeneracy cut 0.0001
# are default-real (single-precision) literals
BERRY_GAMMA = float(np.float32(0.001))
BERRY_DEGTOL = float(np.float32(0.0001))
BERRY_PAIRS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]


def berryct2(model, k, e, U, nocp, gamma=BERRY_GAMMA, degtol=BERRY_DEGTOL):
    """berry_curvature_subs.f90:1-128: b_ab = sum over n <= nocp < i of
    -2 v_a(n,i) conj(v_b(n,i)) / ((E_n - E_i)^2 + gamma^2) with v_a(n,i) = conj(u_n).(h_a u_i)
    (vecconjg, matvec, prodintsq) and h_a from hlm; pairs with |E_i - E_n| < degtol give 0.
    berryct2 passes hlm a kz it never sets; the k-point's own kz is used (2D models have
    R_z = 0). Returns the complex [bxx, bxy, bxz, byy, byz, bzz], summed n outer, i inner."""
    hs = hlm(model, k)
    w = model.w
    b = np.zeros(6, dtype=np.complex128)
    for n in range(nocp):
        vn = np.conj(U[n])
        for i in range(nocp, w):
            v = [np.sum(vn * (h @ U[i])) for h in hs]
            if abs(e[i] - e[n]) < degtol:
                continue
            aux = (e[n] - e[i]) ** 2 + gamma ** 2
            for c, (a, bb) in enumerate(BERRY_PAIRS):
                b[c] += -2.0 * ((v[a] * np.conj(v[bb])) / aux)
    return b


def berry_bz(model, ngrid, mshift):
    """berry_curvature_bz-tool.f90: rows (real(4) kx, ky, kz, Im b_yz, Im b_xz, Im b_xy)."""
    kpts = monkhorst_pack(ngrid[0], ngrid[1], ngrid[2], mshift, model.rlat)
    rows = []
    for k in kpts:
        e, U, nocp = eigsys(model, k)
        b = berryct2(model, k, e, U, nocp)
        rows.append([f32(k[0]), f32(k[1]), f32(k[2]), b[4].imag, b[2].imag, b[1].imag])
    return np.array(rows)


def berry_kpath(model, ks, npts):
    """berry_curvature_kpath-tool.f90: rows (distance, Im b_yz, Im b_xz, Im b_xy) along kpath2."""
    kp, labels = kpathbse(model.rlat, ks, npts)
    rows = []
    for j in range(kp.shape[0]):
        e, U, nocp = eigsys(model, kp[j, 1:])
        b = berryct2(model, kp[j, 1:], e, U, nocp)
        rows.append([kp[j, 0], b[4].imag, b[2].imag, b[1].imag])
    return np.array(rows), labels


def sp_optbz(model, ngrid, mshift, nv, nc, sme):
    """sp_opt_bz-tool.f90:81-175 (spoptpolbz): per k of the mesh, over the pairs c = nocp_k+1 ..
    nocp_k+nc (outer), v = nocp_k-nv+1 .. nocp of the FIRST k-point (inner), the first nc*nv of
    them, h_a = optspbz / cmplx(E_c - E_v, sme) (a default-kind complex: both parts rounded to
    single precision); rows (real(4) kx, ky, kz, sum|h_x|^2, sum|h_y|^2, sum|h_z|^2, sigma+,
    sigma-, dichroism) with norm = f32(1/sqrt 2)."""
    kpts = monkhorst_pack(ngrid[0], ngrid[1], ngrid[2], mshift, model.rlat)
    norm = float(np.float32(1.0) / np.sqrt(np.float32(2.0)))
    nocp1 = eigsys(model, kpts[0])[2]
    rows = []
    for k in kpts:
        e, U, nocp = eigsys(model, k)
        hs = hlm(model, k)
        pairs = [(c, v) for c in range(nocp, nocp + nc) for v in range(nocp - nv, nocp1)][:nc * nv]
        assert len(pairs) == nc * nv
        s = np.zeros(5)
        for c, v in pairs:
            den = complex(f32(e[c] - e[v]), f32(sme))
            h = [np.sum(np.conj(U[c]) * (H @ U[v])) / den for H in hs]
            s[0] += (h[0] * np.conj(h[0])).real
            s[1] += (h[1] * np.conj(h[1])).real
            s[2] += (h[2] * np.conj(h[2])).real
            p = norm * (h[0] + 1j * h[1])
            m = norm * (h[0] - 1j * h[1])
            s[3] += (p * np.conj(p)).real
            s[4] += (m * np.conj(m)).real
        rows.append([f32(k[0]), f32(k[1]), f32(k[2]), *s, (s[3] - s[4]) / (s[3] + s[4])])
    return np.array(rows)


def dostool(model, ngrid, mshift, numdos, sme, orbw=None, dft="V"):
    """tdos-tool.f90: the dos.dat columns (energy, tdos, sumdos, [updos, -dndos,] awdos)."""
    kpts = monkhorst_pack(ngrid[0], ngrid[1], ngrid[2], mshift, model.rlat)
    w = model.w
    ow = np.ones(w) if orbw is None else np.asarray(orbw)
    res = []
    e0, e1 = 0.0, 0.0
    for k in kpts:
        e, U, _ = eigsys(model, k)
        e0, e1 = min(e0, e[0]), max(e1, e[-1])
        for i in range(w):
            cu, cd = spincont(U[i], dft, model.systype)
            res.append((e[i], 1.0, cu, cd, layercont(U[i], ow)))
    res = np.array(res)
    nw = int(numdos)
    en = np.array([e0 + ((e1 - e0) * i) / (numdos - 1.0) for i in range(nw)])
    g = gaussian(en[:, None] - res[None, :, 0], sme)
    caux = 1.0 / kpts.shape[0]
    cols = (g @ res[:, 1:]) * caux
    np_ = model.systype.strip() == "NP"
    spinf = 2.0 if np_ else 1.0
    at, up, dn, aw = spinf * cols[:, 0], cols[:, 1], cols[:, 2], spinf * cols[:, 3]
    dde = (e1 - e0) / (numdos - 1.0)
    sums = np.zeros(nw)
    s = 0.0
    for i in range(nw):
        sums[i] = s
        if i > 0:
            s = s + (dde * (at[i - 1] + at[i]) * 0.5)
    if np_:
        return np.column_stack([en, at, sums, aw])
    return np.column_stack([en, at, sums, up, -dn, aw])
