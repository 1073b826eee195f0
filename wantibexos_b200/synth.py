"""Synthetic Wannier tight-binding models in the WanTiBEXOS params-file format.

The reference reads a "params" file (``subroutines/module_input_read.f90:32-176``):

    systype            (character, e.g. NP / SOC / SP)
    scs                (scissors shift, eV)
    efermi             (Fermi level, eV)
    a1x a1y a1z        (three real-space lattice rows, Angstrom)
    a2x a2y a2z
    a3x a3y a3z
    <header line>      (ignored)
    w                  (number of Wannier orbitals)
    nvec               (number of lattice vectors R)
    deg(1..nvec)       (degeneracies, 15 per line)
    R1 R2 R3 m n Re Im (nvec*w*w rows; row index m fastest, then n, then R)

This module generates the seeded synthetic 2D hexagonal models used by the tests
and the benchmark (no public dataset exists for this path): a=3.2 A,
a1=(a,0,0), a2=(-a/2, a*sqrt(3)/2, 0), a3=(0,0,20); R = i*a1 + j*a2 with hexagonal
distance max(|i|,|j|,|i-j|) <= n_shell (37/61/91 cells for 3/4/5 shells); deg=1;
H(R) for one of each +-R pair is complex Gaussian * 0.2*exp(-|R|/a) eV with
H(-R)=H(R)^dagger; H(0) has onsite energies on the diagonal and a Hermitian
Gaussian*0.2 off-diagonal part.  E_F=0, scs=0, systype NP.

For w > 8 every random coupling (hoppings and the H(0) off-diagonal) is additionally
scaled by sqrt(8/w): the band width of a random w x w coupling grows like sqrt(w), and
with the bare 0.2 eV scale the valence and conduction groups of a w=24 model overlap at
any seed.  The normalisation keeps every material at the band width of the w=8 model,
so that the gap check (nocp = w/2 at every k, gap > 0) can be met.
"""
from __future__ import annotations

import dataclasses
import io
import math
from typing import Optional

import numpy as np

A_LAT = 3.2
C_VAC = 20.0


@dataclasses.dataclass
class TBModel:
    """A Wannier TB model exactly as ``hamiltonian_input_read`` stores it.

    hre/him are (nvec, w, w) arrays with hre[iR, m, n] = Re H_mn(R)
    (``hopmatrices(iR,m,n)``, module_input_read.f90:158-167).
    rlat rows are the real-space lattice vectors (``rlat(i,:)``).
    """
    systype: str
    scs: float
    efermi: float
    rlat: np.ndarray          # (3,3)
    w: int
    rvec: np.ndarray          # (nvec,3) int32
    deg: np.ndarray           # (nvec,) int32
    hre: np.ndarray           # (nvec,w,w) float64
    him: np.ndarray           # (nvec,w,w) float64

    @property
    def nvec(self) -> int:
        return int(self.rvec.shape[0])


def hex_cells(n_shell: int) -> np.ndarray:
    cells = []
    for i in range(-n_shell, n_shell + 1):
        for j in range(-n_shell, n_shell + 1):
            if max(abs(i), abs(j), abs(i - j)) <= n_shell:
                cells.append((i, j, 0))
    out = np.array(cells, dtype=np.int32)
    expect = 1 + 3 * n_shell * (n_shell + 1)
    assert out.shape[0] == expect, (out.shape, expect)
    return out


def hex_rlat(a: float = A_LAT, c: float = C_VAC) -> np.ndarray:
    return np.array([[a, 0.0, 0.0],
                     [-a / 2.0, a * math.sqrt(3.0) / 2.0, 0.0],
                     [0.0, 0.0, c]], dtype=np.float64)


def make_hex_model(w: int, n_shell: int, onsite_lo: tuple, onsite_hi: tuple,
                   seed: int, hop_scale: Optional[float] = None,
                   h0_scale: Optional[float] = None) -> TBModel:
    """Generate one synthetic model (no gap check; see :func:`make_gapped_model`)."""
    norm = math.sqrt(8.0 / w) if w > 8 else 1.0
    hop_scale = 0.2 * norm if hop_scale is None else hop_scale
    h0_scale = 0.2 * norm if h0_scale is None else h0_scale
    rng = np.random.Generator(np.random.PCG64(seed))
    rlat = hex_rlat()
    rvec = hex_cells(n_shell)
    nvec = rvec.shape[0]
    index = {tuple(r): i for i, r in enumerate(rvec.tolist())}
    H = np.zeros((nvec, w, w), dtype=np.complex128)
    done = set()
    for i, r in enumerate(rvec.tolist()):
        key = tuple(r)
        if key == (0, 0, 0) or key in done:
            continue
        mkey = (-r[0], -r[1], -r[2])
        Rc = r[0] * rlat[0] + r[1] * rlat[1] + r[2] * rlat[2]
        scale = hop_scale * math.exp(-np.linalg.norm(Rc) / A_LAT)
        M = (rng.standard_normal((w, w)) + 1j * rng.standard_normal((w, w))) * scale
        H[i] = M
        H[index[mkey]] = M.conj().T
        done.add(key)
        done.add(mkey)
    i0 = index[(0, 0, 0)]
    nlo = w // 2
    lo = rng.uniform(onsite_lo[0] - onsite_lo[1], onsite_lo[0] + onsite_lo[1], nlo)
    hi = rng.uniform(onsite_hi[0] - onsite_hi[1], onsite_hi[0] + onsite_hi[1], w - nlo)
    onsite = np.concatenate([lo, hi])
    U = (rng.standard_normal((w, w)) + 1j * rng.standard_normal((w, w))) * h0_scale
    H0 = np.triu(U, 1)
    H0 = H0 + H0.conj().T
    H0[np.diag_indices(w)] = onsite
    H[i0] = H0
    return TBModel(systype="NP", scs=0.0, efermi=0.0, rlat=rlat, w=w, rvec=rvec,
                   deg=np.ones(nvec, dtype=np.int32),
                   hre=np.ascontiguousarray(H.real), him=np.ascontiguousarray(H.imag))


def _bands_on_mesh(model: TBModel, n: int) -> np.ndarray:
    """Exact (double, no float32 phase) band energies on an n x n mesh: for the gap check only."""
    b = 2 * math.pi * np.linalg.inv(model.rlat).T
    Rc = model.rvec @ model.rlat
    H = model.hre + 1j * model.him
    ev = []
    for i in range(n):
        for j in range(n):
            k = b[0] * i / n + b[1] * j / n
            ph = np.exp(1j * (Rc @ k))
            Hk = np.tensordot(ph, H, axes=(0, 0))
            ev.append(np.linalg.eigvalsh(Hk))
    return np.array(ev)


def qwz_model(u: float = -1.0, a: float = 1.0) -> TBModel:
    """Qi-Wu-Zhang two-band Chern insulator on a square lattice (lattice constant a):
    H(k) = sin(k_x a) sx + sin(k_y a) sy + (u + cos(k_x a) + cos(k_y a)) sz, i.e. H(0) = u sz,
    H(+x) = (sz - i sx)/2, H(+y) = (sz - i sy)/2 and H(-R) = H(R)^dagger. The lower band has
    Chern number +-1 for 0 < |u| < 2 and 0 for |u| > 2 (a known-answer model for the Berry
    curvature; E_F = 0 lies in the gap)."""
    sx = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    sy = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    sz = np.array([[1, 0], [0, -1]], dtype=np.complex128)
    hx = 0.5 * sz - 0.5j * sx
    hy = 0.5 * sz - 0.5j * sy
    cells = [((0, 0, 0), u * sz), ((1, 0, 0), hx), ((-1, 0, 0), hx.conj().T),
             ((0, 1, 0), hy), ((0, -1, 0), hy.conj().T)]
    rvec = np.array([c[0] for c in cells], dtype=np.int32)
    H = np.array([c[1] for c in cells])
    return TBModel(systype="NP", scs=0.0, efermi=0.0,
                   rlat=np.array([[a, 0.0, 0.0], [0.0, a, 0.0], [0.0, 0.0, 20.0]]), w=2, rvec=rvec,
                   deg=np.ones(len(cells), dtype=np.int32), hre=H.real.copy(), him=H.imag.copy())


def make_gapped_model(w: int, n_shell: int, onsite_lo: tuple, onsite_hi: tuple,
                      seed: int, check_mesh: int = 12, max_tries: int = 64) -> TBModel:
    """Re-seed (seed, seed+1, ...) until nocp = w/2 at every k of the check mesh and the gap > 0."""
    for t in range(max_tries):
        m = make_hex_model(w, n_shell, onsite_lo, onsite_hi, seed + t)
        ev = _bands_on_mesh(m, check_mesh)
        nneg = (ev <= 0.0).sum(axis=1)
        if np.all(nneg == w // 2) and ev[:, w // 2].min() > ev[:, w // 2 - 1].max():
            return m
    raise RuntimeError("no gapped synthetic model found")


# Seeded workloads: sizes follow the five benchmark configurations of this path.
CONFIGS = {
    # w, shells, onsite (centre, half-width) low / high, seed
    "c1": dict(w=8, n_shell=3, lo=(-1.5, 0.3), hi=(1.5, 0.3), seed=1001),
    "c2": dict(w=24, n_shell=5, lo=(-1.8, 0.4), hi=(1.8, 0.4), seed=2001),
    "c4_w8": dict(w=8, n_shell=4, lo=(-1.5, 0.3), hi=(1.5, 0.3), seed=4008),
    "c4_w16": dict(w=16, n_shell=4, lo=(-1.5, 0.3), hi=(1.5, 0.3), seed=4016),
    "c4_w24": dict(w=24, n_shell=4, lo=(-1.5, 0.3), hi=(1.5, 0.3), seed=4024),
    "c4_w40": dict(w=40, n_shell=4, lo=(-1.5, 0.3), hi=(1.5, 0.3), seed=4040),
}


def config_model(name: str) -> TBModel:
    c = CONFIGS[name]
    return make_gapped_model(c["w"], c["n_shell"], c["lo"], c["hi"], c["seed"])


def _fmt(x: float) -> str:
    return repr(float(x))


def params_text(model: TBModel, header: str = "synthetic hexagonal model") -> str:
    """Render ``model`` in the params-file layout (full double precision)."""
    out = io.StringIO()
    out.write(f"{model.systype}\n{_fmt(model.scs)}\n{_fmt(model.efermi)}\n")
    for i in range(3):
        out.write(" ".join(_fmt(v) for v in model.rlat[i]) + "\n")
    out.write(header + "\n")
    out.write(f"{model.w}\n{model.nvec}\n")
    deg = model.deg.tolist()
    for s in range(0, len(deg), 15):
        out.write(" ".join(f"{d:4d}" for d in deg[s:s + 15]) + "\n")
    for i in range(model.nvec):
        r = model.rvec[i]
        for n in range(model.w):
            for m in range(model.w):
                out.write(f"{r[0]:5d}{r[1]:5d}{r[2]:5d}{m + 1:5d}{n + 1:5d} "
                          f"{_fmt(model.hre[i, m, n])} {_fmt(model.him[i, m, n])}\n")
    return out.getvalue()


def write_params(model: TBModel, path: str, header: str = "synthetic hexagonal model") -> None:
    with open(path, "w") as f:
        f.write(params_text(model, header))


def _tokens_fortran(line: str) -> list:
    """Split one record the way list-directed input does (blanks/commas; '!' is not special,
    but trailing non-numeric text after the needed values is ignored by the callers)."""
    return line.replace(",", " ").split()


def read_params(path: str) -> TBModel:
    """Parse a params file like ``hamiltonian_input_read`` (module_input_read.f90:32-176).

    Supports the default single-block layout and the SP (spin-polarised up/down) merge
    (module_input_read.f90:56-142)."""
    with open(path) as f:
        lines = f.read().splitlines()
    pos = 0

    def rec():
        nonlocal pos
        while pos < len(lines) and lines[pos].strip() == "":
            pos += 1
        if pos >= len(lines):
            raise ValueError("params file ended early")
        s = lines[pos]
        pos += 1
        return s

    def read_ints(n):
        vals = []
        while len(vals) < n:
            vals.extend(int(t) for t in _tokens_fortran(rec()))
        return np.array(vals[:n], dtype=np.int32)

    systype = _tokens_fortran(rec())[0][:4]
    scs = float(_tokens_fortran(rec())[0])
    efermi = float(_tokens_fortran(rec())[0])
    rlat = np.array([[float(t) for t in _tokens_fortran(rec())[:3]] for _ in range(3)])

    def block():
        rec()  # header
        w = int(_tokens_fortran(rec())[0])
        nvec = int(_tokens_fortran(rec())[0])
        deg = read_ints(nvec)
        rvec = np.zeros((nvec, 3), dtype=np.int32)
        hre = np.zeros((nvec, w, w))
        him = np.zeros((nvec, w, w))
        for i in range(nvec):
            for n in range(w):
                for m in range(w):
                    t = _tokens_fortran(rec())
                    rvec[i] = (int(t[0]), int(t[1]), int(t[2]))
                    hre[i, m, n] = float(t[5])
                    him[i, m, n] = float(t[6])
        return w, rvec, deg, hre, him

    if systype.strip() == "SP":
        wu, ru, du, hru, hiu = block()
        wd, rd, dd, hrd, hid = block()
        w = wu + wd
        nvec = ru.shape[0] + rd.shape[0]
        hre = np.zeros((nvec, w, w))
        him = np.zeros((nvec, w, w))
        hre[:ru.shape[0], :wu, :wu] = hru
        him[:ru.shape[0], :wu, :wu] = hiu
        hre[ru.shape[0]:, wu:, wu:] = hrd
        him[ru.shape[0]:, wu:, wu:] = hid
        return TBModel(systype, scs, efermi, rlat, w, np.concatenate([ru, rd]),
                       np.concatenate([du, dd]), hre, him)
    w, rvec, deg, hre, him = block()
    return TBModel(systype, scs, efermi, rlat, w, rvec, deg, hre, him)
