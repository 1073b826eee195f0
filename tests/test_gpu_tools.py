"""Tools that share the per-k eigensolver (the next rows after the BSE path): eigsys for every
band, the DOS smearing kernel, the Berry curvature (berryct2), and the deck-level
band-structure (BANDS=T), DOS (DOS=T) and Berry-curvature (BERRY=T, BERRY_BZ=T) runs against
the CPU oracle."""
import copy
import subprocess

import numpy as np
import pytest

from oracle import wtb_oracle as O
from wantibexos_b200 import build as B
from wantibexos_b200 import synth

pytestmark = pytest.mark.gpu


def test_eigsys_every_band_matches_oracle(gpu_ctx):
    m = synth.config_model("c1")
    kpts = O.monkhorst_pack(5, 5, 1, [0, 0, 0], m.rlat)
    gpu_ctx.set_model(m)
    e, v, no = gpu_ctx.eigsys(kpts)
    for k in range(kpts.shape[0]):
        er, Ur, nr = O.eigsys(m, kpts[k])
        assert no[k] == nr
        assert np.abs(e[k] - er).max() < 1e-8
        sign = np.sign(v[k, :, 0].real * Ur[:, 0].real)
        assert np.abs(v[k] - Ur * sign[:, None]).max() < 1e-9


def test_dos_kernel_matches_numpy(gpu_ctx):
    rng = np.random.default_rng(3)
    etb = rng.uniform(-3, 3, 5000)
    wts = rng.uniform(0, 1, (5000, 3))
    en = np.linspace(-3.5, 3.5, 301)
    gpu_ctx.set_model(synth.config_model("c1"))
    got = gpu_ctx.dos(etb, wts, 250, en, 0.05)
    want = (O.gaussian(en[:, None] - etb[None, :], 0.05) @ wts) / 250.0
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_berry_curvature_matches_oracle(gpu_ctx):
    """wtbg_berry (berryct2 on the device) against the oracle restatement, c1 and QWZ models."""
    cases = [(synth.config_model("c1"), 4), (synth.qwz_model(-1.0), 6)]
    for m, n in cases:
        kp = O.monkhorst_pack(n, n, 1, [0, 0, 0], m.rlat) + np.array([0.013, -0.021, 0.0])
        gpu_ctx.set_model(m)
        got = gpu_ctx.berry(kp)
        want = np.array([[x.imag for x in O.berryct2(m, k, *O.eigsys(m, k))] for k in kp])
        assert np.abs(got - want).max() <= 1e-9 * max(1.0, np.abs(want).max())


def test_berry_curvature_chern_numbers_on_device(gpu_ctx):
    """Known answer: the QWZ lower band has Chern number +1, -1, 0 for u = -1, +1, -3."""
    for u, chern in ((-1.0, 1.0), (1.0, -1.0), (-3.0, 0.0)):
        m = synth.qwz_model(u)
        gpu_ctx.set_model(m)
        kp = O.monkhorst_pack(48, 48, 1, [0, 0, 0], m.rlat)
        b = gpu_ctx.berry(kp)
        b1, b2, _ = O.recvec(m.rlat[0], m.rlat[1], m.rlat[2])
        area = abs(np.cross(b1, b2)[2])
        assert abs(b[:, 1].sum() * area / len(kp) / (2 * np.pi) - chern) < 1e-4
        assert np.abs(b[:, [0, 3, 5]]).max() < 1e-12   # diagonal components are real


def test_berry_tool_runs_match_oracle(tmp_path):
    """BERRY=T (berry_curv_kpath.dat, KLABELS.dat) and BERRY_BZ=T (berry_curv_bz.dat) decks."""
    m = synth.config_model("c1")
    synth.write_params(m, str(tmp_path / "tb.dat"))
    ks = [(0, 0, 0), (0.5, 0, 0), (0.5, 0, 0), (1 / 3, 1 / 3, 0)]
    (tmp_path / "kpath.dat").write_text("4\n6\n" + "\n".join(f"{a:.10f} {b:.10f} {c:.10f}" for a, b, c in ks) + "\n")
    text = f"""BERRY= T
BERRY_BZ= T
NGX= 5
NGY= 5
NGZ= 1
OUTPUT= "{tmp_path}/"
CALC_DATA= "{tmp_path}/"
PARAMS_FILE= "{tmp_path}/tb.dat"
KPATH_FILE= "{tmp_path}/kpath.dat"
"""
    _run(tmp_path, text)
    kin = [tuple(float(x) for x in l.split()) for l in (tmp_path / "kpath.dat").read_text().splitlines()[2:]]
    want, labels = O.berry_kpath(m, kin, 6)
    lines = (tmp_path / "berry_curv_kpath.dat").read_text().splitlines()
    assert lines[0].split() == ["kp", "yz", "xz", "xy"]
    got = np.array([[float(x) for x in l.split()] for l in lines[1:]])
    assert got.shape == want.shape
    assert np.abs(got - np.round(want, 4)).max() <= 1.0001e-4
    assert np.allclose(_floats(tmp_path / "KLABELS.dat").ravel(), np.array(labels, dtype=np.float32), rtol=1e-6)
    wb = O.berry_bz(m, [5, 5, 1], [0, 0, 0])
    lines = (tmp_path / "berry_curv_bz.dat").read_text().splitlines()
    assert lines[0].split() == ["kx", "ky", "kz", "yz", "xz", "xy"]
    gb = np.array([[float(x) for x in l.split()] for l in lines[1:]])
    assert gb.shape == wb.shape
    assert np.abs(gb - np.round(wb, 4)).max() <= 1.0001e-4


def test_sp_optics_tools_match_oracle(tmp_path):
    """OPT_BZ=T (bz_act_*.dat, dichroism.dat against the oracle) and DIEL=T (sp_optics files
    identical to those of a BSE=T run on the same deck)."""
    m = synth.config_model("c1")
    synth.write_params(m, str(tmp_path / "tb.dat"))
    common = f"""NGX= 5
NGY= 5
NGZ= 1
NBANDSV= 2
NBANDSC= 2
CSHIFT= 0.05
TMCOEF= T
CALC_DATA= "{tmp_path}/"
PARAMS_FILE= "{tmp_path}/tb.dat"
"""
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    _run(tmp_path, "OPT_BZ= T\nDIEL= T\n" + common + f'OUTPUT= "{tmp_path}/a/"\n')
    want = O.sp_optbz(m, [5, 5, 1], [0, 0, 0], 2, 2, float(np.float32(0.05)))
    for c, name in enumerate(["x", "y", "z", "sp", "sm"]):
        got = _floats(tmp_path / "a" / f"bz_act_{name}.dat")
        assert got.shape == (25, 4)
        assert np.array_equal(got[:, :3].astype(np.float32), want[:, :3].astype(np.float32))
        assert np.allclose(got[:, 3], want[:, 3 + c], rtol=1e-10, atol=0)
    got = _floats(tmp_path / "a" / "dichroism.dat")
    assert np.allclose(got[:, 3], want[:, 8], rtol=1e-9, atol=1e-12)
    _run(tmp_path, "BSE= T\n" + common + "COULOMB_POT= V2DRK\nR_0= 40\n" + f'OUTPUT= "{tmp_path}/b/"\n')
    for f in ["sp_optics.dat", "sp_optics-pol.dat", "tm_coef.dat", "tm_coef-pol.dat"]:
        assert (tmp_path / "a" / f).read_text() == (tmp_path / "b" / f).read_text(), f


def _run(tmp_path, text):
    B.build()
    r = subprocess.run([B.DRIVER_EXE], input=text.encode(), capture_output=True, cwd=str(tmp_path), timeout=600)
    assert r.returncode == 0, r.stderr.decode()


def _floats(path, skip_hash=True):
    rows = []
    for line in open(path).read().splitlines():
        t = line.split()
        if not t or (skip_hash and t[0].startswith("#")):
            continue
        rows.append([float(x) for x in t])
    return np.array(rows)


@pytest.mark.parametrize("systype", ["NP", "SOC"])
def test_band_and_dos_runs_match_oracle(tmp_path, systype):
    m = copy.copy(synth.config_model("c1"))
    m.systype = systype
    synth.write_params(m, str(tmp_path / "tb.dat"))
    ow = np.linspace(0.2, 1.0, m.w)
    (tmp_path / "orbw.dat").write_text("\n".join(f"{x:.6f}" for x in ow) + "\n")
    ks = [(0, 0, 0), (0.5, 0, 0), (0.5, 0, 0), (1 / 3, 1 / 3, 0)]
    (tmp_path / "kpath.dat").write_text("4\n7\n" + "\n".join(f"{a:.10f} {b:.10f} {c:.10f}" for a, b, c in ks) + "\n")
    text = f"""BANDS= T
DOS= T
NGX= 6
NGY= 6
NGZ= 1
NEDOS= 201
SIGMA= 0.08
OUTPUT= "{tmp_path}/"
CALC_DATA= "{tmp_path}/"
PARAMS_FILE= "{tmp_path}/tb.dat"
KPATH_FILE= "{tmp_path}/kpath.dat"
ORB_W= "{tmp_path}/orbw.dat"
"""
    _run(tmp_path, text)
    kin = [tuple(float(x) for x in l.split()) for l in (tmp_path / "kpath.dat").read_text().splitlines()[2:]]
    want, labels = O.bandstool(m, kin, 7, orbw=[float(f"{x:.6f}") for x in ow])
    got = _floats(tmp_path / "bands.dat")
    assert got.shape == (m.w * want.shape[1], 4)
    assert np.allclose(got, want.reshape(-1, 4), rtol=2e-6, atol=2e-6)
    assert np.allclose(_floats(tmp_path / "KLABELS.dat").ravel(), np.array(labels, dtype=np.float32), rtol=1e-6)
    dd = O.dostool(m, [6, 6, 1], [0, 0, 0], 201.0, float(np.float32(0.08)), orbw=[float(f"{x:.6f}") for x in ow])
    gd = _floats(tmp_path / "dos.dat")
    assert gd.shape == dd.shape
    assert np.abs(gd - np.round(dd, 4)).max() <= 1.0001e-4
