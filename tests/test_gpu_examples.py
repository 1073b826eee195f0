"""The reference's own example decks through the drop-in (wtb_bse < deck) against the oracle
fixtures (tests/golden/make_examples.py): MoS2 with spin-orbit coupling (w = 22, 147 cells,
near-degenerate Kramers pairs 5.6e-6 eV apart in the band window) for BSE+SPEC (example 3),
BSE_WF (example 6), BSET (example 7), BSE_BND (example 5) and BERRY (example 4), and graphene
(w = 5, 1615 cells) for BANDS with orbital weights (example 1).  The k-meshes are reduced
(RK= 16 and 12) so that the oracle numbers are cheap to make."""
import gzip
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import wtb_oracle as O
from wantibexos_b200 import build as B

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_examples as X  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(HERE, "golden", "examples_golden.npz"))


def params(tmp_path, name):
    p = tmp_path / (name + ".dat")
    with gzip.open(os.path.join(HERE, "golden", name + ".dat.gz"), "rb") as f:
        p.write_bytes(f.read())
    return str(p)


def run(tmp_path, template, model, **kw):
    """wtb_bse < deck in tmp_path; the deck names its files relative to the working directory
    (the reference reads every path into a character(len=70) variable)."""
    B.build()
    out = tmp_path / "out"
    out.mkdir(exist_ok=True)
    params(tmp_path, model)
    text = template.format(out="./out/", params=model + ".dat", **kw)
    r = subprocess.run([B.DRIVER_EXE], input=text.encode(), capture_output=True, cwd=str(tmp_path), timeout=600)
    assert r.returncode == 0, r.stderr.decode()
    return out


def rows(path):
    """Numeric rows of an output file (header lines, with or without '#', skipped)."""
    out = []
    for line in open(path).read().splitlines():
        t = line.split()
        if not t or t[0].startswith("#"):
            continue
        try:
            out.append([float(x) for x in t])
        except ValueError:
            continue
    return np.array(out)


def check_opt_diel(path, W, act, cols):
    got = rows(path)
    want = O.roundtrip_f154(np.column_stack([W] + [act[:, c] for c in cols]))
    d = np.abs(got - want)
    assert got.shape == want.shape
    assert d.max() <= 1.0001e-4 and (d > 0).sum() <= 3, d.max()
    return got


@pytest.fixture(scope="module")
def ex6(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("ex6")
    return run(tmp, X.EX6, "tb_mos2")


def test_example3_bse_files(ex6):
    out = ex6
    got = check_opt_diel(out / "bse_opt_diel.dat", GOLD["ex3_W"], GOLD["ex3_act"], range(6))
    mos2 = X.model("tb_mos2")
    ng = GOLD["ex3_ngrid"]
    d = X.deck(X.EX3)
    # spectrum: from the drop-in's own F15.4 rows (isolates the spectrum kernel), then against
    # the fixture built from the oracle's rows
    mine = O.bsedielraw(mos2.systype, mos2.rlat, ng, got[:, 0], got[:, 1:], d["ebse0"], d["ebsef"], d["numbse"],
                        d["cshift"], d["renorm"])
    for c in ("xx", "yy", "xy"):
        g = rows(out / f"bse_diel_{c}.dat")
        gold = GOLD["ex3_eps_" + c]
        assert np.array_equal(g[:, 0], gold[:, 0])
        scale = np.abs(gold[:, 1:]).max()
        assert np.abs(g[:, 1:] - mine[c][:, 1:]).max() <= 4 * np.spacing(np.float32(scale)), c
        assert np.abs(g[:, 1:] - gold[:, 1:]).max() <= 1e-4 * scale, c
    # post-processing: every optical-constant file from the diel files as written
    e = {c: rows(out / f"bse_diel_{c}.dat") for c in ("xx", "yy", "zz", "xy", "xz", "yz")}
    for q, name in enumerate(("refractive_index", "extinction_coef", "reflectibility", "absorption_coef",
                              "en_loss_func")):
        f = rows(out / f"bse_{name}.dat")
        assert f.shape == (6001, 7), name
        assert np.abs(f[:, 0] - O.roundtrip_f154(e["xx"][:, 0])).max() <= 1.0001e-4
        for k, c in enumerate(("xx", "yy", "zz", "xy", "xz", "yz")):
            want = O.roundtrip_f154(O.optprop(e[c][:, 1], e[c][:, 2], e[c][:, 0])[q])
            have = f[:, 1 + k]
            fin = np.isfinite(want)
            assert np.array_equal(fin, np.isfinite(have)), (name, c)
            if fin.any():
                assert np.abs(have[fin] - want[fin]).max() <= 1.0001e-4, (name, c)
    # lifetimes (exclft, 2D) of the rounded file values
    lt = rows(out / "exciton_lifetime.dat")
    assert lt.shape == (got.shape[0], 5)
    E = got[:, 0]
    F = got[:, 1:4]
    cols = [F.sum(axis=1), F[:, 0], F[:, 1], F[:, 2]]
    for k, f in enumerate(cols):
        want = O.exclft("2D", ng, mos2.rlat, f, E)
        fin = np.isfinite(want)
        assert np.array_equal(fin, np.isfinite(lt[:, 1 + k])), k
        # E15.4 keeps four significant digits: relative rounding up to 5e-4
        assert fin.sum() == 0 or np.all(np.abs(lt[fin, 1 + k] - want[fin]) <= 5.01e-4 * np.abs(want[fin])), k


def test_example3_single_particle_table(ex6):
    mos2 = X.model("tb_mos2")
    r = O.run_bse(mos2, X.deck(X.EX3))
    sp = O.sp_table(r["kpts"], r["eigv"], r["nocp"], r["h"], 2, 2)
    got = rows(ex6 / "sp_optics.dat")
    assert np.abs(got - O.roundtrip_f154(sp[:, 6:13].astype(np.float64))).max() <= 1.0001e-4


def test_example6_exciton_wave_functions(ex6):
    """exc_wf_1..10.dat: per basis state |A|^2 (gauge invariant: the reference's vector phase and
    the per-k band signs drop out) against the oracle's ZHEEV vectors, and the header lines."""
    N = GOLD["ex3_W"].shape[0]
    for n in range(1, 11):
        lines = open(ex6 / f"exc_wf_{n}.dat").read().splitlines()
        assert lines[0].split()[-1] == str(n)
        assert abs(float(lines[1].split(":")[1]) - GOLD["ex3_W"][n - 1]) < 1e-9
        a = rows(ex6 / f"exc_wf_{n}.dat")
        assert a.shape == (N, 8)
        a2 = a[:, 6] ** 2 + a[:, 7] ** 2
        want = GOLD["ex3_A10_abs2"][:, n - 1]
        assert np.abs(a2 - want).max() <= 3e-4 * want.max(), n
        # basis labels: nocp (14 for MoS2), conduction and valence band numbers
        assert set(a[:, 0].astype(int)) == {14}
        assert set(a[:, 4].astype(int)) == {15, 16} and set(a[:, 5].astype(int)) == {13, 14}


def test_example7_temperature_bse(tmp_path):
    out = run(tmp_path, X.EX7, "tb_mos2")
    check_opt_diel(out / "bse_opt_diel.dat", GOLD["ex7_W"], GOLD["ex7_act"], range(6))
    assert " temperature" in open(out / "log_bse-diel.dat").read()


def test_example5_exciton_band_structure(tmp_path):
    (tmp_path / "kp.dat").write_text(X.kpath_text(5))
    out = run(tmp_path, X.EX5, "tb_mos2", kpath="kp.dat")
    exk = GOLD["ex5_exk"]
    got = rows(out / "bands_bse.dat")
    N, nq = exk.shape
    assert got.shape == (N * nq, 2)
    assert np.abs(got[:, 1] - exk.reshape(-1)).max() < 1e-9
    assert np.array_equal(got[:nq, 0].astype(np.float32), GOLD["ex5_qpath"][:, 0].astype(np.float32))


def test_example4_berry_curvature_path(tmp_path):
    (tmp_path / "kp.dat").write_text(X.kpath_text(50))
    out = run(tmp_path, X.EX4, "tb_mos2", kpath="kp.dat")
    want = GOLD["ex4_berry"]
    got = rows(out / "berry_curv_kpath.dat")
    assert got.shape == want.shape
    assert np.all(np.abs(got - np.round(want, 4)) <= 1.0001e-4 + 1e-9 * np.abs(want))


def test_example1_graphene_bands_with_orbital_weights(tmp_path):
    (tmp_path / "kp.dat").write_text(X.kpath_text(50))
    (tmp_path / "c1.dat").write_text("".join(f"{v}\n" for v in X.ORBW_C1))
    out = run(tmp_path, X.EX1, "tb_graphene", kpath="kp.dat", orbw="c1.dat")
    want = GOLD["ex1_bands"]
    got = rows(out / "bands.dat")
    assert got.shape == (want.shape[0] * want.shape[1], 4)
    assert np.allclose(got, want.reshape(-1, 4), rtol=2e-6, atol=2e-6)
