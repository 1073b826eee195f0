"""End to end through the deck-level driver (wtb_bse < deck): the output files of a BSE=T,
SPEC=T, CPOL=T, DTDIAG=T, BSE_WF=T run and of a BSE_BND=T run against the CPU oracle."""
import os
import subprocess

import numpy as np
import pytest

from oracle import wtb_oracle as O
from oracle.deck import parse_deck
from wantibexos_b200 import build as B
from wantibexos_b200 import synth

pytestmark = pytest.mark.gpu


def run_deck(tmp_path, text):
    B.build()
    r = subprocess.run([B.DRIVER_EXE], input=text.encode(), capture_output=True, cwd=str(tmp_path), timeout=600)
    assert r.returncode == 0, r.stderr.decode()


def rows(path, skip=1):
    out = []
    for line in open(path).read().splitlines()[skip:]:
        if line.strip():
            out.append([float(x) for x in line.split()])
    return np.array(out)


def deck_for(tmp_path, extra=""):
    return f"""BSE= T
SPEC= T
NGX= 8
NGY= 8
NGZ= 1
NBANDSV= 2
NBANDSC= 2
COULOMB_POT= V2DRK
R_0= 40
KTOL= 0.001
CSHIFT= 0.05
ENSPECI= 0
ENSPECF= 5
NESPEC= 501
DTDIAG= T
CPOL= T
BSE_WF= T
EXC_WF_I= 1
EXC_WF_F= 2
SYSDIM= "2D"
OUTPUT= "{tmp_path}/"
CALC_DATA= "{tmp_path}/"
PARAMS_FILE= "{tmp_path}/tb.dat"
{extra}"""


def test_bse_run_files(tmp_path):
    m = synth.config_model("c1")
    synth.write_params(m, str(tmp_path / "tb.dat"))
    text = deck_for(tmp_path)
    run_deck(tmp_path, text)
    deck = parse_deck(text)
    ref = O.run_bse(m, deck)
    # bse_opt_diel.dat: W and the six tensor components (F15.4)
    got = rows(tmp_path / "bse_opt_diel.dat")
    want = O.roundtrip_f154(np.column_stack([ref["W"], ref["act"][:, :6]]))
    d = np.abs(got - want)
    assert d.max() <= 1.0001e-4 and (d > 0).sum() <= 3
    got_pol = rows(tmp_path / "bse_opt_diel-pol.dat")
    want_pol = O.roundtrip_f154(np.column_stack([ref["W"], ref["act"][:, [0, 1, 2, 6, 7]]]))
    assert np.abs(got_pol - want_pol).max() <= 1.0001e-4
    # sp_optics.dat: the sorted single-particle table
    sp = O.sp_table(ref["kpts"], ref["eigv"], ref["nocp"], ref["h"], 2, 2)
    got_sp = rows(tmp_path / "sp_optics.dat")
    want_sp = O.roundtrip_f154(sp[:, 6:13].astype(np.float64))
    assert np.abs(got_sp - want_sp).max() <= 1.0001e-4
    # bse_diel_xx.dat from the oracle's file values
    dl = O.bsedielraw(m.systype, m.rlat, ref["ngrid"], want[:, 0], want[:, 1:], 0.0, 5.0, 501.0, deck["cshift"], True)
    for name in ("xx", "yy", "xy"):
        g = rows(tmp_path / f"bse_diel_{name}.dat")
        assert g.shape == (501, 3)
        assert np.abs(g[:, 0] - dl[name][:, 0]).max() < 1e-12
        scale = np.abs(dl[name][:, 1:]).max()
        assert np.abs(g[:, 1:] - dl[name][:, 1:]).max() <= 4e-7 * scale, name
    # post-processing and lifetime files exist with one row per photon energy / exciton
    for f in ("bse_refractive_index.dat", "bse_extinction_coef.dat", "bse_reflectibility.dat",
              "bse_absorption_coef.dat", "bse_en_loss_func.dat", "sp_diel_xx.dat", "sp_refractive_index.dat",
              "bse_diel-pol_sp.dat", "bse_absorption_coef-pol.dat", "sp_diel-pol_sm.dat"):
        assert rows(tmp_path / f).shape[0] == 501, f
    lt = open(tmp_path / "exciton_lifetime.dat").read().splitlines()
    assert len(lt) == 1 + ref["W"].shape[0]
    n, k = O.optprop(dl["xx"][:, 1], dl["xx"][:, 2], dl["xx"][:, 0])[:2]
    g = rows(tmp_path / "bse_refractive_index.dat")
    assert np.abs(g[:, 1] - O.roundtrip_f154(n)).max() <= 1.0001e-4
    # exciton wave-function files
    A1 = open(tmp_path / "exc_wf_1.dat").read().splitlines()
    assert len(A1) == 7 + ref["W"].shape[0]


def test_bse_band_structure_file(tmp_path):
    m = synth.config_model("c1")
    synth.write_params(m, str(tmp_path / "tb.dat"))
    (tmp_path / "kp.dat").write_text("2\n4\n0.0 0.0 0.0\n0.5 0.0 0.0\n")
    text = f"""BSE_BND= T
NGX= 5
NGY= 5
NGZ= 1
NBANDSV= 2
NBANDSC= 2
COULOMB_POT= V2DRK
R_0= 40
KTOL= 0.001
OUTPUT= "{tmp_path}/"
CALC_DATA= "{tmp_path}/"
PARAMS_FILE= "{tmp_path}/tb.dat"
KPATH_BSE= "{tmp_path}/kp.dat"
"""
    run_deck(tmp_path, text)
    deck = parse_deck(text)
    exk, qpath, labels = O.run_bsebnds(m, deck, [(0, 0, 0), (0.5, 0, 0)], 4)
    got = [ln.split() for ln in open(tmp_path / "bands_bse.dat").read().splitlines() if ln.strip()]
    got = np.array([[float(a) for a in r] for r in got])
    N = exk.shape[0]
    assert got.shape == (N * 4, 2)
    assert np.abs(got[:, 1] - exk.reshape(-1)).max() < 1e-9
    assert np.array_equal(got[:4, 0].astype(np.float32), qpath[:, 0].astype(np.float32))


def test_temperature_bse_run_files(tmp_path):
    """BSET=T (bsesolvertemp): bse_opt_diel.dat and sp_optics.dat with the occupation factors
    and the TA= VE scissors, the temperature line in log_bse-diel.dat, no lifetime files."""
    m = synth.config_model("c1")
    synth.write_params(m, str(tmp_path / "tb.dat"))
    text = deck_for(tmp_path, "TEMP= 4000\nTA= VE\nST= 2.0\nPHAVG= 0.02\n").replace("BSE= T", "BSET= T")
    run_deck(tmp_path, text)
    deck = parse_deck(text)
    ref = O.run_bse(m, deck)
    got = rows(tmp_path / "bse_opt_diel.dat")
    want = O.roundtrip_f154(np.column_stack([ref["W"], ref["act"][:, :6]]))
    d = np.abs(got - want)
    assert d.max() <= 1.0001e-4 and (d > 0).sum() <= 3
    sp = O.sp_table(ref["kpts"], ref["eigv"], ref["nocp"], ref["h"], 2, 2, fdeh=ref["fdeh"])
    got_sp = rows(tmp_path / "sp_optics.dat")
    assert np.abs(got_sp - O.roundtrip_f154(sp[:, 6:13].astype(np.float64))).max() <= 1.0001e-4
    log = open(tmp_path / "log_bse-diel.dat").read()
    assert " temperature" in log
    assert (tmp_path / "bse_diel_xx.dat").exists() and not (tmp_path / "exciton_lifetime.dat").exists()
    assert "with temperature, finished" in open(tmp_path / "log.dat").read()
