"""Deck-level selection of the solver forms through wtb_run (libwtbdriver.so):
GPU_SOLVER= DAVIDSON with GPU_PRECISION= BF16X3 against the dense FP64 run of the same deck,
and the dense fallback when the Davidson residual fails (GPU_MAXIT= 2), whose files must be
identical to the dense run's.  Both decks run in this process, so the two dense solves share
the tuned mat-vec chunk and are bit-identical."""
import ctypes as C
import os

import numpy as np
import pytest

from wantibexos_b200 import build as B
from wantibexos_b200 import synth

pytestmark = pytest.mark.gpu

DECK = """BSE= T
SPEC= T
NGX= 10
NGY= 10
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
OUTPUT= "{d}/"
CALC_DATA= "{d}/"
PARAMS_FILE= "{p}"
{extra}"""

FILES = ["bse_opt_diel.dat", "bse_opt_diel-pol.dat", "sp_optics.dat", "bse_diel_xx.dat", "bse_diel_yy.dat",
         "bse_diel_xy.dat", "bse_diel-pol_sp.dat", "bse_refractive_index.dat", "bse_absorption_coef.dat",
         "exciton_lifetime.dat", "exciton_lifetime-pol.dat", "exc_wf_1.dat", "exc_wf_2.dat"]


def wtb_run(text):
    B.build()
    lib = C.CDLL(B.DRIVER_LIB)
    lib.wtb_run.restype = C.c_int
    lib.wtb_run.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_char_p, C.c_int]
    err = C.create_string_buffer(512)
    rc = lib.wtb_run(text.encode(), 0, None, err, 512)
    assert rc == 0, err.value.decode()


def rows(path):
    out = []
    for ln in open(path).read().splitlines():
        t = ln.split()
        if t and not t[0].startswith("#"):
            out.append([float(x) for x in t])
    return np.array(out)


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    base = tmp_path_factory.mktemp("forms")
    p = str(base / "tb.dat")
    synth.write_params(synth.config_model("c1"), p)
    out = {}
    for name, extra in (("dense", ""),
                        ("fast", "GPU_SOLVER= DAVIDSON\nGPU_PRECISION= BF16X3\n"),
                        ("fallback", "GPU_SOLVER= DAVIDSON\nGPU_MAXIT= 2\n")):
        d = base / name
        d.mkdir()
        wtb_run(DECK.format(d=d, p=p, extra=extra))
        out[name] = d
    return out


def test_fallback_files_identical_to_dense(runs):
    log = open(runs["fallback"] / "log_bse-diel.dat").read()
    assert "dense FP64 solve used" in log
    for f in FILES:
        a = open(runs["dense"] / f).read()
        b = open(runs["fallback"] / f).read()
        assert a == b, f


def test_fast_form_matches_dense_run(runs):
    log = open(runs["fast"] / "log_bse-diel.dat").read()
    assert "fast form: lowest" in log and "dense FP64 solve used" not in log
    dense = rows(runs["dense"] / "bse_opt_diel.dat")
    fast = rows(runs["fast"] / "bse_opt_diel.dat")
    assert fast.shape == (32, 7)
    # energies within 0.5 meV (the F15.4 rounding is 0.05 meV); strengths of non-degenerate states
    assert np.abs(fast[:, 0] - dense[:32, 0]).max() <= 5e-4
    # eps2 of xx and yy within 1e-3 of max eps2 at the dense spectrum's peaks
    for c in ("xx", "yy"):
        a = rows(runs["dense"] / f"bse_diel_{c}.dat")
        b = rows(runs["fast"] / f"bse_diel_{c}.dat")
        assert np.array_equal(a[:, 0], b[:, 0])
        e2 = a[:, 2]
        pk = np.where((e2[1:-1] > e2[:-2]) & (e2[1:-1] >= e2[2:]))[0] + 1
        assert np.abs(b[pk, 2] - e2[pk]).max() <= 1e-3 * np.abs(e2).max(), c
    # single-particle table: the precision form's bands differ from FP64 by ~1e-5 eV at most
    assert np.abs(rows(runs["dense"] / "sp_optics.dat") - rows(runs["fast"] / "sp_optics.dat")).max() <= 2.0001e-4
    # exciton wave functions: the lowest state's |A|^2 per basis state agrees with the dense run
    wd = rows(runs["dense"] / "exc_wf_1.dat")
    wf = rows(runs["fast"] / "exc_wf_1.dat")
    assert np.abs((wd[:, -2] ** 2 + wd[:, -1] ** 2) - (wf[:, -2] ** 2 + wf[:, -1] ** 2)).max() < 1e-3
    assert os.path.exists(runs["fast"] / "exciton_lifetime.dat")
