"""The oracle on the reference's own example inputs (examples/example-1, -3 .. -7), against the
committed fixture numbers, and the fixture models against the reference files when the
reference tree is present.  CPU only."""
import gzip
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_examples as X  # noqa: E402

from oracle import wtb_oracle as O  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "examples_golden.npz"))
REF = "/root/reference"


def test_fixture_models_parse_as_the_reference_describes_them():
    mos2 = X.model("tb_mos2")
    gra = X.model("tb_graphene")
    assert (mos2.systype.strip(), mos2.w, mos2.nvec) == ("SOC", 22, 147)
    assert (gra.systype.strip(), gra.w, gra.nvec) == ("NP", 5, 1615)
    assert mos2.efermi == -1.2008 and gra.efermi == -2.8823
    # H(-R) = H(R)^dagger for every cell pair (a Wannier model is Hermitian)
    for m in (mos2, gra):
        idx = {tuple(r): i for i, r in enumerate(m.rvec)}
        for i, r in enumerate(m.rvec[:40]):
            j = idx[tuple(-r)]
            H = m.hre[i] + 1j * m.him[i]
            Hm = m.hre[j] + 1j * m.him[j]
            assert np.abs(H / m.deg[i] - Hm.conj().T / m.deg[j]).max() < 2e-6


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_fixture_files_equal_the_reference_examples():
    for name, src in (("tb_mos2", "examples/example-3/tb_mos2.dat"),
                      ("tb_graphene", "examples/example-1/tb_graphene.dat")):
        with gzip.open(os.path.join(HERE, "golden", name + ".dat.gz"), "rb") as f:
            a = f.read()
        with open(os.path.join(REF, src), "rb") as f:
            assert f.read() == a, name


def test_oracle_reproduces_example_numbers():
    mos2 = X.model("tb_mos2")
    r = O.run_bse(mos2, X.deck(X.EX3))
    assert list(r["ngrid"]) == [6, 6, 1]
    assert np.abs(r["W"] - GOLD["ex3_W"]).max() < 1e-12
    assert np.abs(r["act"] - GOLD["ex3_act"]).max() < 1e-10 * np.abs(GOLD["ex3_act"]).max()
    # the example's physics: the lowest excitons are the bright K/K' pair below the 2.19 eV gap
    assert r["egap"] > r["W"][0] > 2.0 and r["act"][0, 0] > 1.0
    exk, _, _ = O.run_bsebnds(mos2, X.deck(X.EX5), X.KS, 5)
    assert np.abs(exk - GOLD["ex5_exk"]).max() < 1e-12
    b, _ = O.bandstool(X.model("tb_graphene"), X.KS, 50, orbw=X.ORBW_C1, dft="V")
    assert np.array_equal(b, GOLD["ex1_bands"])
