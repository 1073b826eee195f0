"""Builds the example-input fixtures of the parity tests (run in a container that holds the
reference tree; the outputs travel with the repository, the reference does not).

* tb_mos2.dat.gz, tb_graphene.dat.gz: the reference's two example TB models
  (examples/example-3/tb_mos2.dat: MoS2 with spin-orbit coupling, w = 22, 147 cells;
  examples/example-1/tb_graphene.dat: w = 5, 1615 cells), gzip-compressed, content unchanged,
  so that the drop-in's own params reader parses exactly the reference's input text.
* examples_golden.npz: the oracle's numbers for the reference's example decks, at a reduced
  k-mesh (RK= 16 -> 6x6 for BSE, RK= 12 -> 4x4 for BSE_BND) so that the oracle finishes in
  seconds; everything else in the decks is as the examples set it:
    ex3  examples/example-3/example_3.sh:8-34   BSE+SPEC, V2DT2, LC=8, CSHIFT=0.08, DTDIAG
    ex6  examples/example-6/example_6.sh        the same with BSE_WF, EXC_WF_I=1..10
    ex7  examples/example-7/example_7.sh        BSET (TEMP=300, TA=DE, ST=0.036, PHAVG=225)
    ex5  examples/example-5/exemple_5.sh:19-38  BSE_BND on the G-K-K'-G path, 5 points/segment
    ex4  examples/example-4/example_4.sh        BERRY along the same path, 50 points/segment
    ex1  examples/example-1/example_1.sh        BANDS of graphene with ORB_W c1 (1 1 1 1 0)

Usage: python tests/golden/make_examples.py [reference root]
"""
import gzip
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import wtb_oracle as O  # noqa: E402
from oracle.deck import parse_deck  # noqa: E402
from wantibexos_b200 import synth  # noqa: E402

# the decks of the examples (k-mesh reduced as stated above); {out} and {params} are filled
# in by the tests
EX3 = """NTHREADS= 1
SYSDIM= "2D"
DFT= "V"
OUTPUT= "{out}"
CALC_DATA= "{out}"
PARAMS_FILE= "{params}"
MESH_TYPE= "RK2D"
RK= 16
BSE= T
SPEC= T
DTDIAG= T
COULOMB_POT= V2DT2
NBANDSC= 2
NBANDSV= 2
LC= 8.00
CSHIFT= 0.08
ENSPECI= 0.0
ENSPECF= 4.0
"""
EX6 = EX3 + "BSE_WF= T\nEXC_WF_I= 1\nEXC_WF_F= 10\n"
EX7 = EX3.replace("BSE= T", "BSET= T") + "TA= DE\nST= 0.036\nPHAVG= 225\nTEMP= 300\n"
EX5 = """NTHREADS= 1
SYSDIM= "2D"
DFT= "V"
OUTPUT= "{out}"
CALC_DATA= "{out}"
PARAMS_FILE= "{params}"
KPATH_BSE= "{kpath}"
MESH_TYPE= "RK2D"
RK= 12
BSE_BND= T
COULOMB_POT= V2DT2
NBANDSC= 2
NBANDSV= 2
LC= 8.00
"""
EX4 = """NTHREADS= 1
SYSDIM= "2D"
DFT= "V"
OUTPUT= "{out}"
CALC_DATA= "{out}"
PARAMS_FILE= "{params}"
KPATH_FILE= "{kpath}"
BERRY= T
"""
EX1 = """NTHREADS= 1
SYSDIM= "2D"
DFT= "V"
OUTPUT= "{out}"
CALC_DATA= "{out}"
PARAMS_FILE= "{params}"
KPATH_FILE= "{kpath}"
ORB_W= "{orbw}"
BANDS= T
"""
# G K K K' K' G in fractional reciprocal coordinates (the examples' k-path files)
KS = [(0.0, 0.0, 0.0), (0.6667, -0.3333, 0.0), (0.6667, -0.3333, 0.0), (0.3333, 0.3333, 0.0),
      (0.3333, 0.3333, 0.0), (0.0, 0.0, 0.0)]
ORBW_C1 = [1, 1, 1, 1, 0]


def kpath_text(npts):
    return "%d\n%d\n" % (len(KS), npts) + "".join("%.4f %.4f %.4f\n" % k for k in KS)


def model(name):
    """The fixture model (the reference's params text, parsed by the oracle's reader)."""
    import tempfile
    with gzip.open(os.path.join(HERE, name + ".dat.gz"), "rt") as f:
        text = f.read()
    with tempfile.NamedTemporaryFile("w", suffix=".dat", delete=False) as t:
        t.write(text)
    try:
        return synth.read_params(t.name)
    finally:
        os.unlink(t.name)


def deck(text):
    return parse_deck(text.format(out="./", params="x", kpath="x", orbw="x"))


def golden():
    mos2 = model("tb_mos2")
    gra = model("tb_graphene")
    out = {}
    r3 = O.run_bse(mos2, deck(EX6), want_vectors=True)
    out["ex3_ngrid"] = np.array(r3["ngrid"])
    out["ex3_eigv"] = r3["eigv"]
    out["ex3_nocp"] = r3["nocp"]
    out["ex3_W"] = r3["W"]
    out["ex3_act"] = r3["act"]
    out["ex3_A10_abs2"] = np.abs(r3["A"][:, :10]) ** 2
    d3 = deck(EX3)
    E = O.roundtrip_f154(r3["W"])
    F = O.roundtrip_f154(r3["act"][:, :6])
    dl = O.bsedielraw(mos2.systype, mos2.rlat, r3["ngrid"], E, F, d3["ebse0"], d3["ebsef"], d3["numbse"],
                      d3["cshift"], d3["renorm"])
    for c in ("xx", "yy", "xy"):
        out["ex3_eps_" + c] = dl[c]
    r7 = O.run_bse(mos2, deck(EX7))
    out["ex7_W"] = r7["W"]
    out["ex7_act"] = r7["act"]
    exk, qpath, _ = O.run_bsebnds(mos2, deck(EX5), KS, 5)
    out["ex5_exk"] = exk
    out["ex5_qpath"] = qpath
    rows, _ = O.berry_kpath(mos2, KS, 50)
    out["ex4_berry"] = rows
    bands, _ = O.bandstool(gra, KS, 50, orbw=ORBW_C1, dft="V")
    out["ex1_bands"] = bands
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    for name, src in (("tb_mos2", "examples/example-3/tb_mos2.dat"),
                      ("tb_graphene", "examples/example-1/tb_graphene.dat")):
        with open(os.path.join(ref, src), "rb") as f:
            data = f.read()
        with gzip.GzipFile(os.path.join(HERE, name + ".dat.gz"), "wb", compresslevel=9, mtime=0) as g:
            g.write(data)
    np.savez_compressed(os.path.join(HERE, "examples_golden.npz"), **golden())


if __name__ == "__main__":
    main()
