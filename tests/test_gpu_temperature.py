"""Temperature BSE (BSET=T / BSET_BND=T) on the GPU against the CPU oracle: occupation factors
f_v - f_c in the kernel rows, the sp table and one factor of the oscillators, and the
temperature scissors shift (TA= VE). Same tolerances as the plain FP64 parity tests."""
import numpy as np
import pytest

from oracle import wtb_oracle as O
from oracle.deck import parse_deck
from wantibexos_b200 import synth, wtbgpu

pytestmark = pytest.mark.gpu

DECK = """BSET= T
NGX= 10
NGY= 10
NGZ= 1
NBANDSV= 2
NBANDSC= 2
COULOMB_POT= V2DRK
R_0= 40
KTOL= 0.001
CSHIFT= 0.05
DTDIAG= T
CPOL= T
TEMP= 4000
TA= VE
ST= 2.0
PHAVG= 0.02
"""


def coul_of(deck, ngrid):
    return wtbgpu.coulomb_params(deck["coultype"], ngrid, deck["ktol"], deck["ediel"], deck["lc"], deck["ez"],
                                 deck["w"], deck["r0"])


def test_temperature_bse_matches_oracle(gpu_ctx):
    m = synth.config_model("c1")
    deck = parse_deck(DECK)
    ref = O.run_bse(m, deck)
    tcor = O.temperature_shift(deck)
    assert tcor < 0.0
    f = ref["fdeh"]
    assert f.min() < 0.99   # the temperature is high enough to matter (f < 0: inverted occupation)
    gpu_ctx.set_model(O.with_scs(m, m.scs + tcor))
    gpu_ctx.set_temperature(True, deck["temp"])
    eigv, vec, nocp, gap = gpu_ctx.bands(ref["kpts"], deck["nv"], deck["nc"])
    assert np.abs(eigv - ref["eigv"]).max() < 1e-8
    gpu_ctx.velocity(deck["cshift"], want=False)
    sp = gpu_ctx.sp_table()
    want = O.sp_table(ref["kpts"], ref["eigv"], ref["nocp"], ref["h"], deck["nv"], deck["nc"], fdeh=f)
    assert np.allclose(sp, want, rtol=1e-5, atol=1e-6)
    gpu_ctx.bse_build(coul_of(deck, ref["ngrid"]))
    H = gpu_ctx.bse_get_matrix()
    p = O.CoulombParams(deck["coultype"], deck["ktol"], deck["ediel"], deck["lc"], deck["ez"], deck["w"],
                        deck["r0"], ref["ngrid"], m.rlat)
    Hw = O.bse_matrix(p, ref["kpts"], eigv, vec, deck["nv"], deck["nc"],
                      fdeh=O.fdeh_states(eigv, eigv, deck["nv"], deck["nc"], deck["temp"]))
    assert np.abs(np.triu(H) - Hw).max() < 1e-12 * np.abs(Hw).max()
    W, act = gpu_ctx.bse_solve(deck["dtfull"], deck["cpol"])
    assert np.abs(W - ref["W"]).max() < 1e-9
    for c in range(8):
        scale = max(np.abs(ref["act"][:, c]).max(), 1e-30)
        assert np.abs(act[:, c] - ref["act"][:, c]).max() < 1e-7 * scale, c
    # the plain path differs at this temperature
    plain = O.run_bse(m, parse_deck(DECK.replace("BSET= T", "BSE= T")))
    assert np.abs(plain["W"] - ref["W"]).max() > 1e-4
    gpu_ctx.set_temperature(False)


def test_temperature_q_point_matches_oracle(gpu_ctx):
    m = synth.config_model("c1")
    deck = parse_deck(DECK.replace("BSET= T", "BSET_BND= T").replace("NGX= 10", "NGX= 6").replace("NGY= 10", "NGY= 6"))
    mm = O.with_scs(m, m.scs + O.temperature_shift(deck))
    ng = deck["ngrid"]
    kpts = O.monkhorst_pack(ng[0], ng[1], ng[2], deck["mshift"], m.rlat)
    nv, nc = deck["nv"], deck["nc"]
    energy, vector, _, _ = O.bands(mm, kpts, nv, nc)
    qpath, _ = O.kpathbse(m.rlat, [(0, 0, 0), (0.5, 0, 0)], 5)
    p = O.CoulombParams(deck["coultype"], deck["ktol"], deck["ediel"], deck["lc"], deck["ez"], deck["w"],
                        deck["r0"], ng, m.rlat)
    gpu_ctx.set_model(mm)
    gpu_ctx.set_temperature(True, deck["temp"])
    gpu_ctx.bands(kpts, nv, nc)
    for iq in (0, 3):
        q4 = qpath[iq]
        kq = O.monkhorst_pack(ng[0], ng[1], ng[2], deck["mshift"], m.rlat, q=q4[1:])
        eq, vq, _, _ = O.bands(mm, kq, nv, nc)
        f = O.fdeh_states(eq, energy, nv, nc, deck["temp"])
        H = O.bse_matrix_q(p, q4, kpts, energy, vector, eq, vq, nv, nc, fdeh=f)
        w_ref = np.linalg.eigvalsh(H, UPLO="U")
        W = gpu_ctx.bse_q_eigenvalues(kq, q4, coul_of(deck, ng))
        assert np.abs(W - w_ref).max() < 1e-9, iq
    gpu_ctx.set_temperature(False)


def test_zero_temperature_equals_plain(gpu_ctx):
    """T = 0 (taken as 1E-8 K) gives f = 1 for a gapped model: the plain results."""
    m = synth.config_model("c1")
    deck = parse_deck(DECK.replace("TEMP= 4000", "TEMP= 0").replace("TA= VE", "TA= FA"))
    kpts = O.monkhorst_pack(8, 8, 1, deck["mshift"], m.rlat)
    out = []
    for on in (False, True):
        gpu_ctx.set_model(m)
        gpu_ctx.set_temperature(on, 0.0)
        gpu_ctx.bands(kpts, 2, 2, want_vectors=False)
        gpu_ctx.velocity(0.05, want=False)
        gpu_ctx.bse_build(coul_of(deck, [8, 8, 1]))
        out.append(gpu_ctx.bse_solve(True, True))
    gpu_ctx.set_temperature(False)
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-12
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-12 * np.abs(out[0][1]).max()
