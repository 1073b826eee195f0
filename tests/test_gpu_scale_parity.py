"""GPU parity beyond the small config-1 model: the config-2 model (w = 24, 91 cells,
nv = nc = 4) on a 12x12 mesh (N = 2304) through every stage, the config-4 models (w = 16 and
40, 61 cells) and models wider than the shared-memory budget of the per-k kernels (w = 64
and 100, whose work matrices live in global memory), all against the CPU oracle.

Tolerances as in the config-1 parity tests: bands 1e-8 eV, velocities 1e-9 relative after the
per-k band signs, BSE matrix 1e-12 relative (from the same band vectors), exciton energies
1e-9 eV, oscillator strengths 1e-7 of the largest, spectra within a few float32 ulps."""
import functools

import numpy as np
import pytest

from oracle import wtb_oracle as O
from oracle.deck import parse_deck
from wantibexos_b200 import synth, wtbgpu

pytestmark = pytest.mark.gpu

C2S = """BSE= T
SPEC= T
NGX= 12
NGY= 12
NGZ= 1
NBANDSV= 4
NBANDSC= 4
COULOMB_POT= V2DRK
R_0= 30
KTOL= 0.001
CSHIFT= 0.03
ENSPECI= 0
ENSPECF= 6
NESPEC= 2001
DTDIAG= T
CPOL= T
SYSDIM= "2D"
"""


def coul(deck, ngrid):
    return wtbgpu.coulomb_params(deck["coultype"], ngrid, deck["ktol"], deck["ediel"], deck["lc"], deck["ez"],
                                 deck["w"], deck["r0"])


def signs(vg, vo, nv):
    """s_i = sign_c(k) sign_v(k) of every basis state (GPU bands: component 1 real >= 0)."""
    sc = np.sign(vg[:, :, 0].real * vo[:, :, 0].real)
    return (sc[:, nv:, None] * sc[:, None, :nv]).reshape(-1)


@functools.lru_cache(maxsize=None)
def c2s():
    m = synth.config_model("c2")
    deck = parse_deck(C2S)
    ref = O.run_bse(m, deck)
    ctx = wtbgpu.Context(0)
    ctx.set_model(m)
    eigv, vec, nocp, gap = ctx.bands(ref["kpts"], 4, 4)
    h = ctx.velocity(deck["cshift"])
    ctx.bse_build(coul(deck, ref["ngrid"]))
    H = ctx.bse_get_matrix()
    W, act = ctx.bse_solve(True, True)
    g = dict(eigv=eigv, vec=vec, nocp=nocp, gap=gap, h=h, H=H, W=W, act=act, ctx=ctx)
    return m, deck, ref, g


def test_config2_model_bands_and_velocities():
    m, deck, ref, g = c2s()
    assert np.array_equal(g["nocp"], ref["nocp"])
    assert np.abs(g["eigv"] - ref["eigv"]).max() < 1e-8
    assert abs(g["gap"] - ref["egap"]) < 1e-8
    s = signs(g["vec"], ref["vec"], 4)
    assert np.abs(g["h"] - ref["h"] * s[:, None]).max() < 1e-9 * np.abs(ref["h"]).max()


def test_config2_model_bse_matrix():
    m, deck, ref, g = c2s()
    p = O.CoulombParams(deck["coultype"], deck["ktol"], deck["ediel"], deck["lc"], deck["ez"], deck["w"],
                        deck["r0"], ref["ngrid"], m.rlat)
    Hw = O.bse_matrix(p, ref["kpts"], g["eigv"], g["vec"], 4, 4)
    assert np.abs(np.triu(g["H"]) - Hw).max() < 1e-12 * np.abs(Hw).max()


def test_config2_model_excitons_oscillators_spectrum():
    m, deck, ref, g = c2s()
    assert np.abs(g["W"] - ref["W"]).max() < 1e-9
    for c in range(8):
        scale = max(np.abs(ref["act"][:, c]).max(), 1e-30)
        assert np.abs(g["act"][:, c] - ref["act"][:, c]).max() < 1e-7 * scale, c
    E = O.roundtrip_f154(ref["W"])
    F = O.roundtrip_f154(ref["act"][:, :6])
    want = O.bsedielraw(m.systype, m.rlat, ref["ngrid"], E, F, 0.0, 6.0, 2001.0, deck["cshift"], True)
    om, eps = g["ctx"].spectrum(E, F, ref["ngrid"], O.vcell3d(m.rlat), 0.0, 6.0, 2001.0, deck["cshift"], True, 2.0)
    assert np.array_equal(om, want["xx"][:, 0])
    for c, name in enumerate(["xx", "yy", "zz", "xy", "xz", "yz"]):
        for ri in range(2):
            exp = want[name][:, 1 + ri]
            tol = 4 * np.spacing(np.float32(np.abs(exp).max() + 1e-30))
            assert np.abs(eps[:, ri, c].astype(np.float64) - exp).max() <= tol, (name, ri)


def test_config2_model_degenerate_clusters():
    """Oscillator sums over each group of excitons closer than 1e-6 eV (gauge invariant inside a
    degenerate group, whatever basis the solver picks) agree with the oracle."""
    m, deck, ref, g = c2s()
    W = ref["W"]
    cuts = np.concatenate([[0], np.where(np.diff(W) > 1e-6)[0] + 1, [len(W)]])
    for a, b in zip(cuts[:-1], cuts[1:]):
        for c in range(3):
            so = ref["act"][a:b, c].sum()
            sg = g["act"][a:b, c].sum()
            assert abs(sg - so) <= 1e-7 * np.abs(ref["act"][:, c]).max()


@pytest.mark.parametrize("name,n", [("c4_w16", 6), ("c4_w40", 6)])
def test_config4_models_full_path(name, n, gpu_ctx):
    m = synth.config_model(name)
    deck = parse_deck(C2S.replace("NGX= 12", f"NGX= {n}").replace("NGY= 12", f"NGY= {n}")
                      .replace("NBANDSV= 4", "NBANDSV= 2").replace("NBANDSC= 4", "NBANDSC= 2"))
    ref = O.run_bse(m, deck)
    gpu_ctx.set_model(m)
    eigv, vec, nocp, _ = gpu_ctx.bands(ref["kpts"], 2, 2)
    assert np.array_equal(nocp, ref["nocp"])
    assert np.abs(eigv - ref["eigv"]).max() < 1e-8
    h = gpu_ctx.velocity(deck["cshift"])
    s = signs(vec, ref["vec"], 2)
    assert np.abs(h - ref["h"] * s[:, None]).max() < 1e-9 * np.abs(ref["h"]).max()
    gpu_ctx.bse_build(coul(deck, ref["ngrid"]))
    W, act = gpu_ctx.bse_solve(True, True)
    assert np.abs(W - ref["W"]).max() < 1e-9
    assert np.abs(act[:, :3] - ref["act"][:, :3]).max() < 1e-7 * np.abs(ref["act"][:, :3]).max()


def test_config4_bands_on_larger_mesh(gpu_ctx):
    m = synth.config_model("c4_w40")
    kpts = O.monkhorst_pack(12, 12, 1, [0, 0, 0], m.rlat)
    e, v, nocp, gap = O.bands(m, kpts, 3, 3)
    gpu_ctx.set_model(m)
    eg, vg, ng, gg = gpu_ctx.bands(kpts, 3, 3)
    assert np.array_equal(ng, nocp)
    assert np.abs(eg - e).max() < 1e-8
    sign = np.sign(vg[:, :, 0].real * v[:, :, 0].real)
    assert np.abs(vg - v * sign[:, :, None]).max() < 1e-9


@pytest.mark.parametrize("w,shells", [(64, 3), (100, 2)])
def test_models_beyond_shared_memory(w, shells, gpu_ctx):
    """w = 64 and 100: bands, velocities, every band (eigsys of the tools), Berry curvature and a
    BSE solve on a 4x4 mesh, with the per-k work matrices in global memory."""
    m = synth.make_gapped_model(w, shells, (-1.5, 0.3), (1.5, 0.3), 7000 + w)
    deck = parse_deck("BSE= T\nNGX= 4\nNGY= 4\nNGZ= 1\nNBANDSV= 2\nNBANDSC= 2\nCOULOMB_POT= V2DRK\nR_0= 30\n"
                      "CSHIFT= 0.03\nDTDIAG= T\n")
    ref = O.run_bse(m, deck)
    gpu_ctx.set_model(m)
    eigv, vec, nocp, _ = gpu_ctx.bands(ref["kpts"], 2, 2)
    assert np.array_equal(nocp, ref["nocp"])
    assert np.abs(eigv - ref["eigv"]).max() < 1e-8
    h = gpu_ctx.velocity(deck["cshift"])
    s = signs(vec, ref["vec"], 2)
    assert np.abs(h - ref["h"] * s[:, None]).max() < 1e-9 * np.abs(ref["h"]).max()
    gpu_ctx.bse_build(coul(deck, ref["ngrid"]))
    W, act = gpu_ctx.bse_solve(True, False)
    assert np.abs(W - ref["W"]).max() < 1e-9
    assert np.abs(act[:, :2] - ref["act"][:, :2]).max() < 1e-7 * np.abs(ref["act"][:, :2]).max()
    kp = ref["kpts"][:5]
    eig, _, _ = gpu_ctx.eigsys(kp)
    for j in range(5):
        assert np.abs(eig[j] - O.eigsys(m, kp[j])[0]).max() < 1e-8
    b = gpu_ctx.berry(kp)
    for j in range(5):
        e_, U_, nocp_ = O.eigsys(m, kp[j])
        bo = O.berryct2(m, kp[j], e_, U_, nocp_)
        assert np.abs(b[j] - bo.imag).max() < 1e-8 * max(1.0, np.abs(bo.imag).max())
