"""CPU self-checks of the oracle (the restatement of the reference path) and of the deck /
params readers.  No GPU is used here."""
import math

import numpy as np
import pytest
import scipy.linalg.lapack as lapack

from oracle import wtb_oracle as O
from oracle.deck import parse_deck
from wantibexos_b200 import synth


@pytest.fixture(scope="module")
def small():
    m = synth.config_model("c1")
    kpts = O.monkhorst_pack(4, 4, 1, [0, 0, 0], m.rlat)
    return m, kpts


def test_float32_literals():
    assert O.PI_F32 == float(np.float32(math.pi))
    # -(0.0904756)*10**(3) in real(4): the literal rounds first, then the product
    assert O.CIC == float(-(np.float32(0.0904756) * np.float32(1000)))
    assert O.CIC == -90.47559356689453
    assert O.GAMA == float(np.float32(180.9))
    assert O.INV_SQRT2_F32 == float(np.float32(0.70710677))
    assert O.RENORM_FACTOR != 0.15 and abs(O.RENORM_FACTOR - 0.15) < 1e-8


def test_synthetic_model_shapes():
    for n, cnt in ((3, 37), (4, 61), (5, 91)):
        assert synth.hex_cells(n).shape[0] == cnt
    m = synth.config_model("c1")
    H = m.hre + 1j * m.him
    idx = {tuple(r): i for i, r in enumerate(m.rvec.tolist())}
    for r, i in idx.items():
        j = idx[(-r[0], -r[1], -r[2])]
        assert np.allclose(H[j], H[i].conj().T)


def test_params_roundtrip(tmp_path):
    m = synth.config_model("c1")
    p = tmp_path / "tb.dat"
    synth.write_params(m, str(p))
    r = synth.read_params(str(p))
    assert r.w == m.w and r.nvec == m.nvec and r.systype == "NP"
    assert np.array_equal(r.rvec, m.rvec)
    assert np.array_equal(r.hre, m.hre) and np.array_equal(r.him, m.him)
    assert np.array_equal(r.rlat, m.rlat)


def test_deck_defaults_and_keys():
    d = parse_deck("")
    assert d["ktol"] == float(np.float32(0.001)) and d["cshift"] == float(np.float32(0.01))
    assert d["coultype"] == "V3D" and d["renorm"] is True and d["nc"] == 1
    d = parse_deck('NTHREADS= 10\nSYSDIM= "2D"\nOUTPUT= "./out/"\nMESH_TYPE= "RK2D"\nRK= 120\n'
                   'BSE= T\nSPEC= T\nDTDIAG= T\nCOULOMB_POT= V2DT2\nNBANDSC= 2\nNBANDSV= 2\n'
                   'LC= 8.00\nCSHIFT= 0.08\nENSPECI= 0.0\nENSPECF= 4.0\nUNKNOWN_KEY= 3\n')
    assert d["sysdim"] == "2D" and d["outputfolder"] == "./out/" and d["rk"] == 120.0
    assert d["bse"] and d["spec"] and d["dtfull"] and d["coultype"] == "V2DT2"
    assert d["lc"] == 8.0 and d["cshift"] == 0.08 and d["ebsef"] == 4.0
    # a key whose value sits on the next record
    d = parse_deck("NGX=\n 7\nNGY= 5\n")
    assert d["ngrid"][:2] == [7, 5]


def test_eigsys_matches_eigh_and_gauge(small):
    m, kpts = small
    for k in kpts[:5]:
        e, U, nocp = O.eigsys(m, k)
        Hk = O.hk(m, k)
        ref = np.linalg.eigvalsh(Hk)
        assert np.abs(e[:nocp] - ref[:nocp]).max() < 1e-12
        assert np.abs(U[:, 0].imag).max() == 0.0          # ZHEEV('V','L'): component 1 real
        assert np.allclose(U.conj() @ Hk @ U.T, np.diag(e[:nocp].tolist() + (e[nocp:] - m.scs).tolist()), atol=1e-12)
        assert nocp == m.w // 2


def test_phase_is_float32(small):
    m, kpts = small
    k = kpts[5]
    R = O._rcart(m)
    p = O.phases(m, k)
    kr = (k[0] * R[:, 0] + k[1] * R[:, 1]) + k[2] * R[:, 2]
    assert np.allclose(p, np.exp(1j * kr), atol=1e-5)
    assert np.array_equal(p.real, np.cos(kr.astype(np.float32).astype(np.float64)))


def test_oscillator_sum_rule_and_gauges(small):
    """sum_n f_n = ||h||^2 (A unitary); energies are gauge invariant; oscillators are
    invariant under valence phases and real sign flips but not under conduction phases
    (the no-conjugate quirk of dielbsev)."""
    m, kpts = small
    nv = nc = 2
    eigv, vec, nocp, _ = O.bands(m, kpts, nv, nc)
    h = O.optsp_all(m, kpts, eigv, vec, nv, nc, 0.05)
    p = O.CoulombParams("V2DRK", 1e-3, [1, 1, 1], 1, 1, 0, 40, [4, 4, 1], m.rlat)
    W, act = O.bse_solve(p, kpts, eigv, vec, h, nv, nc, True, True)
    assert abs(act[:, 0].sum() - (np.abs(h[:, 0]) ** 2).sum()) < 1e-10 * act[:, 0].sum()
    rng = np.random.default_rng(3)

    def rerun(vec2):
        h2 = O.optsp_all(m, kpts, eigv, vec2, nv, nc, 0.05)
        return O.bse_solve(p, kpts, eigv, vec2, h2, nv, nc, True, True)

    ph = np.exp(1j * rng.uniform(0, 2 * np.pi, (len(kpts), nv)))
    v2 = vec.copy()
    v2[:, :nv, :] *= ph[:, :, None]
    W2, act2 = rerun(v2)
    assert np.abs(W2 - W).max() < 1e-10 and np.abs(act2 - act).max() < 1e-8 * act.max()
    v3 = vec.copy()
    v3[:, nv:, :] *= -1.0
    W3, act3 = rerun(v3)
    assert np.abs(act3 - act).max() < 1e-8 * act.max()
    v4 = vec.copy()
    v4[:, nv:, :] *= np.exp(1j * rng.uniform(0, 2 * np.pi, (len(kpts), 1, 1)))
    W4, act4 = rerun(v4)
    assert np.abs(W4 - W).max() < 1e-10
    assert np.abs(act4 - act).max() > 1e-3 * act.max()


def test_bse_matrix_is_hermitian_and_diagonal(small):
    m, kpts = small
    eigv, vec, nocp, _ = O.bands(m, kpts, 2, 2)
    p = O.CoulombParams("V2DRK", 1e-3, [1, 1, 1], 1, 1, 0, 40, [4, 4, 1], m.rlat)
    Hf = O.bse_matrix(p, kpts, eigv, vec, 2, 2, upper_only=False)
    assert np.abs(Hf - Hf.conj().T).max() < 1e-12
    de = (eigv[:, 2:][:, :, None] - eigv[:, :2][:, None, :]).reshape(-1)
    assert np.allclose(np.diag(Hf).real, de)   # V(0) = 0 for V2DRK


def test_v2drk_limits():
    rlat = synth.hex_rlat()
    p = O.CoulombParams("V2DRK", 1e-3, [1, 1, 1], 1.0, 1.0, 0.0, 0.0, [10, 10, 1], rlat)
    q = np.array([[0.05, 0, 0], [0.2, 0.1, 0]])
    vbz = 1.0 / (100 * O.vcell2d(rlat))
    # eps = 1, r0 = 0: bare 2D Coulomb vbz*cic/q
    assert np.allclose(O.coulomb(p, q), vbz * O.CIC / np.linalg.norm(q, axis=1), rtol=1e-12)
    assert O.coulomb(p, np.array([1e-4, 0, 0])) == 0.0


def test_spectrum_lorentzian_and_renorm():
    E = np.array([1.0, 1.5, 2.0])
    F = np.zeros((3, 6))
    F[:, 0] = [1.0, 0.5, 0.25]
    rlat = synth.hex_rlat()
    d = O.bsedielraw("NP", rlat, [4, 4, 1], E, F, 0.0, 3.0, 301.0, 0.05, False)
    om = d["xx"][:, 0]
    eta = 0.05 + 10 * (2.0 - 1.0) / 3
    c = O.GAMA / (16 * O.vcell3d(rlat))
    im = 2 * c * sum(F[i, 0] * eta / ((om - E[i]) ** 2 + eta ** 2) for i in range(3))
    assert np.allclose(d["xx"][:, 2], im, rtol=1e-6)
    r = O.bsedielraw("NP", rlat, [4, 4, 1], E, F, 0.0, 3.0, 301.0, 0.05, True)
    below = om <= E[0] - O.RENORM_FACTOR
    assert np.all(r["xx"][below, 2] == 0) and np.all(r["xx"][:, 2] >= 0)


def test_kpathbse_counts():
    rlat = synth.hex_rlat()
    ks = [(0, 0, 0), (0.5, 0, 0), (0.5, 0, 0), (1 / 3, 1 / 3, 0), (1 / 3, 1 / 3, 0), (0, 0, 0)]
    pts, labels = O.kpathbse(rlat, ks, 21)
    assert pts.shape == (63, 4) and len(labels) == 4
    assert abs(labels[-1] - 1.0) < 1e-12
    t = float(np.float32(np.float32(1) / np.float32(20)))
    assert pts[1, 0] == labels[0] + (pts[20, 0] - pts[0, 0]) * t or abs(pts[1, 0] - pts[20, 0] * t) < 1e-15


def test_zheev_min_workspace_gauge():
    rng = np.random.default_rng(0)
    X = rng.standard_normal((9, 9)) + 1j * rng.standard_normal((9, 9))
    H = X + X.conj().T
    w, v = O.zheev(H, lower=0)
    assert np.abs(v[-1].imag).max() == 0.0      # 'U': last component real
    w, v = O.zheev(H, lower=1)
    assert np.abs(v[0].imag).max() == 0.0       # 'L': first component real


def test_temperature_oracle_reduces_to_plain_at_unit_occupation():
    """With f = 1 (T -> 0 for a gapped model) the temperature kernel, sp table and
    oscillators equal the plain ones; at high T they differ."""
    m = synth.config_model("c1")
    deck = parse_deck("NGX= 6\nNGY= 6\nNGZ= 1\nNBANDSV= 2\nNBANDSC= 2\nCOULOMB_POT= V2DRK\nR_0= 40\n"
                      "KTOL= 0.001\nCSHIFT= 0.05\nDTDIAG= T\nCPOL= T\n")
    kpts = O.monkhorst_pack(6, 6, 1, [0, 0, 0], m.rlat)
    eigv, vec, nocp, _ = O.bands(m, kpts, 2, 2)
    f0 = O.fdeh_states(eigv, eigv, 2, 2, 0.0)
    assert np.all(f0 == 1.0)
    p = O.CoulombParams("V2DRK", 1e-3, [1, 1, 1], 1, 1, 0, 40, [6, 6, 1], m.rlat)
    H0 = O.bse_matrix(p, kpts, eigv, vec, 2, 2)
    H1 = O.bse_matrix(p, kpts, eigv, vec, 2, 2, fdeh=f0)
    assert np.abs(H0 - H1).max() < 1e-15
    fT = O.fdeh_states(eigv, eigv, 2, 2, 5000.0)
    assert fT.min() < 0.95
    HT = O.bse_matrix(p, kpts, eigv, vec, 2, 2, fdeh=fT)
    de = np.real(np.diag(H0)) - np.real(np.diag(H0 - np.diag(np.diag(H0))))
    off = np.triu(H0, 1)
    assert np.allclose(np.triu(HT, 1), off * fT[:, None])
    h = O.optsp_all(m, kpts, eigv, vec, 2, 2, 0.05)
    A = np.linalg.qr(np.random.default_rng(0).standard_normal((h.shape[0], 5)) + 0j)[0]
    assert np.allclose(O.dielbseptemp(A, h[:, 0], h[:, 1], np.ones(h.shape[0])), O.dielbsep(A, h[:, 0], h[:, 1]))
    assert abs(O.gapcortemp(2.0, 0.02, 300.0) - (-2.0 * 0.02 * (1.0 / np.tanh(0.02 / (2 * O.KB_F32 * 300.0)) - 1.0))) < 1e-15
    assert O.gapcortemp2(1.0, 300.0, 300.0) == -(2.0 / (np.exp(1.0) - 1.0))


def test_berry_oracle_gives_qwz_chern_numbers():
    """Known answer for the Berry curvature restatement (berryct2): the lower band of the
    Qi-Wu-Zhang model integrates to Chern number +1 (u = -1), -1 (u = +1) and 0 (u = -3)."""
    for u, chern in ((-1.0, 1.0), (1.0, -1.0), (-3.0, 0.0)):
        m = synth.qwz_model(u)
        kp = O.monkhorst_pack(24, 24, 1, [0, 0, 0], m.rlat)
        s = 0.0
        for k in kp:
            e, U, nocp = O.eigsys(m, k)
            assert nocp == 1
            s += O.berryct2(m, k, e, U, nocp)[1].imag
        b1, b2, _ = O.recvec(m.rlat[0], m.rlat[1], m.rlat[2])
        area = abs(np.cross(b1, b2)[2])
        assert abs(s * area / len(kp) / (2 * np.pi) - chern) < 1e-4


def test_sp_optbz_oracle_identities():
    """spoptpolbz sums: |h_x + i h_y|^2 + |h_x - i h_y|^2 = 2 (|h_x|^2 + |h_y|^2), so
    sigma+ + sigma- = 2 norm^2 (x + y) with norm = f32(1/sqrt 2), and the dichroism lies in [-1, 1]."""
    m = synth.config_model("c1")
    rows = O.sp_optbz(m, [3, 3, 1], [0, 0, 0], 2, 2, float(np.float32(0.05)))
    norm = float(np.float32(1.0) / np.sqrt(np.float32(2.0)))
    assert rows.shape == (9, 9)
    assert np.allclose(rows[:, 6] + rows[:, 7], 2 * norm ** 2 * (rows[:, 3] + rows[:, 4]), rtol=1e-12)
    assert np.all(np.abs(rows[:, 8]) <= 1.0)
    assert np.all(rows[:, 3:8] >= 0.0)
