"""CPU checks of the learned warm start's oracle: its analytic gradient against central finite
differences in float64, and the bf16 rounding helper."""
import numpy as np

from oracle import mlp_oracle as MO


def test_oracle_gradient_matches_finite_differences():
    p = MO.init_params(1, scale_last=1.0).astype(np.float64)
    F, CAR, A = MO.random_problem(40, 2, 3)
    L, g = MO.loss_grad(p, F, CAR, A, 2, bf16=False)
    assert L > 0
    idx = [5, 100, MO.WD * MO.NF + 3, MO.WD * MO.NF + MO.WD + 777, len(p) - 400, len(p) - 3]
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (MO.loss_grad(p + e, F, CAR, A, 2, bf16=False)[0] - MO.loss_grad(p - e, F, CAR, A, 2, bf16=False)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_loss_is_zero_at_an_orthonormal_basis_of_the_targets():
    # X = A exactly (coefficients on the constant carrier) gives L = 0
    rows = 40
    rng = np.random.default_rng(0)
    Z = rng.standard_normal((rows, MO.NS)) + 1j * rng.standard_normal((rows, MO.NS))
    A = np.linalg.qr(Z)[0]
    O = np.zeros((rows, MO.NO))
    O[:, 0::2 * MO.NCAR] = A.real
    O[:, 1::2 * MO.NCAR] = A.imag
    CAR = np.zeros((MO.NCAR, rows), dtype=np.complex128)
    CAR[0] = 1.0
    X = MO.combine(O, CAR)
    assert np.allclose(X, A)


def test_bf16_round_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-30], dtype=np.float32)
    r = MO.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7
    assert abs(r[3] + 3.140625) < 1e-12
    assert abs(r[4] - 1e-30) / 1e-30 < 2 ** -8
