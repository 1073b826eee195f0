"""CPU oracle of the learned warm start (test infrastructure only: imported by tests/).

The reference has no learned component; this module restates, in float64 numpy, the network
and loss that the GPU kernels of ``wtbg_net_*`` implement, so their gradients can be checked:

  features F (M x 32) -> Z1 = F W1^T + b1 -> H1 = silu(Z1)      (W1: 512 x 32)
                      -> Z2 = H1 W2^T + b2 -> H2 = silu(Z2)     (W2: 512 x 512)
                      -> O  = H2 W3^T + b3                       (W3: 320 x 512)
  X[i, s] = sum_c (O[i, 2(5s+c)] + 1j O[i, 2(5s+c)+1]) * CAR[c, i]         (32 states, 5 carriers)
  per sample: L = min over unitary R of ||X - A R||_F^2 = tr(X^H X) - 2 ||A^H X||_* + 32
  (R = U V^H from the SVD of A^H X), averaged over 32 * nsamp; dL/dX = 2 (X - A R).

``bf16=True`` rounds what the GPU keeps in bf16 (weights, F, H1, H2, dO, dZ2, dZ1) so the two
agree to accumulation order; ``bf16=False`` is the exact float64 function, whose gradient is
checked against finite differences.
"""
from __future__ import annotations

import numpy as np

NF, WD, NS, NCAR = 32, 512, 32, 5
NO = NS * NCAR * 2
SIZES = [("W1", (WD, NF)), ("b1", (WD,)), ("W2", (WD, WD)), ("b2", (WD,)), ("W3", (NO, WD)), ("b3", (NO,))]


def unflatten(p):
    out, o = {}, 0
    for name, shp in SIZES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    return out


def flatten(d):
    return np.concatenate([np.ravel(d[name]) for name, _ in SIZES])


def bf16_round(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def combine(O, CAR):
    M = O.shape[0]
    Oc = O.reshape(M, NS, NCAR, 2)
    coef = Oc[..., 0] + 1j * Oc[..., 1]                 # (M, NS, NCAR)
    return np.einsum("msc,cm->ms", coef, CAR)           # (M, NS)


def loss_grad(p, F, CAR, A, nsamp, bf16=True):
    """Loss and flat gradient. F (M, 32), CAR (5, M) complex, A (32, M) complex."""
    P = unflatten(p)
    rnd = bf16_round if bf16 else (lambda x: np.asarray(x, dtype=np.float64))
    W1, W2, W3 = rnd(P["W1"]), rnd(P["W2"]), rnd(P["W3"])
    F = rnd(F)
    M = F.shape[0]
    rows = M // nsamp
    Z1 = F @ W1.T + P["b1"]
    H1 = rnd(silu(Z1))
    Z2 = H1 @ W2.T + P["b2"]
    H2 = rnd(silu(Z2))
    O = H2 @ W3.T + P["b3"]
    X = combine(O, np.asarray(CAR, dtype=np.complex128))
    At = np.asarray(A, dtype=np.complex128).T            # (M, NS)
    scale = 1.0 / (NS * nsamp)
    loss = 0.0
    GX = np.zeros_like(X)
    for s in range(nsamp):
        sl = slice(s * rows, (s + 1) * rows)
        Xs, As = X[sl], At[sl]
        Pm = As.conj().T @ Xs
        U, sv, Vh = np.linalg.svd(Pm)
        R = U @ Vh
        loss += np.real(np.vdot(Xs, Xs)) - 2.0 * sv.sum() + NS
        GX[sl] = 2.0 * (Xs - As @ R)
    loss *= scale
    GX *= scale
    # dO: Re(conj(G) car), -Im(conj(G) car)
    t = np.einsum("ms,cm->msc", GX.conj(), np.asarray(CAR, dtype=np.complex128))
    dO = np.stack([t.real, -t.imag], axis=-1).reshape(M, NO)
    db3 = dO.sum(0)
    dOr = rnd(dO)
    dW3 = dOr.T @ H2
    dH2 = dOr @ W3
    dZ2 = dH2 * dsilu(Z2)
    db2 = dZ2.sum(0)
    dZ2r = rnd(dZ2)
    dW2 = dZ2r.T @ H1
    dH1 = dZ2r @ W2
    dZ1 = dH1 * dsilu(Z1)
    db1 = dZ1.sum(0)
    dW1 = rnd(dZ1).T @ F
    g = flatten({"W1": dW1, "b1": db1, "W2": dW2, "b2": db2, "W3": dW3, "b3": db3})
    return float(loss), g


def init_params(seed=0, scale_last=0.1):
    rng = np.random.default_rng(seed)
    d = {"W1": rng.standard_normal((WD, NF)) * np.sqrt(2.0 / NF), "b1": np.zeros(WD),
         "W2": rng.standard_normal((WD, WD)) * np.sqrt(2.0 / WD), "b2": np.zeros(WD),
         "W3": rng.standard_normal((NO, WD)) * scale_last * np.sqrt(1.0 / WD), "b3": np.zeros(NO)}
    return flatten(d).astype(np.float32)


def random_problem(rows, nsamp, seed=0):
    """Features, carriers and per-sample orthonormal targets for gradient checks."""
    rng = np.random.default_rng(seed)
    M = rows * nsamp
    F = rng.standard_normal((M, NF)).astype(np.float32) * 0.5
    ph = np.exp(1j * rng.uniform(0, 2 * np.pi, (NCAR, M)))
    ph[0] = 1.0
    CAR = ph.astype(np.complex64)
    A = np.zeros((NS, M), dtype=np.complex64)
    for s in range(nsamp):
        Z = rng.standard_normal((rows, NS)) + 1j * rng.standard_normal((rows, NS))
        Q, _ = np.linalg.qr(Z)
        A[:, s * rows:(s + 1) * rows] = Q.T
    return F, CAR, A
