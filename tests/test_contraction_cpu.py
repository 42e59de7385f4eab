"""Host-side checks of the Green's contraction the x-pencil kernel evaluates.

The kernel never forms B(k): it applies sum_b B_ab(k) Y_b through the per-k
stress Sig = sum_b Y_b sigma^b.  Restated here in numpy with the same
formula and compared with the oracle's B table (a restatement of Bmatrix)."""
import numpy as np

import pfdd_oracle as O
from pfdd_b200 import configs


def green_apply(xn, xb, dslip, C44, C12, C11, k, Y):
    mu, ll, young, xnu = O.voigt_constants(C44, C12, C11)
    eps = np.einsum("ai,aj->aij", xb, xn) / dslip
    tr = np.trace(eps, axis1=1, axis2=2)
    sig = C44 * (eps + eps.transpose(0, 2, 1)) + C12 * tr[:, None, None] * np.eye(3)
    Sig = np.einsum("b,bij->ij", Y, sig)
    k2 = k @ k
    if k2 == 0:
        return np.zeros(len(Y), dtype=complex)
    U = Sig @ k
    V = k @ U
    t = np.einsum("aij,j->ai", sig, k)
    p = t @ k
    es = np.einsum("aij,ij->a", eps, Sig)
    return (es - (2 * (t @ U) / k2 - p * V / ((1 - xnu) * k2 * k2)) / (2 * C44)) / mu


def test_structured_green_operator_equals_B_table():
    w = configs.fcc_workload(6, 4, 4, n_loops=1, seed=1)
    C44, C12, C11 = w.material.elastic()
    BB = O.bmatrix(w.nx, w.ny, w.nz, w.four, w.xn, w.xb, C44, C12, C11, w.material.dslip)
    fx, fy, fz = O.frequencies(w.nx, w.ny, w.nz, w.four)
    rng = np.random.default_rng(0)
    for (i, j, l) in [(0, 0, 0), (1, 2, 3), (3, 1, 2), (5, 3, 0), (2, 0, 1)]:
        Y = rng.standard_normal(12) + 1j * rng.standard_normal(12)
        k = np.array([fx[i, j, l], fy[i, j, l], fz[i, j, l]])
        got = green_apply(w.xn, w.xb, w.material.dslip, C44, C12, C11, k, Y)
        want = BB[:, :, i, j, l] @ Y
        assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())


def test_B_properties():
    w = configs.loop_workload(n=8)
    C44, C12, C11 = w.material.elastic()
    BB = O.bmatrix(w.nx, w.ny, w.nz, w.four, w.xn, w.xb, C44, C12, C11, w.material.dslip)
    assert np.abs(BB[:, :, 0, 0, 0]).max() == 0.0                       # B(0) = 0
    assert np.abs(BB - BB.transpose(1, 0, 2, 3, 4)).max() < 1e-14        # symmetric in (a, b)
    neg = lambda n: (-np.arange(n)) % n
    Bm = BB[:, :, neg(8)][:, :, :, neg(8)][:, :, :, :, neg(8)]
    inner = (slice(None), slice(None), slice(1, 4), slice(1, 4), slice(1, 4))
    assert np.abs(BB[inner] - Bm[inner]).max() < 1e-14                    # even off the Nyquist planes
    assert np.abs(BB - Bm).max() > 1e-3                                   # but not on them
