"""The FP32 path's own sin(pi y) / cos(pi y) polynomials (sincospi_poly in
csrc/pfdd_kernels.cuh), evaluated here in FP32 with the same operation order
(fused multiply-adds emulated exactly in FP64, then rounded) against the
exact values: within 2 ulp of |value| (absolute 2^-24 floor near zeros)."""
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "phase-field-dislocation-dynamics-pfdd-2.x_b200", "csrc", "pfdd_kernels.cuh")


def _coefficients():
    text = open(SRC).read()
    body = text[text.index("void sincospi_poly"):]
    body = body[body.index("const float t"):body.index("\n}\n")]
    nums = [float(x) for x in re.findall(r"(-?\d+\.\d+)f", body)]
    # order in the source: -0.5, then S (deg 3 .. 0 as written), C (deg 4 .. 0)
    return nums


def _fma(a, b, c):
    # a*b + c rounded once: exact in FP64 for FP32 inputs (24+24 bit product)
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def sincospi_poly(y):
    nums = _coefficients()
    s3, s2, s1, s0 = [np.float32(v) for v in nums[1:5]]
    c4, c3, c2, c1, c0 = [np.float32(v) for v in nums[5:10]]
    y = np.float32(y)
    n = np.float32(np.rint(np.float32(2.0) * y))
    t = _fma(n, np.float32(-0.5), y)
    u = np.float32(t * t)
    ps = _fma(u, s3, s2)
    ps = _fma(u, ps, s1)
    ps = _fma(u, ps, s0)
    sv = np.float32(t * ps)
    pc = _fma(u, c4, c3)
    pc = _fma(u, pc, c2)
    pc = _fma(u, pc, c1)
    cv = _fma(u, pc, c0)
    q = n.astype(np.int64) & 3
    ss = np.where(q & 1, cv, sv)
    cs = np.where(q & 1, sv, cv)
    ss = np.where(q & 2, -ss, ss)
    cs = np.where((q + 1) & 2, -cs, cs)
    return ss.astype(np.float32), cs.astype(np.float32)


def test_coefficients_parsed():
    nums = _coefficients()
    assert len(nums) == 10 and nums[0] == -0.5 and nums[4] == np.float32(np.pi) and nums[9] == 1.0


def test_within_two_ulp():
    rng = np.random.default_rng(3)
    y = np.concatenate([np.linspace(-8, 8, 400001), rng.uniform(-3, 5, 200000), rng.uniform(-1e5, 1e5, 50000),
                        np.arange(-40, 41) * 0.25]).astype(np.float32)
    s, c = sincospi_poly(y)
    yd = y.astype(np.float64)
    # exact sin(pi y), cos(pi y) for the FP32 input, with the argument reduced in FP64 first
    r = yd - 2.0 * np.round(yd / 2.0)
    es, ec = np.sin(np.pi * r), np.cos(np.pi * r)
    for got, ex in ((s, es), (c, ec)):
        tol = 2.0 * np.spacing(np.maximum(np.abs(ex), 2.0 ** -24).astype(np.float32)).astype(np.float64)
        err = np.abs(got.astype(np.float64) - ex)
        assert (err <= tol).all(), (err / tol).max()
