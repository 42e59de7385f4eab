"""Strain and stress diagnostics on the GPU (pfdd_gpu_strain_stress, through
the C ABI) against the numpy restatement of the reference's strain, stress
and average routines (itself pinned to the compiled reference in
test_oracle_vs_reference.py), on the state the GPU reached.

Tolerance: FP64 1e-10 of each field's largest magnitude; FP32 2e-4."""
import numpy as np
import pytest

import pfdd_oracle as O
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def _workload(make):
    if make == "loop":
        return configs.loop_workload(n=16, nz=8, radius=4.0, seed=5, sigma_mpa=250.0)
    if make == "fcc":
        return configs.fcc_workload(8, 6, 4, n_loops=1, seed=3)
    return configs.frank_read_workload(nx=16, ny=16, nz=8, seg=4)   # 60-degree grid, mask, full Im carrier


def _sigma_rot(w):
    prim = np.asarray(w.prim, float)
    return O.rotate_stress(w.sigma, prim, np.linalg.inv(prim), np.linalg.det(prim))


@pytest.mark.parametrize("make", ["loop", "fcc", "skew"])
@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_strain_stress_matches_oracle(make, prec):
    w = _workload(make)
    with capi.Stepper.from_workloads([w], precision=prec) as st:
        st.set_state(0, w.xi0)
        st.advance(3)
        re, im = st.get_state(0)
        eps, sig, ave_eps, ave_sig = st.strain_stress(0)
        _, _, ave_eps2, ave_sig2 = st.strain_stress(0, fields=False)
        st.advance(1)   # the spectrum buffer was reused: stepping on must still work
    C44, C12, C11 = w.material.elastic()
    eo, so, aeo, aso, _ = O.strain_stress(w.nx, w.ny, w.nz, w.four, w.xn, w.xb, w.material.dslip, C44, C12, C11,
                                          _sigma_rot(w), re + 1j * im)
    tol = 1e-10 if prec == capi.FP64 else 2e-4
    se, ss = np.abs(eo.real).max(), np.abs(so).max()
    assert np.abs(eps - eo.real).max() <= tol * se
    assert np.abs(sig - so).max() <= tol * ss
    assert np.abs(ave_eps - aeo).max() <= tol * se
    assert np.abs(ave_sig - aso).max() <= tol * ss
    # without fields the stress average is formed from the sums it is linear in
    # (<strain> and <Re xi>): the same averages to round-off
    np.testing.assert_allclose(ave_eps2, ave_eps, rtol=0, atol=1e-12 * se)
    np.testing.assert_allclose(ave_sig2, ave_sig, rtol=0, atol=1e-12 * ss)
