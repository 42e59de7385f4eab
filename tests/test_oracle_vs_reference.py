"""Live pin: the numpy oracle and the reference sources compiled in
oracle/_ref (make -C oracle/ref_build) on fresh seeded inputs, plus the FFTW-2
API stand-in against numpy.fft.  Skipped where the oracle binary is absent."""
import ctypes
import os

import numpy as np
import pytest

import pfdd_oracle as O
import ref_runner
from common import oracle_instance
from pfdd_b200 import configs

needs_ref = pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("seed,n,nz,sig", [(1, 16, 8, 150.0), (2, 12, 12, 400.0)])
def test_oracle_equals_reference_live(seed, n, nz, sig):
    w = configs.loop_workload(n=n, nz=nz, radius=n / 4.0, seed=seed, sigma_mpa=sig)
    r = ref_runner.run_reference(w, 5)
    su = r["setup"]
    np.testing.assert_allclose(su["xn"], w.xn, atol=1e-15)
    np.testing.assert_allclose(su["xb"], w.xb, atol=1e-15)
    xi, nrm, ave = O.run(oracle_instance(w), w.xi0, 5)
    assert np.abs(xi - r["xi"]).max() <= 1e-12
    np.testing.assert_allclose(nrm, r["xinorm"], rtol=1e-11)
    np.testing.assert_allclose(ave, r["xiave"], rtol=1e-11)


@needs_ref
def test_bmatrix_restatement_equals_reference_table():
    w = configs.fcc_workload(8, 6, 4, n_loops=1, seed=3)
    r = ref_runner.run_reference(w, 1, want_B=True)
    C44, C12, C11 = w.material.elastic()
    BB = O.bmatrix(w.nx, w.ny, w.nz, w.four, w.xn, w.xb, C44, C12, C11, w.material.dslip)
    # the reference stores BB[b][a][k]; B is symmetric in (a, b)
    assert np.abs(BB - r["BB"]).max() <= 1e-13 * max(1.0, np.abs(BB).max())


@pytest.mark.skipif(not os.path.exists(os.path.join(ref_runner.REF_DIR, "libfftshim.so")),
                    reason="FFT stand-in not built")
@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 12, 10), (32, 48, 64), (7, 9, 11)])
def test_fftw_api_stand_in_matches_numpy(shape):
    lib = ctypes.CDLL(os.path.join(ref_runner.REF_DIR, "libfftshim.so"))
    lib.pfdd_shim_fft3d.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 5
    rng = np.random.default_rng(0)
    for h in (1, 3):
        a = rng.standard_normal(shape + (h,)) + 1j * rng.standard_normal(shape + (h,))
        for sign in (-1, 1):
            b = np.ascontiguousarray(a.copy())
            lib.pfdd_shim_fft3d(b.ctypes.data, *shape, h, sign)
            ref = np.fft.fftn(a, axes=(0, 1, 2)) if sign < 0 else np.fft.ifftn(a, axes=(0, 1, 2)) * np.prod(shape)
            assert np.abs(b - ref).max() <= 1e-13 * np.abs(ref).max()
