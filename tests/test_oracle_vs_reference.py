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


@needs_ref
@pytest.mark.parametrize("make", ["loop", "fcc", "skew"])
def test_strain_stress_restatement_equals_reference(make):
    """Strain and stress diagnostics (Fmatrix, strain, stressfree_strain,
    total_average_strain, stress) of the state after 3 GL steps."""
    if make == "loop":
        w = configs.loop_workload(n=16, nz=8, radius=4.0, seed=5, sigma_mpa=250.0)
    elif make == "fcc":
        w = configs.fcc_workload(8, 6, 4, n_loops=1, seed=3)
    else:
        w = configs.frank_read_workload(nx=16, ny=16, nz=8, seg=4)
    r = ref_runner.run_reference(w, 3, want_stress=True)
    su = r["setup"]
    C44, C12, C11 = su["C44"], su["C12"], su["C11"]
    eps, sigma, ave_eps, ave_sigma, avepst = O.strain_stress(
        w.nx, w.ny, w.nz, su["four"], su["xn"], su["xb"], su["dslip"], C44, C12, C11, su["sigma_rot"], r["xi"])
    scale_e = max(1e-30, np.abs(r["eps"]).max())
    scale_s = max(1e-30, np.abs(r["sigma"].real).max())
    assert np.abs(eps - r["eps"]).max() <= 1e-12 * scale_e
    assert np.abs(sigma - r["sigma"].real).max() <= 1e-12 * scale_s
    assert np.abs(r["sigma"].imag).max() == 0.0
    np.testing.assert_allclose(avepst, r["avepst"], rtol=1e-12, atol=1e-12 * np.abs(avepst).max())
    # the averages are means of fields of either sign: compare on the fields' scale
    assert np.abs(ave_eps - r["ave_eps"]).max() <= 1e-12 * scale_e
    assert np.abs(ave_sigma - r["ave_sigma"]).max() <= 1e-12 * scale_s


@needs_ref
@pytest.mark.parametrize("make", ["loop", "skew"])
def test_bcc_perfect_core_equals_reference(make):
    """Core model 5: the core force weighted by the edge/screw angle of the
    gradient of Re xi (orthogonal grid, and the 60-degree grid where the
    in-place `four` transform of the gradient matters)."""
    if make == "loop":
        w = configs.loop_workload(n=16, nz=8, radius=4.0, seed=8, sigma_mpa=250.0)
    else:
        w = configs.frank_read_workload(nx=16, ny=16, nz=8, seg=4)
    w.core_flag = 5
    r = ref_runner.run_reference(w, 4)
    xi, nrm, ave = O.run(oracle_instance(w), w.xi0, 4)
    assert np.abs(xi - r["xi"]).max() <= 1e-12
    np.testing.assert_allclose(nrm, r["xinorm"], rtol=1e-10)


@needs_ref
@pytest.mark.parametrize("flag", [1, 6])
def test_non_schmid_and_usfe_angle_tau_equal_reference(flag):
    """resolSS_non_Schmid (the projections on the MRSSP at angle_to_110 and
    the plane 60 degrees from it, weights w1..w3) with the perfect core and
    with the USFE(angle, tau) core whose amplitude follows sigma_rot[2][1]."""
    w = configs.bcc_screw_workload(n=16, nz=8, core_flag=flag)
    r = ref_runner.run_reference(w, 4)
    su = r["setup"]
    assert su["non_schmid"][0] == 1
    np.testing.assert_array_equal(su["non_schmid"][1], w.non_schmid)
    np.testing.assert_array_equal(su["usfe_fit"], configs.TA_USFE_FIT)
    inst = oracle_instance(w)
    np.testing.assert_allclose(inst.tau, su["tau"], rtol=1e-13)
    sr = O.rotate_stress(w.sigma, w.prim, np.linalg.inv(w.prim), 1.0)
    schmid = O.resolved_shear(sr, w.xn, w.xb, w.material.dslip)
    assert abs(schmid[0] - inst.tau[0]) > 0.1 * abs(schmid[0])
    xi, nrm, ave = O.run(inst, w.xi0, 4)
    assert np.abs(xi - r["xi"]).max() <= 1e-12
    np.testing.assert_allclose(nrm, r["xinorm"], rtol=1e-11)
    np.testing.assert_allclose(ave, r["xiave"], rtol=1e-11)


@needs_ref
def test_usfe_angle_tau_follows_each_stress_state():
    """Core model 6 over three stress states of a sigma_yz ramp: the amplitude
    is re-evaluated from each state's sigma_rot[2][1]."""
    from common import oracle_run_golden
    w = configs.bcc_screw_workload(n=12, nz=8, core_flag=6, seed=4, angle=-15.0)
    w.dsigma = configs._sigma("yz", 6e-3)
    r = ref_runner.run_reference(w, 2, stress_states=3)
    xi, nrm, ave = oracle_run_golden(w, {"xi0": w.xi0, "sigma": w.sigma, "dsigma": w.dsigma,
                                         "stress_states": 3, "steps": 2})
    assert np.abs(xi - r["xi"]).max() <= 1e-12
    np.testing.assert_allclose(ave, r["xiave"], rtol=1e-11)


@needs_ref
@pytest.mark.parametrize("make", ["bcc", "frank_read"])
def test_core_profile_equals_reference(make):
    """project_core_energy (delta and the ddelta line) of the state after
    three steps, for one system (app 1SBCC) and two (Frank-Read, 60-degree grid)."""
    if make == "bcc":
        w = configs.bcc_screw_workload(n=16, nz=8, core_flag=1)
    else:
        w = configs.frank_read_workload(nx=16, ny=16, nz=8, seg=4)
        w.non_schmid = (5.0, 0.1, 0.2, 0.3)
    r = ref_runner.run_reference(w, 3, want_profile=True)
    xi, _, _ = O.run(oracle_instance(w), w.xi0, 3)
    np.testing.assert_allclose(xi, r["xi"], rtol=0, atol=1e-12)
    d, dd = O.core_profile(xi.real, w.xb, r["delta"].shape[0])
    assert np.abs(d - r["delta"]).max() <= 1e-12
    assert np.abs(dd - r["ddelta"]).max() <= 1e-12


@needs_ref
def test_conductivity_fields_equal_reference():
    """The defined part of the conductivity iteration (forwardcond, divcurrent,
    backwardcond's transforms, current and conductivity) of a seeded complex
    state on a Cu/W multilayer.  (The reference's driving term reads its layer
    table before writing it, so condxi after an update is not comparable.)"""
    cc = configs.cond_case()
    w = cc.workload
    A, B = O.CondMaterial(**cc.A), O.CondMaterial(**cc.B)
    eff, lay = O.cond_layers(A, B, w.ny, cc.temperature)
    rng = np.random.default_rng(1)
    c0 = (rng.standard_normal((w.nx, w.ny, w.nz)) + 1j * rng.standard_normal((w.nx, w.ny, w.nz))) * 1e-16
    r = ref_runner.run_reference_cond(cc.deck(), w.nx, w.ny, w.nz, 1, state=c0)
    a, b, j, cond = O.cond_fields(c0, w.four, eff, cc.El_y, configs.EPSILON_ZERO)
    assert np.abs(a - r["a"]).max() <= 1e-13 * np.abs(r["a"]).max()
    assert np.abs(b - r["b"]).max() <= 1e-13 * np.abs(r["b"]).max()
    # sigma_eff carries the cancellation of the grain-boundary series
    assert np.abs(j - r["j"]).max() <= 1e-10 * np.abs(r["j"]).max()
    assert abs(cond / r["conductivity"][0] - 1.0) <= 1e-10
