"""GPU parity: the CUDA path (through the C ABI) against the numpy oracle.

Tolerances: FP64 path max |dxi| <= 1e-10 (per step and over 100 steps);
FP32 path relative L2 of Re xi <= 2e-5 after 100 steps.
"""
import numpy as np
import pytest

import pfdd_oracle as O
from common import oracle_instance, small_loop
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def _run_gpu(ws, steps, precision=capi.FP64, states=None, stress_states=1, imag=capi.IMAG_AUTO):
    with capi.Stepper.from_workloads(ws, precision=precision, imag_mode=imag) as st:
        for i, w in enumerate(ws):
            s = w.xi0 if states is None else states[i]
            st.set_state(i, np.real(s), np.imag(s) if np.iscomplexobj(s) else None)
        st.advance(steps, stress_states)
        out = [st.get_state(i) for i in range(len(ws))]
        hist = [st.history(i) for i in range(len(ws))]
    return out, hist


@pytest.mark.parametrize("n,steps", [(16, 1), (16, 10), (32, 100)])
def test_fp64_loop_matches_oracle(n, steps):
    w = small_loop(n)
    inst = oracle_instance(w)
    ref, nrm, ave = O.run(inst, w.xi0, steps)
    (re, im), (hn, ha) = [x[0] for x in _run_gpu([w], steps)]
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10
    np.testing.assert_allclose(hn, nrm, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(ha, ave, rtol=1e-10, atol=1e-10)


def test_fp64_anisotropic_grid_and_sizes():
    # non-cubic grid with a factor-3 axis
    w = configs.loop_workload(n=16, radius=3.0)
    w2 = configs.Workload("aniso", 24, 16, 12, w.app, w.xn, w.xb, w.four, w.prim, w.material, 3, w.sigma,
                          0.5, np.random.default_rng(3).uniform(-0.2, 1.0, size=(3, 24, 16, 12)))
    inst = oracle_instance(w2)
    ref, _, _ = O.run(inst, w2.xi0, 5)
    (re, im), _ = [x[0] for x in _run_gpu([w2], 5)]
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10


@pytest.mark.parametrize("flag", [capi.CORE_PERFECT, capi.CORE_SINE, capi.CORE_MPEA, capi.CORE_SINE_FIELD])
def test_fp64_core_models(flag):
    w = small_loop(16)
    rng = np.random.default_rng(11)
    if flag == capi.CORE_MPEA:
        w.site = rng.uniform(0.1, 0.3, size=(w.S, w.nx, w.ny, w.nz))
    elif flag == capi.CORE_SINE_FIELD:
        w.site = np.exp(0.15 * rng.standard_normal((w.S, w.nx, w.ny, w.nz)))
    if flag == capi.CORE_PERFECT:
        w.material.An = 0.3
    w.core_flag = flag
    inst = oracle_instance(w)
    ref, _, _ = O.run(inst, w.xi0, 6)
    (re, im), _ = [x[0] for x in _run_gpu([w], 6)]
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10


@pytest.mark.parametrize("make", ["loop", "skew"])
def test_bcc_perfect_core(make):
    """Core model 5: angle-weighted core force from the gradient of Re xi,
    on an orthogonal grid and on the 60-degree masked grid."""
    if make == "loop":
        w = configs.loop_workload(n=16, nz=8, radius=4.0, seed=8, sigma_mpa=250.0)
    else:
        w = configs.frank_read_workload(nx=16, ny=16, nz=8, seg=4)
    w.core_flag = capi.CORE_BCC_PERFECT
    ref, _, _ = O.run(oracle_instance(w), w.xi0, 10)
    (re, im), _ = [x[0] for x in _run_gpu([w], 10)]
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10
    (r32, _), _ = [x[0] for x in _run_gpu([w], 10, precision=capi.FP32)]
    assert np.linalg.norm(r32 - ref.real) / np.linalg.norm(ref.real) <= 2e-5


def test_fp64_mask_and_complex_state():
    w = small_loop(16)
    rng = np.random.default_rng(5)
    w.xo = (rng.uniform(size=(w.S, 16, 16, 16)) < 0.3).astype(np.float64)
    xi0 = w.xi0 + 1j * rng.uniform(-0.01, 0.01, size=w.xi0.shape)
    inst = oracle_instance(w)
    ref, _, _ = O.run(inst, xi0, 8)
    (re, im), _ = [x[0] for x in _run_gpu([w], 8, states=[xi0])]
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10


def test_fp64_multi_instance_mixed_sizes():
    ws = [small_loop(16, seed=1), configs.loop_workload(n=32, radius=6.0, seed=2, sigma_mpa=350.0),
          configs.loop_workload(n=24, radius=4.0, seed=3, sigma_mpa=120.0)]
    outs, _ = _run_gpu(ws, 7)
    for w, (re, im) in zip(ws, outs):
        ref, _, _ = O.run(oracle_instance(w), w.xi0, 7)
        assert np.abs(re - ref.real).max() <= 1e-10
        assert np.abs(im - ref.imag).max() <= 1e-10


def test_fp32_loop_error_bound():
    w = small_loop(32)
    inst = oracle_instance(w)
    ref, _, _ = O.run(inst, w.xi0, 100)
    (re, im), _ = [x[0] for x in _run_gpu([w], 100, precision=capi.FP32)]
    rel = np.linalg.norm(re - ref.real) / np.linalg.norm(ref.real)
    assert rel <= 2e-5, rel


def test_fp64_stress_ramp_states():
    w = small_loop(16)
    w.dsigma = np.zeros((3, 3))
    w.dsigma[0, 2] = w.dsigma[2, 0] = 1e-3
    # 3 stress states x 2 iterations each, sigma += dsigma between states
    xi = w.xi0.astype(complex)
    sig = w.sigma.copy()
    for s in range(3):
        w2 = configs.Workload(w.name, w.nx, w.ny, w.nz, w.app, w.xn, w.xb, w.four, w.prim, w.material,
                              w.core_flag, sig.copy(), w.cd_dt, w.xi0)
        xi, _, _ = O.run(oracle_instance(w2), xi, 2)
        sig = sig + w.dsigma
    (re, im), _ = [x[0] for x in _run_gpu([w], 2, stress_states=3)]
    assert np.abs(re - xi.real).max() <= 1e-10
    assert np.abs(im - xi.imag).max() <= 1e-10


@pytest.mark.parametrize("prec,tol", [(capi.FP64, 1e-10), (capi.FP32, 5e-5)])
def test_nyquist_carrier_equals_full(prec, tol):
    """Im xi carried only on the Nyquist planes (no mask) gives the same Re and
    Im xi as carrying the full second field, and both match the oracle."""
    w = small_loop(32)
    ref, nrm, _ = O.run(oracle_instance(w), w.xi0, 30)
    outs = {}
    for mode in (capi.IMAG_NYQUIST, capi.IMAG_FULL):
        (re, im), (hn, _) = [x[0] for x in _run_gpu([w], 30, precision=prec, imag=mode)]
        outs[mode] = (re, im)
        scale = np.abs(ref.real).max()
        assert np.abs(re - ref.real).max() <= tol * scale
        assert np.abs(im - ref.imag).max() <= tol * scale
        np.testing.assert_allclose(hn, nrm, rtol=1e-9 if prec == capi.FP64 else 1e-3)
    assert np.abs(outs[capi.IMAG_NYQUIST][0] - outs[capi.IMAG_FULL][0]).max() <= tol


def test_nyquist_rejects_imaginary_state():
    w = small_loop(16)
    with capi.Stepper.from_workloads([w], imag_mode=capi.IMAG_NYQUIST) as st:
        with pytest.raises(capi.PfddError) as e:
            st.set_state(0, w.xi0, np.full(w.xi0.shape, 1e-3))
        assert e.value.code == -1


def test_nyquist_rejects_mask():
    w = small_loop(16)
    w.xo = np.zeros((w.S, 16, 16, 16))
    with pytest.raises(capi.PfddError):
        capi.Stepper.from_workloads([w], imag_mode=capi.IMAG_NYQUIST)


@pytest.mark.parametrize("make", ["loop", "skew"])
def test_bcc_perfect_energy(make):
    """Energy with core model 5: usf' cof(theta) sin^2(pi xi) summed with the
    elastic and applied terms, FP64, against the oracle."""
    if make == "loop":
        w = configs.loop_workload(n=16, nz=8, radius=4.0, seed=8, sigma_mpa=250.0)
    else:
        w = configs.frank_read_workload(nx=16, ny=16, nz=8, seg=4)
    w.core_flag = capi.CORE_BCC_PERFECT
    inst = oracle_instance(w)
    xi, _, _ = O.run(inst, w.xi0, 5)
    want = O.total_energy(inst, xi)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        st.advance(5)
        got = st.energy(0)
    for g, e in zip(got, want):
        assert abs(g - e) <= 1e-10 * max(1.0, abs(e)), (got, want)


def test_extended_core_energy():
    """Energy with core model 2 (three-system Fourier GSFE, the Ni preset of
    the reference-written fixture): the plane's fcore, FP64, against the oracle,
    and its gradient is the update's drift (energy decreases per step)."""
    from common import load_golden
    w, fx = load_golden("fcc12_extended")
    inst = oracle_instance(w)
    xi, _, _ = O.run(inst, fx["xi0"], 3)
    want = O.total_energy(inst, xi)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, np.real(fx["xi0"]), np.imag(fx["xi0"]))
        st.advance(3)
        got = st.energy(0)
        st.advance(1)
        later = st.energy(0)
    for g, e in zip(got, want):
        assert abs(g - e) <= 1e-10 * max(1.0, abs(e)), (got, want)
    assert sum(later) < sum(got)
