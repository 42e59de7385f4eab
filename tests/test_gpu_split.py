"""GPU parity of the split plane passes (each (field, x) plane on a 2-CTA
cluster, half the rows per CTA, the first radix-2 y stage through distributed
shared memory), forced with PFDD_PLANE_SPLIT=1 at sizes the oracle runs in
seconds, against the same oracle and tolerances as the whole-plane path:
FP64 max |dxi| <= 1e-10, FP32 relative L2 <= 2e-5 on the loop workload.

ny = 18 makes ny/2 odd, so the ky = ny/2 Nyquist row lands on rank 1.
"""
import numpy as np
import pytest

import pfdd_oracle as O
from common import adjoint_l2, oracle_instance, small_loop
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["1", "0"], ids=["split", "whole"])
def split_env(request, monkeypatch):
    monkeypatch.setenv("PFDD_PLANE_SPLIT", request.param)
    return request.param


def _run(ws, steps, precision=capi.FP64, states=None, imag=capi.IMAG_AUTO, stress_states=1):
    with capi.Stepper.from_workloads(ws, precision=precision, imag_mode=imag) as st:
        for i, w in enumerate(ws):
            s = w.xi0 if states is None else states[i]
            st.set_state(i, np.real(s), np.imag(s) if np.iscomplexobj(s) else None)
        st.advance(steps, stress_states)
        out = [st.get_state(i) for i in range(len(ws))]
        hist = [st.history(i) for i in range(len(ws))]
    return out, hist


def _aniso(nx, ny, nz, seed=3):
    w = configs.loop_workload(n=16, radius=3.0)
    xi0 = np.random.default_rng(seed).uniform(-0.2, 1.0, size=(3, nx, ny, nz))
    return configs.Workload("aniso", nx, ny, nz, w.app, w.xn, w.xb, w.four, w.prim, w.material, 3, w.sigma,
                            0.5, xi0)


@pytest.mark.parametrize("imag", [capi.IMAG_NYQUIST, capi.IMAG_FULL])
def test_split_loop_fp64(split_env, imag):
    w = small_loop(16)
    inst = oracle_instance(w)
    ref, nrm, ave = O.run(inst, w.xi0, 12)
    (re, im), (hn, ha) = [x[0] for x in _run([w], 12, imag=imag)]
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10
    np.testing.assert_allclose(hn, nrm, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(ha, ave, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("shape", [(16, 18, 8), (12, 6, 12), (8, 24, 16)])
def test_split_odd_half_rows_fp64(split_env, shape):
    w = _aniso(*shape)
    inst = oracle_instance(w)
    ref, _, _ = O.run(inst, w.xi0, 6)
    (re, im), _ = [x[0] for x in _run([w], 6)]
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10


def test_split_mask_complex_state_fp64(split_env):
    w = small_loop(16)
    rng = np.random.default_rng(5)
    w.xo = (rng.uniform(size=(w.S, 16, 16, 16)) < 0.3).astype(np.float64)
    xi0 = w.xi0 + 1j * rng.uniform(-0.01, 0.01, size=w.xi0.shape)
    inst = oracle_instance(w)
    ref, _, _ = O.run(inst, xi0, 8)
    (re, im), _ = [x[0] for x in _run([w], 8, states=[xi0])]
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10


def test_split_group_fp64(split_env):
    # three instances of one group (one launch per kernel), different stresses
    ws = []
    for k, s in enumerate((150.0, 250.0, 350.0)):
        ws.append(small_loop(16, seed=100 + k, sigma_mpa=s))
    out, _ = _run(ws, 7)
    for w, (re, im) in zip(ws, out):
        ref, _, _ = O.run(oracle_instance(w), w.xi0, 7)
        assert np.abs(re - ref.real).max() <= 1e-10
        assert np.abs(im - ref.imag).max() <= 1e-10


def test_split_energy_fp64(split_env):
    w = small_loop(16)
    inst = oracle_instance(w)
    ref, _, _ = O.run(inst, w.xi0, 5)
    want = O.total_energy(inst, ref)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        st.advance(5)
        got = st.energy(0)
    for g, e in zip(got, want):
        assert abs(g - e) <= 1e-10 * max(1.0, abs(e)), (got, want)


def test_split_fp32_loop(split_env):
    w = small_loop(32)
    inst = oracle_instance(w)
    ref, _, _ = O.run(inst, w.xi0, 100)
    (re, _), _ = [x[0] for x in _run([w], 100, precision=capi.FP32)]
    rel = np.linalg.norm(re - ref.real) / np.linalg.norm(ref.real)
    assert rel <= 2e-5


def test_split_fp32_fcc_error_like_whole(monkeypatch):
    # 12 FCC systems: FP32 rounding is amplified near the loop cores; the
    # split layout must not add error beyond the whole-plane path's
    w = configs.fcc_workload(32, 32, 16, n_loops=3, seed=7)
    inst = oracle_instance(w)
    ref, _, _ = O.run(inst, w.xi0, 30)
    rel = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("PFDD_PLANE_SPLIT", mode)
        (re, _), _ = [x[0] for x in _run([w], 30, precision=capi.FP32)]
        rel[mode] = np.linalg.norm(re - ref.real) / np.linalg.norm(ref.real)
    assert rel["0"] <= 5e-5 and rel["1"] <= 5e-5, rel
    assert rel["1"] <= 1.5 * rel["0"] + 1e-6, rel


def test_split_adjoint_matches_whole(monkeypatch):
    # the adjoint pass (reductions of four sums) agrees between the two layouts
    w = small_loop(16)
    rng = np.random.default_rng(2)
    target = np.real(w.xi0) + 0.01 * rng.standard_normal(w.xi0.shape)
    res = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("PFDD_PLANE_SPLIT", mode)
        with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
            st.set_state(0, w.xi0)
            res[mode] = adjoint_l2(st, 0, 6, 3, target)
    for a, b in zip(res["0"], res["1"]):
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-14)
