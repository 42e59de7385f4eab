"""Non-Schmid resolved shear stress and the USFE(angle, tau) core (model 6)
on the GPU through the C ABI, against the numpy oracle (itself pinned to the
reference in test_oracle_vs_reference.py and by tests/golden/bcc_non_schmid).

Tolerances: FP64 max |dxi| <= 1e-10; FP32 relative L2 of Re xi <= 2e-5;
energies 1e-10 relative; adjoint stress gradients 2e-6 relative against
central finite differences of the oracle."""
import dataclasses

import numpy as np
import pytest

import pfdd_oracle as O
from common import adjoint_l2, oracle_instance, oracle_run_golden
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def _run(ws, steps, precision=capi.FP64, stress_states=1):
    with capi.Stepper.from_workloads(ws, precision=precision) as st:
        for i, w in enumerate(ws):
            st.set_state(i, w.xi0)
        st.advance(steps, stress_states)
        return [st.get_state(i) for i in range(len(ws))]


@pytest.mark.parametrize("flag", [1, 6])
def test_non_schmid_matches_oracle(flag):
    w = configs.bcc_screw_workload(n=16, nz=8, core_flag=flag)
    ref, _, _ = O.run(oracle_instance(w), w.xi0, 10)
    (re, im), = _run([w], 10)
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10
    (r32, _), = _run([w], 10, precision=capi.FP32)
    assert np.linalg.norm(r32 - ref.real) / np.linalg.norm(ref.real) <= 2e-5


def test_usfe_amplitude_per_stress_state_and_instance():
    """Two instances in one batched group with different loads over a ramp of
    three stress states: each instance's core amplitude follows its own
    sigma_rot[2][1] in every state."""
    ws = []
    for k, s in enumerate((250.0, 400.0)):
        w = configs.bcc_screw_workload(n=16, nz=8, core_flag=6, seed=20 + k, sigma_mpa=s)
        w.dsigma = configs._sigma("yz", (3e-3, -2e-3)[k])
        ws.append(w)
    got = _run(ws, 3, stress_states=3)
    for w, (re, im) in zip(ws, got):
        ref, _, _ = oracle_run_golden(w, {"xi0": w.xi0, "sigma": w.sigma, "dsigma": w.dsigma,
                                          "stress_states": 3, "steps": 3})
        assert np.abs(re - ref.real).max() <= 1e-10
        assert np.abs(im - ref.imag).max() <= 1e-10


def test_usfe_energy_matches_oracle():
    w = configs.bcc_screw_workload(n=16, nz=8, core_flag=6)
    inst = oracle_instance(w)
    xi, _, _ = O.run(inst, w.xi0, 5)
    want = O.total_energy(inst, xi)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        st.advance(5)
        got = st.energy(0)
    for g, e in zip(got, want):
        assert abs(g - e) <= 1e-10 * max(1.0, abs(e)), (got, want)


N_STEPS, CKPT = 8, 3


def _loss_oracle(w, target, c, h):
    idx = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)][c]
    sig = w.sigma.copy()
    sig[idx] += h
    if idx[0] != idx[1]:
        sig[idx[::-1]] += h
    xi, _, _ = O.run(oracle_instance(dataclasses.replace(w, sigma=sig)), w.xi0, N_STEPS)
    return float(np.sum((xi.real - target) ** 2))


def test_adjoint_stress_gradient_non_schmid_usfe():
    """dJ/dsigma through the non-Schmid projections and, for sigma_yz, the
    stress dependence of the model 6 amplitude."""
    w = configs.bcc_screw_workload(n=16, nz=8, core_flag=6, sigma_mpa=350.0)
    w2 = configs.bcc_screw_workload(n=16, nz=8, core_flag=6, sigma_mpa=200.0)
    target, _, _ = O.run(oracle_instance(w2), w.xi0, N_STEPS)
    target = target.real
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        loss, dp, ds = adjoint_l2(st, 0, N_STEPS, CKPT, target)
    assert abs(loss - _loss_oracle(w, target, 0, 0.0)) <= 1e-10 * max(1.0, loss)
    h = 1e-9
    for c in (4, 5):   # sigma_xz, sigma_yz (sigma_yz moves the amplitude)
        fd = (_loss_oracle(w, target, c, h) - _loss_oracle(w, target, c, -h)) / (2 * h)
        assert abs(ds[c] - fd) <= 2e-6 * abs(fd), (c, ds[c], fd)


@pytest.mark.parametrize("make,planes", [("bcc", 1), ("frank_read", 2), ("fcc", 4)])
def test_core_profile_matches_oracle(make, planes):
    """pfdd_gpu_core_profile (project_core_energy) after 4 steps: Re xi for
    one and two systems, the projection on b_1 for twelve FCC systems."""
    if make == "bcc":
        w = configs.bcc_screw_workload(n=16, nz=8, core_flag=6)
    elif make == "frank_read":
        w = configs.frank_read_workload(nx=16, ny=16, nz=8, seg=4)
        w.non_schmid = (5.0, 0.1, 0.2, 0.3)
    else:
        w = configs.fcc_workload(16, 12, 8, n_loops=3, seed=5)
    xi, _, _ = O.run(oracle_instance(w), w.xi0, 4)
    d_ref, dd_ref = O.core_profile(xi.real, w.xb, planes)
    for prec, tol in ((capi.FP64, 1e-10), (capi.FP32, 2e-4)):
        with capi.Stepper.from_workloads([w], precision=prec) as st:
            st.set_state(0, w.xi0)
            st.advance(4)
            d, dd = st.core_profile(0, planes)
        scale = max(1.0, np.abs(d_ref).max())
        assert np.abs(d - d_ref).max() <= tol * scale
        assert np.abs(dd - dd_ref).max() <= 2 * tol * scale
