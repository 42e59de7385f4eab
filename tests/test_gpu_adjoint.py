"""Adjoint of the GL step through the C ABI (pfdd_gpu_adjoint_forward /
_backward, pfdd_gpu_adjoint), seeded with dL/dRe xi_N.

The test-harness loss J = sum (Re xi_N - target)^2 after N steps
(common.adjoint_l2) and a linear loss; gradients with respect to
(isf, usf) and sigma are checked against FP64 central finite differences of
J computed with the numpy oracle (an independent restatement of the
reference step).  Tolerance: 2e-6 relative (FP64), 2e-3 (FP32 vs FP64).
The torch.autograd.Function wrapper lives only here, in the test harness."""
import numpy as np
import pytest

import pfdd_oracle as O
from common import adjoint_l2, oracle_instance
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu

N_STEPS, CKPT = 12, 5


def _workload(mask=False):
    w = configs.loop_workload(n=16, nz=8, radius=4.0, seed=31, sigma_mpa=250.0)
    if mask:
        rng = np.random.default_rng(2)
        w.xo = (rng.uniform(size=(w.S, w.nx, w.ny, w.nz)) < 0.25).astype(float)
    return w


def _target(w):
    w2 = configs.loop_workload(n=16, nz=8, radius=4.0, seed=31, sigma_mpa=200.0)
    w2.material.isf, w2.material.usf = 0.040, 0.160
    w2.xo = w.xo
    xi, _, _ = O.run(oracle_instance(w2), w.xi0, N_STEPS)
    return xi.real


def _loss_oracle(w, target, isf=None, usf=None, dsig=0.0):
    m = configs.Material(**{k: getattr(w.material, k) for k in ("preset", "mu", "young", "b", "isf", "usf", "An",
                                                                 "dslip")})
    if isf is not None:
        m.isf = isf
    if usf is not None:
        m.usf = usf
    sig = w.sigma.copy()
    sig[0, 2] += dsig
    sig[2, 0] += dsig
    w2 = configs.Workload(w.name, w.nx, w.ny, w.nz, w.app, w.xn, w.xb, w.four, w.prim, m, w.core_flag, sig,
                          w.cd_dt, w.xi0, xo=w.xo)
    xi, _, _ = O.run(oracle_instance(w2), w.xi0, N_STEPS)
    return float(np.sum((xi.real - target) ** 2))


def _gpu_adjoint(w, target, prec=capi.FP64):
    with capi.Stepper.from_workloads([w], precision=prec) as st:
        st.set_state(0, w.xi0)
        loss, dp, ds = adjoint_l2(st, 0, N_STEPS, CKPT, target)
        re, _ = st.get_state(0)
    return loss, dp, ds, re


@pytest.mark.parametrize("mask", [False, True])
def test_adjoint_matches_finite_differences(mask):
    w = _workload(mask)
    target = _target(w)
    loss, dp, ds, re = _gpu_adjoint(w, target)
    L0 = _loss_oracle(w, target)
    assert abs(loss - L0) <= 1e-10 * max(1.0, L0)
    # the handle ends at xi_N
    ref, _, _ = O.run(oracle_instance(w), w.xi0, N_STEPS)
    assert np.abs(re - ref.real).max() <= 1e-10
    h_isf, h_usf, h_sig = 1e-6 * w.material.isf, 1e-6 * w.material.usf, 1e-9
    fd_isf = (_loss_oracle(w, target, isf=w.material.isf + h_isf) -
              _loss_oracle(w, target, isf=w.material.isf - h_isf)) / (2 * h_isf)
    fd_usf = (_loss_oracle(w, target, usf=w.material.usf + h_usf) -
              _loss_oracle(w, target, usf=w.material.usf - h_usf)) / (2 * h_usf)
    fd_sxz = (_loss_oracle(w, target, dsig=h_sig) - _loss_oracle(w, target, dsig=-h_sig)) / (2 * h_sig)
    assert abs(dp[0] - fd_isf) <= 2e-6 * abs(fd_isf), (dp[0], fd_isf)
    assert abs(dp[1] - fd_usf) <= 2e-6 * abs(fd_usf), (dp[1], fd_usf)
    assert abs(ds[4] - fd_sxz) <= 2e-6 * abs(fd_sxz), (ds[4], fd_sxz)


def test_adjoint_fp32_close_to_fp64():
    w = _workload()
    target = _target(w)
    l64, dp64, ds64, _ = _gpu_adjoint(w, target, capi.FP64)
    l32, dp32, ds32, _ = _gpu_adjoint(w, target, capi.FP32)
    assert abs(l32 - l64) <= 2e-3 * l64
    assert np.abs(dp32 - dp64).max() <= 2e-3 * np.abs(dp64).max()
    assert np.abs(ds32 - ds64).max() <= 2e-3 * np.abs(ds64).max()


def test_autograd_function_wrapper():
    """A torch.autograd.Function over the C-ABI adjoint (test harness only)."""
    import torch

    w0 = _workload()
    target = _target(w0)

    class PfddLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, isf, usf):
            w = _workload()
            w.material.isf, w.material.usf = float(isf), float(usf)
            loss, dp, _, _ = _gpu_adjoint(w, target)
            ctx.save_for_backward(torch.tensor(dp))
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            (dp,) = ctx.saved_tensors
            return g * dp[0], g * dp[1]

    isf = torch.tensor(w0.material.isf, dtype=torch.float64, requires_grad=True)
    usf = torch.tensor(w0.material.usf, dtype=torch.float64, requires_grad=True)
    loss = PfddLoss.apply(isf, usf)
    loss.backward()
    _, dp, _, _ = _gpu_adjoint(w0, target)
    assert float(isf.grad) == pytest.approx(dp[0], rel=1e-12)
    assert float(usf.grad) == pytest.approx(dp[1], rel=1e-12)


def test_store_all_equals_checkpointed():
    """ckpt_every >= n_steps keeps every forward state (no recomputation) and
    gives the checkpointed call's loss and gradients."""
    w = _workload(False)
    target = _target(w)
    a = _gpu_adjoint(w, target)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        loss, dp, ds = adjoint_l2(st, 0, N_STEPS, N_STEPS, target)
        re, _ = st.get_state(0)
    assert abs(loss - a[0]) <= 1e-12 * abs(a[0])
    np.testing.assert_allclose(dp, a[1], rtol=1e-12, atol=0)
    np.testing.assert_allclose(ds, a[2], rtol=1e-12, atol=1e-12 * np.abs(a[2]).max())
    assert np.abs(re - a[3]).max() == 0.0


def test_general_seed_linear_loss_and_reused_tape():
    """A seed that is not an L2 residual: L = sum W * Re xi_N with a fixed
    random weight W (dL/dRe xi_N = W), checked against FP64 central finite
    differences of the oracle's L; a second backward pass on the same tape
    with another seed equals a fresh one-call adjoint with that seed."""
    w = _workload()
    W = np.random.default_rng(4).standard_normal((w.S, w.nx, w.ny, w.nz))

    def L(isf=None, usf=None, dsig=0.0):
        m = configs.Material(**{k: getattr(w.material, k) for k in ("preset", "mu", "young", "b", "isf", "usf",
                                                                     "An", "dslip")})
        m.isf = w.material.isf if isf is None else isf
        m.usf = w.material.usf if usf is None else usf
        sig = w.sigma.copy()
        sig[0, 2] += dsig
        sig[2, 0] += dsig
        w2 = configs.Workload(w.name, w.nx, w.ny, w.nz, w.app, w.xn, w.xb, w.four, w.prim, m, w.core_flag, sig,
                              w.cd_dt, w.xi0)
        xi, _, _ = O.run(oracle_instance(w2), w.xi0, N_STEPS)
        return float(np.sum(W * xi.real))

    W2 = np.random.default_rng(5).standard_normal(W.shape)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        st.adjoint_forward(0, N_STEPS, CKPT)
        dp, ds = st.adjoint_backward(0, W)
        dp2, ds2 = st.adjoint_backward(0, W2)
        st.set_state(0, w.xi0)
        dp2b, ds2b = st.adjoint(0, N_STEPS, CKPT, W2)
        # the tape is gone once the state changes
        st.set_state(0, w.xi0)
        with pytest.raises(capi.PfddError) as e:
            st.adjoint_backward(0, W)
        assert e.value.code == -7
    h_isf, h_usf, h_sig = 1e-6 * w.material.isf, 1e-6 * w.material.usf, 1e-9
    fd_isf = (L(isf=w.material.isf + h_isf) - L(isf=w.material.isf - h_isf)) / (2 * h_isf)
    fd_usf = (L(usf=w.material.usf + h_usf) - L(usf=w.material.usf - h_usf)) / (2 * h_usf)
    fd_sxz = (L(dsig=h_sig) - L(dsig=-h_sig)) / (2 * h_sig)
    assert abs(dp[0] - fd_isf) <= 2e-6 * abs(fd_isf), (dp[0], fd_isf)
    assert abs(dp[1] - fd_usf) <= 2e-6 * abs(fd_usf), (dp[1], fd_usf)
    assert abs(ds[4] - fd_sxz) <= 2e-6 * abs(fd_sxz), (ds[4], fd_sxz)
    np.testing.assert_array_equal(dp2, dp2b)
    np.testing.assert_array_equal(ds2, ds2b)
