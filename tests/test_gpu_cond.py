"""The conductivity sub-problem on the GPU (pfdd_gpu_cond_*) against the
oracle's restatement (tests/test_oracle_vs_reference.py pins its defined part
to the reference).  Tolerances: FP64 condxi and statistics 1e-10 relative;
FP32 condxi 1e-4 of its scale, conductivity 1e-6."""
import numpy as np
import pytest

import pfdd_oracle as O
from common import oracle_instance
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def _case(nx=8, ny=32, nz=8):
    cc = configs.cond_case(nx=nx, ny=ny, nz=nz)
    eff, lay = capi.cond_layers(cc.A, cc.B, ny, cc.temperature)
    rng = np.random.default_rng(2)
    c0 = (rng.standard_normal((nx, ny, nz)) + 1j * rng.standard_normal((nx, ny, nz))) * 1e-16
    return cc, eff, lay, c0


def _oracle(cc, eff, lay, c0, n):
    c, out = c0, []
    for _ in range(n):
        c, nrm, ave, cond = O.cond_step(c, cc.workload.four, eff, lay, cc.El_y, configs.EPSILON_ZERO, 1.0)
        out.append((nrm, ave, cond))
    return c, np.array(out)


# (8, 32, 8) and (16, 24, 12) run split planes (2-CTA clusters: too few planes
# for the SMs), (384, 16, 8) whole-plane CTAs
@pytest.mark.parametrize("shape", [(8, 32, 8), (16, 24, 12), (384, 16, 8)])
def test_cond_step_matches_oracle(shape):
    cc, eff, lay, c0 = _case(*shape)
    ref, st_ref = _oracle(cc, eff, lay, c0, 3)
    for prec, tol, tc in ((capi.FP64, 1e-10, 1e-10), (capi.FP32, 1e-4, 1e-6)):
        with capi.Stepper.from_workloads([cc.workload], precision=prec) as st:
            st.cond_enable(0, eff, lay, cc.El_y, configs.EPSILON_ZERO, 1.0)
            st.cond_set_state(0, c0)
            stats = st.cond_step(0, 3)
            got = st.cond_get_state(0)
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= tol * scale
        np.testing.assert_allclose(stats[:, 2], st_ref[:, 2], rtol=tc)
        if prec == capi.FP64:
            np.testing.assert_allclose(stats[:, 0], st_ref[:, 0], rtol=1e-9)
            np.testing.assert_allclose(stats[:, 1], st_ref[:, 1], rtol=1e-9, atol=1e-9 * np.abs(st_ref[:, 1]).max())


def test_cond_beside_the_gl_step():
    """SolveGLCond's pattern: one GL step of the dislocation field and one
    conductivity iteration per stress state; neither field disturbs the other."""
    cc, eff, lay, c0 = _case()
    w = cc.workload
    ref_c, _ = _oracle(cc, eff, lay, c0, 3)
    ref_xi, _, _ = O.run(oracle_instance(w), w.xi0, 3)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        st.cond_enable(0, eff, lay, cc.El_y, configs.EPSILON_ZERO, 1.0)
        st.cond_set_state(0, c0)
        for _ in range(3):
            st.advance(1)
            st.cond_step(0, 1)
        re, im = st.get_state(0)
        got = st.cond_get_state(0)
    assert np.abs(re - ref_xi.real).max() <= 1e-10
    assert np.abs(im - ref_xi.imag).max() <= 1e-10
    assert np.abs(got - ref_c).max() <= 1e-10 * np.abs(ref_c).max()


def test_cond_requires_enable():
    cc, eff, lay, c0 = _case()
    with capi.Stepper.from_workloads([cc.workload], precision=capi.FP64) as st:
        with pytest.raises(capi.PfddError):
            st.cond_step(0, 1)
