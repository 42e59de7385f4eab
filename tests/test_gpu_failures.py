"""Failure detection on the GPU, made to happen without faulting anything.

The reference stops on every error through Error::all / Error::one, which
print and exit or MPI_Abort (src/error.cpp:34-69), and it leaves its GL loop
on convergence or when xi falls below ximin (src/solve_GL.cpp:137-147).
Here each failure comes back as a status code and the handle stays usable:

* a non-finite order parameter (a NaN placed in the host state) is found by
  the step's reduction and returns PFDD_EDIVERGED;
* a bounded device wait that runs out returns PFDD_ETIMEOUT: the test switch
  PFDD_STALL_BULK_WAITS=1 makes every plane-pass CTA's copy barrier withhold
  one arrival, so the first wait gives up after its short limit; the CTA then
  waits for its copies to land and abandons the plane;
* a device allocation that fails returns PFDD_ENOMEM: the test hook
  PFDD_FAIL_ALLOC_ABOVE=<bytes> refuses larger allocations as cudaMalloc does
  when memory runs out.

After each, the same handle (or a new one) is set to a fresh state and must
step to the oracle's result (FP64, 1e-10)."""
import os

import numpy as np
import pytest

import pfdd_oracle as O
from common import adjoint_l2, oracle_instance, small_loop
from pfdd_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _code(fn):
    with pytest.raises(capi.PfddError) as e:
        fn()
    return e.value.code


class _env:
    def __init__(self, **kv):
        self.kv = kv

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kv}
        os.environ.update({k: str(v) for k, v in self.kv.items()})

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _check_steps(st, w, steps=3):
    ref, _, _ = O.run(oracle_instance(w), w.xi0, steps)
    st.set_state(0, w.xi0)
    st.advance(steps)
    re, im = st.get_state(0)
    assert np.abs(re - ref.real).max() <= TOL
    assert np.abs(im - ref.imag).max() <= TOL


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_nan_state_reports_diverged_and_handle_recovers(prec):
    w = small_loop(16)
    bad = w.xi0.copy()
    bad[1, 3, 4, 5] = np.nan
    with capi.Stepper.from_workloads([w], precision=prec) as st:
        st.set_state(0, bad)
        assert _code(lambda: st.advance(2)) == -5
        if prec == capi.FP64:
            _check_steps(st, w)
        else:
            st.set_state(0, w.xi0)
            st.advance(3)
            assert np.isfinite(st.get_state(0)[0]).all()


@pytest.mark.parametrize("split", ["0", "1"])
@pytest.mark.parametrize("imag", [capi.IMAG_NYQUIST, capi.IMAG_FULL])
def test_stalled_copy_wait_reports_timeout_and_handle_recovers(split, imag):
    w = small_loop(16)
    with _env(PFDD_PLANE_SPLIT=split):
        st = capi.Stepper.from_workloads([w], precision=capi.FP64, imag_mode=imag)
    try:
        st.set_state(0, w.xi0)
        with _env(PFDD_STALL_BULK_WAITS=1):
            assert _code(lambda: st.advance(4)) == -8           # graph-replayed steps
            assert _code(lambda: st.energy(0)) == -8
        _check_steps(st, w)
        e = st.energy(0)
        assert all(np.isfinite(e))
    finally:
        st.close()


def test_stalled_wait_in_strain_stress_and_adjoint():
    w = small_loop(16)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        st.advance(2)
        with _env(PFDD_STALL_BULK_WAITS=1):
            assert _code(lambda: st.strain_stress(0, fields=False)) == -8
            assert _code(lambda: adjoint_l2(st, 0, 3, 2, np.zeros_like(w.xi0))) == -8
        _check_steps(st, w)
        _, _, ae, asg = st.strain_stress(0, fields=False)
        assert np.isfinite(ae).all() and np.isfinite(asg).all()


def test_failed_allocation_reports_enomem():
    w = small_loop(16)
    with _env(PFDD_FAIL_ALLOC_ABOVE=4096):
        assert _code(lambda: capi.Stepper.from_workloads([w], precision=capi.FP64)) == -2
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        # the adjoint's checkpoint buffers are allocated on its first call
        with _env(PFDD_FAIL_ALLOC_ABOVE=1 << 16):
            assert _code(lambda: adjoint_l2(st, 0, 4, 2, np.zeros_like(w.xi0))) == -2
        _check_steps(st, w)
        loss, dp, ds = adjoint_l2(st, 0, 4, 2, np.zeros_like(w.xi0))
        assert np.isfinite(loss) and np.isfinite(dp).all() and np.isfinite(ds).all()
