"""Asynchronous state snapshots (pfdd_gpu_snapshot_begin / _wait): the copy
of the state after step 3 runs beside steps 4..7 and equals the oracle's
state after 3 steps (FP64, 1e-10); the stepping itself is unchanged."""
import numpy as np
import pytest

import pfdd_oracle as O
from common import oracle_instance, small_loop
from pfdd_b200 import capi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("imag,pinned", [(capi.IMAG_FULL, True), (capi.IMAG_NYQUIST, True),
                                         (capi.IMAG_NYQUIST, False)])
def test_snapshot_beside_the_next_steps(imag, pinned):
    _snapshot_case(imag, pinned, capi.FP64, 1e-10)


def test_snapshot_fp32_equals_get_state():
    """FP32 handle: the snapshot holds exactly what get_state returns at the
    same step (the same conversion to FP64)."""
    import torch
    w = small_loop(16)
    n = w.S * w.N
    re = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    im = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    with capi.Stepper.from_workloads([w], precision=capi.FP32) as st:
        st.set_state(0, w.xi0)
        st.advance(3)
        r3, i3 = st.get_state(0)
        st.snapshot_begin(0, re, im)
        st.advance(2)
        st.snapshot_wait(0)
    assert np.array_equal(re, r3.reshape(-1))
    assert np.array_equal(im, i3.reshape(-1))


def _snapshot_case(imag, pinned, prec, tol):
    import torch
    w = small_loop(16)
    n = w.S * w.N
    if pinned:
        re = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
        im = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    else:
        re, im = np.empty(n), np.empty(n)
    inst = oracle_instance(w)
    ref3, _, _ = O.run(inst, w.xi0, 3)
    ref7, _, _ = O.run(inst, ref3, 4)
    with capi.Stepper.from_workloads([w], precision=prec, imag_mode=imag) as st:
        st.set_state(0, w.xi0)
        st.advance(3)
        st.snapshot_begin(0, re, im)
        st.advance(4)
        st.snapshot_wait(0)
        first = re.copy()
        r7, i7 = st.get_state(0)
        # a second snapshot into the same device buffer
        st.snapshot_begin(0, re, None)
        st.snapshot_wait(0)
        second = re.copy()
    shape = (w.S, w.nx, w.ny, w.nz)
    assert np.abs(first.reshape(shape) - ref3.real).max() <= tol
    assert np.abs(second.reshape(shape) - ref7.real).max() <= tol
    assert np.abs(r7 - ref7.real).max() <= tol
    assert np.abs(i7 - ref7.imag).max() <= tol
    # the first snapshot's imaginary part was not overwritten by the second call
    assert np.abs(im.reshape(shape) - ref3.imag).max() <= tol
