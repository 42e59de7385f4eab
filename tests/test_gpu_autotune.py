"""The x-pencil tile autotuner (pfdd_gpu_autotune): timing trials between
two advances keep the state (spectrum rebuilt, Nyquist carrier and stop flag
restored), the chosen width per batched group is one the grid divides into,
and the stepping afterwards matches an untuned handle and the oracle (FP64)."""
import numpy as np
import pytest

import pfdd_oracle as O
from common import oracle_instance, small_loop
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("imag", [capi.IMAG_NYQUIST, capi.IMAG_FULL])
def test_autotune_between_advances_keeps_the_state(imag):
    w = configs.fcc_workload(32, 32, 16, n_loops=3, seed=4)
    with capi.Stepper.from_workloads([w], precision=capi.FP64, imag_mode=imag) as st:
        st.set_state(0, w.xi0)
        st.advance(7)
        re0, im0 = st.get_state(0)
    with capi.Stepper.from_workloads([w], precision=capi.FP64, imag_mode=imag) as st:
        st.set_state(0, w.xi0)
        st.advance(3)
        chosen = st.autotune(reps=2)
        st.advance(4)
        re1, im1 = st.get_state(0)
    assert chosen[0] >= 1 and (chosen[0] & (chosen[0] - 1)) == 0
    assert np.abs(re1 - re0).max() <= 1e-13
    assert np.abs(im1 - im0).max() <= 1e-13
    ref, _, _ = O.run(oracle_instance(w), w.xi0, 7)
    assert np.abs(re1 - ref.real).max() <= 1e-10
    assert np.abs(im1 - ref.imag).max() <= 1e-10


def test_autotune_batched_groups():
    ws = [small_loop(16, seed=1), configs.loop_workload(n=32, radius=6.0, seed=2, sigma_mpa=350.0),
          small_loop(16, seed=3)]
    for prec, tol in ((capi.FP64, 1e-10), (capi.FP32, None)):
        with capi.Stepper.from_workloads(ws, precision=prec) as st:
            for i, w in enumerate(ws):
                st.set_state(i, w.xi0)
            chosen = st.autotune(reps=2)
            st.advance(5)
            out = [st.get_state(i) for i in range(len(ws))]
        assert chosen[0] == chosen[2]          # one group, one width
        for w, (re, im) in zip(ws, out):
            ref, _, _ = O.run(oracle_instance(w), w.xi0, 5)
            if tol is not None:
                assert np.abs(re - ref.real).max() <= tol
            else:
                assert np.linalg.norm(re - ref.real) / np.linalg.norm(ref.real) <= 2e-5
