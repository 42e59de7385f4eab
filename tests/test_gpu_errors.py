"""Argument checks of the entry points added around the step: each refuses
with its status code and leaves the handle usable (no exit, unlike the
reference's Error::all)."""
import numpy as np
import pytest

from common import small_loop
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def _code(fn):
    with pytest.raises(capi.PfddError) as e:
        fn()
    return e.value.code


def test_non_schmid_needs_three_systems_or_fewer():
    w = configs.fcc_workload(8, 8, 8, n_loops=1, seed=3)
    w.non_schmid = (0.0, 0.1, 0.1, 0.1)
    assert _code(lambda: capi.Stepper.from_workloads([w], precision=capi.FP64)) == -1


def test_refusals_leave_the_handle_usable():
    w = small_loop(16)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        assert _code(lambda: st.core_profile(0, 2)) == -1           # 3 systems: one projected plane
        assert _code(lambda: st.autotune(reps=0)) == -1
        assert _code(lambda: st.cond_get_state(0)) == -7            # cond_enable not called
        assert _code(lambda: st.snapshot_begin(0, None, None)) == -1
        st.advance(2)
        re, _ = st.get_state(0)
        d, dd = st.core_profile(0, 1)
    assert np.isfinite(re).all() and d.shape == (1, 16, 16, 16) and dd.shape == (1, 16)
