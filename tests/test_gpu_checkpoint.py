"""Resume from a binary checkpoint on the GPU: a run that is saved after 7
steps, then loaded into a fresh handle of the same descriptor, continues bit
for bit as the uninterrupted run (FP32 and FP64, Nyquist and full carriers,
and a stress ramp whose sigma is part of the state).  A checkpoint of another
grid or precision, or a corrupted one, is refused and the handle keeps its
state."""
import os

import numpy as np
import pytest

from common import small_loop
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [capi.FP32, capi.FP64])
@pytest.mark.parametrize("imag", [capi.IMAG_NYQUIST, capi.IMAG_FULL])
def test_resume_is_bit_identical(tmp_path, prec, imag):
    w = small_loop(16)
    w.dsigma = np.zeros((3, 3))
    w.dsigma[0, 2] = w.dsigma[2, 0] = 2e-4
    path = str(tmp_path / "mid.ckp")
    with capi.Stepper.from_workloads([w], precision=prec, imag_mode=imag) as a:
        a.set_state(0, w.xi0)
        a.advance(7)
        a.checkpoint_save(0, path)
        a.advance(3, stress_states=2)
        want = a.get_state(0)
        want_tau = a.tau(0)
    with capi.Stepper.from_workloads([w], precision=prec, imag_mode=imag) as b:
        b.checkpoint_load(0, path)
        b.advance(3, stress_states=2)
        got = b.get_state(0)
        got_tau = b.tau(0)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    assert np.array_equal(got_tau, want_tau)


def test_refused_checkpoints_leave_the_state(tmp_path):
    w = small_loop(16)
    other = configs.loop_workload(n=32, radius=6.0)
    p_other = str(tmp_path / "other.ckp")
    with capi.Stepper.from_workloads([other], precision=capi.FP64) as o:
        o.checkpoint_save(0, p_other)
    p32 = str(tmp_path / "fp32.ckp")
    with capi.Stepper.from_workloads([w], precision=capi.FP32) as o:
        o.checkpoint_save(0, p32)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        st.advance(2)
        before = st.get_state(0)
        good = str(tmp_path / "good.ckp")
        st.checkpoint_save(0, good)
        bad = str(tmp_path / "bad.ckp")
        raw = bytearray(open(good, "rb").read())
        raw[300] ^= 0x04
        open(bad, "wb").write(bytes(raw))
        for p in (p_other, p32, bad, str(tmp_path / "missing.ckp")):
            with pytest.raises(capi.PfddError) as e:
                st.checkpoint_load(0, p)
            assert e.value.code == -1
        after = st.get_state(0)
        assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])


def test_carrier_is_layout_independent(tmp_path, monkeypatch):
    """The file holds the Nyquist carrier of Im xi in frequency order, so a
    checkpoint written by a handle whose planes run split over 2-CTA
    clusters (its y transforms then keep a different slot order) resumes in
    a handle with whole planes: the continued run matches the writer's own
    continuation to FP64 round-off (the two layouts sum in different orders)."""
    w = small_loop(16)
    path = str(tmp_path / "split.ckp")
    monkeypatch.setenv("PFDD_PLANE_SPLIT", "1")
    with capi.Stepper.from_workloads([w], precision=capi.FP64, imag_mode=capi.IMAG_NYQUIST) as a:
        a.set_state(0, w.xi0)
        a.advance(6)
        a.checkpoint_save(0, path)
        a.advance(6)
        want = a.get_state(0)
    monkeypatch.setenv("PFDD_PLANE_SPLIT", "0")
    with capi.Stepper.from_workloads([w], precision=capi.FP64, imag_mode=capi.IMAG_NYQUIST) as b:
        b.checkpoint_load(0, path)
        b.advance(6)
        got = b.get_state(0)
    scale = max(np.abs(want[0]).max(), np.abs(want[1]).max())
    assert np.abs(got[0] - want[0]).max() <= 1e-10 * scale
    assert np.abs(got[1] - want[1]).max() <= 1e-10 * scale
    assert np.abs(want[1]).max() > 1e-6   # the carrier is not trivially zero
