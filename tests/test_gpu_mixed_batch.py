"""Mixed-size batches in one launch per pass.

Instances that differ only in their grid size (a random-alloy batch of
several sizes) advance with three launches per step in all: the x-pencil
pass, the plane pass and the reduction each cover every instance of every
size, blockIdx mapped to (size group, instance, plane or tile) through a
prefix table.  Checked: FP64 against the oracle per instance (1e-10), FP32
against the one-launch-per-group layout (PFDD_MERGE=0) and the oracle,
per-instance tolerance stops inside the shared launches, and the launch count.
(The reference batches only the slip systems of one grid, FFTW's `howmany`
in forward_mode2, src/fft_fftw_slab.cpp:1966-1994.)"""
import os

import numpy as np
import pytest

import pfdd_oracle as O
from common import oracle_instance
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def _batch():
    sizes = (16, 24, 32, 16, 24)
    return [configs.alloy_instance(n, seed=700 + i, sigma_mpa=120.0 + 60.0 * i) for i, n in enumerate(sizes)]


def _run(ws, steps, prec, merge=True, tol=0.0, states=1):
    old = os.environ.get("PFDD_MERGE")
    if not merge:
        os.environ["PFDD_MERGE"] = "0"
    try:
        st = capi.Stepper.from_workloads(ws, precision=prec)
    finally:
        if old is None:
            os.environ.pop("PFDD_MERGE", None)
        else:
            os.environ["PFDD_MERGE"] = old
    with st:
        for i, w in enumerate(ws):
            st.set_state(i, w.xi0)
        stats = st.advance(steps, states, tol)
        outs = [st.get_state(i) for i in range(len(ws))]
        hist = [st.history(i)[0] for i in range(len(ws))]
        _, lps = st.profile(1)
    return outs, stats, hist, lps


def test_mixed_sizes_fp64_match_the_oracle_in_three_launches():
    ws = _batch()
    outs, _, _, lps = _run(ws, 7, capi.FP64)
    assert lps == 3
    for w, (re, im) in zip(ws, outs):
        ref, _, _ = O.run(oracle_instance(w), w.xi0, 7)
        assert np.abs(re - ref.real).max() <= 1e-10
        assert np.abs(im - ref.imag).max() <= 1e-10


def test_mixed_sizes_fp32_merged_equals_per_group_layout():
    ws = _batch()
    a, _, _, la = _run(ws, 20, capi.FP32, merge=True)
    b, _, _, lb = _run(ws, 20, capi.FP32, merge=False)
    assert la == 3 and lb == 9          # three size groups
    for w, (ra, _), (rb, _) in zip(ws, a, b):
        ref, _, _ = O.run(oracle_instance(w), w.xi0, 20)
        for r in (ra, rb):
            assert np.linalg.norm(r - ref.real) / np.linalg.norm(ref.real) <= 2e-5


def test_tolerance_stops_per_instance_in_shared_launches():
    """A tolerance that stops some instances before others: each stops at the
    step the oracle does, the others run on in the same launches."""
    ws = _batch()
    norms = []
    for w in ws:
        inst = oracle_instance(w)
        xi = w.xi0.astype(complex)
        ns = []
        for _ in range(30):
            xi, nrm, _ = O.gl_step(inst, xi)
            ns.append(nrm)
        norms.append(np.array(ns))
    # stops one instance near step 15; the others when they reach it, or not
    tol = float(min(n[14] for n in norms)) * 1.0000001
    outs, stats, hist, _ = _run(ws, 30, capi.FP64, tol=tol)
    done = []
    for w, (re, _), h, s, ns in zip(ws, outs, hist, stats, norms):
        below = np.nonzero(ns < tol)[0]
        n = int(below[0]) + 1 if len(below) else 30
        ref, _, _ = O.run(oracle_instance(w), w.xi0, n)
        assert s[2] == n == len(h)
        assert np.abs(re - ref.real).max() <= 1e-10
        done.append(n)
    assert min(done) <= 15 and max(done) > min(done)
