"""The compiled reference run with its set-up spread over forked processes and
its FFT stand-in over threads gives bit-identical results.

bench.py's reference arm times the 256x256x128, 12-system grid, whose
one-process set-up (Bmatrix and Fmatrix, src/fft_fftw_slab.cpp:466-732) takes
tens of minutes; the harness can run those loops on one-x-plane slabs in
forked processes (PFDD_ORACLE_SETUP_PROCS) and the FFTW-2 stand-in its
transforms on threads (PFDD_SHIM_THREADS).  Neither changes an operation, so
B(k), the strain/stress tables and every step's xi must come out bit for bit
as in the one-process, one-thread run."""
import os

import numpy as np
import pytest

import ref_runner
from pfdd_b200 import configs

pytestmark = pytest.mark.skipif(not ref_runner.available(), reason="reference oracle not built")


def _run(procs, threads, w, steps):
    old = {k: os.environ.get(k) for k in ("PFDD_ORACLE_SETUP_PROCS", "PFDD_SHIM_THREADS")}
    os.environ["PFDD_ORACLE_SETUP_PROCS"] = str(procs)
    os.environ["PFDD_SHIM_THREADS"] = str(threads)
    try:
        return ref_runner.run_reference(w, steps, want_B=True, want_stress=True)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize("make", ["fcc12", "skew_mask"])
def test_forked_setup_and_threaded_fft_are_bit_identical(make):
    if make == "fcc12":
        w = configs.fcc_workload(12, 16, 8, n_loops=2, seed=3)
    else:
        w = configs.frank_read_workload(nx=16, ny=12, nz=8, seg=4)
    a = _run(1, 1, w, 3)
    b = _run(3, 4, w, 3)
    assert np.array_equal(a["BB"], b["BB"])
    assert np.array_equal(a["xi"], b["xi"])
    assert np.array_equal(a["xinorm"], b["xinorm"])
    for k in ("eps", "sigma", "ave_eps", "ave_sigma"):
        assert np.array_equal(a[k], b[k]), k
