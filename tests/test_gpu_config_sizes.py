"""GPU parity at the sizes of the benchmark configurations.

The small-grid parity tests exercise every kernel variant; these run the
CUDA path (through the C ABI) against the numpy oracle -- itself pinned to
the compiled reference -- at the grid sizes the measurements use, so the
FFT plans of 48, 64, 96, 128, 256 and 512 points, the split and whole-plane
passes and the FP32 compile-time plans are all checked where they run:

  loop 64^3 x 3 (plain FP64)      max |dxi| <= 1e-10 after 1, 10 and 100 steps,
                                  xinorm / xiave of every step
  alloy 48^3 and 96^3 x 3         FP64 <= 1e-10, FP32 rel. L2 <= 2e-5 (10 steps)
  edge 128 x 128 x 32 x 3         FP64 <= 1e-10 (10 steps)
  FCC 128 x 128 x 64 x 12         FP64 <= 1e-10, FP32 rel. L2 <= 2e-5 (3 steps;
                                  the 12-system pencil and the 128-point plans of
                                  the 256^2 x 128 grid)
  Frank-Read 512 x 512 x 64 x 2   FP64 <= 1e-10, FP32 rel. L2 <= 2e-5 (2 steps),
  (60-degree grid, mask)          full complex carrier
  loop 64^3 x 3                   FP32 vs the FP64 GPU path (equal to the oracle
                                  per step above) after 2000 steps: rel. L2 of
                                  Re xi <= 1e-5
  FCC 256 x 256 x 128 x 12        FP32 vs FP64 <= 1e-5 after 10 steps; after 2000
                                  steps no further than an FP64 run perturbed by
                                  1e-7 (this trajectory amplifies perturbations)

The reference's counterparts are the update and transforms these grids run
through: update_order_parameter and forward/backward_mode1
(src/fft_fftw_slab.cpp:1746-1790, 1953-2052).
"""
import gc

import numpy as np
import pytest

import pfdd_oracle as O
from common import oracle_instance
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 2e-5


def _oracle_states(w, checkpoints):
    """Oracle states (complex) and per-step xinorm / xiave at the given step counts."""
    inst = oracle_instance(w)
    xi = w.xi0.astype(np.complex128)
    out, norms, aves = {}, [], []
    for n in range(1, max(checkpoints) + 1):
        xi, xn, xa = O.gl_step(inst, xi)
        norms.append(xn)
        aves.append(xa)
        if n in checkpoints:
            out[n] = xi.copy()
    del inst
    gc.collect()
    return out, np.array(norms), np.array(aves)


def _gpu_states(w, checkpoints, precision=capi.FP64):
    out = {}
    hist_n, hist_a = [], []
    with capi.Stepper.from_workloads([w], precision=precision) as st:
        st.set_state(0, w.xi0)
        done = 0
        for n in sorted(checkpoints):
            st.advance(n - done)
            hn, ha = st.history(0)
            hist_n += list(hn)
            hist_a += list(ha)
            done = n
            out[n] = st.get_state(0)
    return out, np.array(hist_n), np.array(hist_a)


def _max_abs(got, ref):
    re, im = got
    return max(np.abs(re - ref.real).max(), np.abs(im - ref.imag).max())


def _rel_l2(got, ref):
    return np.linalg.norm(got[0] - ref.real) / np.linalg.norm(ref.real)


def test_loop64_fp64_1_10_100_steps():
    w = configs.loop_workload()        # 64^3, 3 systems, r = 12, noise 1e-3 (seed 576), 200 MPa
    cps = (1, 10, 100)
    ref, nrm, ave = _oracle_states(w, cps)
    got, hn, ha = _gpu_states(w, cps)
    for n in cps:
        assert _max_abs(got[n], ref[n]) <= TOL64, n
    np.testing.assert_allclose(hn, nrm, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(ha, ave, rtol=1e-10, atol=1e-9)


@pytest.mark.parametrize("n", [48, 96])
def test_alloy_instance_fp64_and_fp32(n):
    w = configs.alloy_instance(n, seed=99000 + n, sigma_mpa=275.0)   # per-site lognormal GSFE field
    ref, _, _ = _oracle_states(w, (10,))
    got, _, _ = _gpu_states(w, (10,))
    assert _max_abs(got[10], ref[10]) <= TOL64
    got32, _, _ = _gpu_states(w, (10,), precision=capi.FP32)
    assert _rel_l2(got32[10], ref[10]) <= TOL32


def test_edge128_fp64_10_steps():
    w = configs.edge_workload()
    ref, _, _ = _oracle_states(w, (10,))
    got, _, _ = _gpu_states(w, (10,))
    assert _max_abs(got[10], ref[10]) <= TOL64


def test_fcc12_128x128x64_fp64_and_fp32_3_steps():
    w = configs.fcc_workload(128, 128, 64, n_loops=6, seed=5)
    ref, nrm, _ = _oracle_states(w, (3,))
    got, hn, _ = _gpu_states(w, (3,))
    assert _max_abs(got[3], ref[3]) <= TOL64
    np.testing.assert_allclose(hn, nrm, rtol=1e-10)
    got32, _, _ = _gpu_states(w, (3,), precision=capi.FP32)
    assert _rel_l2(got32[3], ref[3]) <= TOL32


def test_frank_read_512x512x64_fp64_and_fp32():
    w = configs.frank_read_workload()   # 60-degree grid, 2 systems, pinned 64-cell segment (mask)
    # a loaded state: the ramp's 600 MPa end point applied at once
    w.sigma = w.dsigma * 20000
    w.dsigma = np.zeros((3, 3))
    ref, _, _ = _oracle_states(w, (2,))
    got, _, _ = _gpu_states(w, (2,))
    assert _max_abs(got[2], ref[2]) <= TOL64
    got32, _, _ = _gpu_states(w, (2,), precision=capi.FP32)
    assert _rel_l2(got32[2], ref[2]) <= TOL32


def _fp_runs(w, runs, checkpoints):
    """{name: {step: Re xi}} for runs = {name: (precision, initial state)}."""
    out = {}
    for name, (prec, x0) in runs.items():
        out[name] = {}
        with capi.Stepper.from_workloads([w], precision=prec) as st:
            st.set_state(0, x0)
            done = 0
            for c in checkpoints:
                st.advance(c - done)
                done = c
                out[name][c] = st.get_state(0, imag=False)[0]
    return out


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_loop64_fp32_against_fp64_after_2000_steps():
    w = configs.loop_workload()
    r = _fp_runs(w, {"fp64": (capi.FP64, w.xi0), "fp32": (capi.FP32, w.xi0)}, (2000,))
    assert _rel(r["fp32"][2000], r["fp64"][2000]) <= 1e-5


def test_fcc256_fp32_error_bounded_by_the_dynamics():
    """On the 256x256x128, 12-system FCC deck the trajectory itself amplifies
    any perturbation: an FP64 run started 1e-7 (normal, seeded) away ends 0.16
    (relative L2) away after 2000 steps, as far as the FP32 run does.  So the
    FP32 path is checked where the dynamics have not amplified its rounding,
    <= 1e-5 relative L2 after 10 steps, and after 2000 steps against that
    FP64 control: no further from the FP64 run than the perturbed FP64 run."""
    w = configs.fcc_workload()
    pert = 1e-7 * np.random.default_rng(1).standard_normal(w.xi0.shape)
    r = _fp_runs(w, {"fp64": (capi.FP64, w.xi0), "fp32": (capi.FP32, w.xi0),
                     "fp64_pert": (capi.FP64, w.xi0 + pert)}, (10, 2000))
    assert _rel(r["fp32"][10], r["fp64"][10]) <= 1e-5
    assert _rel(r["fp32"][2000], r["fp64"][2000]) <= _rel(r["fp64_pert"][2000], r["fp64"][2000])
