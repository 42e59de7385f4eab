"""Long horizons: the FP32 path against the FP64 path over 2000 steps (the
FP64 GPU path equals the FP64 oracle to 1e-10 per step in the parity tests,
so it stands in for the oracle where the numpy step would take minutes).
Checks the three agreements the step is held to: relative L2 of Re xi
<= 1e-5, the dislocation line's position, and the total energy."""
import numpy as np
import pytest

from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def _run(w, steps, prec):
    with capi.Stepper.from_workloads([w], precision=prec) as st:
        st.set_state(0, w.xi0)
        st.advance(steps)
        re, im = st.get_state(0)
        e = st.energy(0)
    return re, im, e


def _line_position(re_plane):
    """x where Re xi_0 falls through 1/2 along each y row, nearest the
    starting line x = nx/2 (linear between the bracketing sites)."""
    nx, ny = re_plane.shape
    pos = np.empty(ny)
    for j in range(ny):
        col = re_plane[:, j]
        cross = [i for i in range(1, nx) if col[i - 1] >= 0.5 > col[i]]
        assert cross, "no falling crossing in row %d" % j
        i = min(cross, key=lambda c: abs(c - nx // 2))
        a, b = col[i - 1], col[i]
        pos[j] = (i - 1) + (a - 0.5) / (a - b)
    return pos


def test_fp32_l2_after_2000_steps():
    w = configs.loop_workload(n=32, radius=7.0, seed=12, sigma_mpa=250.0)
    r32, _, _ = _run(w, 2000, capi.FP32)
    r64, _, _ = _run(w, 2000, capi.FP64)
    assert np.linalg.norm(r32 - r64) / np.linalg.norm(r64) <= 1e-5


def test_edge_position_and_energy_after_1000_steps():
    w = configs.edge_workload(64, 64, 16, perturb=6, sigma_mpa=150.0)
    r32, _, e32 = _run(w, 1000, capi.FP32)
    r64, _, e64 = _run(w, 1000, capi.FP64)
    z = w.nz // 2
    p32, p64 = _line_position(r32[0, :, :, z]), _line_position(r64[0, :, :, z])
    # the line moved and both precisions put it at the same place
    p0 = _line_position(w.xi0[0, :, :, z])
    assert np.abs(p64 - p0).max() > 0.5
    assert np.abs(p32 - p64).max() <= 1e-3
    # total energy (elastic + core + applied, FP64 reductions in both paths)
    assert abs(sum(e32) - sum(e64)) <= 1e-5 * abs(sum(e64))
