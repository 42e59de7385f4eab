"""Batched groups, CUDA-graph replay, tolerance stops and the energy reduction."""
import numpy as np
import pytest

import pfdd_oracle as O
from common import oracle_instance, small_loop
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def test_group_of_alloy_instances_matches_oracle():
    """Same grid, different stresses and lognormal GSFE fields: one group."""
    ws = [configs.alloy_instance(16, seed=40 + i, sigma_mpa=100.0 + 90.0 * i) for i in range(4)]
    with capi.Stepper.from_workloads(ws, precision=capi.FP64) as st:
        for i, w in enumerate(ws):
            st.set_state(i, w.xi0)
        st.advance(9)
        outs = [st.get_state(i) for i in range(4)]
        _, lps = st.profile(1)
        assert lps == 3          # one group: 3 launches per step for all 4 instances
    for w, (re, im) in zip(ws, outs):
        ref, _, _ = O.run(oracle_instance(w), w.xi0, 9)
        assert np.abs(re - ref.real).max() <= 1e-10
        assert np.abs(im - ref.imag).max() <= 1e-10


def _oracle_with_tol(w, max_iter, states, tol):
    xi = w.xi0.astype(complex)
    sig = w.sigma.copy()
    norms = []
    for _ in range(states):
        w2 = configs.Workload(w.name, w.nx, w.ny, w.nz, w.app, w.xn, w.xb, w.four, w.prim, w.material,
                              w.core_flag, sig.copy(), w.cd_dt, w.xi0)
        inst = oracle_instance(w2)
        for _ in range(max_iter):
            xi, n, _ = O.gl_step(inst, xi)
            norms.append(n)
            if n < tol:
                break
        sig = sig + w.dsigma
    return xi, np.array(norms)


@pytest.mark.parametrize("graphs", [True, False])
def test_tolerance_stops_across_stress_states(graphs):
    w = small_loop(16)
    w.dsigma = np.zeros((3, 3))
    w.dsigma[0, 2] = w.dsigma[2, 0] = 2e-4
    ref, nrm = _oracle_with_tol(w, 40, 3, tol=0.3)
    assert len(nrm) < 120       # the tolerance ends some stress states early
    with capi.Stepper.from_workloads([w], precision=capi.FP64, use_graphs=graphs) as st:
        st.set_state(0, w.xi0)
        (xn, xa, done, conv), = st.advance(40, 3, 0.3)
        re, im = st.get_state(0)
        hn, _ = st.history(0)
    assert done == len(nrm)
    np.testing.assert_allclose(hn, nrm, rtol=1e-9)
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10


@pytest.mark.parametrize("graphs", [True, False])
def test_tolerance_stops_in_short_stress_states(graphs):
    """Several short stress states per graph: an instance that stops on the
    tolerance resumes in the next state from the spectrum its last plane pass
    left (the forward spectrum does not depend on the stress)."""
    w = small_loop(16)
    w.dsigma = np.zeros((3, 3))
    w.dsigma[0, 2] = w.dsigma[2, 0] = 2e-4
    _, free = _oracle_with_tol(w, 6, 1, tol=0.0)
    tol = float(free[3]) * (1 + 1e-6)   # the first state stops after 4 steps
    ref, nrm = _oracle_with_tol(w, 6, 5, tol=tol)
    assert len(nrm) < 30
    with capi.Stepper.from_workloads([w], precision=capi.FP64, use_graphs=graphs) as st:
        st.set_state(0, w.xi0)
        (xn, xa, done, conv), = st.advance(6, 5, tol)
        re, im = st.get_state(0)
        hn, _ = st.history(0)
    assert done == len(nrm)
    np.testing.assert_allclose(hn, nrm, rtol=1e-9)
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10


def test_graph_and_direct_launches_agree():
    ws = [small_loop(16, seed=1), small_loop(16, seed=2), configs.loop_workload(n=24, radius=4.0, seed=3)]
    res = []
    for graphs in (True, False):
        with capi.Stepper.from_workloads(ws, precision=capi.FP32, use_graphs=graphs) as st:
            for i, w in enumerate(ws):
                st.set_state(i, w.xi0)
            st.advance(37)
            res.append([st.get_state(i)[0] for i in range(3)])
    for a, b in zip(*res):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("mask", [False, True])
def test_energy_matches_oracle(mask):
    w = small_loop(16)
    if mask:
        w.xo = np.zeros((w.S, 16, 16, 16))
        w.xo[:, :, :4] = 1.0
    inst = oracle_instance(w)
    xi, _, _ = O.run(inst, w.xi0, 7)
    want = O.total_energy(inst, xi)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        st.advance(7)
        got = st.energy(0)
    for g, e in zip(got, want):
        assert abs(g - e) <= 1e-10 * max(1.0, abs(e)), (got, want)


def test_energy_gradient_is_the_drift():
    """dE/dxi equals the update's drift term: E decreases by ~cd |drift|^2 per step."""
    w = small_loop(16)
    inst = oracle_instance(w)
    with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
        st.set_state(0, w.xi0)
        e0 = sum(st.energy(0))
        st.advance(1)
        (xn, _, _, _), = [(*s,) for s in [st.advance(1)[0]]]
        e2 = sum(st.energy(0))
    assert e2 < e0


def test_two_live_handles_of_different_sizes():
    """A handle created for a small grid while a large-grid handle is alive
    leaves the large one's kernels launchable (per-kernel shared-memory limits
    are process-wide and only ever raised)."""
    big = configs.loop_workload(n=32, radius=6.0, seed=2, sigma_mpa=350.0)
    small = configs.bcc_screw_workload(n=16, nz=8, core_flag=6)
    with capi.Stepper.from_workloads([big], precision=capi.FP64) as sa:
        sa.set_state(0, big.xi0)
        with capi.Stepper.from_workloads([small], precision=capi.FP64) as sb:
            sb.set_state(0, small.xi0)
            sb.advance(2)
            sa.advance(3)
            re, im = sa.get_state(0)
    ref, _, _ = O.run(oracle_instance(big), big.xi0, 3)
    assert np.abs(re - ref.real).max() <= 1e-10
    assert np.abs(im - ref.imag).max() <= 1e-10
