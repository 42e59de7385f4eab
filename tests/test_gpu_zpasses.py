"""The register-resident z passes of the plane pass against the generic
staged passes of the same library.

The update and adjoint plane passes take three register-resident z passes
(complex-to-real pairs with the inverse stage B; the inverse stage A, the
per-site update and the forward stage A; the forward stage B with the
real-to-complex pairs) for the sine-family core models on two-stage z plans
when enough rows are in flight; PFDD_ZFUSED=0 in the environment at handle
creation keeps the generic passes everywhere.  Both are the same arithmetic
in another order, so states, per-step statistics and adjoint gradients agree
to round-off, here on grids that take the register-resident passes: whole and
split planes, an obstacle mask with the imaginary field carried, the per-site
GSFE multiplier (core model 103), radix-3 stages (96^3), FP32 and FP64."""
import numpy as np
import pytest

from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu


def _loop(n=128, nz=64, mask=False):
    w = configs.loop_workload(n=n, nz=nz, radius=n / 5.0, seed=5, sigma_mpa=250.0)
    if mask:
        rng = np.random.default_rng(3)
        w.xo = (rng.uniform(size=(w.S, w.nx, w.ny, w.nz)) < 0.2).astype(float)
    return w


def _advance(monkeypatch, zfused, w, prec, steps, split=None):
    monkeypatch.setenv("PFDD_ZFUSED", "1" if zfused else "0")
    if split is None:
        monkeypatch.delenv("PFDD_PLANE_SPLIT", raising=False)
    else:
        monkeypatch.setenv("PFDD_PLANE_SPLIT", "1" if split else "0")
    with capi.Stepper.from_workloads([w], precision=prec) as st:
        st.set_state(0, w.xi0, getattr(w, "xi0_im", None))
        st.advance(steps)
        re, im = st.get_state(0)
        nrm, ave = st.history(0)
    return re, im, nrm, ave


CASES = [
    ("loop 128x128x64, whole planes", lambda: _loop(), None),
    ("loop 128x128x64, split planes", lambda: _loop(), True),
    ("loop 128x128x64, mask + Im field", lambda: _loop(mask=True), None),
    ("alloy 64^3, per-site GSFE, whole planes", lambda: configs.alloy_instance(64, 17, 250.0), False),
    ("alloy 96^3, radix-3 z stage, whole planes", lambda: configs.alloy_instance(96, 23, 250.0), False),
]


@pytest.mark.parametrize("prec,tol", [(capi.FP64, 1e-11), (capi.FP32, 2e-5)])
@pytest.mark.parametrize("name,make,split", CASES, ids=[c[0] for c in CASES])
def test_register_resident_z_passes_match_generic(monkeypatch, prec, tol, name, make, split):
    w = make()
    steps = 20
    a = _advance(monkeypatch, True, w, prec, steps, split)
    b = _advance(monkeypatch, False, w, prec, steps, split)
    scale = max(np.abs(b[0]).max(), 1.0)
    assert np.abs(a[0] - b[0]).max() <= tol * scale, name
    assert np.abs(a[1] - b[1]).max() <= tol * scale, name
    assert len(a[2]) == len(b[2]) == steps
    np.testing.assert_allclose(a[2], b[2], rtol=10 * tol, atol=0)
    np.testing.assert_allclose(a[3], b[3], rtol=10 * tol, atol=10 * tol * np.abs(b[3]).max())
    # the dynamics moved the state: the comparison is not of two unchanged inputs
    assert np.abs(b[0] - w.xi0).max() > 1e-4
    # and the two forms did run: their plane sums add the sites in other orders
    assert not np.array_equal(a[2], b[2])


@pytest.mark.parametrize("split", [None, True])
def test_adjoint_gradients_match_generic(monkeypatch, split):
    """dL/d(isf, usf) and dL/dsigma of L = sum W Re xi_N (checkpointed
    adjoint, 12 steps, a checkpoint every 5) through both z pass forms, FP64."""
    w = _loop()
    W = np.random.default_rng(8).standard_normal((w.S, w.nx, w.ny, w.nz))
    out = []
    for zf in (True, False):
        monkeypatch.setenv("PFDD_ZFUSED", "1" if zf else "0")
        if split is None:
            monkeypatch.delenv("PFDD_PLANE_SPLIT", raising=False)
        else:
            monkeypatch.setenv("PFDD_PLANE_SPLIT", "1")
        with capi.Stepper.from_workloads([w], precision=capi.FP64) as st:
            st.set_state(0, w.xi0)
            out.append(st.adjoint(0, 12, 5, W))
    (dp_a, ds_a), (dp_b, ds_b) = out
    np.testing.assert_allclose(dp_a, dp_b, rtol=1e-10, atol=0)
    np.testing.assert_allclose(ds_a, ds_b, rtol=1e-10, atol=1e-10 * np.abs(ds_b).max())
    assert np.abs(dp_b).max() > 0
