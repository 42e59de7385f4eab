"""The numpy oracle against fixtures written by the reference itself
(tests/golden/make_golden.py runs the reference sources compiled in
oracle/_ref): loop/FCC decks, a masked skewed Frank-Read deck with complex
state, perfect / MPEA / extended / pyrII cores, a stress ramp, and a BCC deck with
the non-Schmid resolved shear stress and the USFE(angle, tau) core over a
stress ramp."""
import numpy as np
import pytest

from common import golden_names, load_golden, oracle_run_golden


@pytest.mark.parametrize("name", golden_names())
def test_oracle_reproduces_reference_fixture(name):
    w, fx = load_golden(name)
    xi, norms, aves = oracle_run_golden(w, fx)
    scale = max(1.0, float(np.abs(fx["xi"]).max()))
    assert np.abs(xi - fx["xi"]).max() <= 1e-12 * scale
    np.testing.assert_allclose(norms, fx["xinorm"], rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(aves, fx["xiave"], rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("name", golden_names())
def test_fixture_tau_matches_restated_resolve(name):
    import pfdd_oracle as O
    w, fx = load_golden(name)
    invprim = np.linalg.inv(w.prim)
    sr = O.rotate_stress(fx["sigma"], w.prim, invprim, np.linalg.det(w.prim))
    if "non_schmid" in fx:
        tau = O.resolved_shear_non_schmid(sr, fx["xb"], float(fx["dslip"]), *fx["non_schmid"])
    else:
        tau = O.resolved_shear(sr, fx["xn"], fx["xb"], float(fx["dslip"]))
    if int(fx["stress_states"]) == 1:
        np.testing.assert_allclose(tau, fx["tau"], rtol=1e-13, atol=1e-16)
