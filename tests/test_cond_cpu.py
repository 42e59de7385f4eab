"""Host side of the conductivity sub-problem: pfdd_cond_layers (the per-y
conductivity of backwardcond) through the C ABI against the oracle's
restatement, no GPU needed."""
import numpy as np
import pytest

import pfdd_oracle as O
from pfdd_b200 import capi, configs


@pytest.mark.parametrize("ny,grains,temperature,pint", [(32, (3, 2), 350.0, 0.4), (48, (1, 1), 300.0, 0.5),
                                                        (30, (4, 1), 420.0, 1.0), (16, (2, 5), 280.0, 0.2)])
def test_cond_layers_abi_equals_oracle(ny, grains, temperature, pint):
    cc = configs.cond_case(ny=ny, grains=grains, temperature=temperature)
    cc.A["pinterface"] = pint
    eff, lay = capi.cond_layers(cc.A, cc.B, ny, temperature)
    e0, l0 = O.cond_layers(O.CondMaterial(**cc.A), O.CondMaterial(**cc.B), ny, temperature)
    np.testing.assert_allclose(lay, l0, rtol=1e-15)
    np.testing.assert_allclose(eff, e0, rtol=1e-12)
    # two materials alternate along y with A.Nlayers periods
    assert len(set(np.round(lay, 6))) == 2


def test_cond_layers_rejects_empty_period():
    cc = configs.cond_case(ny=8)
    cc.A["Nlayers"] = 16
    with pytest.raises(capi.PfddError):
        capi.cond_layers(cc.A, cc.B, 8, 300.0)
