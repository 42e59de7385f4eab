"""Shared test helpers: build oracle instances for configs.Workload objects."""
import numpy as np

import pfdd_oracle as O
from pfdd_b200 import configs


def oracle_instance(w, core_flag=None, An=None, extra=None):
    C44, C12, C11 = w.material.elastic()
    BB = O.bmatrix(w.nx, w.ny, w.nz, w.four, w.xn, w.xb, C44, C12, C11, w.material.dslip)
    mu, ll, young, xnu = O.voigt_constants(C44, C12, C11)
    flag = w.core_flag if core_flag is None else core_flag
    kw = dict(isf=w.material.isf, usf=w.material.usf, An=w.material.An if An is None else An)
    if extra:
        kw.update(extra)
    core = O.CoreModel(flag, mu, w.material.dslip, w.material.b, site=w.site, **kw)
    invprim = np.linalg.inv(w.prim)
    sr = O.rotate_stress(w.sigma, w.prim, invprim, np.linalg.det(w.prim))
    tau = O.resolved_shear(sr, w.xn, w.xb, w.material.dslip)
    return O.Instance(w.nx, w.ny, w.nz, BB, tau, w.cd_dt, core, xo=w.xo)


def small_loop(n=16, seed=576, sigma_mpa=200.0):
    return configs.loop_workload(n=n, radius=n * 12.0 / 64.0, seed=seed, sigma_mpa=sigma_mpa)
