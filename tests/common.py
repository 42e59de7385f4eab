"""Shared test helpers: build oracle instances for configs.Workload objects."""
import dataclasses

import numpy as np

import pfdd_oracle as O
from pfdd_b200 import configs


def oracle_instance(w, core_flag=None, An=None, extra=None):
    C44, C12, C11 = w.material.elastic()
    BB = O.bmatrix(w.nx, w.ny, w.nz, w.four, w.xn, w.xb, C44, C12, C11, w.material.dslip)
    mu, ll, young, xnu = O.voigt_constants(C44, C12, C11)
    flag = w.core_flag if core_flag is None else core_flag
    kw = dict(isf=w.material.isf, usf=w.material.usf, An=w.material.An if An is None else An)
    ce = getattr(w, "core_extra", None) or {}
    for key in ("c", "aa", "bb"):
        if key in ce:
            kw[key] = tuple(float(v) for v in ce[key])
    if extra:
        kw.update(extra)
    geom = (w.four, w.xn, w.xb) if flag == 5 else None
    invprim = np.linalg.inv(w.prim)
    sr = O.rotate_stress(w.sigma, w.prim, invprim, np.linalg.det(w.prim))
    ns = getattr(w, "non_schmid", None)
    if flag == 6:
        kw["An"] = O.usfe_angle_tau(sr, mu, w.material.usfe_fit, ns[0] if ns else 0.0)
    core = O.CoreModel(flag, mu, w.material.dslip, w.material.b, site=w.site, geom=geom, **kw)
    if ns is not None:
        tau = O.resolved_shear_non_schmid(sr, w.xb, w.material.dslip, *ns)
    else:
        tau = O.resolved_shear(sr, w.xn, w.xb, w.material.dslip)
    return O.Instance(w.nx, w.ny, w.nz, BB, tau, w.cd_dt, core, xo=w.xo)


def small_loop(n=16, seed=576, sigma_mpa=200.0):
    return configs.loop_workload(n=n, radius=n * 12.0 / 64.0, seed=seed, sigma_mpa=sigma_mpa)


def golden_names():
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    return sorted(f[:-4] for f in os.listdir(here) if f.endswith(".npz"))


def load_golden(name):
    """(workload, fixture dict) for tests/golden/<name>.npz, with every constant
    exactly as the reference used it."""
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    fx = dict(np.load(os.path.join(here, name + ".npz")))
    m = configs.Material(b=float(fx["b"]), dslip=float(fx["dslip"]), isf=float(fx["isf"]),
                         usf=float(fx["usf"]), An=float(fx["An"]), mu=float(fx["C44"]),
                         elastic_override=(float(fx["C44"]), float(fx["C12"]), float(fx["C11"])),
                         usfe_fit=tuple(fx["usfe_fit"]) if "usfe_fit" in fx else None)
    w = configs.Workload(name, int(fx["nx"]), int(fx["ny"]), int(fx["nz"]), str(fx["app"]), fx["xn"], fx["xb"],
                         fx["four"], fx["prim"], m, int(fx["core_flag"]), fx["sigma"], float(fx["cd_dt"]),
                         fx["xi0"], xo=fx.get("xo"), site=fx.get("site"), dsigma=fx["dsigma"],
                         core_extra={"c": fx["c"], "aa": fx["aa"], "bb": fx["bb"]},
                         non_schmid=tuple(fx["non_schmid"]) if "non_schmid" in fx else None)
    return w, fx


def oracle_run_golden(w, fx):
    """Run the numpy oracle over the fixture's stress states and steps."""
    xi = np.asarray(fx["xi0"], dtype=np.complex128)
    sig = np.array(fx["sigma"], dtype=float)
    norms, aves = [], []
    for _ in range(int(fx["stress_states"])):
        w2 = dataclasses.replace(w, sigma=sig.copy())
        xi, n, a = O.run(oracle_instance(w2), xi, int(fx["steps"]))
        norms += list(n)
        aves += list(a)
        sig = sig + np.asarray(fx["dsigma"])
    return xi, np.array(norms), np.array(aves)


def adjoint_l2(st, inst, n_steps, ckpt_every, target):
    """J = sum (Re xi_N - target)^2 and its gradients through the general-seed
    adjoint (test-harness loss): the forward tape, then the seed
    dJ/dRe xi_N = 2 (Re xi_N - target).  Returns (J, dJ/dparams, dJ/dsigma)."""
    st.adjoint_forward(inst, n_steps, ckpt_every)
    xr, _ = st.get_state(inst, imag=False)
    r = xr - np.asarray(target)
    dp, ds = st.adjoint_backward(inst, 2.0 * r)
    return float(np.sum(r * r)), dp, ds
