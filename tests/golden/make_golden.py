"""Write tests/golden/*.npz from the reference itself.

Each fixture is one small deck run through the reference sources compiled by
oracle/ref_build (oracle/_ref/pfdd_ref_harness): the input state, the
constants the reference actually used (slip vectors after set_slip, elastic
constants, GSFE constants, tau, CD), and its output xi plus per-step xinorm and
xiave.  Run from the repository root:

    make -C oracle/ref_build && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "phase-field-dislocation-dynamics-pfdd-2.x_b200"))

import ref_runner  # noqa: E402
from pfdd_b200 import configs as C  # noqa: E402


def case_loop_sine():
    w = C.loop_workload(n=16, nz=8, radius=4.0, seed=11)
    return w, 6, {}


def case_fcc12_sine():
    w = C.fcc_workload(12, 8, 8, n_loops=3, seed=5)
    return w, 4, {}


def case_frank_read_mask():
    w = C.frank_read_workload(16, 16, 8, seg=8)
    w.sigma = C._sigma("yz", 0.02)
    rng = np.random.default_rng(3)
    w.xi0 = w.xi0 + 1j * rng.uniform(-1e-3, 1e-3, size=w.xi0.shape)
    return w, 5, {}


def case_loop_perfect():
    w, steps, kw = case_loop_sine()
    w.core_flag = 1
    w.material.An = 0.4
    return w, 4, kw


def case_loop_mpea():
    w, steps, kw = case_loop_sine()
    w.core_flag = 7
    rng = np.random.default_rng(9)
    w.site = rng.uniform(0.05, 0.4, size=(w.S, w.nx, w.ny, w.nz))
    return w, 4, {"mpea": w.site}


def case_fcc12_extended():
    w = C.fcc_workload(8, 8, 8, n_loops=2, seed=21)
    w.core_flag = 2
    w.material.deck_line = "material preset Ni"
    rng = np.random.default_rng(4)
    w.xi0 = w.xi0 + rng.uniform(-0.05, 0.05, size=w.xi0.shape)
    return w, 3, {"set_b": False}


def case_pyrII():
    # the Mg preset sets no Burgers vector (material.cpp:369-396); use b = a
    w = C.loop_workload(n=8, radius=2.0, seed=2)
    w.core_flag = 4
    w.material.deck_line = "material preset Mg"
    w.material.b = 3.19e-10
    return w, 3, {}


def case_ramp():
    w = C.loop_workload(n=16, nz=8, radius=4.0, seed=13)
    w.dsigma = C._sigma("xz", 1e-3)
    return w, 2, {"stress_states": 3}


def case_bcc_non_schmid():
    # Ta, one BCC system, non-Schmid tau and the USFE(angle, tau) core over a
    # ramp of sigma_yz: the core amplitude changes with every stress state
    w = C.bcc_screw_workload(n=16, nz=8, core_flag=6)
    w.dsigma = C._sigma("yz", 4e-3)
    return w, 3, {"stress_states": 3}


CASES = {
    "loop_sine": case_loop_sine,
    "fcc12_sine": case_fcc12_sine,
    "frank_read_mask": case_frank_read_mask,
    "loop_perfect": case_loop_perfect,
    "loop_mpea": case_loop_mpea,
    "fcc12_extended": case_fcc12_extended,
    "pyrII": case_pyrII,
    "ramp": case_ramp,
    "bcc_non_schmid": case_bcc_non_schmid,
}


def run_case(name):
    w, steps, kw = CASES[name]()
    r = ref_runner.run_reference(w, steps, **kw)
    su = r["setup"]
    out = dict(
        nx=w.nx, ny=w.ny, nz=w.nz, S=w.S, steps=steps, stress_states=kw.get("stress_states", 1),
        app=w.app, core_flag=su["core_flag"], cd_dt=su["CD"] * su["timestep"],
        xn=su["xn"], xb=su["xb"], four=su["four"], prim=w.prim, sigma=w.sigma, dsigma=w.dsigma,
        C44=su["C44"], C12=su["C12"], C11=su["C11"], b=su["b"], dslip=su["dslip"],
        isf=su["isf"], usf=su["usf"], An=su["An"],
        c=np.array([su["c%d" % i] for i in range(7)]), aa=np.array([su["aa%d" % i] for i in range(5)]),
        bb=np.array([su["bb%d" % i] for i in range(1, 5)]),
        tau=su["tau"], xi0=np.asarray(w.xi0, dtype=np.complex128), xi=r["xi"],
        xinorm=r["xinorm"], xiave=r["xiave"],
    )
    if w.xo is not None:
        out["xo"] = w.xo
    if w.site is not None:
        out["site"] = w.site
    if w.non_schmid is not None:
        out["non_schmid"] = np.asarray(su["non_schmid"][1])
    if w.core_flag == 6:
        out["usfe_fit"] = np.asarray(su["usfe_fit"])
    return out


def main():
    names = sys.argv[1:] or list(CASES)
    for name in names:
        fx = run_case(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **fx)
        print(name, "steps", fx["steps"], "max|xi|", float(np.abs(fx["xi"]).max()),
              "max|Im xi|", float(np.abs(fx["xi"].imag).max()))


if __name__ == "__main__":
    main()
