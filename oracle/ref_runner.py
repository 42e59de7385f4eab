"""Run the compiled reference (oracle/_ref/pfdd_ref_harness) on a workload.

TEST INFRASTRUCTURE ONLY: used by tests/ and by the golden-fixture script to
obtain the reference's own results; never part of the product path.
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
HARNESS = os.path.join(REF_DIR, "pfdd_ref_harness")


def available() -> bool:
    return os.access(HARNESS, os.X_OK)


def parse_setup(path):
    out = {"slip": {}, "tau": {}, "four": {}, "sigma_rot": {}}
    with open(path) as f:
        for line in f:
            w = line.split()
            if not w:
                continue
            if w[0] == "usfe_fit":
                out["usfe_fit"] = [float(v) for v in w[1:]]
            elif w[0] == "non_schmid":
                out["non_schmid"] = (int(w[1]), [float(v) for v in w[2:]])
            elif w[0] in ("slip", "four", "sigma_rot", "tau"):
                out[w[0]][int(w[1])] = [float(v) for v in w[2:]]
            elif w[0] in ("nx", "ny", "nz", "S", "core_flag", "iterations"):
                out[w[0]] = int(w[1])
            else:
                out[w[0]] = float(w[1])
    S = out["S"]
    out["xn"] = np.array([out["slip"][a][:3] for a in range(S)])
    out["xb"] = np.array([out["slip"][a][3:] for a in range(S)])
    out["tau"] = np.array([out["tau"][a][0] for a in range(S)])
    out["four"] = np.array([out["four"][i] for i in range(3)])
    out["sigma_rot"] = np.array([out["sigma_rot"][i] for i in range(3)])
    return out


def _raise_stack():
    # Bmatrix keeps an S*S*N double array on the stack (fft_fftw_slab.cpp:475)
    import resource
    try:
        soft, hard = resource.getrlimit(resource.RLIMIT_STACK)
        resource.setrlimit(resource.RLIMIT_STACK, (hard, hard))
    except Exception:
        pass


def run_reference(workload, steps, state=None, xo=None, mpea=None, sets=(), want_B=False,
                  timing=False, workdir=None, timeout=3600, set_b=True, stress_states=None, want_stress=False,
                  want_profile=False):
    """Run `steps` GL iterations of the reference on `workload`.

    state: complex or real array [S, nx, ny, nz] (default workload.xi0).
    Returns dict with xi (complex [S,nx,ny,nz]), xinorm, xiave, setup, and
    optionally BB [S,S,nx,ny,nz], the timing record, (want_profile) the
    project_core_energy arrays delta [NP,nx,ny,nz] and the ddelta line [NP,nx]
    at j = ny/2, k = nz/2 of the final state, and (want_stress) the
    strain/stress diagnostics of the final state: eps and sigma [3,3,nx,ny,nz]
    complex (data_eps, data_sigma), ave_eps, ave_sigma, avepst [3,3].
    """
    if not available():
        raise RuntimeError("reference oracle not built: make -C oracle/ref_build")
    own_tmp = workdir is None
    tmp = workdir or tempfile.mkdtemp(prefix="pfdd_ref_")
    try:
        return _run(workload, steps, state, xo, mpea, sets, want_B, timing, tmp, timeout, set_b, stress_states,
                    want_stress, want_profile)
    finally:
        if own_tmp:
            import shutil
            shutil.rmtree(tmp, ignore_errors=True)


def _run(workload, steps, state, xo, mpea, sets, want_B, timing, tmp, timeout, set_b, stress_states,
         want_stress=False, want_profile=False):
    S, nx, ny, nz = workload.S, workload.nx, workload.ny, workload.nz
    deck = os.path.join(tmp, "in.deck")
    with open(deck, "w") as f:
        f.write(workload.deck(steps, run_T=stress_states or 1))
    st = workload.xi0 if state is None else state
    st = np.asarray(st)
    inter = np.empty((S * nx * ny * nz, 2))
    inter[:, 0] = np.real(st).reshape(-1)
    inter[:, 1] = np.imag(st).reshape(-1) if np.iscomplexobj(st) else 0.0
    inter.tofile(os.path.join(tmp, "xi0.bin"))
    args = [HARNESS, "-deck", deck] + ([] if stress_states else ["-steps", str(steps)]) + [
            "-state_in", os.path.join(tmp, "xi0.bin"),
            "-state_out", os.path.join(tmp, "xi.bin"),
            "-stats_out", os.path.join(tmp, "stats.txt"),
            "-setup_out", os.path.join(tmp, "setup.txt")]
    xo = workload.xo if xo is None else xo
    if xo is not None:
        np.asarray(xo, dtype=np.float64).tofile(os.path.join(tmp, "xo.bin"))
        args += ["-xo_in", os.path.join(tmp, "xo.bin")]
    if mpea is not None:
        np.asarray(mpea, dtype=np.float64).tofile(os.path.join(tmp, "mpea.bin"))
        args += ["-mpea_in", os.path.join(tmp, "mpea.bin")]
    m = workload.material
    base = (("b", m.b), ("dslip", m.dslip)) if set_b else ()
    for k, v in base + tuple(sets):
        args += ["-set", k, repr(float(v))]
    args += ["-set", "CD", repr(float(workload.cd_dt))]
    if want_B:
        args += ["-B_out", os.path.join(tmp, "B.bin")]
    if want_stress:
        args += ["-stress_out", os.path.join(tmp, "stress.bin")]
    if want_profile:
        args += ["-profile_out", os.path.join(tmp, "profile.bin")]
    if timing:
        args += ["-timing"]
    env = dict(os.environ)
    proc = subprocess.run(args, cwd=tmp, capture_output=True, text=True, timeout=timeout, env=env,
                          preexec_fn=_raise_stack)
    if proc.returncode != 0:
        raise RuntimeError("reference harness failed (%d):\n%s\n%s" % (proc.returncode, proc.stdout[-3000:],
                                                                      proc.stderr[-3000:]))
    xi = np.fromfile(os.path.join(tmp, "xi.bin")).reshape(S, nx, ny, nz, 2)
    stats = np.loadtxt(os.path.join(tmp, "stats.txt"), ndmin=2)
    out = {
        "xi": xi[..., 0] + 1j * xi[..., 1],
        "xinorm": stats[:, 1] if stats.size else np.zeros(0),
        "xiave": stats[:, 2] if stats.size else np.zeros(0),
        "setup": parse_setup(os.path.join(tmp, "setup.txt")),
        "stdout": proc.stdout,
    }
    if want_B:
        out["BB"] = np.fromfile(os.path.join(tmp, "B.bin")).reshape(S, S, nx, ny, nz)
    if want_stress:
        raw = np.fromfile(os.path.join(tmp, "stress.bin"))
        n = 2 * 9 * nx * ny * nz
        # layout of data_eps / data_sigma: 2*(r + ida N + idb 3N) (fft_fftw_slab.cpp:3455-3459)
        to_field = lambda a: (a[0::2] + 1j * a[1::2]).reshape(3, 3, nx, ny, nz).transpose(1, 0, 2, 3, 4)
        out["eps"] = to_field(raw[:n])
        out["sigma"] = to_field(raw[n:2 * n])
        out["ave_eps"] = raw[2 * n:2 * n + 9].reshape(3, 3)
        out["ave_sigma"] = raw[2 * n + 9:2 * n + 18].reshape(3, 3)
        out["avepst"] = raw[2 * n + 18:2 * n + 27].reshape(3, 3)
    if want_profile:
        raw = np.fromfile(os.path.join(tmp, "profile.bin"))
        NP = int(raw[0])
        n = nx * ny * nz
        out["delta"] = raw[1:1 + NP * n].reshape(NP, nx, ny, nz)
        out["ddelta"] = raw[1 + NP * n:1 + NP * n + NP * nx].reshape(NP, nx)
    if timing:
        import json
        for line in proc.stdout.splitlines()[::-1]:
            if line.startswith("{") and "loop_s" in line:
                out["timing"] = json.loads(line)
                break
    return out


def run_reference_cond(deck_text, nx, ny, nz, steps, state=None, timeout=600):
    """Run `steps` iterations of the reference's conductivity sub-problem
    (forwardcond, divcurrent, backwardcond, update_conduct_order_param,
    prepare_next_conditr) on a cond100B deck.  Returns condxi (complex
    [nx, ny, nz]), per-iteration conductivity, condxinorm, condxiave, and the
    first iteration's unnormalised inverse transforms a, b and current j."""
    if not available():
        raise RuntimeError("reference oracle not built: make -C oracle/ref_build")
    tmp = tempfile.mkdtemp(prefix="pfdd_cond_")
    try:
        deck = os.path.join(tmp, "in.deck")
        with open(deck, "w") as f:
            f.write(deck_text)
        N = nx * ny * nz
        args = [HARNESS, "-deck", deck, "-cond_steps", str(steps), "-cond_out", os.path.join(tmp, "cond.bin")]
        if state is not None:
            st = np.asarray(state, dtype=np.complex128).reshape(-1)
            inter = np.empty((N, 2))
            inter[:, 0] = st.real
            inter[:, 1] = st.imag
            inter.tofile(os.path.join(tmp, "c0.bin"))
            args += ["-cond_in", os.path.join(tmp, "c0.bin")]
        proc = subprocess.run(args, cwd=tmp, capture_output=True, text=True, timeout=timeout,
                              preexec_fn=_raise_stack)
        if proc.returncode != 0:
            raise RuntimeError("reference harness failed (%d):\n%s\n%s" % (
                proc.returncode, proc.stdout[-3000:], proc.stderr[-3000:]))
        raw = np.fromfile(os.path.join(tmp, "cond.bin"))
        c = raw[:2 * N].reshape(nx, ny, nz, 2)
        rec = raw[2 * N:2 * N + 3 * steps].reshape(steps, 3)
        f = raw[2 * N + 3 * steps:].reshape(3, nx, ny, nz, 2)
        cplx = f[..., 0] + 1j * f[..., 1]
        return {"condxi": c[..., 0] + 1j * c[..., 1], "conductivity": rec[:, 0], "condxinorm": rec[:, 1],
                "condxiave": rec[:, 2], "a": cplx[0], "b": cplx[1], "j": cplx[2], "stdout": proc.stdout}
    finally:
        import shutil
        shutil.rmtree(tmp, ignore_errors=True)
