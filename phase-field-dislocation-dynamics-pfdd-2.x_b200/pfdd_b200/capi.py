"""ctypes binding of libpfdd_b200.so (C ABI in include/pfdd_b200.h).

This is the Python-side mirror of the boundary the reference's host code binds
(its FFT style object replaced by the library): the same descriptors and calls
a C++ FftStyle plugin makes.  The library is loaded from
this package directory; when it is missing, or no sm_100 device exists, every
call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfdd_b200.so")
MAX_SLIP = 12

PFDD_OK = 0
ERRORS = {-1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "EUNSUPPORTED", -5: "EDIVERGED", -6: "ENODEVICE",
          -7: "ESTATE", -8: "ETIMEOUT"}
FP64, FP32 = 0, 1
IMAG_AUTO, IMAG_FULL, IMAG_NYQUIST = 0, 1, 2
CORE_PERFECT, CORE_EXTENDED, CORE_SINE, CORE_PYRII, CORE_USFE_ANGLE, CORE_MPEA, CORE_SINE_FIELD = 1, 2, 3, 4, 6, 7, 103
CORE_BCC_PERFECT = 5

# every symbol include/pfdd_b200.h declares
EXPORTS = [
    "pfdd_gpu_create", "pfdd_gpu_set_state", "pfdd_gpu_set_state_interleaved", "pfdd_gpu_get_state",
    "pfdd_gpu_get_state_interleaved", "pfdd_gpu_advance", "pfdd_gpu_step_history", "pfdd_gpu_energy",
    "pfdd_gpu_tau", "pfdd_gpu_set_stress", "pfdd_gpu_info", "pfdd_gpu_last_error", "pfdd_gpu_destroy", "pfdd_gpu_version",
    "pfdd_gpu_set_stream", "pfdd_gpu_profile", "pfdd_gpu_adjoint", "pfdd_gpu_adjoint_forward",
    "pfdd_gpu_adjoint_backward", "pfdd_gpu_strain_stress",
    "pfdd_gpu_core_profile", "pfdd_gpu_autotune", "pfdd_gpu_snapshot_begin", "pfdd_gpu_snapshot_wait", "pfdd_cond_layers", "pfdd_gpu_cond_enable", "pfdd_gpu_cond_set_state",
    "pfdd_gpu_cond_get_state", "pfdd_gpu_cond_step", "pfdd_checkpoint_write", "pfdd_checkpoint_read",
    "pfdd_gpu_checkpoint_save", "pfdd_gpu_checkpoint_load", "pfdd_gl_step_noalloc",
]
KERNELS = ["fwd_planes", "xpencil", "step_planes", "finalize"]

D33 = ctypes.c_double * 3 * 3
DS3 = ctypes.c_double * 3 * MAX_SLIP
DP = ctypes.POINTER(ctypes.c_double)


class InstanceDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("n_slip", ctypes.c_int),
        ("four", D33), ("prim", D33), ("xn", DS3), ("xb", DS3),
        ("C44", ctypes.c_double), ("C12", ctypes.c_double), ("C11", ctypes.c_double),
        ("dslip", ctypes.c_double), ("b", ctypes.c_double), ("cd_dt", ctypes.c_double),
        ("core_flag", ctypes.c_int),
        ("isf", ctypes.c_double), ("usf", ctypes.c_double), ("An", ctypes.c_double),
        ("c", ctypes.c_double * 7), ("aa", ctypes.c_double * 5), ("bb", ctypes.c_double * 4),
        ("site_gsfe", DP), ("xo", DP),
        ("sigma", D33), ("dsigma", D33),
        ("non_schmid", ctypes.c_int), ("angle_to_110", ctypes.c_double),
        ("w1", ctypes.c_double), ("w2", ctypes.c_double), ("w3", ctypes.c_double),
        ("usfe_fit", ctypes.c_double * 5),
    ]


class CondMaterial(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("condsigma", "alpha_resistivity", "mfpel", "alpha_mfpel", "dlayer",
                                               "Rgrain", "beta_disloc", "rho_disloc")] + [
        ("Ngrains", ctypes.c_int), ("Nlayers", ctypes.c_int), ("pinterface", ctypes.c_double)]


class CondDesc(ctypes.Structure):
    _fields_ = [("sigma_eff", DP), ("sigma_layer", DP), ("El_y", ctypes.c_double),
                ("epsilonzero", ctypes.c_double), ("timestep", ctypes.c_double)]


class CondStats(ctypes.Structure):
    _fields_ = [("condxinorm", ctypes.c_double), ("condxiave", ctypes.c_double), ("conductivity", ctypes.c_double)]


class CheckpointInfo(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("n_slip", ctypes.c_int),
                ("fields", ctypes.c_int), ("precision", ctypes.c_int), ("imag_mode", ctypes.c_int),
                ("advanced", ctypes.c_int), ("field_bytes", ctypes.c_size_t), ("carrier_bytes", ctypes.c_size_t),
                ("sigma", D33), ("dsigma", D33), ("steps", ctypes.c_ulonglong)]


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("imag_mode", ctypes.c_int), ("device", ctypes.c_int),
                ("use_graphs", ctypes.c_int), ("check_finite", ctypes.c_int)]


class StepStats(ctypes.Structure):
    _fields_ = [("xinorm", ctypes.c_double), ("xiave", ctypes.c_double), ("steps_done", ctypes.c_int),
                ("converged", ctypes.c_int)]


class PfddError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("pfdd status %d (%s): %s" % (code, ERRORS.get(code, "?"), msg))
        self.code = code


_lib = None


def load(path: str = LIB_PATH):
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError("libpfdd_b200.so not built at %s (run __graft_entry__.build())" % path)
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    lib.pfdd_gpu_create.argtypes = [ctypes.POINTER(InstanceDesc), ctypes.c_int, ctypes.POINTER(Options),
                                    ctypes.POINTER(vp)]
    lib.pfdd_gpu_set_state.argtypes = [vp, ctypes.c_int, DP, DP]
    lib.pfdd_gpu_set_state_interleaved.argtypes = [vp, ctypes.c_int, DP]
    lib.pfdd_gpu_get_state.argtypes = [vp, ctypes.c_int, DP, DP]
    lib.pfdd_gpu_get_state_interleaved.argtypes = [vp, ctypes.c_int, DP]
    lib.pfdd_gpu_advance.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(StepStats)]
    lib.pfdd_gpu_step_history.argtypes = [vp, ctypes.c_int, DP, DP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.pfdd_gpu_energy.argtypes = [vp, ctypes.c_int, DP, DP, DP]
    lib.pfdd_gpu_strain_stress.argtypes = [vp, ctypes.c_int, DP, DP, DP, DP]
    lib.pfdd_gpu_core_profile.argtypes = [vp, ctypes.c_int, ctypes.c_int, DP, DP]
    lib.pfdd_gpu_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.pfdd_gpu_snapshot_begin.argtypes = [vp, ctypes.c_int, DP, DP]
    lib.pfdd_gpu_snapshot_wait.argtypes = [vp, ctypes.c_int]
    lib.pfdd_cond_layers.argtypes = [ctypes.POINTER(CondMaterial), ctypes.POINTER(CondMaterial), ctypes.c_int,
                                     ctypes.c_double, DP, DP]
    lib.pfdd_gpu_cond_enable.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CondDesc)]
    lib.pfdd_gpu_cond_set_state.argtypes = [vp, ctypes.c_int, DP, DP]
    lib.pfdd_gpu_cond_get_state.argtypes = [vp, ctypes.c_int, DP, DP]
    lib.pfdd_gpu_cond_step.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(CondStats)]
    lib.pfdd_gpu_tau.argtypes = [vp, ctypes.c_int, DP]
    lib.pfdd_checkpoint_write.argtypes = [ctypes.c_char_p, ctypes.POINTER(CheckpointInfo), vp, vp]
    lib.pfdd_checkpoint_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(CheckpointInfo), vp, ctypes.c_size_t, vp,
                                         ctypes.c_size_t]
    lib.pfdd_gpu_checkpoint_save.argtypes = [vp, ctypes.c_int, ctypes.c_char_p]
    lib.pfdd_gpu_checkpoint_load.argtypes = [vp, ctypes.c_int, ctypes.c_char_p]
    lib.pfdd_gl_step_noalloc.argtypes = [ctypes.POINTER(InstanceDesc), vp, vp, DP, vp]
    lib.pfdd_gpu_set_stress.argtypes = [vp, ctypes.c_int, DP]
    lib.pfdd_gpu_adjoint.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, DP, DP, DP]
    lib.pfdd_gpu_adjoint_forward.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.pfdd_gpu_adjoint_backward.argtypes = [vp, ctypes.c_int, DP, DP, DP]
    lib.pfdd_gpu_set_stream.argtypes = [vp, vp]
    lib.pfdd_gpu_profile.argtypes = [vp, ctypes.c_int, DP, ctypes.POINTER(ctypes.c_int)]
    lib.pfdd_gpu_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_size_t)]
    lib.pfdd_gpu_last_error.argtypes = [vp]
    lib.pfdd_gpu_last_error.restype = ctypes.c_char_p
    lib.pfdd_gpu_destroy.argtypes = [vp]
    lib.pfdd_gpu_destroy.restype = None
    lib.pfdd_gpu_version.restype = ctypes.c_char_p
    for name in EXPORTS:
        if name not in ("pfdd_gpu_last_error", "pfdd_gpu_destroy", "pfdd_gpu_version"):
            getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(DP) if a is not None else None


def desc_from_workload(w, core_flag=None, An=None):
    """InstanceDesc for a configs.Workload (constants derived as Material does)."""
    d = InstanceDesc()
    d.nx, d.ny, d.nz, d.n_slip = w.nx, w.ny, w.nz, w.S
    for i in range(3):
        for j in range(3):
            d.four[i][j] = float(w.four[i, j])
            d.prim[i][j] = float(w.prim[i, j])
            d.sigma[i][j] = float(w.sigma[i, j])
            d.dsigma[i][j] = float(w.dsigma[i, j])
    for a in range(w.S):
        for j in range(3):
            d.xn[a][j] = float(w.xn[a, j])
            d.xb[a][j] = float(w.xb[a, j])
    C44, C12, C11 = w.material.elastic()
    d.C44, d.C12, d.C11 = C44, C12, C11
    d.dslip, d.b, d.cd_dt = w.material.dslip, w.material.b, w.cd_dt
    d.core_flag = w.core_flag if core_flag is None else core_flag
    d.isf, d.usf = w.material.isf, w.material.usf
    d.An = w.material.An if An is None else An
    ns = getattr(w, "non_schmid", None)
    if ns is not None:
        d.non_schmid = 1
        d.angle_to_110, d.w1, d.w2, d.w3 = (float(v) for v in ns)
    fit = getattr(w.material, "usfe_fit", None)
    if fit is not None:
        for i in range(5):
            d.usfe_fit[i] = float(fit[i])
    extra = getattr(w, "core_extra", None) or {}
    for key, n in (("c", 7), ("aa", 5), ("bb", 4)):
        if key in extra:
            arr = getattr(d, key)
            for i in range(n):
                arr[i] = float(extra[key][i])
    return d


def cond_material(d):
    m = CondMaterial()
    for name, _ in CondMaterial._fields_:
        setattr(m, name, d.get(name, 0) if name not in ("Ngrains", "Nlayers") else int(d.get(name, 1)))
    return m


def cond_layers(A, B, ny, temperature):
    """pfdd_cond_layers (host): per-y effective and layer conductivity [ny] each."""
    lib = load()
    eff, lay = np.zeros(ny), np.zeros(ny)
    a, b = cond_material(A), cond_material(B)
    st = lib.pfdd_cond_layers(ctypes.byref(a), ctypes.byref(b), ny, float(temperature), _dp(eff), _dp(lay))
    if st != 0:
        raise PfddError(st, "pfdd_cond_layers")
    return eff, lay


class Stepper:
    """Owns one pfdd_gpu handle (one or more instances)."""

    def __init__(self, descs, precision=FP64, imag_mode=IMAG_AUTO, device=0, keep=(), use_graphs=True):
        lib = load()
        self._lib = lib
        self._keep = list(keep)   # host arrays referenced by descriptors during create
        arr = (InstanceDesc * len(descs))(*descs)
        opt = Options(precision, imag_mode, device, 1 if use_graphs else 0, 1)
        h = ctypes.c_void_p()
        st = lib.pfdd_gpu_create(arr, len(descs), ctypes.byref(opt), ctypes.byref(h))
        if st != PFDD_OK:
            raise PfddError(st, lib.pfdd_gpu_last_error(None).decode())
        self.h = h
        self.descs = descs
        self.n = len(descs)

    @classmethod
    def from_workloads(cls, workloads, precision=FP64, imag_mode=IMAG_AUTO, device=0, use_graphs=True):
        descs, keep = [], []
        for w in workloads:
            d = desc_from_workload(w)
            if w.site is not None:
                s = np.ascontiguousarray(w.site, dtype=np.float64).reshape(-1)
                keep.append(s)
                d.site_gsfe = _dp(s)
            if w.xo is not None:
                m = np.ascontiguousarray(w.xo, dtype=np.float64).reshape(-1)
                keep.append(m)
                d.xo = _dp(m)
            descs.append(d)
        st = cls(descs, precision, imag_mode, device, keep, use_graphs)
        st._keep = []
        return st

    def _check(self, st):
        if st != PFDD_OK:
            raise PfddError(st, self._lib.pfdd_gpu_last_error(self.h).decode())

    def set_state(self, inst, re, im=None):
        re = np.ascontiguousarray(re, dtype=np.float64).reshape(-1)
        im = None if im is None else np.ascontiguousarray(im, dtype=np.float64).reshape(-1)
        self._check(self._lib.pfdd_gpu_set_state(self.h, inst, _dp(re), _dp(im)))

    def get_state(self, inst, imag=True):
        """(Re xi, Im xi) as [S, nx, ny, nz] arrays; imag=False: Im is None."""
        d = self.descs[inst]
        n = d.n_slip * d.nx * d.ny * d.nz
        re = np.empty(n)
        im = np.empty(n) if imag else None
        self._check(self._lib.pfdd_gpu_get_state(self.h, inst, _dp(re), _dp(im)))
        shape = (d.n_slip, d.nx, d.ny, d.nz)
        return re.reshape(shape), (im.reshape(shape) if imag else None)

    def advance(self, n_steps, stress_states=1, tol=0.0):
        stats = (StepStats * self.n)()
        self._check(self._lib.pfdd_gpu_advance(self.h, n_steps, stress_states, tol, stats))
        return [(s.xinorm, s.xiave, s.steps_done, s.converged) for s in stats]

    def history(self, inst, cap=1 << 20):
        cnt = ctypes.c_int()
        self._check(self._lib.pfdd_gpu_step_history(self.h, inst, None, None, 0, ctypes.byref(cnt)))
        n = cnt.value
        a = np.empty(max(n, 1))
        b = np.empty(max(n, 1))
        self._check(self._lib.pfdd_gpu_step_history(self.h, inst, _dp(a), _dp(b), n, ctypes.byref(cnt)))
        return a[:n], b[:n]

    def set_stress(self, inst, sigma):
        """Replace instance inst's current applied stress (3x3, units of mu)."""
        s = np.ascontiguousarray(sigma, dtype=np.float64).reshape(9)
        self._check(self._lib.pfdd_gpu_set_stress(self.h, inst, _dp(s)))

    def checkpoint_save(self, inst, path):
        self._check(self._lib.pfdd_gpu_checkpoint_save(self.h, inst, os.fsencode(path)))

    def checkpoint_load(self, inst, path):
        self._check(self._lib.pfdd_gpu_checkpoint_load(self.h, inst, os.fsencode(path)))

    def tau(self, inst):
        t = np.empty(self.descs[inst].n_slip)
        self._check(self._lib.pfdd_gpu_tau(self.h, inst, _dp(t)))
        return t

    def energy(self, inst):
        e = np.empty(3)
        self._check(self._lib.pfdd_gpu_energy(self.h, inst, _dp(e[0:1]), _dp(e[1:2]), _dp(e[2:3])))
        return tuple(e)

    def autotune(self, reps=5):
        """Time every x-pencil tile width per group and keep the fastest;
        returns the chosen width per instance."""
        out = (ctypes.c_int * len(self.descs))()
        self._check(self._lib.pfdd_gpu_autotune(self.h, int(reps), out))
        return list(out)

    def snapshot_begin(self, inst, re, im=None):
        """Start copying the current state into re / im (float64 arrays of
        S*N, ideally page-locked); they are filled when snapshot_wait returns."""
        self._snap = (re, im)   # keep the buffers alive until the wait
        self._check(self._lib.pfdd_gpu_snapshot_begin(self.h, inst, _dp(re), _dp(im) if im is not None else None))

    def snapshot_wait(self, inst):
        self._check(self._lib.pfdd_gpu_snapshot_wait(self.h, inst))

    def cond_enable(self, inst, sigma_eff, sigma_layer, El_y, epsilonzero, timestep=1.0):
        eff = np.ascontiguousarray(sigma_eff, dtype=np.float64)
        lay = np.ascontiguousarray(sigma_layer, dtype=np.float64)
        d = CondDesc(_dp(eff), _dp(lay), float(El_y), float(epsilonzero), float(timestep))
        self._check(self._lib.pfdd_gpu_cond_enable(self.h, inst, ctypes.byref(d)))

    def cond_set_state(self, inst, c):
        c = np.asarray(c)
        re = np.ascontiguousarray(np.real(c), dtype=np.float64).reshape(-1)
        im = np.ascontiguousarray(np.imag(c), dtype=np.float64).reshape(-1)
        self._check(self._lib.pfdd_gpu_cond_set_state(self.h, inst, _dp(re), _dp(im)))

    def cond_get_state(self, inst):
        ds = self.descs[inst]
        n = ds.nx * ds.ny * ds.nz
        re, im = np.zeros(n), np.zeros(n)
        self._check(self._lib.pfdd_gpu_cond_get_state(self.h, inst, _dp(re), _dp(im)))
        return (re + 1j * im).reshape(ds.nx, ds.ny, ds.nz)

    def cond_step(self, inst, n_iters=1):
        """n_iters conductivity iterations: array [n_iters, 3] of
        (condxinorm, condxiave, conductivity)."""
        st = (CondStats * n_iters)()
        self._check(self._lib.pfdd_gpu_cond_step(self.h, inst, n_iters, st))
        return np.array([[s.condxinorm, s.condxiave, s.conductivity] for s in st])

    def core_profile(self, inst, n_planes):
        """project_core_energy of the current state: delta [n_planes, nx, ny, nz]
        and the ddelta line [n_planes, nx] at j = ny/2, k = nz/2."""
        ds = self.descs[inst]
        nx, ny, nz = ds.nx, ds.ny, ds.nz
        d = np.zeros(n_planes * nx * ny * nz)
        dd = np.zeros(n_planes * nx)
        self._check(self._lib.pfdd_gpu_core_profile(self.h, inst, n_planes, _dp(d), _dp(dd)))
        return d.reshape(n_planes, nx, ny, nz), dd.reshape(n_planes, nx)

    def strain_stress(self, inst, fields=True):
        """Strain and stress of the current state (the reference's data_eps /
        data_sigma real parts and ave_eps / ave_sigma): eps, sigma
        [3, 3, nx, ny, nz] (None unless fields) and ave_eps, ave_sigma [3, 3]."""
        d = self.descs[inst]
        nx, ny, nz = d.nx, d.ny, d.nz
        n = nx * ny * nz
        e = np.empty(9 * n) if fields else None
        s = np.empty(9 * n) if fields else None
        ae, asg = np.empty(9), np.empty(9)
        null = ctypes.cast(None, DP)
        self._check(self._lib.pfdd_gpu_strain_stress(self.h, inst, _dp(e) if fields else null,
                                                     _dp(s) if fields else null, _dp(ae), _dp(asg)))
        shape = (3, 3, nx, ny, nz)
        return (e.reshape(shape) if fields else None, s.reshape(shape) if fields else None,
                ae.reshape(3, 3), asg.reshape(3, 3))

    def adjoint_forward(self, inst, n_steps, ckpt_every):
        """Forward run of n_steps kept as the adjoint's tape (checkpoints every
        ckpt_every steps); the instance ends at xi_N as after advance."""
        self._check(self._lib.pfdd_gpu_adjoint_forward(self.h, inst, n_steps, ckpt_every))

    def adjoint_backward(self, inst, dL_dxiN):
        """(dL/d(p0, p1), dL/dsigma[6]) for the seed dL/dRe xi_N [S, nx, ny, nz]."""
        g = np.ascontiguousarray(dL_dxiN, dtype=np.float64).reshape(-1)
        dp = np.zeros(2)
        ds = np.zeros(6)
        self._check(self._lib.pfdd_gpu_adjoint_backward(self.h, inst, _dp(g), _dp(dp), _dp(ds)))
        return dp, ds

    def adjoint(self, inst, n_steps, ckpt_every, dL_dxiN):
        """Forward tape and backward pass in one call, for a seed known beforehand."""
        g = np.ascontiguousarray(dL_dxiN, dtype=np.float64).reshape(-1)
        dp = np.zeros(2)
        ds = np.zeros(6)
        self._check(self._lib.pfdd_gpu_adjoint(self.h, inst, n_steps, ckpt_every, _dp(g), _dp(dp), _dp(ds)))
        return dp, ds

    def set_stream(self, stream_handle):
        """Run on a caller stream (an int cudaStream_t, e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self._lib.pfdd_gpu_set_stream(self.h, ctypes.c_void_p(stream_handle or None)))

    def profile(self, n_steps):
        """Mean device ms per launch of each kernel class over n_steps GL iterations."""
        ms = np.zeros(len(KERNELS))
        lps = ctypes.c_int()
        self._check(self._lib.pfdd_gpu_profile(self.h, n_steps, _dp(ms), ctypes.byref(lps)))
        return dict(zip(KERNELS, ms)), lps.value

    def info(self):
        n = ctypes.c_int()
        b = ctypes.c_size_t()
        self._check(self._lib.pfdd_gpu_info(self.h, ctypes.byref(n), ctypes.byref(b)))
        return n.value, b.value

    def close(self):
        if getattr(self, "h", None):
            self._lib.pfdd_gpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
