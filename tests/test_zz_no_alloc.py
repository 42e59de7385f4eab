"""The allocation-free single-step entry point, pfdd_gl_step_noalloc.

It exists for callers that cannot call cudaMalloc (host codes whose runtime
owns all device memory through its own pool, long-running or real-time hosts
that must not allocate after start-up).  Its scratch is a fixed device
array inside the library, so this test checks it the way such a caller uses
it: device buffers owned by the caller, two steps in a row through the C ABI,
each compared with the handle-based entry point (pfdd_gpu_advance) on the same
input, to the FP64 tolerance of the other parity tests (1e-10).  The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from common import small_loop
from pfdd_b200 import capi, configs

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _handle_steps(w, xi0, n):
    """States after 1..n steps from the handle path (FP64, Im as full field)."""
    out = []
    with capi.Stepper.from_workloads([w], precision=capi.FP64, imag_mode=capi.IMAG_FULL) as st:
        st.set_state(0, xi0.real, xi0.imag)
        for _ in range(n):
            st.advance(1)
            re, im = st.get_state(0)
            out.append(np.concatenate([re.reshape(-1), im.reshape(-1)]))
    return out


@pytest.mark.parametrize("make", ["loop", "bcc_non_schmid"])
def test_noalloc_matches_handle_path_two_calls(make):
    import torch
    lib = capi.load()
    lib.pfdd_gl_step_noalloc.argtypes = [ctypes.POINTER(capi.InstanceDesc), ctypes.c_void_p, ctypes.c_void_p,
                                         capi.DP, ctypes.c_void_p]
    lib.pfdd_gl_step_noalloc.restype = ctypes.c_int
    # the second deck: non-Schmid tau and the USFE(angle, tau) core (model 6)
    w = small_loop(32) if make == "loop" else configs.bcc_screw_workload(n=16, nz=8, core_flag=6)
    rng = np.random.default_rng(17)
    xi0 = w.xi0 + 1j * rng.uniform(-1e-3, 1e-3, size=w.xi0.shape)
    expect = _handle_steps(w, xi0, 2)

    desc = capi.desc_from_workload(w)
    dev = torch.device("cuda:0")
    a = torch.from_numpy(np.concatenate([xi0.real.reshape(-1), xi0.imag.reshape(-1)])).to(dev)
    b = torch.empty_like(a)
    stream = torch.cuda.current_stream().cuda_stream
    stats = np.zeros(2)
    for call in range(2):
        torch.cuda.synchronize()
        rc = lib.pfdd_gl_step_noalloc(ctypes.byref(desc), ctypes.c_void_p(a.data_ptr()),
                                      ctypes.c_void_p(b.data_ptr()), stats.ctypes.data_as(capi.DP),
                                      ctypes.c_void_p(stream))
        assert rc == 0, rc
        got = b.cpu().numpy()
        assert np.abs(got - expect[call]).max() <= TOL
        assert np.isfinite(stats).all() and stats[0] > 0
        a, b = b, a


def test_noalloc_rejects_grid_beyond_static_scratch():
    lib = capi.load()
    lib.pfdd_gl_step_noalloc.argtypes = [ctypes.POINTER(capi.InstanceDesc), ctypes.c_void_p, ctypes.c_void_p,
                                         capi.DP, ctypes.c_void_p]
    lib.pfdd_gl_step_noalloc.restype = ctypes.c_int
    w = small_loop(16)
    desc = capi.desc_from_workload(w)
    desc.nx = desc.ny = desc.nz = 128     # 3 systems, Re+Im: about 100 MB of spectrum
    import torch
    a = torch.zeros(16, dtype=torch.float64, device="cuda:0")   # not touched: the size check comes first
    b = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    rc = lib.pfdd_gl_step_noalloc(ctypes.byref(desc), ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                  None, None)
    assert rc == -1
