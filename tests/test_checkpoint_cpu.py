"""The binary checkpoint format on the host (no device): a round trip keeps
every byte, and a file that was truncated, altered in its payload or header,
or is not a checkpoint at all is refused with PFDD_EINVAL while the caller's
buffers stay untouched.  (The reference has no resumable state; its only
copies are temp_stor_data / reset_data, src/fft_fftw_slab.cpp:1891-1925.)"""
import ctypes
import os

import numpy as np
import pytest

from pfdd_b200 import capi


def _info(nx=8, ny=6, nz=4, S=3, prec=capi.FP32, carrier=40):
    i = capi.CheckpointInfo()
    i.nx, i.ny, i.nz, i.n_slip, i.fields, i.precision = nx, ny, nz, S, S, prec
    i.imag_mode, i.advanced = capi.IMAG_NYQUIST, 1
    i.field_bytes = S * nx * ny * nz * (4 if prec == capi.FP32 else 8)
    i.carrier_bytes = carrier
    for a in range(3):
        for b in range(3):
            i.sigma[a][b] = 0.001 * (3 * a + b)
            i.dsigma[a][b] = 1e-6 * (a - b)
    i.steps = 1234
    return i


def _write(path, info, fields, carrier):
    lib = capi.load()
    return lib.pfdd_checkpoint_write(os.fsencode(path), ctypes.byref(info), fields.ctypes.data_as(ctypes.c_void_p),
                                     carrier.ctypes.data_as(ctypes.c_void_p) if carrier is not None else None)


def _read(path, fcap, ccap):
    lib = capi.load()
    out = capi.CheckpointInfo()
    f = np.full(fcap, 0xAB, dtype=np.uint8)
    c = np.full(max(ccap, 1), 0xCD, dtype=np.uint8)
    rc = lib.pfdd_checkpoint_read(os.fsencode(path), ctypes.byref(out), f.ctypes.data_as(ctypes.c_void_p), fcap,
                                  c.ctypes.data_as(ctypes.c_void_p) if ccap else None, ccap)
    return rc, out, f, c


def test_round_trip(tmp_path):
    info = _info()
    rng = np.random.default_rng(0)
    fields = rng.integers(0, 256, info.field_bytes, dtype=np.uint8)
    carrier = rng.integers(0, 256, info.carrier_bytes, dtype=np.uint8)
    p = tmp_path / "a.ckp"
    assert _write(p, info, fields, carrier) == 0
    assert os.path.getsize(p) == 256 + info.field_bytes + info.carrier_bytes
    rc, out, f, c = _read(p, info.field_bytes, info.carrier_bytes)
    assert rc == 0
    assert np.array_equal(f, fields) and np.array_equal(c[:info.carrier_bytes], carrier)
    for k in ("nx", "ny", "nz", "n_slip", "fields", "precision", "imag_mode", "advanced", "field_bytes",
              "carrier_bytes", "steps"):
        assert getattr(out, k) == getattr(info, k), k
    assert [[out.sigma[a][b] for b in range(3)] for a in range(3)] == \
           [[info.sigma[a][b] for b in range(3)] for a in range(3)]
    # the header alone
    hdr = capi.CheckpointInfo()
    assert capi.load().pfdd_checkpoint_read(os.fsencode(p), ctypes.byref(hdr), None, 0, None, 0) == 0
    assert hdr.field_bytes == info.field_bytes


@pytest.mark.parametrize("damage", ["payload_bit", "header_bit", "truncated", "appended", "magic"])
def test_damaged_file_is_refused(tmp_path, damage):
    info = _info(prec=capi.FP64, carrier=0)
    fields = np.arange(info.field_bytes, dtype=np.uint8)
    p = tmp_path / "b.ckp"
    assert _write(p, info, fields, None) == 0
    raw = bytearray(open(p, "rb").read())
    if damage == "payload_bit":
        raw[256 + 17] ^= 0x10
    elif damage == "header_bit":
        raw[20] ^= 0x01          # ny
    elif damage == "truncated":
        raw = raw[:-8]
    elif damage == "appended":
        raw += b"\0"
    else:
        raw[0:8] = b"NOTACKPT"
    open(p, "wb").write(bytes(raw))
    rc, _, f, _ = _read(p, info.field_bytes, 0)
    assert rc == -1
    assert (f == 0xAB).all()     # untouched


def test_missing_file_and_small_buffer(tmp_path):
    rc, _, _, _ = _read(tmp_path / "none.ckp", 16, 0)
    assert rc == -1
    info = _info(carrier=0)
    fields = np.zeros(info.field_bytes, dtype=np.uint8)
    p = tmp_path / "c.ckp"
    assert _write(p, info, fields, None) == 0
    rc, _, _, _ = _read(p, info.field_bytes - 1, 0)
    assert rc == -1
