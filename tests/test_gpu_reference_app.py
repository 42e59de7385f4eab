"""The reference's own application driving the GPU through the drop-in styles.

The reference's main.cpp and sources, linked with the library's FFT style
`b200` and solve style `GLgpu` (the package's reference_plugin/, built by
`make -C oracle/ref_build b200`), run the reference's example decks
(src/in.fcc-pfdd: app 1L1S100B, perfect core, Ni, sigma_xz = 0.03;
src/in.bcc-pfdd: app 2d-bcc-1lOrtho on the rotated BCC grid; both 32^3 with
strain/stress diagnostics and a text dump) with only the two style lines
swapped (tests/golden/decks/, written by tests/golden/make_decks.py).  The
same decks with the stock styles run through the unmodified reference build:
its own main.cpp for the FCC deck; for the BCC deck the oracle harness, which
runs the deck the same way but first gives App::num_planes a value -- the
stock application crashes on that deck because app 2d-bcc-1lOrtho never sets
it (app_2d_bcc_ortho_1loop.cpp; FFTW_Slab::allocate sizes arrays by it,
fft_fftw_slab.cpp:140-199).  The b200 style sets it the same way.
Every dump snapshot (xi and the six stress components per site) and every
stats line (the diagnostics' averages) must agree to the text's printed
precision (%g, 6 digits): the GPU's FP64 path equals the reference to 1e-10 in
xi, so what differs is the last printed digit at most.

Deck -> Input::fft_style / Input::solve_style (src/input.cpp:693-727) ->
FFT_B200 (FftStyle, src/fft_fftw_slab.h:16-17) / SolveGLGPU (SolveStyle,
src/solve_GL.h:16-17) -> libpfdd_b200.so.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_APP = os.path.join(ROOT, "oracle", "_ref", "pfdd_ref")
REF_HARNESS = os.path.join(ROOT, "oracle", "_ref", "pfdd_ref_harness")
B200_APP = os.path.join(ROOT, "oracle", "_ref", "pfdd_ref_b200")
DECKS = os.path.join(ROOT, "tests", "golden", "decks")


def _raise_stack():
    import resource
    try:
        soft, hard = resource.getrlimit(resource.RLIMIT_STACK)
        resource.setrlimit(resource.RLIMIT_STACK, (hard, hard))
    except Exception:
        pass


def _run(app, deck_text, tmp):
    with open(os.path.join(tmp, "in.deck"), "w") as f:
        f.write(deck_text)
    if app == REF_HARNESS:   # the deck as the reference runs it, stats not logged
        args = [app, "-deck", "in.deck"]
    else:
        args = [app, "-in", "in.deck", "-log", "log.txt", "-screen", "none"]
    p = subprocess.run(args, cwd=tmp, capture_output=True, text=True, timeout=900, preexec_fn=_raise_stack)
    assert p.returncode == 0, (os.path.basename(app), p.returncode, p.stdout[-2000:], p.stderr[-2000:])
    stats = _stats(os.path.join(tmp, "log.txt")) if app != REF_HARNESS else None
    return _dump(os.path.join(tmp, "dump.txt")), stats, p.stdout


def _dump(path):
    """[(timestep, array of the ATOMS rows)] of a text dump."""
    snaps, lines = [], open(path).read().splitlines()
    i = 0
    while i < len(lines):
        if lines[i].startswith("ITEM: TIMESTEP"):
            ts = int(lines[i + 1].split()[0])
            n = int(lines[i + 3])
            rows = np.array([[float(v) for v in l.split()] for l in lines[i + 9:i + 9 + n]])
            snaps.append((ts, rows))
            i += 9 + n
        else:
            i += 1
    return snaps


def _stats(path):
    """Numeric stats lines of the log (iteration, ..., diagnostics), the
    elapsed-time column (index 2) dropped."""
    out = []
    for line in open(path):
        w = line.split()
        if len(w) > 3:
            try:
                v = [float(x) for x in w]
            except ValueError:
                continue
            out.append(v[:2] + v[3:])
    return np.array(out)


def _close(a, b, what, groups):
    """a equals b to the printed precision (%g, 6 digits: 2e-5 relative) within
    each group of columns that hold one quantity; entries that are round-off
    around zero (the reference's FP64 FFTs leave ~1e-16 in Im xi, ~1e-19 of the
    strain scale in near-zero averages; the GPU's Nyquist carrier leaves exact
    zeros) are compared against 1e-9 of the group's scale."""
    for cols in groups:
        x, y = a[:, cols], b[:, cols]
        scale = max(np.abs(y).max(), 1e-300)
        err = np.abs(x - y) / np.maximum(np.abs(y), 1e-9 * scale)
        assert err.max() <= 2e-5, (what, cols, float(err.max()), np.unravel_index(np.argmax(err), err.shape))


# dump columns: x y z | xir1 xii1 | pxx pyy pzz pxy pxz pyz
DUMP_GROUPS = ([0, 1, 2], [3, 4], [5, 6, 7, 8, 9, 10])
# stats columns (elapsed time dropped): iteration, time | six strain averages | six stress averages
STATS_GROUPS = ([0, 1], [2, 3, 4, 5, 6, 7], [8, 9, 10, 11, 12, 13])


@pytest.mark.parametrize("deck,ref_app", [("in.fcc-pfdd", REF_APP), ("in.bcc-pfdd", REF_HARNESS)])
def test_reference_deck_through_the_drop_in_styles(deck, ref_app):
    if not all(os.access(p, os.X_OK) for p in (ref_app, B200_APP)):
        pytest.fail("reference applications not built (make -C oracle/ref_build all b200)")
    ref_text = open(os.path.join(DECKS, deck + ".ref")).read()
    b200_text = open(os.path.join(DECKS, deck + ".b200")).read()
    with tempfile.TemporaryDirectory() as t1, tempfile.TemporaryDirectory() as t2:
        ref_dump, ref_stats, _ = _run(ref_app, ref_text, t1)
        gpu_dump, gpu_stats, _ = _run(B200_APP, b200_text, t2)
    assert [s[0] for s in ref_dump] == [s[0] for s in gpu_dump] and len(ref_dump) >= 4
    for (ts, a), (_, b) in zip(gpu_dump, ref_dump):
        assert a.shape == b.shape
        _close(a, b, "dump step %d" % ts, DUMP_GROUPS)
    if ref_stats is not None:
        assert gpu_stats.shape == ref_stats.shape and len(ref_stats) >= 40
        _close(gpu_stats, ref_stats, "stats", STATS_GROUPS)


def test_fp32_and_gpu_diagnostics_track_the_reference():
    """`precision fp32 diag gpu`: the FP32 step follows the reference run (xi
    columns), and the GPU strain/stress fill the stress columns.  Their values
    are those of the state after each output step (pfdd_gpu_strain_stress,
    checked against the oracle in test_gpu_strain_stress.py); the reference's
    loop prints the strain of the state before the step with the eigenstrain
    of the state after it, which differ at a moving core by the step's
    change times the elastic constants, so only their finiteness and scale
    are compared here."""
    if not (os.access(REF_APP, os.X_OK) and os.access(B200_APP, os.X_OK)):
        pytest.fail("reference applications not built (make -C oracle/ref_build all b200)")
    deck = "in.fcc-pfdd"
    ref_text = open(os.path.join(DECKS, deck + ".ref")).read()
    b200_text = open(os.path.join(DECKS, deck + ".b200")).read().replace("precision fp64", "precision fp32 diag gpu")
    with tempfile.TemporaryDirectory() as t1, tempfile.TemporaryDirectory() as t2:
        ref_dump, _, _ = _run(REF_APP, ref_text, t1)
        gpu_dump, _, _ = _run(B200_APP, b200_text, t2)
    assert [s[0] for s in ref_dump] == [s[0] for s in gpu_dump]
    (_, a), (_, b) = gpu_dump[-1], ref_dump[-1]
    xi_err = np.abs(a[:, 3:5] - b[:, 3:5]).max()
    assert xi_err <= 1e-4, xi_err
    assert np.isfinite(a[:, 5:]).all()
    ra, rb = np.abs(a[:, 5:]).max(), np.abs(b[:, 5:]).max()
    assert 0.5 * rb <= ra <= 2.0 * rb, (ra, rb)
