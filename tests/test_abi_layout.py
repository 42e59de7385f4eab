"""The ctypes mirror of pfdd_instance_desc has the C header's layout: a
C program compiled from include/pfdd_b200.h prints each field's offset."""
import ctypes
import os
import shutil
import subprocess
import tempfile

import pytest

from pfdd_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_instance_desc_layout_matches_header():
    names = [f[0] for f in capi.InstanceDesc._fields_]
    src = ['#include <stddef.h>', '#include <stdio.h>', '#include "pfdd_b200.h"', 'int main(void) {',
           '  printf("%zu\\n", sizeof(pfdd_instance_desc));']
    src += ['  printf("%%zu\\n", offsetof(pfdd_instance_desc, %s));' % n for n in names]
    src += ['  return 0;', '}']
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "layout.c")
        exe = os.path.join(tmp, "layout")
        with open(c, "w") as f:
            f.write("\n".join(src) + "\n")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = [int(v) for v in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()]
    assert out[0] == ctypes.sizeof(capi.InstanceDesc)
    for n, off in zip(names, out[1:]):
        assert getattr(capi.InstanceDesc, n).offset == off, n
