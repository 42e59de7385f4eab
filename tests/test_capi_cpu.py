"""The C-ABI library without a GPU: it loads, exports every entry point
include/pfdd_b200.h declares, and create fails cleanly (no compute calls)."""
import os
import re

import pytest

from pfdd_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "pfdd_b200.h")).read()
    decl = r"^(?:pfdd_status|void|const char \*)\s*(pfdd_[a-z_0-9]+)\s*\("
    return sorted(set(re.findall(decl, txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_symbols()
    assert "pfdd_gpu_create" in names and len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(capi.EXPORTS) <= set(names)


def test_version_string():
    assert capi.load().pfdd_gpu_version().startswith(b"pfdd_b200")


def test_create_without_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from pfdd_b200 import configs
    w = configs.loop_workload(n=8)
    with pytest.raises(capi.PfddError) as e:
        capi.Stepper.from_workloads([w])
    assert e.value.code in (-6, -3)
    assert capi.load().pfdd_gpu_last_error(None)
