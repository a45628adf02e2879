"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "sdft_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sdft_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_all_symbols(pkg):
    lib = ctypes.CDLL(pkg.LIB_PATH)
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_is_reported_cleanly(pkg, sys1):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(pkg.SdftError) as e:
        pkg.Context(*sys1["grid"], sys1["ka"], sys1["kb"], sys1["kc"], sys1["hmat"], max_states=2)
    assert e.value.code == 6  # SDFT_ERR_NODEVICE


def test_host_validation(pkg):
    with pytest.raises(pkg.SdftError):
        pkg.calcChebyCoeff(0, 1.0, 0.0, 1000.0, 0.0)
