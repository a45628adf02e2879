"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import numpy as np
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


@pytest.mark.parametrize("kw", [dict(alp=0.0), dict(rmax=-1.0), dict(ishift=3), dict(ishift=2, rheal=0.0),
                                dict(ishift=2, rheal=30.0), dict(rmax=400.0), dict(natm=0)])
def test_ewald_real_arguments_checked_before_the_device(pkg, kw):
    """sdft_ewald_real refuses bad arguments with SDFT_ERR_ARG before it
    touches a device: a non-positive splitting parameter or cutoff, an unknown
    shift option, a switching width outside (0, rmax], a cutoff spanning more
    than 16 cells, no atoms."""
    h = np.eye(3) * 10.0
    a = dict(alp=0.5, rmax=20.0, ishift=0, rheal=1.0, natm=2)
    a.update(kw)
    pos = np.zeros((max(a["natm"], 1), 3))
    q = np.ones(a["natm"])
    with pytest.raises(pkg.SdftError) as e:
        pkg.ewald_real(h, pos[:a["natm"]] if a["natm"] else pos[:0], q, a["alp"], a["rmax"], a["ishift"], a["rheal"])
    assert e.value.code == 1  # SDFT_ERR_ARG


ADAPTED = ("filterChebyPolyHerm", "filterNewtonPolyHerm", "normHCheby", "normHNewtonHerm", "calcChebyMoments",
           "calcCoefForceWrapSCF", "rhoCalcRealStoHybrid")


def test_piny_adapter_source_is_guarded():
    """Without -DSDFT_PINY_ADAPTER the adapter translation unit is empty, so a
    build without a PINY tree never needs PINY's headers."""
    src = open(os.path.join(ROOT, "stochastic-density-functional-theory-piny_b200", "csrc", "piny",
                            "sdft_piny_adapter.c")).read()
    body = re.sub(r"/\*.*?\*/", "", src, flags=re.S).strip()
    assert body.startswith("#ifdef SDFT_PINY_ADAPTER") and body.endswith("#endif")
    for name in ADAPTED + ("genNoiseOrbitalReal", "sdft_piny_noise"):
        assert re.search(r"\nvoid " + name + r"\(", src), name


def test_piny_adapter_replaces_the_reference_definitions():
    """In the adapter test library (reference objects + adapter), each
    replaced routine has exactly one strong definition: the adapter's."""
    import subprocess
    path = os.path.join(ROOT, "oracle", "_ref", "libpinyref_adapter.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref/libpinyref_adapter.so not built (needs the reference tree at build time)")
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    kinds = {}
    for line in out.splitlines():
        parts = line.split()
        if len(parts) == 3:
            kinds.setdefault(parts[2], []).append(parts[1])
    for name in ADAPTED:
        assert kinds.get(name) == ["T"], (name, kinds.get(name))
    # the library loads (the device library is found through its runpath)
    ctypes.CDLL(path)


@pytest.mark.parametrize("grid,prec,ncut,code", [
    ((25, 24, 24), 0, None, 5),    # an edge that is not 2^a 3^b
    ((24, 24, 256), 0, None, 5),   # an edge above 128
    ((24, 24, 24), 7, None, 1),    # no such precision mode
    ((24, 24, 24), 0, 1, 1),       # a sphere of one coefficient
])
def test_context_arguments_checked_before_the_device(pkg, sys1, grid, prec, ncut, code):
    """Sizes and modes the kernels do not cover are refused on the host, with
    the reference-style status code, before any device is touched."""
    ka, kb, kc = (sys1[k][:ncut] if ncut else sys1[k] for k in ("ka", "kb", "kc"))
    with pytest.raises(pkg.SdftError) as e:
        pkg.Context(*grid, ka, kb, kc, sys1["hmat"], precision=prec, max_states=2)
    assert e.value.code == code
