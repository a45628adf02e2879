"""sdft_piny_adapter_finalize (csrc/piny/sdft_piny_adapter.c) releases every
system's context; the next adapted call builds it again.  A module of its own,
run after test_gpu_piny_adapter.py, because it drops the contexts that module's
fixtures made."""
import os

import numpy as np
import pytest

from conftest import rel_l2
from oracle import ref as R

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cfg1_reference.npz")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(adapter=True), reason="oracle/_ref/libpinyref_adapter.so not built")]


def test_adapter_finalize_and_recreate(sys1, monkeypatch):
    gold = dict(np.load(GOLD))
    monkeypatch.setenv("SDFT_PINY_PRECISION", "fp64")
    r = R.RefSys(sys1, 8, adapter=True)
    fr, fi, _ = r.hpsi(gold["in_re"], gold["in_im"])
    R.lib(adapter=True).sdft_piny_adapter_finalize()
    gr, gi, _ = r.hpsi(gold["in_re"], gold["in_im"])
    cat = np.concatenate
    assert rel_l2(cat([gr, gi]), cat([fr, fi])) < 1e-15
    assert rel_l2(cat([gr, gi]), cat([gold["hpsi_re"], gold["hpsi_im"]])) < 1e-12
