"""Pin the numpy density mixer (oracle/mixer.py) to the reference's own
genDensityMix (stodft/diis.c) and checkpointOutput
(stodft/checkpointIO.c), compiled in oracle/_ref."""
import numpy as np
import pytest

from oracle import mixer as OM
from oracle import ref as R

pytestmark = pytest.mark.skipif(not R.available(), reason="reference-compiled oracle (oracle/_ref) not built")

PARAMS = dict(num_diis=4, num_step_mix=2, mix_ratio_big=0.3, mix_ratio_sm=0.5, mix_ratio_sm2=0.7)


def _densities(n, steps, seed=3):
    """A converging sequence of corrected densities: a fixed profile plus a
    decaying random error per step."""
    rng = np.random.default_rng(seed)
    base = 0.02 + 0.01 * np.sin(np.linspace(0.0, 40.0, n)) ** 2
    return [base + (0.6 ** k) * 1e-3 * rng.standard_normal(n) for k in range(steps)]


@pytest.mark.parametrize("params", [PARAMS, dict(PARAMS, num_diis=1, num_step_mix=0),
                                    dict(PARAMS, num_diis=7, num_step_mix=1)])
def test_mixing_matches_reference(params):
    n, steps = 4096, 14
    ref = R.RefMixer(n, **params)
    orc = OM.DensityMixer(n, **params)
    for k, rho in enumerate(_densities(n, steps)):
        a = ref.step(k, rho)
        b = orc.step(k, rho)
        if k <= params["num_step_mix"]:
            assert np.array_equal(a, b), k  # bank / simple mix: same operations
        else:
            assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a)), k


def test_checkpoint_bytes_match_reference(tmp_path):
    n = 1000
    ref = R.RefMixer(n, **PARAMS)
    orc = OM.DensityMixer(n, **PARAMS)
    for k, rho in enumerate(_densities(n, 3)):
        ref.step(k, rho)
        out = orc.step(k, rho)
    cell = (10.26, 11.0, 9.5)
    path = ref.checkpoint(tmp_path, cell)
    with open(path) as f:
        text_ref = f.read()
    vol = cell[0] * (cell[1] * cell[2])  # getdeth of a diagonal cell
    assert text_ref == orc.checkpoint_text(out, vol)
    assert text_ref.splitlines()[0] == "2 2" and len(text_ref.splitlines()) == 1 + n * (1 + 3 + 2)
