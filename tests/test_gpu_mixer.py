"""Device density mixer (genDensityMix, stodft/diis.c) and its checkpoint
files (stodft/checkpointIO.c) against the numpy oracle, which
tests/test_mixer_pin.py pins to the reference's own C."""
import numpy as np
import pytest

from oracle import mixer as OM

pytestmark = pytest.mark.gpu

PARAMS = dict(num_diis=4, num_step_mix=2, mix_ratio_big=0.3, mix_ratio_sm=0.5, mix_ratio_sm2=0.7)


def _densities(n, steps, seed=3):
    rng = np.random.default_rng(seed)
    base = 0.02 + 0.01 * np.sin(np.linspace(0.0, 40.0, n)) ** 2
    return [base + (0.6 ** k) * 1e-3 * rng.standard_normal(n) for k in range(steps)]


@pytest.mark.parametrize("n,params", [(1000, PARAMS), (96 ** 3, PARAMS), (5000, dict(PARAMS, num_diis=1, num_step_mix=0)),
                                      (5000, dict(PARAMS, num_diis=7, num_step_mix=1))])
def test_device_mixer_matches_oracle(pkg, n, params):
    dev = pkg.DensityMixer(n, **params)
    orc = OM.DensityMixer(n, **params)
    rho = np.zeros(n)
    try:
        for k, rc in enumerate(_densities(n, 14)):
            a = dev.step(k, rc, rho)
            b = orc.step(k, rc)
            if k == 0:
                assert not a.any()  # rho_up untouched at step 0
            elif k <= params["num_step_mix"]:
                assert np.array_equal(a, b), k
            else:
                assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)), k
                assert np.allclose(dev.state()[2], orc.coef, rtol=0, atol=1e-10)
    finally:
        dev.close()


def test_checkpoint_file_bytes_and_restart(pkg, tmp_path):
    n = 2000
    dev = pkg.DensityMixer(n, **PARAMS)
    orc = OM.DensityMixer(n, **PARAMS)
    seq = _densities(n, 9)
    cell = (10.26, 11.0, 9.5)
    vol = cell[0] * (cell[1] * cell[2])
    try:
        for k in range(3):
            out = dev.step(k, seq[k])
            ref = orc.step(k, seq[k])
        p = tmp_path / "density-checkpoint"
        dev.write_checkpoint(p, out, vol)
        assert p.read_text() == orc.checkpoint_text(ref, vol)
        # DIIS steps, checkpoint, restart into a fresh mixer: same continuation
        for k in range(3, 6):
            out = dev.step(k, seq[k])
        dev.write_checkpoint(p, out, vol)
        again = pkg.DensityMixer(n, **PARAMS)
        try:
            rho_file = again.read_checkpoint(p)
            assert np.array_equal(rho_file, np.array([float("%.16g" % v) for v in out * vol]))
            assert again.state()[:2] == (5, 4)
            # the restarted mixer's rho_old is the file density (as checkpointInput leaves it);
            # give the original the same rho_old by reading the file too, then both continue alike
            dev.read_checkpoint(p)
            for k in range(6, 9):
                a = dev.step(k, seq[k])
                b = again.step(k, seq[k])
                assert np.array_equal(a, b), k
        finally:
            again.close()
    finally:
        dev.close()


def test_device_pointers(pkg):
    import torch
    n = 5000
    seq = _densities(n, 5)
    dev = pkg.DensityMixer(n, **PARAMS)
    host = pkg.DensityMixer(n, **PARAMS)
    try:
        out_d = torch.zeros(n, dtype=torch.float64, device="cuda")
        for k, rc in enumerate(seq):
            rc_d = torch.from_numpy(rc).cuda()
            dev.step(k, rc_d.data_ptr(), out_d.data_ptr())
            b = host.step(k, rc)
            if k > 0:
                assert np.array_equal(out_d.cpu().numpy(), b), k
    finally:
        dev.close()
        host.close()
