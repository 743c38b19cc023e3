"""The equilibration test of runMCMC's automatic equilibration
(NewtonSteps.py:395-442): the oracle's restatement of scipy.stats.spearmanr
(scipy 1.18.1: average ranks, Pearson r of the ranks, two-sided Student-t
p-value) against scipy itself, the critical |r| that stands for p > 0.02,
and the device-side equilibration loop of NewtonSteps (ranks and their
correlations on the device) against the host loop, on the CPU test device:
same checkpoints, same verdicts, same correlations."""
import numpy as np
import pytest
from scipy.stats import rankdata, spearmanr

from oracle import oracle


def _energy_sets(seed):
    rng = np.random.default_rng(seed)
    n = 4096
    base = rng.normal(0, 3, n).astype("<f4")
    out = []
    for lag_corr in (0.9, 0.3, 0.05, 0.0, -0.02):
        nxt = (lag_corr * base + np.sqrt(1 - lag_corr ** 2) * rng.normal(0, 3, n)).astype("<f4")
        out.append((base, nxt))
    tied = np.round(base).astype("<f4")
    out.append((tied, np.round(out[2][1]).astype("<f4")))
    z = base.copy()
    z[:100] = 0.0
    z[100:200] = -0.0  # equal to +0 for ranking
    out.append((z, out[3][1]))
    return out


def test_oracle_spearman_equals_scipy():
    for seed in range(3):
        for a, b in _energy_sets(seed):
            np.testing.assert_array_equal(oracle.rank_average(a), rankdata(a))
            r, p = oracle.spearman(a, b)
            rs, ps = spearmanr(a, b)
            assert abs(r - rs) < 1e-12 and abs(p - ps) <= 1e-9 * ps + 1e-300, (r, rs, p, ps)


def test_constant_energies_have_no_correlation():
    a = np.full(512, 2.5, "<f4")
    b = np.random.default_rng(1).normal(size=512).astype("<f4")
    r, p = oracle.spearman(a, b)
    assert np.isnan(r) and np.isnan(p)
    assert not (p > 0.02)  # the reference's test then continues


@pytest.mark.parametrize("n", [100, 4096, 1 << 20])
def test_rcrit_is_the_p_threshold(n):
    rc = oracle.spearman_rcrit(n)
    from mi3gpu_b200.NewtonSteps import _spearman_p
    for f in (0.5, 0.9, 0.999, 1.001, 1.1, 2.0):
        r = rc * f
        assert (abs(r) < rc) == (_spearman_p(r, n) > 0.02), (n, f)
        assert (abs(-r) < rc) == (_spearman_p(-r, n) > 0.02)


def test_device_equilibration_loop_matches_host_loop(monkeypatch):
    """runMCMC with equiltime 'auto' on one device: the device path (ranks
    on the device) takes the same sampler calls and reports the same
    correlations as the host path (energies collected, scipy.spearmanr)."""
    from mi3gpu_b200 import GPU_node
    from mi3gpu_b200 import NewtonSteps as NS
    from mi3gpu_b200.potts import synthetic_ground_truth
    from tests.fake_device import FakeMCMCGPU
    L, q, N = 8, 3, 512
    J = synthetic_ground_truth(L, q, seed=9, contact_sigma=0.8)
    out = {}
    for path in ("device", "host"):
        g = FakeMCMCGPU(L, q, N, seed=4)
        gpus = GPU_node([g])
        gpus.initMCMC(2 * L)
        gpus.setSeqs('main', np.zeros((N, L), '<u1'))
        if path == "host":
            monkeypatch.setattr(GPU_node, "deviceRanks", lambda self: False)
        p = NS.Param(equiltime='auto', min_equil=16, max_equil=4096, trackequil=0, outdir=None, beta=None,
                     device_resident=False, nsteps=2 * L)
        logs = []
        bim, bic, es, e_rho, _, step = NS.runMCMC(gpus, J, 'run_0', p, logs.append)
        out[path] = (step, e_rho, [x for x in logs if 'Step' in x])
        monkeypatch.undo()
    (sd, rd, ld), (sh, rh, lh) = out["device"], out["host"]
    assert sd == sh and len(ld) == len(lh)
    np.testing.assert_allclose([r for r, _ in rd], [r for r, _ in rh], rtol=0, atol=1e-12)
    np.testing.assert_allclose([p for _, p in rd], [p for _, p in rh], rtol=1e-9, atol=1e-300)
    assert [x.split('r=')[-1] for x in ld] == [x.split('r=')[-1] for x in lh]
