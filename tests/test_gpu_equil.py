"""GPU parity of the device-side equilibration test: average ranks bit for
bit against the oracle's restatement of scipy.stats.rankdata, the rank
correlation within 1e-12 of scipy.stats.spearmanr, the device verdict equal
to the reference's "p1 > 0.02 and p2 > 0.02", and runMCMC's automatic
equilibration (NewtonSteps.py:395-442) taking the same sampler calls with
the same correlations whether the test runs on the device or, as in the
reference, on the host."""
import numpy as np
import pytest
from scipy.stats import spearmanr

from oracle import oracle
from mi3gpu_b200 import GPU_node, MCMCGPU, _lib
from tests._util import dev, empty, host, stream

pytestmark = pytest.mark.gpu


def _ranks(x):
    n = x.shape[0]
    ws = empty((int(_lib.query("mi3_rank_workspace", n)) // 8 + 2,), np.int64)
    r = empty((n,), np.float32)
    dx = dev(x)
    _lib.call("mi3_rank_average", dx.data_ptr(), n, r.data_ptr(), ws.data_ptr(), ws.numel() * 8, stream())
    return r, host(r)


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 50, n).astype("<f4")
    yield x
    yield np.round(x / 10).astype("<f4")       # many ties
    z = x.copy()
    z[: n // 3] = 0.0
    z[n // 3: n // 2] = -0.0                  # -0 ties with +0
    yield z
    yield np.full(n, 7.0, "<f4")               # constant


@pytest.mark.parametrize("n", [1, 2, 3, 2047, 2048, 4097, 100003, 1 << 20])
def test_rank_average_bitexact(cuda, n):
    for x in _inputs(n, n):
        _, r = _ranks(x)
        np.testing.assert_array_equal(r, oracle.rank_average(x).astype("<f4"))


@pytest.mark.parametrize("n", [4096, 1 << 20])
def test_rank_corr_and_verdict_match_scipy(cuda, n):
    rng = np.random.default_rng(3)
    base = rng.normal(0, 3, n).astype("<f4")
    vecs = [base] + [(c * base + np.sqrt(1 - c * c) * rng.normal(0, 3, n)).astype("<f4")
                     for c in (0.5, 0.01, 0.0005, 0.0)]
    vecs.append(np.full(n, 1.0, "<f4"))
    ranks = [_ranks(v)[0] for v in vecs]
    ws = empty((int(_lib.query("mi3_rank_corr_workspace")) // 8 + 2,), np.float64)
    rc = oracle.spearman_rcrit(n)
    flag = empty((1,), np.int32)
    for i in range(1, len(vecs)):
        r1 = empty((1,), np.float64)
        r2 = empty((1,), np.float64)
        _lib.call("mi3_rank_corr", ranks[i].data_ptr(), ranks[0].data_ptr(), n, r1.data_ptr(), ws.data_ptr(),
                  ws.numel() * 8, stream())
        _lib.call("mi3_rank_corr", ranks[i].data_ptr(), ranks[i - 1].data_ptr(), n, r2.data_ptr(),
                  ws.data_ptr(), ws.numel() * 8, stream())
        _lib.call("mi3_equil_decide", r1.data_ptr(), r2.data_ptr(), rc, flag.data_ptr(), stream())
        a, b = float(host(r1)[0]), float(host(r2)[0])
        (ra, pa), (rb, pb) = spearmanr(vecs[i], vecs[0]), spearmanr(vecs[i], vecs[i - 1])
        if np.isnan(ra):
            assert np.isnan(a)
        else:
            assert abs(a - ra) < 1e-12, (a, ra)
        if np.isnan(rb):
            assert np.isnan(b)
        else:
            assert abs(b - rb) < 1e-12, (b, rb)
        assert int(host(flag)[0]) == int(pa > 0.02 and pb > 0.02), (i, pa, pb)


def test_runmcmc_auto_equilibration_device_equals_host(cuda, monkeypatch):
    from mi3gpu_b200 import NewtonSteps as NS
    from mi3gpu_b200.potts import synthetic_ground_truth
    L, q, N = 48, 4, 16384
    J = synthetic_ground_truth(L, q, seed=1000)
    out = {}
    for path in ("device", "host"):
        g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 8)
        gpus = GPU_node([g])
        gpus.initMCMC(4 * L)
        gpus.setSeqs('main', np.zeros((N, L), '<u1'))
        if path == "host":
            monkeypatch.setattr(GPU_node, "deviceRanks", lambda self: False)
        p = NS.Param(equiltime='auto', min_equil=32, max_equil=4096, trackequil=0, outdir=None, beta=None,
                     device_resident=False, nsteps=4 * L)
        logs = []
        _, _, es, e_rho, _, step = NS.runMCMC(gpus, J, 'run_0', p, logs.append)
        out[path] = (step, e_rho, [x for x in logs if 'Step' in x], es)
        monkeypatch.undo()
    (sd, rd, ld, ed), (sh, rh, lh, eh) = out["device"], out["host"]
    print("equilibrated after", sd, "sampler calls;", ld[-1])
    assert sd == sh and len(ld) == len(lh)
    np.testing.assert_array_equal(ed, eh)  # same trajectory
    np.testing.assert_allclose([r for r, _ in rd], [r for r, _ in rh], rtol=0, atol=1e-12)
    assert [x.split('r=')[-1] for x in ld] == [x.split('r=')[-1] for x in lh]
