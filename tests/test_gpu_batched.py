"""Batched rounds (one CUDA-graph launch per round for many problems)
against the host-driven loop: same seeds, same kernels, same results."""
import numpy as np
import pytest

from mi3gpu_b200 import potts
from mi3gpu_b200.mcmcGPU import MCMCGPU

pytestmark = pytest.mark.gpu


def _target(L, q, seed):
    from mi3gpu_b200.inference import make_target
    return make_target(L, q, 4096, seed=seed, sweeps=64)[0]


def test_batched_graph_matches_host_loop(cuda, monkeypatch):
    """Two problems of different shapes in one graph: J after three rounds,
    the SSR of every round and the Newton step counts equal those of
    inference.infer (device-resident, walkers carried over) bit for bit;
    the consensus energies are switched off in the host loop, since the
    graph uses the direct energy kernel."""
    from mi3gpu_b200.batched import BatchedRounds, Problem
    from mi3gpu_b200.inference import infer
    monkeypatch.setattr(MCMCGPU, 'CONS_ENERGY_MAX_ACTIVE', -1.0)
    shapes = [(20, 4, 2048, 11), (13, 21, 2048, 12)]
    targets = [_target(L, q, s) for L, q, N, s in shapes]
    kw = dict(gamma=4e-3, damping=1e-2)
    probs = [Problem(t, L, q, N, seed=s) for t, (L, q, N, s) in zip(targets, shapes)]
    br = BatchedRounds(probs, lJ=1e-3, newton_max=256, sweeps=8, sweeps_first=32, reseed='none', **kw)
    for _ in range(3):
        br.run_round()
    for pr, t, (L, q, N, s) in zip(probs, targets, shapes):
        res = infer(t, L, q, N, 3, sweeps=8, sweeps_first=32, newtonsteps=256, reg=('l1z', (1e-3,)), seed=s,
                    log=lambda *a: None, reseed='none', device_resident=True, **kw)
        assert [h['ssr'] for h in pr.history] == [h['ssr'] for h in res['history']]
        assert [h['newton_steps'] for h in pr.history] == [h['newton_steps'] for h in res['history']]
        Jb = pr.gpu.bufs['J'].cpu().numpy()[:L * (L - 1) // 2 * q * q].reshape(-1, q * q)
        np.testing.assert_array_equal(Jb, res['J'])
    br.close()


def test_batched_tuned_many_shapes(cuda, tmp_path):
    """Five problems (q in {4, 8, 21}, uneven L and walkers) with autotuned
    kernel schedules: every round finishes with finite statistics, the
    Newton loops stop by the Neff rule, and the SSR falls."""
    from mi3gpu_b200.autotune import Autotuner
    from mi3gpu_b200.batched import BatchedRounds, random_problems
    probs = random_problems(5, seed=77, L_range=(12, 40), walkers_log2=(11, 13), msa=2048)
    br = BatchedRounds(probs, gamma=4e-3, damping=1e-2, lJ=1e-3, newton_max=256, sweeps=8, sweeps_first=64,
                       tuner=Autotuner(tmp_path / "tune.json"))
    recs = [br.run_round() for _ in range(4)]
    for k, pr in enumerate(probs):
        ssr = [h['ssr'] for h in pr.history]
        assert all(np.isfinite(ssr)) and all(h['newton_steps'] >= 0 for h in pr.history)
        assert ssr[-1] < ssr[0], (k, ssr)
    assert all(r['gpu_ms'] > 0 for r in recs)
    br.close()


def test_batched_graph_equilibrates_like_host_loop(cuda, monkeypatch):
    """Equilibration inside the graph (IF node per checkpoint, rank test on
    the device): for two problems in one graph, the sampler calls each
    round settles on, its SSR, the Newton step counts and J after three
    rounds equal those of inference.infer with equiltime='auto' (the
    host-driven loop running the same rank test on the device)."""
    from mi3gpu_b200.batched import BatchedRounds, Problem
    from mi3gpu_b200.inference import infer
    monkeypatch.setattr(MCMCGPU, 'CONS_ENERGY_MAX_ACTIVE', -1.0)
    shapes = [(20, 4, 2048, 11), (13, 21, 2048, 12)]
    targets = [_target(L, q, s) for L, q, N, s in shapes]
    kw = dict(gamma=4e-3, damping=1e-2)
    eq = dict(min_equil=64, max_equil=512)
    probs = [Problem(t, L, q, N, seed=s) for t, (L, q, N, s) in zip(targets, shapes)]
    br = BatchedRounds(probs, lJ=1e-3, newton_max=256, reseed='none', equil=eq, **kw)
    for _ in range(3):
        br.run_round()
    for pr, t, (L, q, N, s) in zip(probs, targets, shapes):
        res = infer(t, L, q, N, 3, equiltime='auto', nsteps=8 * L, newtonsteps=256, reg=('l1z', (1e-3,)), seed=s,
                    log=lambda *a: None, reseed='none', device_resident=True, **eq, **kw)
        assert [h['mcmc_calls'] for h in pr.history] == [h['equil_calls'] for h in res['history']]
        assert all(64 <= h['mcmc_calls'] <= 512 for h in pr.history)
        assert [h['ssr'] for h in pr.history] == [h['ssr'] for h in res['history']]
        assert [h['newton_steps'] for h in pr.history] == [h['newton_steps'] for h in res['history']]
        Jb = pr.gpu.bufs['J'].cpu().numpy()[:L * (L - 1) // 2 * q * q].reshape(-1, q * q)
        np.testing.assert_array_equal(Jb, res['J'])
    br.close()
