"""Multi-rank host path on CPU (gloo, world_size 2): walkers shard across
ranks with disjoint RNG spans, and the only Newton-phase exchanges -- the
sum of bimarginal counts / weighted bimarginals, the min of dE and the FP64
weight sums -- reproduce the single-process results."""
import os
import socket
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, L, q, n_per, out):
    import torch
    import torch.distributed as dist
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    rng = np.random.default_rng(0)
    seqs = rng.integers(0, q, size=(world * n_per, L)).astype("<u1")
    w = rng.uniform(0.2, 2.0, size=world * n_per).astype("<f4")
    dE = rng.normal(0, 1, size=world * n_per).astype("<f4")
    mine = slice(rank * n_per, (rank + 1) * n_per)
    mem = oracle.pack_seqs(seqs[mine])
    # RNG span of this rank (GPU_node.initMCMC with one device per rank)
    span = (2 ** 63) // world
    states = oracle.init_rng(n_per, rank * span, span // (2 * n_per))
    counts = torch.from_numpy(oracle.bicounts(mem, L, q).astype(np.int64))
    dist.all_reduce(counts)
    wm = torch.from_numpy(oracle.weighted_marg_f64(w[mine], mem, L, q))
    dist.all_reduce(wm)
    mn = torch.tensor([oracle.min_floats(dE[mine])], dtype=torch.float64)
    dist.all_reduce(mn, op=dist.ReduceOp.MIN)
    st = torch.from_numpy(oracle.weight_stats_f64(w[mine]))
    dist.all_reduce(st)
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put(dict(counts=counts.numpy(), wm=wm.numpy(), mn=float(mn.item()), st=st.numpy(),
                     tmax=float(t.item())))
    out.put(dict(rank=rank, first_state=states[0].copy(), last_state=states[-1].copy()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reductions_match_single_process():
    from oracle import oracle
    L, q, n_per, world = 12, 5, 256, 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, L, q, n_per, out)) for r in range(world)]
    for p in ps:
        p.start()
    res = [out.get(timeout=120) for _ in range(world + 1)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    red = next(r for r in res if "counts" in r)
    rng = np.random.default_rng(0)
    seqs = rng.integers(0, q, size=(world * n_per, L)).astype("<u1")
    w = rng.uniform(0.2, 2.0, size=world * n_per).astype("<f4")
    dE = rng.normal(0, 1, size=world * n_per).astype("<f4")
    mem = oracle.pack_seqs(seqs)
    np.testing.assert_array_equal(red["counts"], oracle.bicounts(mem, L, q))
    np.testing.assert_allclose(red["wm"], oracle.weighted_marg_f64(w, mem, L, q), rtol=1e-12)
    assert red["mn"] == oracle.min_floats(dE)
    np.testing.assert_allclose(red["st"], oracle.weight_stats_f64(w), rtol=1e-12)
    assert red["tmax"] == 2.0
    # rank r's walkers start at RNG distance r * 2^63 / world
    span = (2 ** 63) // world
    for r in (x for x in res if "rank" in x):
        expect = oracle.init_rng(1, r["rank"] * span, span // (2 * n_per))[0]
        np.testing.assert_array_equal(r["first_state"], expect)


def _newton_worker(rank, world, port, out, mode='all', device_resident=False):
    """iterNewton through RankNode over two FakeMCMCGPU halves of the
    walkers; rank 0 reports the result."""
    import torch.distributed as dist
    from mi3gpu_b200 import NewtonSteps, potts
    from mi3gpu_b200.distributed import RankNode
    from tests.fake_device import FakeMCMCGPU
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    L, q, N = 8, 3, 1024
    n_per = N // world
    J = potts.synthetic_ground_truth(L, q, seed=5, contact_sigma=0.4)
    seqs = np.random.default_rng(4).integers(0, q, size=(N, L)).astype('<u1')
    g = FakeMCMCGPU(L, q, n_per, seed=2 + rank)
    node = RankNode(g)
    node.initMCMC(4 * L)
    node.initJstep()
    node.setSeqs('main', seqs[rank * n_per:(rank + 1) * n_per])
    node.setBuf('J', J)
    node.calcBicounts('main')
    f0 = node.collect('bicount') / N
    target = potts.mutation_pc(f0 * np.exp(np.random.default_rng(3).normal(0, 0.2, f0.shape)), N).astype('<f4')
    target /= target.sum(axis=1, keepdims=True)
    node.setBuf('bi target', target)
    p = NewtonSteps.Param(bimarg=target, gamma0=4e-3, newtonSteps=12, pcdamping=1e-2, fracNeff=0.5,
                          nwalkers=N, reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep=mode,
                          device_resident=device_resident)
    steps, Jt, bt = NewtonSteps.iterNewton(p, f0, node, lambda *a: None)
    if device_resident:  # J += dJ in place, then shared from rank 0
        Jt, bt = g.bufs['J'].copy(), g.bufs['bi'].copy()
    out.put(dict(rank=rank, steps=steps, J=Jt, bi=bt, f0=f0, target=target))
    dist.barrier()
    dist.destroy_process_group()


def _newton_worker_head_gpu(rank, world, port, out):
    _newton_worker(rank, world, port, out, mode='head_gpu', device_resident=True)


def _guarded(fn, rank, world, port, out):
    """Report a worker's exception instead of leaving the parent waiting."""
    try:
        fn(rank, world, port, out)
    except BaseException as e:  # noqa: BLE001 - forwarded to the test
        out.put(dict(rank=rank, error=repr(e)))
        raise


def test_two_rank_newton_phase_matches_single_process():
    """The Newton phase with walkers split over two gloo ranks (bimarginals
    summed, min dE and FP64 weight sums reduced across ranks) takes the same
    steps and reaches the same couplings as one process holding all walkers;
    both ranks end with identical couplings."""
    from mi3gpu_b200 import GPU_node, NewtonSteps
    from tests.fake_device import FakeMCMCGPU
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_guarded, args=(_newton_worker, r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted([out.get(timeout=180) for _ in range(2)], key=lambda r: r["rank"])
    assert not any("error" in r for r in res), res
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    np.testing.assert_array_equal(res[0]["J"], res[1]["J"])
    assert res[0]["steps"] == res[1]["steps"]
    # one process with all walkers
    from mi3gpu_b200 import potts
    L, q, N = 8, 3, 1024
    J = potts.synthetic_ground_truth(L, q, seed=5, contact_sigma=0.4)
    seqs = np.random.default_rng(4).integers(0, q, size=(N, L)).astype('<u1')
    g = FakeMCMCGPU(L, q, N, seed=2)
    node = GPU_node([g])
    node.initMCMC(4 * L)
    node.initJstep()
    node.setSeqs('main', seqs)
    node.setBuf('J', J)
    node.calcBicounts('main')
    np.testing.assert_allclose(node.collect('bicount') / N, res[0]["f0"])
    node.setBuf('bi target', res[0]["target"])
    p = NewtonSteps.Param(bimarg=res[0]["target"], gamma0=4e-3, newtonSteps=12, pcdamping=1e-2, fracNeff=0.5,
                          nwalkers=N, reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep='all')
    steps, Jt, bt = NewtonSteps.iterNewton(p, res[0]["f0"], node, lambda *a: None)
    assert steps == res[0]["steps"]
    np.testing.assert_allclose(res[0]["J"], Jt, rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(res[0]["bi"], bt, rtol=1e-4, atol=1e-6)


def test_two_rank_head_gpu_newton_phase_equals_single_process():
    """distribute_jstep='head_gpu' over two gloo ranks: every rank gathers
    all walkers (one broadcast per rank) and runs the head device's Newton
    phase with no collective in the loop; the couplings, bimarginals and
    step count equal, bit for bit, those of one process holding all walkers,
    and rank 0's J is shared with rank 1."""
    from mi3gpu_b200 import GPU_node, NewtonSteps, potts
    from tests.fake_device import FakeMCMCGPU
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_guarded, args=(_newton_worker_head_gpu, r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted([out.get(timeout=180) for _ in range(2)], key=lambda r: r["rank"])
    assert not any("error" in r for r in res), res
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    np.testing.assert_array_equal(res[0]["J"], res[1]["J"])
    assert res[0]["steps"] == res[1]["steps"]
    L, q, N = 8, 3, 1024
    J = potts.synthetic_ground_truth(L, q, seed=5, contact_sigma=0.4)
    seqs = np.random.default_rng(4).integers(0, q, size=(N, L)).astype('<u1')
    g = FakeMCMCGPU(L, q, N, seed=2)
    node = GPU_node([g])
    node.initMCMC(4 * L)
    node.initJstep()
    node.setSeqs('main', seqs)
    node.setBuf('J', J)
    node.setBuf('bi target', res[0]["target"])
    p = NewtonSteps.Param(bimarg=res[0]["target"], gamma0=4e-3, newtonSteps=12, pcdamping=1e-2, fracNeff=0.5,
                          nwalkers=N, reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep='all')
    steps, Jt, bt = NewtonSteps.iterNewton(p, res[0]["f0"], node, lambda *a: None)
    assert steps == res[0]["steps"]
    np.testing.assert_array_equal(res[0]["J"], Jt)
    np.testing.assert_array_equal(res[0]["bi"], bt)


def _rounds_worker_files(rank, world, port, out):
    _rounds_worker(rank, world, port, out, files=True)


def _rounds_worker(rank, world, port, out, files=False):
    """Two device-resident rounds (sampling on each rank's own walkers,
    Newton phase reduced across ranks) through RankNode; with files, the
    run directories and per-rank checkpoints as well."""
    import torch.distributed as dist
    from mi3gpu_b200 import NewtonSteps, potts
    from mi3gpu_b200.distributed import RankNode
    from tests.fake_device import FakeMCMCGPU
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    L, q, n_per = 6, 3, 256
    truth = potts.synthetic_ground_truth(L, q, seed=9, contact_sigma=0.5)
    target = potts.mutation_pc(np.full((L * (L - 1) // 2, q * q), 1.0 / (q * q)) *
                               np.exp(np.random.default_rng(1).normal(0, 0.3, (L * (L - 1) // 2, q * q))),
                               1000).astype('<f4')
    target /= target.sum(axis=1, keepdims=True)
    g = FakeMCMCGPU(L, q, n_per, seed=4 + rank)
    node = RankNode(g)
    node.initMCMC(4 * L)
    node.initJstep()
    p = NewtonSteps.Param()
    p.update(dict(bimarg=target, gamma0=4e-3, newtonSteps=16, pcdamping=1e-2, fracNeff=0.9, nwalkers=node.nwalkers,
                  reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep='all', L=L, q=q,
                  couplings=np.zeros((L * (L - 1) // 2, q * q), '<f4'), nsteps=4 * L, equiltime=4, trackequil=0,
                  outdir=None, mcmcsteps=2, newton_delta=8, reseed='none', rngseed=3, init_indep=True,
                  device_resident=True, unimarg=potts.getUnimarg(target)))
    if files:
        d = Path(os.environ["MSA_TEST_DIR"])
        p.update(outdir=d / "out", checkpoint=d / "ck", alpha="ABC")
    node.prepare_indep(p.unimarg)
    J = NewtonSteps.newtonMCMC(p, node, 0, 0, lambda *a: None)
    res = dict(rank=rank, J=J, ssr=[h['ssr'] for h in p.history], steps=[h['newton_steps'] for h in p.history],
               N=node.nwalkers)
    if files:
        from mi3gpu_b200 import checkpoint
        st = checkpoint.load(checkpoint.rank_path(p.checkpoint, node))
        res['ck_walkers'] = st['devices'][0]['seq main']
        res['walkers'] = g.bufs['seq main'].copy()
    out.put(res)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_device_resident_rounds_agree():
    """Rounds over two ranks: each samples its own walkers (disjoint RNG
    spans), the Newton phase is reduced across ranks, and both ranks end
    every round with the same statistics and the same couplings."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_guarded, args=(_rounds_worker, r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted([out.get(timeout=180) for _ in range(2)], key=lambda r: r["rank"])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert not any("error" in r for r in res), res
    assert res[0]["N"] == res[1]["N"] == 512
    assert res[0]["ssr"] == res[1]["ssr"] and res[0]["steps"] == res[1]["steps"]
    assert all(np.isfinite(res[0]["ssr"]))
    np.testing.assert_array_equal(res[0]["J"], res[1]["J"])


def _msa_worker(rank, world, port, out):
    """RankNode's MSA files: writeSeqs gathers every rank's walkers and rank
    0 writes them in rank order; loadSeqs hands each rank its share."""
    import torch.distributed as dist
    from mi3gpu_b200.distributed import RankNode
    from tests.fake_device import FakeMCMCGPU
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    L, q, n_per = 7, 4, 512
    seqs = np.random.default_rng(3).integers(0, q, size=(world * n_per, L)).astype('<u1')
    g = FakeMCMCGPU(L, q, n_per, seed=1 + rank)
    node = RankNode(g)
    node.setSeqs('main', seqs[rank * n_per:(rank + 1) * n_per])
    path = Path(os.environ["MSA_TEST_DIR"]) / "walkers"
    node.writeSeqs(path, 'main', "ACGT", zipf=True)
    dist.barrier()
    g.bufs['seq main'][...] = 0
    node.loadSeqs(path, 'main', "ACGT")
    try:
        node.head_node
        refused = False
    except Exception:
        refused = True
    out.put(dict(rank=rank, mine=g.getBuf('seq main').read(), refused=refused))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_msa_files(tmp_path, monkeypatch):
    from mi3gpu_b200 import seqload
    monkeypatch.setenv("MSA_TEST_DIR", str(tmp_path))
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_guarded, args=(_msa_worker, r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted([out.get(timeout=180) for _ in range(2)], key=lambda r: r["rank"])
    assert not any("error" in r for r in res), res
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    seqs = np.random.default_rng(3).integers(0, 4, size=(1024, 7)).astype('<u1')
    np.testing.assert_array_equal(seqload.loadSeqs(tmp_path / "walkers", "ACGT")[0], seqs)
    for r in res:
        np.testing.assert_array_equal(r["mine"], seqs[r["rank"] * 512:(r["rank"] + 1) * 512])
        assert r["refused"]


def test_two_rank_rounds_write_run_directories_once_and_checkpoint_per_rank(tmp_path, monkeypatch):
    """With outdir and checkpoints over two ranks: the run directories hold
    the reference's files (written by rank 0; the walker file gathers both
    ranks' walkers in rank order), and each rank checkpoints its own
    walkers in its own file."""
    from mi3gpu_b200 import seqload
    monkeypatch.setenv("MSA_TEST_DIR", str(tmp_path))
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_guarded, args=(_rounds_worker_files, r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted([out.get(timeout=180) for _ in range(2)], key=lambda r: r["rank"])
    assert not any("error" in r for r in res), res
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for run in ("run_0", "run_1"):
        for f in ("J.npy", "jstep", "newtonsteps", "info.txt", "seqs", "nsteps"):
            assert (tmp_path / "out" / run / f).exists(), (run, f)
    assert sorted(x.name for x in tmp_path.iterdir()) == ["ck.rank0", "ck.rank1", "out"]
    from oracle import oracle
    walkers = seqload.loadSeqs(tmp_path / "out" / "run_1" / "seqs", "ABC")[0]
    both = np.concatenate([oracle.unpack_seqs(r["walkers"], 6) for r in res])
    np.testing.assert_array_equal(walkers, both)
    for r in res:
        np.testing.assert_array_equal(r["ck_walkers"], r["walkers"])
    assert not np.array_equal(res[0]["walkers"], res[1]["walkers"])


def _failing_rank_worker(rank, world, port, out):
    """iterNewton over two ranks in which rank 1's device fails at its 4th
    weighted-bimarginal call (a fake of the failing call raising, as a CUDA
    error surfaces from MCMCGPU); the process group's timeout is short."""
    import datetime
    import torch.distributed as dist
    from mi3gpu_b200 import NewtonSteps, potts
    from mi3gpu_b200.distributed import RankNode
    from tests.fake_device import FakeMCMCGPU

    class FailingDevice(FakeMCMCGPU):
        calls = 0

        def weightedMarg(self, seqbufname='main'):
            FailingDevice.calls += 1
            if FailingDevice.calls == 4:
                raise RuntimeError("injected device failure on rank 1")
            return super().weightedMarg(seqbufname)

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    L, q, N = 8, 3, 1024
    n_per = N // world
    J = potts.synthetic_ground_truth(L, q, seed=5, contact_sigma=0.4)
    seqs = np.random.default_rng(4).integers(0, q, size=(N, L)).astype('<u1')
    g = (FailingDevice if rank == 1 else FakeMCMCGPU)(L, q, n_per, seed=2 + rank)
    node = RankNode(g)
    node.initMCMC(4 * L)
    node.initJstep()
    node.setSeqs('main', seqs[rank * n_per:(rank + 1) * n_per])
    node.setBuf('J', J)
    node.calcBicounts('main')
    f0 = node.collect('bicount') / N
    target = potts.mutation_pc(f0 * np.exp(np.random.default_rng(3).normal(0, 0.2, f0.shape)), N).astype('<f4')
    target /= target.sum(axis=1, keepdims=True)
    node.setBuf('bi target', target)
    p = NewtonSteps.Param(bimarg=target, gamma0=4e-3, newtonSteps=12, pcdamping=1e-2, fracNeff=0.5,
                          nwalkers=N, reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep='all')
    NewtonSteps.iterNewton(p, f0, node, lambda *a: None)
    out.put(dict(rank=rank, finished=True))


def test_two_rank_failure_ends_every_rank_with_an_error():
    """A rank whose device call fails mid Newton phase raises; the other
    rank, blocked in the next collective, ends with an error from the
    process group instead of waiting for good (the reference aborts every
    MPI rank when one exits, Mi3.py:249-258).  No GPU is involved."""
    import time
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    t0 = time.time()
    ps = [ctx.Process(target=_guarded, args=(_failing_rank_worker, r, 2, port, out)) for r in range(2)]
    for p in ps:
        p.start()
    try:
        res = sorted([out.get(timeout=120) for _ in range(2)], key=lambda r: r["rank"])
    finally:
        for p in ps:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert "injected device failure" in res[1].get("error", ""), res
    assert "error" in res[0] and "finished" not in res[0], res
    assert all(p.exitcode != 0 for p in ps)
    assert time.time() - t0 < 120
