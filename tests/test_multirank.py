"""Multi-rank host path on CPU (gloo, world_size 2): walkers shard across
ranks with disjoint RNG spans, and the only Newton-phase exchanges -- the
sum of bimarginal counts / weighted bimarginals, the min of dE and the FP64
weight sums -- reproduce the single-process results."""
import os
import socket

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
