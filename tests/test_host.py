"""Host-side logic without a GPU: sequence packing, the shared site list,
GPU_node fan-out/merge and the NewtonSteps loop, driven over a CPU fake
device (tests/fake_device.py)."""
import numpy as np
import pytest

from oracle import oracle
from mi3gpu_b200 import GPU_node, NewtonSteps, potts
from mi3gpu_b200.mcmcGPU import MCMCGPU, histogram_heuristic, wgsize_heuristic
from tests.fake_device import FakeMCMCGPU


def test_pack_unpack_match_oracle():
    rng = np.random.default_rng(0)
    for L in (1, 3, 4, 5, 48, 93):
        seqs = rng.integers(0, 21, size=(64, L)).astype('<u1')
        g = MCMCGPU.__new__(MCMCGPU)
        g.L, g.SWORDS, g.SBYTES = L, (L - 1) // 4 + 1, 4 * ((L - 1) // 4 + 1)
        mem = g.packSeqs_4(seqs)
        np.testing.assert_array_equal(mem, oracle.pack_seqs(seqs))
        np.testing.assert_array_equal(g.unpackSeqs_4(mem), seqs)


def test_heuristics_match_reference_values():
    assert histogram_heuristic(4) == (256, 512)
    assert histogram_heuristic(8) == (64, 512)
    assert histogram_heuristic(21) == (8, 128)
    assert wgsize_heuristic(21) == 512 and wgsize_heuristic(4) == 256


def test_position_list_refill_schedule():
    """A new block of 1024*nsteps sites is drawn on the first call and every
    1024 calls; all devices draw the same sequence (mcmcGPU.py:447-458)."""
    a = FakeMCMCGPU(10, 3, 512, seed=7)
    b = FakeMCMCGPU(10, 3, 512, seed=7)
    a.initMCMC(4, 0, 2 ** 62)
    b.initMCMC(4, 2 ** 62, 2 ** 62)
    offs = [a.updateRngPos() for _ in range(2050)]
    assert offs[0] == 0 and offs[1] == 4 and offs[1023] == 4092 and offs[1024] == 0
    for _ in range(2050):
        b.updateRngPos()
    np.testing.assert_array_equal(a.bufs['randpos'], b.bufs['randpos'])
    ref = np.random.RandomState(7)
    blocks = [ref.randint(0, 10, size=4096) for _ in range(3)]
    np.testing.assert_array_equal(a.bufs['randpos'], blocks[2])


def test_gpu_node_rng_spans_disjoint():
    gpus = GPU_node([FakeMCMCGPU(6, 3, 512, seed=1, gpunum=k) for k in range(3)])
    gpus.initMCMC(8)
    spans = []
    for g in gpus.gpus:
        for w in range(g.nwalkers):
            for v in range(2):
                start = g.rng_offset + (2 * w + v) * g.walker_span
                spans.append((start, start + g.walker_span))
    spans.sort()
    assert all(a[1] <= b[0] for a, b in zip(spans, spans[1:]))
    assert spans[-1][1] <= 2 ** 63


def test_merge_bimarg_multi_device_equals_pooled():
    rng = np.random.default_rng(2)
    L, q = 9, 4
    seqs = rng.integers(0, q, size=(3 * 512, L)).astype('<u1')
    gpus = GPU_node([FakeMCMCGPU(L, q, 512, seed=1, gpunum=k) for k in range(3)])
    gpus.setSeqs('main', seqs)
    w = rng.uniform(0.5, 1.5, size=3 * 512).astype('<f4')
    for k, g in enumerate(gpus.gpus):
        g.initJstep()
        g.bufs['weights'] = w[512 * k:512 * (k + 1)]
    gpus.weightedMarg('main')
    gpus.merge_bimarg()
    pooled = oracle.weighted_marg_f64(w, oracle.pack_seqs(seqs), L, q)
    pooled /= pooled.sum(axis=1, keepdims=True)
    for g in gpus.gpus:
        np.testing.assert_allclose(g.bufs['bi'], pooled, rtol=2e-6)
    gpus.calcBicounts('main')
    np.testing.assert_array_equal(gpus.collect('bicount'), oracle.bicounts(oracle.pack_seqs(seqs), L, q))


def _param(L, q, N, target, J, newtonSteps=20):
    p = NewtonSteps.Param()
    p.update(dict(bimarg=target, gamma0=4e-3, newtonSteps=newtonSteps, pcdamping=1e-2, fracNeff=0.9,
                  nwalkers=N, reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep='all', L=L, q=q,
                  couplings=J, nsteps=4 * L, equiltime=4, trackequil=0, outdir=None, mcmcsteps=2,
                  newton_delta=8, reseed='independent', rngseed=3))
    return p


def test_iterNewton_over_fake_device_moves_toward_target():
    L, q, N = 8, 3, 1024
    rng = np.random.default_rng(4)
    J = potts.synthetic_ground_truth(L, q, seed=5, contact_sigma=0.4)
    g = FakeMCMCGPU(L, q, N, seed=2)
    gpus = GPU_node([g])
    gpus.initMCMC(4 * L)
    gpus.initJstep()
    gpus.setSeqs('main', rng.integers(0, q, size=(N, L)).astype('<u1'))
    gpus.setBuf('J', J)
    gpus.calcBicounts('main')
    f0 = gpus.collect('bicount') / N
    target = potts.mutation_pc(np.clip(f0 * np.exp(rng.normal(0, 0.3, f0.shape)), 1e-6, None)
                               / np.sum(f0, axis=1, keepdims=True), N).astype('<f4')
    target /= target.sum(axis=1, keepdims=True)
    gpus.setBuf('bi target', target)
    logs = []
    p = _param(L, q, N, target, J)
    steps, trialJ, bim = NewtonSteps.iterNewton(p, f0, gpus, logs.append)
    assert steps >= 1
    # predicted bimarginals are closer to the target than the start
    assert potts.bimarg_stats(target, bim)[1] < potts.bimarg_stats(target, f0.astype('<f4'))[1]
    np.testing.assert_allclose(trialJ, g.bufs['J'], rtol=0, atol=0)
    # fused weights path gives the same result
    g2 = FakeMCMCGPU(L, q, N, seed=2)
    gpus2 = GPU_node([g2])
    gpus2.initMCMC(4 * L)
    gpus2.initJstep()
    g2.bufs['seq main'] = g.bufs['seq main'].copy()
    gpus2.setBuf('J', J)
    gpus2.setBuf('bi target', target)
    s2, J2, b2 = NewtonSteps.iterNewton(_param(L, q, N, target, J), f0, gpus2, lambda *a: None, fused=True)
    assert s2 == steps
    np.testing.assert_array_equal(J2, trialJ)


def _two_device_node(L, q, n_per, seqs, J, target):
    gs = [FakeMCMCGPU(L, q, n_per, seed=2 + k, gpunum=k) for k in range(2)]
    node = GPU_node(gs)
    node.initMCMC(4 * L)
    node.initJstep()
    node.setSeqs('main', seqs)
    node.setBuf('J', J)
    node.setBuf('bi target', target)
    return node


@pytest.mark.parametrize("device_resident", [False, True])
def test_head_gpu_newton_phase_equals_one_device_over_all_walkers(device_resident):
    """distribute_jstep='head_gpu' (NewtonSteps.py:181-195): two devices'
    walkers gathered, in device order, into the head device's large buffer;
    the Newton phase there takes the same steps to the same couplings, bit
    for bit, as one device holding all walkers in its main buffer, and the
    other device receives the new J."""
    L, q, n_per = 8, 3, 512
    N = 2 * n_per
    rng = np.random.default_rng(4)
    J = potts.synthetic_ground_truth(L, q, seed=5, contact_sigma=0.4)
    seqs = rng.integers(0, q, size=(N, L)).astype('<u1')
    f0 = oracle.bicounts(oracle.pack_seqs(seqs), L, q) / N
    target = potts.mutation_pc(f0 * np.exp(rng.normal(0, 0.2, f0.shape)), N).astype('<f4')
    target /= target.sum(axis=1, keepdims=True)
    node = _two_device_node(L, q, n_per, seqs, J, target)
    p = _param(L, q, N, target, J, newtonSteps=12)
    p.update(distribute_jstep='head_gpu', device_resident=device_resident)
    logs = []
    steps, Jt, bt = NewtonSteps.iterNewton(p, f0, node, logs.append)
    assert "Transferring sequences to gpu 0" in logs
    head = node.gpus[0]
    assert head.nstoredseqs == N
    np.testing.assert_array_equal(head.getBuf('seq large').read(), seqs)
    if device_resident:
        Jt, bt = head.bufs['J'].copy(), head.bufs['bi'].copy()
        np.testing.assert_array_equal(node.gpus[1].bufs['J'], Jt)

    one = GPU_node([FakeMCMCGPU(L, q, N, seed=2)])
    one.initMCMC(4 * L)
    one.initJstep()
    one.setSeqs('main', seqs)
    one.setBuf('J', J)
    one.setBuf('bi target', target)
    s1, J1, b1 = NewtonSteps.iterNewton(_param(L, q, N, target, J, newtonSteps=12), f0, one, lambda *a: None)
    assert steps == s1
    np.testing.assert_array_equal(Jt, J1)
    np.testing.assert_array_equal(bt, b1)


def test_head_node_newton_phase_equals_all_on_the_same_devices():
    """distribute_jstep='head_node' on one node: the walkers pass through
    the large buffers split as np.split would, which for one node is the
    same split as the main buffers, so the result equals 'all' bit for
    bit."""
    L, q, n_per = 6, 3, 512
    N = 2 * n_per
    rng = np.random.default_rng(7)
    J = potts.synthetic_ground_truth(L, q, seed=6, contact_sigma=0.4)
    seqs = rng.integers(0, q, size=(N, L)).astype('<u1')
    f0 = oracle.bicounts(oracle.pack_seqs(seqs), L, q) / N
    target = potts.mutation_pc(f0 * np.exp(rng.normal(0, 0.2, f0.shape)), N).astype('<f4')
    target /= target.sum(axis=1, keepdims=True)
    res = []
    for mode in ('all', 'head_node'):
        node = _two_device_node(L, q, n_per, seqs, J, target)
        p = _param(L, q, N, target, J, newtonSteps=10)
        p.update(distribute_jstep=mode)
        res.append(NewtonSteps.iterNewton(p, f0, node, lambda *a: None))
    assert res[0][0] == res[1][0]
    np.testing.assert_array_equal(res[0][1], res[1][1])
    np.testing.assert_array_equal(res[0][2], res[1][2])


def test_large_buffer_bookkeeping_and_errors():
    """storeSeqs appends after the stored part, clearLargeSeqs forgets it,
    overfilling raises (mcmcGPU.py:934-983); an unknown distribute_jstep
    is rejected."""
    L, q, n = 6, 3, 512
    g = FakeMCMCGPU(L, q, n, seed=1)
    node = GPU_node([g])
    rng = np.random.default_rng(2)
    seqs = rng.integers(0, q, size=(n, L)).astype('<u1')
    node.setSeqs('main', seqs)
    node.initLargeBufs(n + n // 2)
    assert node.nseq == {'main': n, 'large': n + n // 2}
    node.storeSeqs()
    extra = rng.integers(0, q, size=(n // 2, L)).astype('<u1')
    g.storeSeqs(extra)
    np.testing.assert_array_equal(g.getBuf('seq large').read(), np.concatenate([seqs, extra]))
    with pytest.raises(Exception, match="past end"):
        g.storeSeqs(extra[:1])
    node.clearLargeSeqs()
    assert g.nstoredseqs == 0
    p = _param(L, q, n, np.zeros((L * (L - 1) // 2, q * q), '<f4'), np.zeros((L * (L - 1) // 2, q * q), '<f4'))
    p.update(distribute_jstep='everywhere')
    node.initJstep()
    with pytest.raises(ValueError, match="distribute_jstep"):
        NewtonSteps.iterNewton(p, None, node, lambda *a: None)


def test_newtonMCMC_rounds_over_fake_device():
    L, q, N = 6, 3, 512
    J0 = np.zeros((L * (L - 1) // 2, q * q), '<f4')
    truth = potts.synthetic_ground_truth(L, q, seed=9, contact_sigma=0.5)
    g = FakeMCMCGPU(L, q, N, seed=4)
    gpus = GPU_node([g])
    gpus.initMCMC(4 * L)
    gpus.initJstep()
    gpus.setBuf('J', truth)
    gpus.setSeqs('main', np.zeros((N, L), '<u1'))
    for _ in range(30):
        gpus.runMCMC()
    gpus.calcBicounts('main')
    target = potts.mutation_pc(gpus.collect('bicount') / N, N).astype('<f4')
    p = _param(L, q, N, target, J0, newtonSteps=16)
    p.unimarg = potts.getUnimarg(target)
    gpus.prepare_indep(p.unimarg)
    logs = []
    J = NewtonSteps.newtonMCMC(p, gpus, 0, 0, logs.append)
    assert J.shape == J0.shape and np.isfinite(J).all() and np.abs(J).max() > 0
    assert len(p.history) == 2 and all(np.isfinite(h['ssr']) for h in p.history)


@pytest.mark.parametrize("device_resident", [False, True])
def test_run_directories_in_reference_format_and_finish(tmp_path, device_resident):
    """With outdir, every round writes what the reference writes
    (NewtonSteps.py:76-94, 610-687): J.npy, newtonsteps, jstep, info.txt,
    the walkers as a bzip2 MSA 'seqs' in the reference's text format,
    nsteps, predictedBimarg.npy and perturbedJ.npy, in run_X directories
    named as the reference names them; finish() then continues from the
    last one as --finish does (Mi3.py:373-402): its J, jstep and
    newtonsteps, and its walkers loaded from 'seqs'."""
    from mi3gpu_b200 import seqload
    L, q, N = 6, 3, 512
    J0 = np.zeros((L * (L - 1) // 2, q * q), '<f4')
    truth = potts.synthetic_ground_truth(L, q, seed=9, contact_sigma=0.5)

    def node():
        g = FakeMCMCGPU(L, q, N, seed=4)
        gpus = GPU_node([g])
        gpus.initMCMC(4 * L)
        gpus.initJstep()
        return g, gpus

    g, gpus = node()
    gpus.setBuf('J', truth)
    gpus.setSeqs('main', np.zeros((N, L), '<u1'))
    for _ in range(30):
        gpus.runMCMC()
    gpus.calcBicounts('main')
    target = potts.mutation_pc(gpus.collect('bicount') / N, N).astype('<f4')
    p = _param(L, q, N, target, J0, newtonSteps=16)
    p.update(unimarg=potts.getUnimarg(target), reseed='none', device_resident=device_resident, outdir=tmp_path,
             alpha="ABC", mcmcsteps=3)
    gpus.prepare_indep(p.unimarg)
    NewtonSteps.newtonMCMC(p, gpus, 0, 0, lambda *a: None)
    runs = sorted(x.name for x in tmp_path.glob('run_*'))
    assert runs == ['run_0', 'run_1', 'run_2']
    for r in runs:
        d = tmp_path / r
        for f in ('J.npy', 'newtonsteps', 'jstep', 'info.txt', 'seqs', 'nsteps', 'predictedBimarg.npy',
                  'perturbedJ.npy'):
            assert (d / f).exists(), (r, f)
        assert (d / 'seqs').read_bytes()[:3] == b"BZh"
    seqs, ids, _ = seqload.loadSeqs(tmp_path / 'run_2' / 'seqs', "ABC")
    assert seqs.shape == (N, L) and ids is None
    np.testing.assert_array_equal(seqs, oracle.unpack_seqs(g.bufs['seq main'], L))

    # finish: a fresh process continues from run_2 (rerunning it)
    g2, gpus2 = node()
    gpus2.prepare_indep(p.unimarg)
    p2 = _param(L, q, N, target, None, newtonSteps=1)
    p2.update(unimarg=p.unimarg, reseed='none', device_resident=device_resident, outdir=tmp_path, alpha="ABC",
              mcmcsteps=2)  # nothing left to run: only the state is restored
    logs = []
    J = NewtonSteps.finish(p2, gpus2, logs.append)
    assert "Continuing from" in logs[0] and logs[0].endswith('run_2')
    np.testing.assert_array_equal(p2.couplings, np.load(tmp_path / 'run_2' / 'J.npy'))
    assert p2.newtonSteps == int((tmp_path / 'run_2' / 'newtonsteps').read_text())
    np.testing.assert_array_equal(oracle.unpack_seqs(g2.bufs['seq main'], L), seqs)
    if not device_resident:
        np.testing.assert_array_equal(J, p2.couplings)
    jstep = (tmp_path / 'run_2' / 'jstep').read_text()
    p2.mcmcsteps = 3  # now run the last round again, from the same jstep
    NewtonSteps.finish(p2, gpus2, lambda *a: None)
    assert (tmp_path / 'run_2' / 'jstep').read_text() == jstep
    assert len(p2.history) == 1 and p2.history[0]['run'] == 'run_2'


def test_device_resident_rounds_match_host_rounds():
    """The device-resident round loop (J kept on the device, gauge and SSR
    computed there) follows the same trajectory as the reference-shaped
    host loop over the same device calls."""
    L, q, N = 6, 3, 512
    J0 = np.zeros((L * (L - 1) // 2, q * q), '<f4')
    truth = potts.synthetic_ground_truth(L, q, seed=9, contact_sigma=0.5)
    out = {}
    for dev in (False, True):
        g = FakeMCMCGPU(L, q, N, seed=4)
        gpus = GPU_node([g])
        gpus.initMCMC(4 * L)
        gpus.initJstep()
        gpus.setBuf('J', truth)
        gpus.setSeqs('main', np.zeros((N, L), '<u1'))
        for _ in range(30):
            gpus.runMCMC()
        gpus.calcBicounts('main')
        target = potts.mutation_pc(gpus.collect('bicount') / N, N).astype('<f4')
        p = _param(L, q, N, target, J0, newtonSteps=16)
        p.unimarg = potts.getUnimarg(target)
        p.reseed = 'none'
        p.device_resident = dev
        gpus.prepare_indep(p.unimarg)
        logs = []
        J = NewtonSteps.newtonMCMC(p, gpus, 0, 0, logs.append)
        out[dev] = (J, [h['ssr'] for h in p.history], [h['newton_steps'] for h in p.history])
    (Jh, sh, nh), (Jd, sd, nd) = out[False], out[True]
    assert nh == nd
    np.testing.assert_allclose(sd, sh, rtol=1e-5)
    np.testing.assert_allclose(Jd, Jh, rtol=1e-4, atol=1e-6)


def test_autotuner_cache_roundtrip_and_concurrent_writers(tmp_path):
    """The tuning cache survives a reload, tolerates a corrupt file and is
    written atomically through per-process temporaries."""
    import json
    import os
    from mi3gpu_b200.autotune import Autotuner
    path = tmp_path / "tune.json"
    a = Autotuner(path)
    a.table["dev/metropolis/L10/q4/N512"] = {"plan": [128, 12, 2]}
    a._save()
    assert Autotuner(path).table == a.table
    assert not any(p.name.endswith(".tmp") for p in tmp_path.iterdir())
    path.write_text("{not json")
    assert Autotuner(path).table == {}
    # two writers: each renames its own temporary, the file stays complete
    b, c = Autotuner(path), Autotuner(path)
    b.table["x"] = {"kernel": "smem"}
    c.table["y"] = {"kernel": "tc"}
    b._save()
    c._save()
    assert json.loads(path.read_text()) in (b.table, c.table)
    assert os.path.exists(path)


def _ckpt_run(tmp_path, rounds, dev, reseed, resume_from=None, ckpt_name="ck.pkl"):
    from mi3gpu_b200 import checkpoint
    L, q, N = 6, 3, 512
    truth = potts.synthetic_ground_truth(L, q, seed=9, contact_sigma=0.5)
    g = FakeMCMCGPU(L, q, N, seed=4)
    gpus = GPU_node([g])
    gpus.initMCMC(4 * L)
    gpus.initJstep()
    gpus.setBuf('J', truth)
    gpus.setSeqs('main', np.zeros((N, L), '<u1'))
    for _ in range(20):
        gpus.runMCMC()
    gpus.calcBicounts('main')
    target = potts.mutation_pc(gpus.collect('bicount') / N, N).astype('<f4')
    p = _param(L, q, N, target, np.zeros((L * (L - 1) // 2, q * q), '<f4'), newtonSteps=16)
    p.unimarg = potts.getUnimarg(target)
    p.reseed, p.device_resident, p.init_indep, p.mcmcsteps = reseed, dev, True, rounds
    p.checkpoint = str(tmp_path / ckpt_name)
    gpus.prepare_indep(p.unimarg)
    state = checkpoint.load(resume_from) if resume_from else None
    J = NewtonSteps.newtonMCMC(p, gpus, 0, 0, lambda *a: None, resume=state)
    return J, p.history


@pytest.mark.parametrize("dev", [False, True])
@pytest.mark.parametrize("reseed", ["none", "independent", "single_random"])
def test_checkpoint_resume_is_bit_identical(tmp_path, dev, reseed):
    """Three rounds straight vs two rounds, a checkpoint, and the third round
    continued from it in a fresh process state: the same couplings and the
    same history, bit for bit."""
    J3, h3 = _ckpt_run(tmp_path, 3, dev, reseed, ckpt_name="a.pkl")
    _ckpt_run(tmp_path, 2, dev, reseed, ckpt_name="b.pkl")
    J3b, h3b = _ckpt_run(tmp_path, 3, dev, reseed, resume_from=tmp_path / "b.pkl", ckpt_name="c.pkl")
    np.testing.assert_array_equal(J3b, J3)
    assert [h['ssr'] for h in h3b] == [h['ssr'] for h in h3]
    assert [h['newton_steps'] for h in h3b] == [h['newton_steps'] for h in h3]


def test_checkpoint_rejects_other_shapes(tmp_path):
    from mi3gpu_b200 import checkpoint
    _ckpt_run(tmp_path, 1, False, "none", ckpt_name="s.pkl")
    state = checkpoint.load(tmp_path / "s.pkl")
    state['shape'] = (7, 3, 512)
    with pytest.raises(ValueError):
        checkpoint.restore(state, GPU_node([FakeMCMCGPU(6, 3, 512, seed=1)]), NewtonSteps.Param(L=6, q=3),
                           np.random.RandomState(0))


def test_auto_equilibration_runs_and_stops():
    """equiltime='auto' (NewtonSteps.py:395-442): loops double until two
    successive energy snapshots are uncorrelated with the current one
    (Spearman p > 0.02) after min_equil calls, or max_equil is reached."""
    L, q, N = 6, 3, 512
    truth = potts.synthetic_ground_truth(L, q, seed=9, contact_sigma=0.5)
    g = FakeMCMCGPU(L, q, N, seed=4)
    gpus = GPU_node([g])
    gpus.initMCMC(2 * L)
    gpus.initJstep()
    p = _param(L, q, N, np.full((L * (L - 1) // 2, q * q), 1.0 / (q * q), '<f4'), truth, newtonSteps=4)
    p.equiltime, p.min_equil, p.max_equil = 'auto', 16, 64
    logs = []
    gpus.setSeqs('main', np.zeros((N, L), '<u1'))
    out = NewtonSteps.runMCMC(gpus, truth, 'run_00', p, logs.append)
    steps = out[5]
    assert 16 <= steps <= 64 + 32
    assert any("Equilibrated" in s or "Max Steps" in s for s in logs)
    assert out[3] is not None and len(out[3]) >= 2  # energy autocorrelations recorded


def _round_setup(L=6, q=3, N=512, seed=4):
    J0 = np.zeros((L * (L - 1) // 2, q * q), '<f4')
    truth = potts.synthetic_ground_truth(L, q, seed=9, contact_sigma=0.5)
    g = FakeMCMCGPU(L, q, N, seed=seed)
    gpus = GPU_node([g])
    gpus.initMCMC(4 * L)
    gpus.initJstep()
    gpus.setBuf('J', truth)
    gpus.setSeqs('main', np.zeros((N, L), '<u1'))
    for _ in range(30):
        gpus.runMCMC()
    gpus.calcBicounts('main')
    target = potts.mutation_pc(gpus.collect('bicount') / N, N).astype('<f4')
    p = _param(L, q, N, target, J0, newtonSteps=16)
    p.unimarg = potts.getUnimarg(target)
    gpus.prepare_indep(p.unimarg)
    return g, gpus, p


@pytest.mark.parametrize("device_resident", [False, True])
def test_preopt_runs_a_newton_phase_on_the_loaded_walkers(tmp_path, device_resident):
    """param.preopt (NewtonSteps.py:274-296, 716-720): one Newton phase on
    the walkers in the main buffers before round 0, written to 'preopt/',
    its steps counted in the jstep of run 0; reseed 'none' then keeps those
    walkers (no independent restart)."""
    g, gpus, p = _round_setup()
    loaded = g.bufs['seq main'].copy()
    p.update(preopt=True, reseed='none', init_indep=True, outdir=tmp_path, alpha="ABC", mcmcsteps=2,
             device_resident=device_resident)
    seen = []
    orig = NewtonSteps.MCMCstep

    def spy(runName, Jstep, couplings, param, gpus_, log):
        seen.append((runName, Jstep, g.bufs['seq main'].copy()))
        return orig(runName, Jstep, couplings, param, gpus_, log)
    NewtonSteps.MCMCstep = spy
    try:
        logs = []
        NewtonSteps.newtonMCMC(p, gpus, 0, 0, logs.append)
    finally:
        NewtonSteps.MCMCstep = orig
    assert "Pre-Optimization:" in logs
    for f in ('info.txt', 'seqs', 'predictedBimarg.npy', 'perturbedJ.npy'):
        assert (tmp_path / 'preopt' / f).exists(), f
    assert seen[0][1] > 0  # run 0 starts after the pre-optimisation's steps
    assert (tmp_path / 'run_0' / 'jstep').read_text() == str(seen[0][1])
    np.testing.assert_array_equal(seen[0][2], loaded)


def test_reseed_msa_restarts_every_round_from_the_seed_msa():
    """reseed 'msa' (NewtonSteps.py:761-762): every round starts from the
    seed sequences (uploaded once, restored on the device afterwards)."""
    L, q, N = 6, 3, 512
    g, gpus, p = _round_setup(L, q, N)
    seedmsa = potts.repeatseqs(np.random.default_rng(8).integers(0, q, size=(100, L)).astype('<u1'), N)
    assert seedmsa.shape == (N, L)
    p.update(reseed='msa', seedmsa=seedmsa, mcmcsteps=3)
    seen = []
    orig = NewtonSteps.MCMCstep

    def spy(runName, Jstep, couplings, param, gpus_, log):
        seen.append(g.bufs['seq main'].copy())
        return orig(runName, Jstep, couplings, param, gpus_, log)
    NewtonSteps.MCMCstep = spy
    try:
        NewtonSteps.newtonMCMC(p, gpus, 0, 0, lambda *a: None)
    finally:
        NewtonSteps.MCMCstep = orig
    assert len(seen) == 3
    for s in seen:
        np.testing.assert_array_equal(s, oracle.pack_seqs(seedmsa))
    assert not np.array_equal(g.bufs['seq main'], oracle.pack_seqs(seedmsa))  # the walkers did move


@pytest.mark.parametrize("max_equil", [16, 64, 100, 512, 32768])
def test_equil_schedule_matches_host_loop(max_equil):
    """The checkpoints the round graph captures (batched.equil_schedule) are
    those runMCMC's loop reaches: 8 calls, then 8, 16, 32, ... more, the
    last one the first at or past max_equil."""
    from mi3gpu_b200.batched import equil_schedule
    host, step, loops = [], 8, 8
    while True:
        host.append((step, loops))
        step += loops
        if step >= max_equil:
            break
        loops *= 2
    sched = equil_schedule(max_equil)
    assert sched == host
    c0, n = sched[-1]
    assert c0 + n >= max_equil and (len(sched) == 1 or sched[-2][0] + sched[-2][1] < max_equil)


@pytest.mark.parametrize("device_resident", [False, True])
@pytest.mark.filterwarnings("ignore::RuntimeWarning")  # numpy on the planted NaN / Inf
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_iterNewton_raises_divergence_on_non_finite_input(bad, device_resident):
    """A NaN or Inf in the target bimarginals makes dJ, and with it the
    reweighting weights exp(-E(dJ)), non-finite; the Newton phase stops with
    the reference's divergence error (NewtonSteps.py:257-260) instead of
    carrying the bad values into the next round.  (The check is on the
    weights, as in the reference: a bad J that never reaches dJ is not
    caught here either, nor a -Inf target, which only zeroes the weights of
    the sequences it touches; the model bimarginals are recounted from the
    walkers at the start of the phase.)"""
    L, q, N = 8, 3, 512
    rng = np.random.default_rng(7)
    J = potts.synthetic_ground_truth(L, q, seed=5, contact_sigma=0.4)
    g = FakeMCMCGPU(L, q, N, seed=2)
    gpus = GPU_node([g])
    gpus.initMCMC(4 * L)
    gpus.initJstep()
    gpus.setSeqs('main', rng.integers(0, q, size=(N, L)).astype('<u1'))
    gpus.setBuf('J', J)
    gpus.calcBicounts('main')
    f0 = gpus.collect('bicount') / N
    target = potts.mutation_pc(f0, N).astype('<f4')
    target /= target.sum(axis=1, keepdims=True)
    target = target.copy()
    target[2, 1] = bad
    gpus.setBuf('bi target', target)
    p = _param(L, q, N, target, J)
    p.device_resident = device_resident
    with pytest.raises(Exception, match="Divergence"):
        NewtonSteps.iterNewton(p, f0, gpus, lambda *a: None)


def test_batched_round_positions_and_rewind_follow_updateRngPos():
    """The batched rounds draw each round's site lists ahead of the graph
    launch (Problem.round_positions) and, after an in-graph equilibration
    that stopped early, rewind the stream to the calls actually made
    (position_state / set_position_state).  Host logic: the sites equal
    those MCMCGPU.updateRngPos hands to one sampler call after another,
    across a refill of the 1024-call block, and a rewind followed by fewer
    calls continues exactly where that many calls end."""
    from mi3gpu_b200.batched import Problem
    L, q, nsteps = 5, 3, 8

    def stub(seed):
        g = FakeMCMCGPU(L, q, 32, seed=seed)
        g.initMCMC(nsteps, 0, 2 ** 63)
        p = Problem.__new__(Problem)
        p.gpu, p.L, p.nsteps = g, L, nsteps
        return p

    ref = FakeMCMCGPU(L, q, 32, seed=11)
    ref.initMCMC(nsteps, 0, 2 ** 63)

    def ref_calls(n):
        out = []
        for _ in range(n):
            off = ref.updateRngPos()
            out.append(ref.bufs['randpos'][off:off + nsteps].copy())
        return np.concatenate(out)

    p = stub(11)
    np.testing.assert_array_equal(p.round_positions(1000), ref_calls(1000))
    st = p.position_state()
    ahead = p.round_positions(100)  # the longest schedule; call 1025 refills the block
    p.set_position_state(st)
    used = p.round_positions(40)  # the calls the equilibration actually made
    np.testing.assert_array_equal(used, ahead[:40 * nsteps])
    np.testing.assert_array_equal(used, ref_calls(40))
    np.testing.assert_array_equal(p.round_positions(70), ref_calls(70))  # 1110 calls in both


def test_untuned_sampler_plan_dispatch():
    """MCMCGPU.sampler_plan without tuning: the skewed-lane kernel from q=16
    with at least one CTA of 512 walkers per SM (512 walkers per CTA while
    L + 31 <= 288, else 256), the row kernel's built-in plan otherwise; an
    autotuned plan overrides both."""
    def plan(L, q, N, tuned=None):
        g = MCMCGPU.__new__(MCMCGPU)
        g.L, g.q, g.nseq = L, q, {'main': N}
        if tuned:
            g.metro_plan = tuned
        return g.sampler_plan()
    assert plan(232, 21, 1 << 20) == ('skew', 512)
    assert plan(257, 21, 1 << 20) == ('skew', 512)
    assert plan(258, 21, 1 << 20) == ('skew', 256)
    assert plan(512, 21, 1 << 21) == ('skew', 256)
    assert plan(546, 21, 1 << 21) == (0, 0, 0)  # L + 31 > 576
    assert plan(232, 8, 1 << 20) == (0, 0, 0)  # q < 16
    assert plan(232, 21, 148 * 512 - 32) == (0, 0, 0)  # fewer than one CTA per SM
    assert plan(232, 21, (1 << 20) + 16) == (0, 0, 0)  # not a multiple of 32
    assert plan(232, 21, 1 << 20, tuned=[512, 24, 3]) == (512, 24, 3)
    assert plan(99, 4, 1 << 18, tuned=['skew', 768]) == ('skew', 768)


@pytest.mark.parametrize("L,q,sigma", [(48, 4, 0.5), (60, 21, 0.5), (99, 4, 0.8)])
def test_synthetic_ground_truth_matches_its_definition(L, q, sigma):
    """The benchmark workloads' ground truth (fields N(0,1), couplings
    N(0, 0.05^2) plus N(0, sigma^2) on 3L distinct pairs with j - i >= 4,
    in the reference's fieldless-even gauge): reproducible from its seed,
    already in that gauge, and its zero-sum couplings single out exactly
    3L strong pairs, all at least 4 sites apart."""
    J = potts.synthetic_ground_truth(L, q, seed=1000 + L, contact_sigma=sigma)
    assert J.dtype == np.float32 and J.shape == (L * (L - 1) // 2, q * q)
    np.testing.assert_array_equal(J, potts.synthetic_ground_truth(L, q, seed=1000 + L, contact_sigma=sigma))
    zeros = np.zeros((L, q))
    h2, J2 = potts.fieldlessGaugeEven(zeros, J.astype(np.float64))
    np.testing.assert_allclose(J2, J, atol=1e-5)  # the gauge transform is a no-op on it
    _, J0 = potts.zeroGauge(zeros, J.astype(np.float64))
    norm = np.sqrt((J0 ** 2).sum(axis=1))
    # zero-sum projections: the 3L contacts (norm ~ sigma (q-1)) sit well
    # above the background (~ 0.05 (q-1)): a gap after the 3L-th largest
    order = np.argsort(norm)[::-1]
    assert norm[order[3 * L - 1]] > 1.8 * norm[order[3 * L]]
    strong = order[:3 * L]
    i, j = potts.pair_indices(L)
    assert (j[strong] - i[strong] >= 4).all()


def test_profile_log_lines_in_the_reference_format(tmp_path):
    """MCMCGPU.logProfile (mcmcGPU.py:224-237): completed commands become
    'EVT name start end bytes' lines in ns relative to the first profiled
    command, appended to the device's log file; commands still running stay
    queued for the next call.  CUDA events are replaced by stand-ins with
    the same query / elapsed_time interface."""
    from collections import deque

    class Evt:
        def __init__(self, ms, done=True):
            self.ms, self.done = ms, done

        def query(self):
            return self.done

        def elapsed_time(self, other):
            return other.ms - self.ms

    g = MCMCGPU.__new__(MCMCGPU)
    g.profile, g.logfn = True, str(tmp_path / "gpu-0.log")
    t0 = Evt(10.0)
    g._t0evt = t0
    running = Evt(10.5, done=False)
    g.events = deque([(t0, Evt(10.25), "mcmc", None), (Evt(10.25), Evt(10.3), "setBuf J", 4096),
                      (Evt(10.3), running, "energies", None)])
    assert g.logProfile() == ["EVT mcmc 0 250000 ", "EVT setBuf J 250000 300000 4096"]
    assert len(g.events) == 1
    running.done = True
    assert g.logProfile() == ["EVT energies 300000 500000 "]
    assert (tmp_path / "gpu-0.log").read_text().splitlines() == [
        "EVT mcmc 0 250000 ", "EVT setBuf J 250000 300000 4096", "EVT energies 300000 500000 "]
    g.profile = False
    assert g.logProfile() is None
