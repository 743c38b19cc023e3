"""The MCMCGPU runtime (the reference's per-device class) on the GPU against
the same calls on the CPU fake device (tests/fake_device.py, built on the
oracle): same seeds, same position lists, same results."""
import numpy as np
import pytest

from mi3gpu_b200 import GPU_node, MCMCGPU, NewtonSteps, potts
from tests.fake_device import FakeMCMCGPU

pytestmark = pytest.mark.gpu


def _pair(L, q, N, seed=11):
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, seed)
    f = FakeMCMCGPU(L, q, N, seed)
    return GPU_node([g]), GPU_node([f]), g, f


def test_runtime_sampling_matches_fake_device(cuda):
    L, q, N = 30, 6, 1024
    gpus, fakes, g, f = _pair(L, q, N)
    rng = np.random.default_rng(1)
    J = potts.synthetic_ground_truth(L, q, seed=3, contact_sigma=0.4)
    seqs = rng.integers(0, q, size=(N, L)).astype('<u1')
    for node in (gpus, fakes):
        node.initMCMC(2 * L)
        node.initJstep()
        node.setSeqs('main', seqs)
        node.setBuf('J', J)
        for _ in range(3):
            node.runMCMC()
    np.testing.assert_array_equal(gpus.collect('seq main'), fakes.collect('seq main'))
    np.testing.assert_array_equal(g.getBuf('rngstates').read().view(np.uint32).reshape(N, 4),
                                  f.bufs['rngstates'])
    for node in (gpus, fakes):
        node.calcEnergies('main')
        node.calcBicounts('main')
    np.testing.assert_array_equal(gpus.collect('bicount'), fakes.collect('bicount'))
    e, ef = gpus.collect('E main'), fakes.collect('E main')
    assert (np.abs(e - ef) / np.maximum(1, np.abs(ef))).max() <= 1e-5
    Ju = g.getBuf('Junpacked').read()
    assert Ju.shape == (L * L, q * q)
    from mi3gpu_b200.mcmcGPU import unpackJ_CPU
    full = unpackJ_CPU(J)
    off = ~np.eye(L, dtype=bool).reshape(-1)
    np.testing.assert_array_equal(Ju[off], full[off])


def test_runtime_gen_indep_and_newton(cuda):
    L, q, N = 24, 4, 2048
    gpus, fakes, g, f = _pair(L, q, N, seed=5)
    truth = potts.synthetic_ground_truth(L, q, seed=7, contact_sigma=0.5)
    uni = np.random.default_rng(2).dirichlet(np.ones(q), size=L)
    for node in (gpus, fakes):
        node.initMCMC(4 * L)
        node.initJstep()
        node.prepare_indep(uni)
        node.gen_indep('main')
    np.testing.assert_array_equal(gpus.collect('seq main'), fakes.collect('seq main'))
    for node in (gpus, fakes):
        node.setBuf('J', truth)
        for _ in range(4):
            node.runMCMC()
    np.testing.assert_array_equal(gpus.collect('seq main'), fakes.collect('seq main'))
    gpus.calcBicounts('main')
    f0 = gpus.collect('bicount') / N
    target = potts.mutation_pc(f0 * np.exp(np.random.default_rng(3).normal(0, 0.2, f0.shape)), N).astype('<f4')
    target /= target.sum(axis=1, keepdims=True)
    res = []
    for node in (gpus, fakes):
        node.setBuf('bi target', target)
        p = NewtonSteps.Param(bimarg=target, gamma0=4e-3, newtonSteps=12, pcdamping=1e-2, fracNeff=0.5,
                              nwalkers=N, reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep='all')
        res.append(NewtonSteps.iterNewton(p, f0, node, lambda *a: None))
    (s1, J1, b1), (s2, J2, b2) = res
    assert s1 == s2 == 11
    # float32 energies of dJ (device: exact sum rounded once; fake: double)
    # feed exp(): trajectories agree to float precision
    np.testing.assert_allclose(J1, J2, rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(b1, b2, rtol=1e-4, atol=1e-6)


def test_runtime_regularizers_dispatch(cuda):
    L, q, N = 9, 4, 512
    gpus, fakes, g, f = _pair(L, q, N)
    gpus.initMCMC(L)
    gpus.initJstep()
    rng = np.random.default_rng(4)
    n = (L * (L - 1) // 2, q * q)
    gpus.setBuf('bi', rng.dirichlet(np.ones(q * q), size=n[0]).astype('<f4'))
    gpus.setBuf('J', rng.normal(0, 0.1, size=n).astype('<f4'))
    gpus.setBuf('Xlambdas', np.full(n[0], 0.05, '<f4'))
    for name, args in [('l1z', (0.01,)), ('l2z', (0.01,)), ('SCADJ', (0.02, 4.0)), ('X', (0.05,)), ('Xij', ()),
                       ('SCADX', (2.0, 0.05, 4.0)), ('expX', (0.3,)), ('ddE', (0.01,)), ('SCADddE', (0.01, 0.02))]:
        gpus.setBuf('dJ', rng.normal(0, 0.02, size=n).astype('<f4'))
        before = gpus.collect('dJ')[0] if isinstance(gpus.collect('dJ'), list) else gpus.collect('dJ')
        gpus.reg(name, (4e-3, 1e-2) + args)
        after = gpus.collect('dJ')
        assert np.isfinite(after).all() and not np.array_equal(after, before), name


def test_device_resident_rounds_on_gpu(cuda):
    """Rounds with J kept on the device (FP64 gauge and statistics there)
    follow the reference-shaped host loop: same Newton step counts, SSR per
    round within float rounding of the gauge, and J after the last round."""
    from mi3gpu_b200.inference import infer
    L, q, N = 20, 4, 4096
    truth = potts.synthetic_ground_truth(L, q, seed=21, contact_sigma=0.5)
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 5)
    node = GPU_node([g])
    node.initMCMC(4 * L)
    node.setBuf('J', truth)
    node.setSeqs('main', np.zeros((N, L), '<u1'))
    for _ in range(40):
        node.runMCMC()
    node.calcBicounts('main')
    target = potts.mutation_pc(node.collect('bicount') / N, N).astype('<f4')
    res = {}
    for dev in (False, True):
        logs = []
        res[dev] = infer(target, L, q, N, 3, sweeps=32, newtonsteps=64, gamma=4e-3, damping=1e-2,
                         reg=('l1z', (1e-3,)), seed=3, log=logs.append, reseed='none', device_resident=dev)
    hh, hd = res[False]['history'], res[True]['history']
    assert [h['newton_steps'] for h in hh] == [h['newton_steps'] for h in hd]
    np.testing.assert_allclose([h['ssr'] for h in hd], [h['ssr'] for h in hh], rtol=1e-3)
    np.testing.assert_allclose(res[True]['J'], res[False]['J'], rtol=1e-3, atol=1e-5)


def test_sampler_plans_same_trajectory_and_autotuner(cuda, tmp_path):
    """Every plan of the sampler -- the skewed-lane kernel's and every tile
    plan of the row-streaming kernel -- gives the same walkers and RNG states
    (the plan changes only the schedule); the autotuner picks one of them,
    caches it and installs it on the device object."""
    import torch
    from mi3gpu_b200 import _lib
    from mi3gpu_b200.autotune import Autotuner, sampler_plans
    for L, q, N in [(37, 21, 1024), (48, 4, 2048)]:
        g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 3)
        node = GPU_node([g])
        node.initMCMC(2 * L)
        node.setBuf('J', potts.synthetic_ground_truth(L, q, seed=L, contact_sigma=0.4))
        node.setSeqs('main', np.random.default_rng(L).integers(0, q, size=(N, L)).astype('<u1'))
        g.unpackJ(kind='rows')
        g.unpackJ(kind='tiles')
        pos = torch.from_numpy(np.random.default_rng(q).integers(0, L, size=3 * L).astype(np.int32)).to(g.device)
        seq0, rng0 = g.bufs['seq main'].clone(), g.bufs['rngstates'].clone()
        outs = []
        for plan in [(0, 0, 0)] + sampler_plans(L, q, N):
            seq, rng = seq0.clone(), rng0.clone()
            st = torch.zeros(1, dtype=torch.int32, device=g.device)
            g.sampler_call(0, pos.data_ptr(), 3 * L, seq.data_ptr(), rng.data_ptr(), st.data_ptr(),
                           g.stream.cuda_stream, plan=plan)
            g.stream.synchronize()
            assert int(st.item()) == 0
            outs.append((plan, seq, rng))
        for plan, seq, rng in outs[1:]:
            assert torch.equal(seq, outs[0][1]) and torch.equal(rng, outs[0][2]), plan
        cache = tmp_path / "tune.json"
        t = Autotuner(cache)
        chosen = t.tune(g)
        assert tuple(chosen["metropolis_plan"]) in set(sampler_plans(L, q, N))
        assert chosen["count_kernel"] in ("smem", "tc")
        # tuning left the chain where it was; a run with the tuned plan works
        assert torch.equal(g.bufs['seq main'], seq0)
        node.runMCMC()
        g.wait()
        assert Autotuner(cache).table == t.table


def test_checkpoint_resume_on_gpu_bit_identical(cuda, tmp_path):
    """On the device: three rounds straight equal two rounds + checkpoint +
    a third round continued from it in new device objects."""
    from mi3gpu_b200 import checkpoint
    L, q, N = 20, 4, 2048
    truth = potts.synthetic_ground_truth(L, q, seed=31, contact_sigma=0.5)

    def run(rounds, path, resume=None):
        g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 17)
        node = GPU_node([g])
        node.initMCMC(4 * L)
        node.initJstep()
        node.setBuf('J', truth)
        node.setSeqs('main', np.zeros((N, L), '<u1'))
        for _ in range(20):
            node.runMCMC()
        node.calcBicounts('main')
        target = potts.mutation_pc(node.collect('bicount') / N, N).astype('<f4')
        uni = potts.getUnimarg(target)
        p = NewtonSteps.Param()
        p.update(dict(bimarg=target, gamma0=4e-3, newtonSteps=64, pcdamping=1e-2, fracNeff=0.9, nwalkers=N,
                      reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep='all', L=L, q=q,
                      couplings=potts.independent_couplings(uni), nsteps=4 * L, equiltime=8, trackequil=0,
                      outdir=None, mcmcsteps=rounds, newton_delta=32, reseed='none', rngseed=5, unimarg=uni,
                      fused=True, init_indep=True, device_resident=True, checkpoint=str(path)))
        node.prepare_indep(uni)
        J = NewtonSteps.newtonMCMC(p, node, 0, 0, lambda *a: None,
                                   resume=checkpoint.load(resume) if resume else None)
        return J, [h['ssr'] for h in p.history]

    J3, s3 = run(3, tmp_path / "a.pkl")
    run(2, tmp_path / "b.pkl")
    J3b, s3b = run(3, tmp_path / "c.pkl", resume=tmp_path / "b.pkl")
    np.testing.assert_array_equal(J3b, J3)
    assert s3b == s3


def test_reference_setup_and_init_signatures(cuda):
    """Mi3.py's device set-up calls, with the reference's signatures:
    setup_GPU_context(scriptpath, scriptfile, param, log) and
    initGPU(devnum, cldat, device, nwalkers, param, log)."""
    from mi3gpu_b200 import initGPU, setup_GPU_context
    logs = []
    p = NewtonSteps.Param(L=12, q=4, gpuspec='0', wgsize=512, outdir=None, rngseed=3, profile=False, beta=None)
    cldat, devices, (info, buildlog) = setup_GPU_context(None, None, p, logs.append)
    assert len(devices) == 1 and "sm_100a" in info
    gpus = GPU_node([initGPU(i, cldat, d, 1024, p, logs.append) for i, d in enumerate(devices)])
    gpus.initMCMC(48)
    gpus.setBuf('J', potts.synthetic_ground_truth(12, 4, seed=1, contact_sigma=0.3))
    gpus.setSeqs('main', np.zeros((1024, 12), '<u1'))
    gpus.runMCMC()
    gpus.wait()
    assert gpus.collect('seq main').shape == (1024, 12)
    with pytest.raises(Exception):
        setup_GPU_context(None, None, NewtonSteps.Param(gpuspec='99'), logs.append)


def test_bounded_wait_gives_up_and_context_survives(cuda):
    """The device-side failure path, exercised without a fault: a wait on an
    mbarrier that nothing completes gives up after its limit (or as soon as
    the CTA's abort flag rises), writes MI3_STATUS_TIMEOUT_FULL, and the
    kernel returns; the device keeps working and MCMCGPU turns the status
    word into an exception."""
    import torch
    from mi3gpu_b200 import _lib
    dev = torch.device('cuda', 0)
    s = torch.cuda.current_stream(dev).cuda_stream
    for limit, abort in [(50_000_000, 0), (1_000_000_000, 20_000_000)]:
        st = torch.zeros(1, dtype=torch.int32, device=dev)
        waited = torch.zeros(1, dtype=torch.int64, device=dev)
        _lib.call('mi3_probe_bounded_wait', st.data_ptr(), limit, abort, waited.data_ptr(), s)
        torch.cuda.synchronize(dev)
        assert int(st.item()) == 1  # MI3_STATUS_TIMEOUT_FULL
        w = int(waited.item())
        if abort:
            assert abort <= w < limit // 2, w
        else:
            assert limit <= w < 20 * limit, w
    # the context still runs kernels
    L, q, N = 12, 4, 512
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 3)
    node = GPU_node([g])
    node.initMCMC(2 * L)
    node.setBuf('J', potts.synthetic_ground_truth(L, q, seed=2, contact_sigma=0.3))
    node.setSeqs('main', np.zeros((N, L), '<u1'))
    node.runMCMC()
    node.wait()
    # a status word set by a kernel surfaces as an exception on the host
    _lib.call('mi3_probe_bounded_wait', g._ptr('status'), 10_000_000, 0, waited.data_ptr(), g.stream.cuda_stream)
    with pytest.raises(RuntimeError):
        g.wait()
    with pytest.raises(_lib.Mi3Error):
        _lib.call('mi3_probe_bounded_wait', st.data_ptr(), 3_000_000_000, 0, waited.data_ptr(), s)


@pytest.mark.parametrize("q", [5, 21])
def test_large_buffer_kernels_match_main(cuda, q):
    """The large sequence buffer (mcmcGPU.py:284-303, 934-999): walkers
    stored from 'seq main' and from the host, read back truncated to the
    stored part; energies, counts (both count kernels at q=5), weights,
    weight statistics and weighted bimarginals over its stored columns
    equal the same calls over a main buffer holding the same walkers, bit
    for bit; restoreSeqs copies stored columns back into 'seq main'."""
    from oracle import oracle
    L, N = 37, 1024
    n_extra = 1024
    rng = np.random.default_rng(q)
    J = potts.synthetic_ground_truth(L, q, seed=8, contact_sigma=0.4)
    seqs = rng.integers(0, q, size=(N, L)).astype('<u1')
    extra = rng.integers(0, q, size=(n_extra, L)).astype('<u1')
    both = np.concatenate([seqs, extra])
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 3)
    g.initMCMC(L, 0, 2 ** 62)
    g.initJstep()
    g.setBuf('seq main', seqs)
    g.setBuf('J', J)
    g.initLargeBufs(N + n_extra + 512)  # 512 columns left unused
    g.storeSeqs()
    g.storeSeqs(extra)
    assert g.nstoredseqs == N + n_extra
    np.testing.assert_array_equal(g.getBuf('seq large').read(), both)
    assert g.getBuf('seq large', truncateLarge=False).read().shape == (N + n_extra + 512, L)
    # the same walkers in the main buffer of a second device object
    h = MCMCGPU((0, 0), L, q, N + n_extra, 512, None, 1024, 3)
    h.initMCMC(L, 0, 2 ** 62)
    h.initJstep()
    h.setBuf('seq main', both)
    h.setBuf('J', J)
    for dev, buf in ((g, 'large'), (h, 'main')):
        dev.calcEnergies(buf)
    Eg, Eh = g.getBuf('E large').read(), h.getBuf('E main').read()
    assert Eg.shape == (N + n_extra,)
    np.testing.assert_array_equal(Eg, Eh)
    for tensor in ([False, True] if q in MCMCGPU.TENSOR_COUNT_Q else [False]):
        g.calcBicounts('large', tensor=tensor)
        np.testing.assert_array_equal(g.getBuf('bicount').read(), oracle.bicounts(oracle.pack_seqs(both), L, q))
    g.bicounts_to_bimarg('large')
    h.calcBicounts('main')
    h.bicounts_to_bimarg('main')
    np.testing.assert_array_equal(g.getBuf('bi').read(), h.getBuf('bi').read())
    dE = rng.normal(0, 0.5, size=N + n_extra).astype('<f4')
    g.setBuf('E large', np.concatenate([dE, np.full(512, -50, '<f4')]))  # unused tail must not count
    g.nstoredseqs = N + n_extra
    h.setBuf('E main', dE)
    for dev, buf, ebuf in ((g, 'large', 'E large'), (h, 'main', 'E main')):
        dev.min_buf(ebuf)
        dev.dE_to_weights(buf, 0.25)
        dev.weight_statistics(buf)
        dev.updateConsensus(buf)
        dev.weightedMarg(buf)
    assert g.getBuf('minout').read()[0] == h.getBuf('minout').read()[0] == min(0.0, float(dE.min()))
    np.testing.assert_array_equal(g.getBuf('weights large').read(), h.getBuf('weights').read())
    np.testing.assert_array_equal(g.getBuf('weightstats64').read(), h.getBuf('weightstats64').read())
    np.testing.assert_array_equal(g.getBuf('bi').read(), h.getBuf('bi').read())
    g.restoreSeqs(offset=n_extra)
    np.testing.assert_array_equal(g.getBuf('seq main').read(), both[n_extra:n_extra + N])
    with pytest.raises(Exception, match="past end"):
        g.storeSeqs(extra[:600])


@pytest.mark.parametrize("device_resident", [False, True])
def test_head_gpu_newton_phase_equals_all(cuda, device_resident):
    """distribute_jstep='head_gpu' on one device: the Newton phase over the
    walkers copied into the large buffer takes the same steps to the same
    couplings, bit for bit, as 'all' over the main buffer."""
    L, q, N = 28, 5, 2048
    truth = potts.synthetic_ground_truth(L, q, seed=17, contact_sigma=0.5)
    seqs = np.random.default_rng(5).integers(0, q, size=(N, L)).astype('<u1')
    res = []
    for mode in ('all', 'head_gpu'):
        g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 9)
        node = GPU_node([g])
        node.initMCMC(4 * L)
        node.initJstep()
        node.setSeqs('main', seqs)
        node.setBuf('J', truth)
        for _ in range(3):
            node.runMCMC()
        node.calcBicounts('main')
        f0 = node.collect('bicount') / N
        target = potts.mutation_pc(f0 * np.exp(np.random.default_rng(3).normal(0, 0.2, f0.shape)),
                                   N).astype('<f4')
        target /= target.sum(axis=1, keepdims=True)
        node.setBuf('bi target', target)
        p = NewtonSteps.Param(bimarg=target, gamma0=4e-3, newtonSteps=16, pcdamping=1e-2, fracNeff=0.5,
                              nwalkers=N, reg='l1z', regarg=(1e-3,), beta=None, distribute_jstep=mode,
                              device_resident=device_resident)
        steps, Jt, bt = NewtonSteps.iterNewton(p, f0, node, lambda *a: None, fused=True)
        if device_resident:
            Jt, bt = g.getBuf('J').read(), g.getBuf('bi').read()
        res.append((steps, Jt, bt))
    assert res[0][0] == res[1][0] >= 1
    np.testing.assert_array_equal(res[0][1], res[1][1])
    np.testing.assert_array_equal(res[0][2], res[1][2])


def test_device_bimarginals_pass_the_reference_checks(cuda):
    """Bimarginals the device produces -- counted (bicounts_to_bimarg) and
    weighted then renormalised (weightedMarg + renormalize_bimarg) -- pass
    the reference's consistency checks (potts_common.py:50-76)."""
    L, q, N = 33, 21, 4096
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 5)
    node = GPU_node([g])
    node.initMCMC(2 * L)
    node.initJstep()
    node.setSeqs('main', np.random.default_rng(3).integers(0, q, size=(N, L)).astype('<u1'))
    node.setBuf('J', potts.synthetic_ground_truth(L, q, seed=4, contact_sigma=0.5))
    for _ in range(4):
        node.runMCMC()
    node.calcBicounts('main')
    node.bicounts_to_bimarg('main')
    potts.validate_bimarg(node.collect('bi'))
    g.setBuf('weights', np.random.default_rng(6).uniform(0.1, 3.0, size=N).astype('<f4'))
    node.weightedMarg('main')
    node.renormalize_bimarg()
    potts.validate_bimarg(node.collect('bi'))


def test_seed_snapshot_restores_walkers_on_device(cuda):
    """snapshotSeqs / restoreSnapshot (the seed MSA of reseed 'msa'): a
    device copy of the walkers, put back after sampling moved them."""
    L, q, N = 19, 21, 1024
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 2)
    node = GPU_node([g])
    node.initMCMC(2 * L)
    seed = potts.repeatseqs(np.random.default_rng(1).integers(0, q, size=(300, L)).astype('<u1'), N)
    node.setSeqs('main', seed)
    snap = node.snapshotSeqs()
    node.setBuf('J', potts.synthetic_ground_truth(L, q, seed=2, contact_sigma=0.5))
    node.runMCMC()
    assert not np.array_equal(node.collect('seq main'), seed)
    node.restoreSnapshot(snap)
    np.testing.assert_array_equal(node.collect('seq main'), seed)
