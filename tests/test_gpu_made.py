"""Learned proposal (MADE) kernels against a PyTorch-CPU oracle of the same
network (float64 autograd), and exactness of the independence MH step.  The
sampler tests here run the SIMT sampler (FP32 activations); the tensor-core
sampler has its own tests (test_gpu_made_tc.py)."""
import itertools

import numpy as np
import pytest
import torch

from oracle import oracle
from mi3gpu_b200 import GPU_node, MCMCGPU, potts
from mi3gpu_b200.learned import LearnedSampler, MadeProposal, made_masks

pytestmark = pytest.mark.gpu


def _cpu_made(made, seqs):
    """float64 CPU forward of the MADE with the device's bf16-rounded
    weights; returns (log q per sequence, parameter tensors with grads)."""
    P = {k: made.pc[k].detach().cpu().double().requires_grad_(True) for k in made.PARAMS}
    L, q = made.L, made.q
    X = torch.nn.functional.one_hot(torch.as_tensor(seqs, dtype=torch.long), q).reshape(len(seqs), L * q).double()
    a1 = torch.relu(X @ P["W1T"] + P["b1"])
    a2 = torch.relu(a1 @ P["W2"].T + P["b2"])
    logits = (a2 @ P["W3"].T + P["b3"]).reshape(len(seqs), L, q)
    lp = torch.log_softmax(logits, dim=-1)
    logq = lp.gather(2, torch.as_tensor(seqs, dtype=torch.long)[..., None])[..., 0].sum(1)
    return logq, P


def _made(L, q, H, seed=0, lr=1e-2):
    m = MadeProposal(L, q, H=H, device=0, seed=seed, lr=lr, sampler="simt", gemm="simt")
    rng = np.random.default_rng(seed + 7)
    for k in ("b1", "b2", "b3"):
        m.p[k].copy_(torch.as_tensor(rng.normal(0, 0.3, size=m.p[k].shape), dtype=torch.float32))
    m.round_params()
    return m


def _boltzmann(J, L, q):
    allseq = np.array(list(itertools.product(range(q), repeat=L)), dtype="<u1")
    E = oracle.energies_f64(J, oracle.pack_seqs(allseq), L, q)
    p = np.exp(-(E - E.min()))
    return allseq, p / p.sum()


def _zscores(seqs, p, L, q):
    idx = (seqs.astype(int) * q ** np.arange(L - 1, -1, -1)).sum(1)
    N = len(seqs)
    freq = np.bincount(idx, minlength=q ** L) / N
    return np.abs(freq - p) / np.sqrt(p * (1 - p) / N + 1e-12)


def test_masks_autoregressive():
    """Output site i is reachable only from input sites j < i."""
    L, q, H = 6, 3, 40
    mW1T, mW2, mW3, m1, m2 = made_masks(L, q, H)
    M = (mW3 @ mW2 @ mW1T.T > 0).reshape(L, q, L, q)  # output (i,a) <- input (j,b)
    for i in range(L):
        for j in range(L):
            assert bool(M[i, :, j, :].any()) == (j < i)


def test_made_forward_backward_vs_torch(cuda):
    L, q, H, B = 7, 3, 48, 128
    made = _made(L, q, H)
    seqs = np.random.default_rng(1).integers(0, q, size=(B, L)).astype("<u1")
    mem = torch.as_tensor(oracle.pack_seqs(seqs).view(np.int32), device="cuda")
    act = made.forward(mem, B, 0, B)
    lq_dev = act["logq"].cpu().double()
    made.backward(mem, B, 0, B, act)
    torch.cuda.synchronize()
    lq_cpu, P = _cpu_made(made, seqs)
    np.testing.assert_allclose(lq_dev.numpy(), lq_cpu.detach().numpy(), rtol=1e-5, atol=1e-4)
    (-lq_cpu.mean()).backward()
    for k in made.PARAMS:
        g = made.g[k].cpu().double()
        ref = P[k].grad
        if k in made.mask:
            ref = ref * made.mask[k].cpu().double()
        scale = ref.abs().max().item() + 1e-12
        assert (g - ref).abs().max().item() <= 1e-4 * scale + 1e-7, k


def test_made_adam_vs_torch(cuda):
    L, q, H, B = 5, 4, 32, 64
    made = _made(L, q, H, seed=3)
    seqs = np.random.default_rng(2).integers(0, q, size=(B, L)).astype("<u1")
    mem = torch.as_tensor(oracle.pack_seqs(seqs).view(np.int32), device="cuda")
    ref = {k: made.p[k].detach().cpu().clone().requires_grad_(True) for k in made.PARAMS}
    opt = torch.optim.Adam(list(ref.values()), lr=made.lr, betas=(0.9, 0.999), eps=1e-8)
    for _ in range(3):
        act = made.forward(mem, B, 0, B)
        made.backward(mem, B, 0, B, act)
        grads = {k: made.g[k].cpu().clone() for k in made.PARAMS}
        made.adam_step()
        for k in made.PARAMS:
            ref[k].grad = grads[k]
        opt.step()
        with torch.no_grad():  # masked weights stay exactly zero in the device update
            for k in made.mask:
                ref[k].mul_(made.mask[k].cpu())
    torch.cuda.synchronize()
    for k in made.PARAMS:
        np.testing.assert_allclose(made.p[k].cpu().numpy(), ref[k].detach().numpy(), rtol=1e-5, atol=1e-6)


def test_made_sampler_logq_and_teacher_forcing(cuda):
    L, q, H, N = 9, 4, 64, 4096
    made = _made(L, q, H, seed=5)
    sw = (L - 1) // 4 + 1
    seq = torch.zeros(sw * N, dtype=torch.int32, device="cuda")
    lq_s = torch.zeros(N, device="cuda")
    lq_t = torch.zeros(N, device="cuda")
    made.sample(seq, N, lq_s, seed=123)
    made.sample(seq, N, lq_t, seed=0, given=True)
    torch.cuda.synchronize()
    np.testing.assert_allclose(lq_s.cpu().numpy(), lq_t.cpu().numpy(), rtol=1e-5, atol=1e-5)
    seqs = oracle.unpack_seqs(seq.cpu().numpy().view(np.uint32).reshape(sw, N), L)
    assert seqs.max() < q
    lq_cpu, _ = _cpu_made(made, seqs)
    np.testing.assert_allclose(lq_s.cpu().numpy(), lq_cpu.detach().numpy(), rtol=1e-4, atol=1e-4)


def test_made_sampler_distribution(cuda):
    """All q^L sequences of a tiny model: sample frequencies match q(s)."""
    L, q, H, N = 3, 3, 16, 1 << 17
    made = _made(L, q, H, seed=8)
    seq = torch.zeros(N, dtype=torch.int32, device="cuda")
    lq = torch.zeros(N, device="cuda")
    made.sample(seq, N, lq, seed=99)
    seqs = oracle.unpack_seqs(seq.cpu().numpy().view(np.uint32).reshape(1, N), L)
    allseq = np.array(list(itertools.product(range(q), repeat=L)), dtype="<u1")
    lq_all, _ = _cpu_made(made, allseq)
    p = np.exp(lq_all.detach().numpy())
    assert abs(p.sum() - 1) < 1e-6
    assert _zscores(seqs, p, L, q).max() < 5.0


def test_made_training_reduces_nll(cuda):
    """Data with strong nearest-neighbour correlation: the trained network's
    NLL falls well below the site-independent value."""
    L, q, H, N = 12, 4, 64, 16384
    rng = np.random.default_rng(3)
    s = np.zeros((N, L), dtype="<u1")
    s[:, 0] = rng.integers(0, q, N)
    for i in range(1, L):
        keep = rng.random(N) < 0.8
        s[:, i] = np.where(keep, s[:, i - 1], rng.integers(0, q, N))
    mem = torch.as_tensor(oracle.pack_seqs(s).view(np.int32), device="cuda")
    made = MadeProposal(L, q, H=H, device=0, seed=1, lr=1e-2)
    hist = made.train(mem, N, epochs=12, batch=1024)
    indep = L * np.log(q)                       # every marginal is uniform
    cond = -(0.85 * np.log(0.85) + 3 * 0.05 * np.log(0.05))
    exact = np.log(q) + (L - 1) * cond          # entropy of the data model
    assert hist[-1] < hist[0]
    assert hist[-1] < exact + 0.5 * (indep - exact)


def test_independence_mh_leaves_boltzmann_invariant(cuda):
    """Tiny Potts model (all q^L states enumerable): (1) walkers started at
    exact Boltzmann samples stay Boltzmann under repeated proposal steps of
    an untrained network (detailed balance); (2) proposals interleaved with
    sweeps from a fixed start reach exp(-E)/Z."""
    L, q, N = 4, 3, 1 << 15
    J = potts.synthetic_ground_truth(L, q, seed=4, contact_sigma=0.6, background_sigma=0.6)
    allseq, p = _boltzmann(J, L, q)
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 5)
    gpus = GPU_node([g])
    gpus.initMCMC(L)
    gpus.setBuf('J', J)
    made = _made(L, q, 16, seed=2)
    ls = LearnedSampler(g, made, every=1, min_accept=0.0)
    rng = np.random.default_rng(11)
    gpus.setSeqs('main', allseq[rng.choice(len(p), size=N, p=p)])
    rates = [ls.propose() for _ in range(20)]
    assert min(rates) > 0.02
    assert _zscores(gpus.collect('seq main'), p, L, q).max() < 5.0
    gpus.setSeqs('main', np.zeros((N, L), '<u1'))
    rates = ls.sweeps(60)
    assert min(rates) > 0.02
    assert _zscores(gpus.collect('seq main'), p, L, q).max() < 5.0


def test_trained_proposal_decorrelates_faster_per_sweep(cuda):
    """What the trained network gains: on a strongly coupled model the energy
    autocorrelation after the same number of sweeps is lower when proposal
    steps (network trained on the equilibrated walkers) are interleaved."""
    L, q, N, H = 40, 4, 1 << 15, 128
    J = potts.synthetic_ground_truth(L, q, seed=12, contact_sigma=0.9)
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 6)
    gpus = GPU_node([g])
    gpus.initMCMC(L)
    gpus.prepare_indep(np.full((L, q), 1.0 / q))
    gpus.gen_indep('main')
    gpus.setBuf('J', J)
    for _ in range(400):
        g.runMCMC()
    made = MadeProposal(L, q, H=H, device=0, seed=3, lr=3e-3)
    hist = made.train(g.bufs['seq main'], N, epochs=20, batch=2048)
    assert hist[-1] < hist[0]
    start, start_rng = g.bufs['seq main'].clone(), g.bufs['rngstates'].clone()

    def rho_after(with_proposals, sweeps=16):
        g.bufs['seq main'].copy_(start)
        g.bufs['rngstates'].copy_(start_rng)
        gpus.calcEnergies('main')
        E0 = gpus.collect('E main').astype(np.float64).copy()
        ls = LearnedSampler(g, made, every=2, min_accept=0.0, seed=9)
        rates = []
        for k in range(sweeps):
            g.runMCMC()
            if with_proposals and (k + 1) % 2 == 0:
                rates.append(ls.propose())
        gpus.calcEnergies('main')
        E1 = gpus.collect('E main').astype(np.float64)
        return np.corrcoef(E0, E1)[0, 1], rates

    rho_plain, _ = rho_after(False)
    rho_learned, rates = rho_after(True)
    assert np.mean(rates) > 0.05
    assert rho_learned < rho_plain - 0.05, (rho_plain, rho_learned, np.mean(rates))
