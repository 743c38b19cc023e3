"""Tensor-core MADE sampler (csrc/made_tc.cu): log q against a float64 CPU
forward of the same network (activations rounded to bf16 where the tensor
cores read them), log q of drawn sequences reproduced exactly by the
teacher-forced pass, the distribution of the draws, and exactness of the
independence MH step with tensor-core proposals."""
import itertools

import numpy as np
import pytest
import torch

from oracle import oracle
from mi3gpu_b200 import GPU_node, MCMCGPU, potts
from mi3gpu_b200.learned import LearnedSampler, MadeProposal

pytestmark = pytest.mark.gpu


def _bf16(x):
    return x.float().to(torch.bfloat16).double()


def _cpu_made_tc(made, seqs):
    """float64 forward with a1 and a2 rounded to bf16, as the sampler reads them."""
    P = {k: made.pc[k].detach().cpu().double() for k in made.PARAMS}
    L, q = made.L, made.q
    X = torch.nn.functional.one_hot(torch.as_tensor(seqs, dtype=torch.long), q).reshape(len(seqs), L * q).double()
    a1 = _bf16(torch.relu(X @ P["W1T"] + P["b1"]))
    a2 = _bf16(torch.relu(a1 @ P["W2"].T + P["b2"]))
    logits = (a2 @ P["W3"].T + P["b3"]).reshape(len(seqs), L, q)
    lp = torch.log_softmax(logits, dim=-1)
    return lp.gather(2, torch.as_tensor(seqs, dtype=torch.long)[..., None])[..., 0].sum(1).numpy()


def _made(L, q, H, seed=0, G=None, wscale=1.0):
    m = MadeProposal(L, q, H=H, device=0, seed=seed, sampler="tc", G=G)
    rng = np.random.default_rng(seed + 7)
    for k in ("b1", "b2", "b3"):
        m.p[k].copy_(torch.as_tensor(rng.normal(0, 0.3, size=m.p[k].shape), dtype=torch.float32))
    for k in ("W1T", "W2", "W3"):
        m.p[k].mul_(wscale)
    m.round_params()
    return m


def _zmax(seqs, p, L, q, min_expected=10):
    """Largest |z| of the state frequencies against p, over the states
    expected at least min_expected times and over the pooled rest (one
    walker in a state of probability 1e-7 is not evidence of a bias)."""
    N = len(seqs)
    idx = (seqs.astype(int) * q ** np.arange(L - 1, -1, -1)).sum(1)
    freq = np.bincount(idx, minlength=q ** L) / N
    big = N * p >= min_expected
    z = np.abs(freq[big] - p[big]) / np.sqrt(p[big] * (1 - p[big]) / N)
    P, F = p[~big].sum(), freq[~big].sum()
    z_rest = abs(F - P) / np.sqrt(max(P * (1 - P), 1e-12) / N) if P > 0 else 0.0
    return max(z.max(), z_rest)


def _draw(made, N, seed, buflen=None):
    L = made.L
    sw = (L - 1) // 4 + 1
    buflen = buflen or N
    seq = torch.zeros(sw * buflen, dtype=torch.int32, device="cuda")
    lq = torch.zeros(N, device="cuda")
    made.sample(seq, N, lq, seed=seed, buflen=buflen)
    return seq, lq, sw, buflen


@pytest.mark.parametrize("L,q,H,G,N", [
    (5, 4, 32, 4, 1000),       # two blocks, the second without units: logits accumulator only
    (8, 4, 64, 4, 4096),       # two blocks with units: layer-2 product and logits accumulator
    (12, 4, 64, 8, 777),       # ragged tile
    (48, 4, 512, None, 2048),  # twelve blocks of 4 sites
    (99, 4, 512, None, 4096),  # the learned-proposal benchmark's network
    (20, 8, 128, None, 1536),  # q = 8
])
def test_tc_logq_vs_cpu_and_teacher_forcing(cuda, L, q, H, G, N):
    made = _made(L, q, H, seed=L + H, G=G, wscale=2.0)
    seq, lq_s, sw, buflen = _draw(made, N, seed=321, buflen=N + 64)
    lq_t = torch.zeros(N, device="cuda")
    made.sample(seq, N, lq_t, seed=0, given=True, buflen=buflen)
    torch.cuda.synchronize()
    made.check_status()
    # the teacher-forced pass is the same arithmetic: identical log q
    assert torch.equal(lq_s, lq_t)
    seqs = oracle.unpack_seqs(seq.cpu().numpy().view(np.uint32).reshape(sw, buflen)[:, :N], L)
    assert seqs.max() < q
    ref = _cpu_made_tc(made, seqs)
    err = np.abs(lq_s.cpu().numpy() - ref)
    # FP32 sums in another order can round an activation to the next bf16
    # value now and then; everything else agrees to float precision
    assert np.median(err) < 1e-4 * L
    assert err.max() < 2e-2, err.max()


def test_tc_sampler_distribution(cuda):
    """All 4^5 sequences of a two-block model: draw frequencies match q(s)."""
    L, q, H, N = 5, 4, 32, 1 << 18
    made = _made(L, q, H, seed=4, G=4, wscale=3.0)
    seq, lq, sw, buflen = _draw(made, N, seed=17)
    torch.cuda.synchronize()
    seqs = oracle.unpack_seqs(seq.cpu().numpy().view(np.uint32).reshape(sw, N), L)
    allseq = np.array(list(itertools.product(range(q), repeat=L)), dtype="<u1")
    p = np.exp(_cpu_made_tc(made, allseq))
    assert abs(p.sum() - 1) < 1e-5
    assert _zmax(seqs, p, L, q) < 5.0


def test_tc_and_simt_samplers_agree_on_logq(cuda):
    """The same network through both samplers' teacher-forced passes: the
    SIMT one keeps the activations in FP32, so they agree to the bf16
    rounding of the activations."""
    L, q, H, N = 40, 4, 128, 4096
    made = _made(L, q, H, seed=9)
    seq, lq_tc, sw, buflen = _draw(made, N, seed=5)
    lq_simt = torch.zeros(N, device="cuda")
    made.sampler = "simt"
    made.sample(seq, N, lq_simt, seed=0, given=True)
    made.sampler = "tc"
    torch.cuda.synchronize()
    d = (lq_tc - lq_simt).abs().cpu().numpy()
    assert np.median(d) < 0.02 and d.max() < 0.2


def test_tc_proposals_leave_boltzmann_invariant(cuda):
    """Walkers at exact Boltzmann samples of a 4^5-state Potts model stay
    Boltzmann under repeated independence-MH steps with tensor-core
    proposals."""
    L, q, N = 5, 4, 1 << 15
    J = potts.synthetic_ground_truth(L, q, seed=4, contact_sigma=0.6, background_sigma=0.6)
    allseq = np.array(list(itertools.product(range(q), repeat=L)), dtype="<u1")
    E = oracle.energies_f64(J, oracle.pack_seqs(allseq), L, q)
    p = np.exp(-(E - E.min()))
    p /= p.sum()
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 5)
    gpus = GPU_node([g])
    gpus.initMCMC(L)
    gpus.setBuf('J', J)
    made = _made(L, q, 32, seed=2, G=4)
    assert made.sampler == "tc"
    ls = LearnedSampler(g, made, every=1, min_accept=0.0)
    rng = np.random.default_rng(11)
    gpus.setSeqs('main', allseq[rng.choice(len(p), size=N, p=p)])
    rates = [ls.propose() for _ in range(20)]
    assert min(rates) > 0.02
    assert _zmax(gpus.collect('seq main'), p, L, q) < 5.0
