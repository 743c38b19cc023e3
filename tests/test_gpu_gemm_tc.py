"""The BF16 tensor-core GEMM (csrc/gemm_tc.cu) against a float64 product of
the bf16-rounded operands, and the MADE training pass built on it against
float64 autograd."""
import numpy as np
import pytest
import torch

from oracle import oracle
from mi3gpu_b200 import _lib
from mi3gpu_b200.learned import MadeProposal

pytestmark = pytest.mark.gpu


def _bf16(x):
    return x.to(torch.bfloat16).double()


def _gemm(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, alpha, beta):
    nbytes = int(_lib.query("mi3_gemm_bf16_workspace", M, N, K))
    ws = torch.empty(nbytes + 1024, dtype=torch.uint8, device="cuda")
    off = (-ws.data_ptr()) % 1024
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("mi3_gemm_bf16", M, N, K, A.data_ptr(), sam, sak, B.data_ptr(), sbk, sbn, C.data_ptr(), ldc,
              alpha, beta, ws.data_ptr() + off, nbytes, status.data_ptr(), None)
    torch.cuda.synchronize()
    assert int(status.item()) == 0


@pytest.mark.parametrize("M,N,K,ta,tb", [
    (128, 128, 64, False, False),
    (300, 200, 100, False, False),   # ragged in every dimension
    (4096, 512, 396, False, True),   # dlogits . W3 (B read across its rows)
    (396, 512, 4096, True, False),   # dlogits^T . a2 (A transposed)
    (512, 512, 4096, True, False),
    (33, 17, 5, True, True),
])
def test_gemm_bf16_vs_float64(cuda, M, N, K, ta, tb):
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N + K)
    A = torch.randn(K, M, generator=g) if ta else torch.randn(M, K, generator=g)
    B = torch.randn(N, K, generator=g) if tb else torch.randn(K, N, generator=g)
    C0 = torch.randn(M, N, generator=g)
    sam, sak = (1, M) if ta else (K, 1)
    sbk, sbn = (1, K) if tb else (N, 1)
    Ad, Bd, Cd = A.cuda(), B.cuda(), C0.cuda()
    _gemm(M, N, K, Ad, sam, sak, Bd, sbk, sbn, Cd, N, 0.5, -1.0)
    Am = (A.T if ta else A)
    Bm = (B.T if tb else B)
    ref = 0.5 * (_bf16(Am) @ _bf16(Bm)) - C0.double()
    err = (Cd.cpu().double() - ref).abs().max().item()
    scale = (_bf16(Am).abs() @ _bf16(Bm).abs()).max().item()
    assert err <= 1e-5 * scale + 1e-5, (err, scale)


def test_gemm_rejects_bad_workspace(cuda):
    p = 4096
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_gemm_bf16", 128, 128, 64, p, 64, 1, p, 128, 1, p, 128, 1.0, 0.0, p, 16, status.data_ptr(), None)
    assert e.value.code == -4


def _cpu_made(made, seqs):
    P = {k: made.pc[k].detach().cpu().double().requires_grad_(True) for k in made.PARAMS}
    L, q = made.L, made.q
    X = torch.nn.functional.one_hot(torch.as_tensor(seqs, dtype=torch.long), q).reshape(len(seqs), L * q).double()
    a1 = torch.relu(X @ P["W1T"] + P["b1"])
    a2 = torch.relu(a1 @ P["W2"].T + P["b2"])
    logits = (a2 @ P["W3"].T + P["b3"]).reshape(len(seqs), L, q)
    lp = torch.log_softmax(logits, dim=-1)
    logq = lp.gather(2, torch.as_tensor(seqs, dtype=torch.long)[..., None])[..., 0].sum(1)
    return logq, P


@pytest.mark.parametrize("L,q,H,B", [(7, 3, 48, 128), (40, 4, 128, 1024)])
def test_made_training_pass_tc_vs_float64(cuda, L, q, H, B):
    """Forward and backward with the dense products in bf16: log q and every
    gradient within the rounding of bf16 operands.  A weight gradient goes
    through up to three chained bf16 products (dlogits -> dh2 -> gW2), and
    cancellation in the batch sums leaves single entries a few percent of
    the largest gradient off; the gradient as a whole stays within 2%."""
    made = MadeProposal(L, q, H=H, device=0, seed=1, lr=1e-2, gemm="tc")
    rng = np.random.default_rng(L)
    for k in ("b1", "b2", "b3"):
        made.p[k].copy_(torch.as_tensor(rng.normal(0, 0.3, size=made.p[k].shape), dtype=torch.float32))
    made.round_params()
    seqs = rng.integers(0, q, size=(B, L)).astype("<u1")
    mem = torch.as_tensor(oracle.pack_seqs(seqs).view(np.int32), device="cuda")
    act = made.forward(mem, B, 0, B)
    lq_dev = act["logq"].cpu().double()
    made.backward(mem, B, 0, B, act)
    torch.cuda.synchronize()
    made.check_status()
    lq_cpu, P = _cpu_made(made, seqs)
    assert (lq_dev - lq_cpu.detach()).abs().max().item() < 2e-2 * L ** 0.5
    (-lq_cpu.mean()).backward()
    for k in made.PARAMS:
        g = made.g[k].cpu().double()
        ref = P[k].grad
        if k in made.mask:
            ref = ref * made.mask[k].cpu().double()
            assert torch.all(g[made.mask[k].cpu() == 0] == 0), k
        scale = ref.abs().max().item() + 1e-12
        assert (g - ref).abs().max().item() <= 6e-2 * scale + 1e-6, k
        assert (g - ref).norm().item() <= 2e-2 * ref.norm().item() + 1e-6, k
