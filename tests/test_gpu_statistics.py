"""Sampled bimarginals against exact enumeration and against the
reference's own CPU sampler (extras/mcmcCPUgenThreaded.c, built from the
reference tree into oracle/_ref): at L=10, q=4 every one of the 4^10
sequences can be weighted exactly, so both samplers are checked against the
true bimarginals within the finite-sample error of their sample sizes, and
against each other."""
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from mi3gpu_b200 import GPU_node, MCMCGPU

pytestmark = pytest.mark.gpu

L, Q = 10, 4


def _model():
    rng = np.random.default_rng(2024)
    return rng.normal(0, 0.35, size=(L * (L - 1) // 2, Q * Q)).astype("<f4")


def _exact_bimarg(J):
    """Boltzmann bimarginals, P(s) ~ exp(-E(s)), by enumerating 4^10 states."""
    idx = np.arange(Q ** L, dtype=np.int64)
    S = np.stack([(idx // Q ** (L - 1 - k)) % Q for k in range(L)], axis=1)
    i, j = np.triu_indices(L, k=1)
    E = np.zeros(Q ** L)
    for p in range(len(i)):
        E += J[p].astype(np.float64)[S[:, i[p]] * Q + S[:, j[p]]]
    w = np.exp(-(E - E.min()))
    w /= w.sum()
    f = np.empty((len(i), Q * Q))
    for p in range(len(i)):
        f[p] = np.bincount(S[:, i[p]] * Q + S[:, j[p]], weights=w, minlength=Q * Q)
    return f


def _bimarg(seqs):
    i, j = np.triu_indices(L, k=1)
    n = seqs.shape[0]
    return np.stack([np.bincount(seqs[:, a] * Q + seqs[:, b], minlength=Q * Q) / n for a, b in zip(i, j)])


def _expected_ssr(f, n):
    """E[sum (f_hat - f)^2] for n independent samples: sum f (1 - f) / n."""
    return float(np.sum(f * (1 - f)) / n)


def test_gpu_sampler_matches_exact_and_reference_cpu_sampler(cuda):
    J = _model()
    f = _exact_bimarg(J)
    # the B200 sampler: 16384 walkers, 400 sweeps from random sequences
    N = 16384
    g = MCMCGPU((0, 0), L, Q, N, 512, None, 1024, 11)
    node = GPU_node([g])
    node.initMCMC(10 * L)
    node.setBuf('J', J)
    node.setSeqs('main', np.random.default_rng(5).integers(0, Q, size=(N, L)).astype('<u1'))
    for _ in range(40):
        node.runMCMC()
    seqs_gpu = node.collect('seq main')
    f_gpu = _bimarg(seqs_gpu)
    ssr_gpu = float(np.sum((f_gpu - f) ** 2))
    exp_gpu = _expected_ssr(f, N)
    assert ssr_gpu < 1.5 * exp_gpu, (ssr_gpu, exp_gpu)

    # the reference's CPU sampler: 16 independent chains, 40 sweeps of
    # burn-in, then one sample every 10 sweeps
    from oracle import oracle
    exe = oracle.ref_cpu_binary()
    if exe is None:
        pytest.skip("reference CPU sampler not built (oracle/_ref)")
    procs, burn, keep = 16, 4, 256
    alpha = "ABCD"
    rng = np.random.default_rng(6)
    with tempfile.TemporaryDirectory() as td:
        jf = Path(td) / "J.dat"
        J.tofile(jf)
        outs = []
        for p in range(procs):
            start = "".join(alpha[k] for k in rng.integers(0, Q, size=L))
            r = subprocess.run([str(exe), str(jf), str(10 * L), str(burn + keep), alpha, start], check=True,
                               capture_output=True, text=True)
            lines = r.stdout.split()[burn:]
            outs.append(np.array([[alpha.index(c) for c in ln] for ln in lines], dtype=np.int64))
    seqs_cpu = np.concatenate(outs)
    f_cpu = _bimarg(seqs_cpu)
    n_cpu = seqs_cpu.shape[0]
    ssr_cpu = float(np.sum((f_cpu - f) ** 2))
    exp_cpu = _expected_ssr(f, n_cpu)
    # successive samples of one chain are 10 sweeps apart: allow for their
    # correlation
    assert ssr_cpu < 3.0 * exp_cpu, (ssr_cpu, exp_cpu)
    ssr_between = float(np.sum((f_gpu - f_cpu) ** 2))
    assert ssr_between < 3.0 * exp_cpu + 1.5 * exp_gpu, (ssr_between, exp_cpu, exp_gpu)
