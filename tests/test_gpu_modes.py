"""The reference's other modes over the device kernels: the subsequence
splice (copySubseq, mcmc.cl:99-122) bit for bit against the oracle, sequence
energies of any number of sequences (Mi3.py:549-606), and subsequence log
frequencies (Mi3.py:876-976) against the oracle's float64 restatement."""
import numpy as np
import pytest
import torch

from oracle import oracle
from mi3gpu_b200 import MCMCGPU, _lib, potts, seqload
from mi3gpu_b200.inference import sequence_energies, subseq_log_frequencies

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,nsmall,nlarge", [(5, 512, 100), (37, 1024, 3001), (232, 512, 20000)])
def test_copy_subseq_matches_oracle(cuda, L, nsmall, nlarge):
    rng = np.random.default_rng(L)
    small = oracle.pack_seqs(rng.integers(0, 21, size=(nsmall, L)).astype('u1'))
    large = oracle.pack_seqs(rng.integers(0, 21, size=(nlarge, L)).astype('u1'))
    for marks in (rng.integers(0, 2, size=L).astype('u1'), np.zeros(L, 'u1'), np.ones(L, 'u1')):
        seqind = int(rng.integers(0, nsmall))
        dl = torch.from_numpy(large.view(np.int32)).cuda()
        ds = torch.from_numpy(small.view(np.int32)).cuda()
        dm = torch.from_numpy(marks).cuda()
        _lib.call('mi3_copy_subseq', ds.data_ptr(), nsmall, seqind, dm.data_ptr(), dl.data_ptr(), nlarge, L, None)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(dl.cpu().numpy().view(np.uint32),
                                      oracle.copy_subseq(small, seqind, marks, large, L))


def test_copy_subseq_through_mcmcgpu(cuda):
    L, q = 11, 4
    rng = np.random.default_rng(2)
    main = rng.integers(0, q, size=(512, L)).astype('u1')
    big = rng.integers(0, q, size=(700, L)).astype('u1')
    g = MCMCGPU((0, 0), L, q, 512, 512, None, 1024, 0)
    g.initLargeBufs(700)
    g.initSubseq()
    g.setBuf('seq main', main)
    g.setBuf('seq large', big)
    marks = np.zeros(L, 'u1')
    marks[[0, 3, 4, 10]] = 1
    g.markPos(marks)
    g.copySubseq(77)
    want = big.copy()
    want[:, marks.astype(bool)] = main[77, marks.astype(bool)]
    np.testing.assert_array_equal(g.getBuf('seq large').read(), want)
    with pytest.raises(Exception, match="past end"):
        g.copySubseq(512)


def test_sequence_energies_any_count(cuda, tmp_path):
    L, q = 29, 21
    J = potts.synthetic_ground_truth(L, q, seed=3, contact_sigma=0.5)
    seqs = np.random.default_rng(4).integers(0, q, size=(1237, L)).astype('u1')
    ref = oracle.energies_f64(J, oracle.pack_seqs(seqs), L, q)
    for src in (seqs, tmp_path / "seqs"):
        if not isinstance(src, np.ndarray):
            seqload.writeSeqs(src, seqs, seqload.alpha21, ids=[f"s{k}" for k in range(len(seqs))], zipf=True)
        E = sequence_energies(J, src)
        assert E.shape == (1237,) and E.dtype == np.float32
        assert (np.abs(E - ref) / np.maximum(1, np.abs(ref))).max() <= 1e-5


@pytest.mark.parametrize("iterbackgrounds", [False, True])
def test_subseq_log_frequencies_match_oracle(cuda, iterbackgrounds):
    L, q = 14, 4
    J = potts.synthetic_ground_truth(L, q, seed=6, contact_sigma=0.5)
    rng = np.random.default_rng(7)
    n = 600 if not iterbackgrounds else 300  # the default branch needs equal sizes
    bseqs = rng.integers(0, q, size=(n, L)).astype('u1')
    sseqs = rng.integers(0, q, size=(n if not iterbackgrounds else 40, L)).astype('u1')
    fixpos = [2, 3, 9]
    got = subseq_log_frequencies(J, bseqs, sseqs, fixpos, iterbackgrounds, alpha="ACGT")
    want = oracle.subseq_log_frequencies(J, bseqs, sseqs, fixpos, iterbackgrounds, L, q)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-4)


def test_equilibrate_gen_mode_outputs(cuda, tmp_path):
    """The reference's `gen` mode (Mi3.py:724-870): walkers from
    independent-site sequences, fixed or automatic equilibration, and the
    files it writes -- bicounts (text), bimarg.npy, energies.npy, seqs -- all
    consistent with the final walkers (counts bit-exact, energies against
    the FP64 oracle)."""
    from mi3gpu_b200.inference import benchmark_mcmc, equilibrate
    L, q, N = 20, 4, 4096
    J = potts.synthetic_ground_truth(L, q, seed=31, contact_sigma=0.5)
    uni = np.full((L, q), 1.0 / q)
    for equiltime in (6, 'auto'):
        out = tmp_path / str(equiltime)
        bim, bic, E, walkers = equilibrate(J, N, equiltime, unimarg=uni, alpha="ACGT", outdir=out,
                                           log=lambda *a: None)
        mem = oracle.pack_seqs(walkers)
        np.testing.assert_array_equal(bic, oracle.bicounts(mem, L, q))
        np.testing.assert_array_equal(np.loadtxt(out / 'bicounts').astype(np.uint32), bic)
        np.testing.assert_array_equal(np.load(out / 'bimarg.npy'), bim)
        ref = oracle.energies_f64(J, mem, L, q)
        assert (np.abs(np.load(out / 'energies.npy') - ref) / np.maximum(1, np.abs(ref))).max() <= 1e-5
        np.testing.assert_array_equal(seqload.loadSeqs(out / 'seqs', "ACGT")[0], walkers)
    rate = benchmark_mcmc(J, N, L, 3, seedseq=np.zeros(L, 'u1'), log=lambda *a: None)
    assert rate > 1e8
