"""Parity at the reference-sized workload (L=232, q=21, 2^20 walkers),
where the oracle cannot replay every pair in the time a test has:

* bimarginal counts: the shared-memory histogram kernel and the tcgen05
  FP8 one-hot GEMM must agree bit for bit on every pair (countBivariate,
  mcmc.cl:462-516, both ways), each equals numpy's integer count on a
  seeded sample of 96 pairs, and all pairs pass the size-independent
  identities of a count table: every pair sums to N, and summing a pair's
  table over the second residue gives the first site's univariate counts
  (the same for every partner site)."""
import numpy as np
import pytest

from mi3gpu_b200 import GPU_node, MCMCGPU, _lib
from tests._util import empty, host

pytestmark = pytest.mark.gpu

L, Q, N = 232, 21, 1 << 20


def _walkers():
    """2^20 walkers from skewed independent-site marginals, generated on the
    device (gen_indep)."""
    rng = np.random.default_rng(2320)
    f = rng.gamma(0.3, size=(L, Q)) + 1e-3
    f /= f.sum(axis=1, keepdims=True)
    g = MCMCGPU((0, 0), L, Q, N, 512, None, 1024, 77)
    node = GPU_node([g])
    node.initMCMC(2048)
    node.prepare_indep(f.astype('<f4'))
    node.gen_indep('main')
    node.wait()
    return g


def _site(words, i):
    return ((words[i // 4] >> np.uint32(8 * (i % 4))) & np.uint32(0xff)).astype(np.int64)


def test_bicounts_full_size_smem_equals_tcgen05_and_numpy(cuda):
    g = _walkers()
    s = g.stream.cuda_stream if hasattr(g.stream, "cuda_stream") else g.stream
    npairs = L * (L - 1) // 2
    seq = g.packedSeqs('main')
    a = empty((npairs, Q * Q), np.uint32)
    b = empty((npairs, Q * Q), np.uint32)
    b.fill_(-1)
    status = empty((1,), np.int32)
    _lib.call("mi3_bicounts", seq.data_ptr(), N, N, a.data_ptr(), L, Q, s)
    _lib.call("mi3_bicounts_tc", seq.data_ptr(), N, N, b.data_ptr(), L, Q, status.data_ptr(), s)
    ca, cb = host(a, np.uint32), host(b, np.uint32)
    assert int(host(status)[0]) == 0
    np.testing.assert_array_equal(ca, cb)

    assert (ca.sum(axis=1, dtype=np.int64) == N).all()
    words = host(seq, np.uint32)
    ii, jj = np.triu_indices(L, k=1)
    uni = np.stack([np.bincount(_site(words, i), minlength=Q) for i in range(L)])
    c3 = ca.reshape(npairs, Q, Q).astype(np.int64)
    np.testing.assert_array_equal(c3.sum(axis=2), uni[ii])
    np.testing.assert_array_equal(c3.sum(axis=1), uni[jj])

    for p in np.random.default_rng(5).choice(npairs, 96, replace=False):
        ref = np.bincount(_site(words, ii[p]) * Q + _site(words, jj[p]), minlength=Q * Q)
        np.testing.assert_array_equal(ca[p].astype(np.int64), ref)
