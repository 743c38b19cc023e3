"""GPU parity of the skewed-lane sampler (mi3_metropolis_skew): the same
trajectories as the reference's metropolis kernel (mcmc.cl:360-458) restated
by the oracle, bit for bit -- sequences and RNG states after 1 to 300
proposals, for both walker-per-CTA plans, per-walker betas, shapes whose
L + 31 fills the register array exactly (L = 257) or leaves a partial last
chunk -- and the same results as the shared-memory-row kernel
mi3_metropolis on the reference-sized shape."""
import numpy as np
import pytest

from oracle import oracle
from mi3gpu_b200 import _lib
from tests._util import dev as _dev, host, empty, stream, random_model

pytestmark = pytest.mark.gpu

_alive = []


def dev(a):
    t = _dev(a)
    _alive.append(t)
    return t


@pytest.fixture(autouse=True)
def _release():
    yield
    import torch
    torch.cuda.synchronize()
    _alive.clear()


def _seqs(L, q, N, seed):
    return np.random.default_rng(seed).integers(0, q, size=(N, L)).astype("<u1")


def _tiles(J, L, q):
    T = empty((int(_lib.query("mi3_jtiles_floats", L, q)),), np.float32)
    T.fill_(3.0)
    _lib.call("mi3_unpack_j_tiles", dev(J).data_ptr(), T.data_ptr(), L, q, stream())
    return T


@pytest.mark.parametrize("L,q", [(10, 5), (48, 4), (37, 21), (93, 4), (64, 8), (2, 2), (257, 3), (232, 21)])
def test_unpack_j_tiles_bitexact(cuda, L, q):
    J = random_model(L, q, 1)
    T = _tiles(J, L, q)
    np.testing.assert_array_equal(host(T).reshape(-1), oracle.unpack_j_tiles(J, L, q).reshape(-1))


@pytest.mark.parametrize("L,q,N", [(10, 5, 512), (48, 4, 1536), (37, 21, 512), (93, 4, 1536), (64, 8, 512),
                                   (2, 2, 512), (31, 7, 512), (32, 3, 512), (33, 21, 512), (257, 4, 512),
                                   (99, 21, 1536), (60, 21, 1024), (40, 6, 96), (300, 4, 512), (512, 21, 256),
                                   (545, 3, 512)])
@pytest.mark.parametrize("nsteps", [1, 37, 300])
@pytest.mark.parametrize("wpc", [256, 512, 768])
def test_skew_trajectory_bitexact(cuda, L, q, N, nsteps, wpc):
    """N need not be a multiple of the walkers per CTA: the last CTA is then
    partly filled (1024 = 768 + 256, 96 < 512).  Rows longer than
    L + 31 = 288 take 256 walkers per CTA only."""
    if L + 31 > 288 and wpc != 256:
        pytest.skip("512 or 768 walkers per CTA hold rows up to L + 31 = 288")
    J = random_model(L, q, 2, sigma=0.5)
    seqs = _seqs(L, q, N, 3)
    mem = oracle.pack_seqs(seqs)
    st = oracle.init_rng(N, 0, 2 ** 63 // (2 * N))
    pos = np.random.RandomState(11).randint(0, L, size=nsteps + 13).astype("<u4")
    off = 13 if nsteps < 100 else 0
    T = _tiles(J, L, q)
    dmem, dst, dpos = dev(mem), dev(st), dev(pos)
    status = empty((1,), np.int32)
    _lib.call("mi3_metropolis_skew", T.data_ptr(), dst.data_ptr(), off, dpos.data_ptr(), nsteps, None, 1.0,
              dmem.data_ptr(), N, L, q, wpc, 1, status.data_ptr(), stream())
    g_mem, g_st = host(dmem, np.uint32), host(dst, np.uint32)
    assert int(host(status)[0]) == 0
    o_mem, o_st = mem.copy(), st.copy()
    oracle.metropolis(J, o_st, pos, off, nsteps, o_mem, L, q)
    np.testing.assert_array_equal(g_st, o_st)
    np.testing.assert_array_equal(g_mem, o_mem)
    assert (g_mem != mem).any()


def test_skew_betas(cuda):
    L, q, N, nsteps = 20, 6, 512, 64
    J = random_model(L, q, 4, sigma=0.6)
    mem = oracle.pack_seqs(_seqs(L, q, N, 5))
    st = oracle.init_rng(N, 77, 10 ** 9)
    pos = np.random.RandomState(1).randint(0, L, size=nsteps).astype("<u4")
    betas = np.linspace(0.2, 2.0, N).astype("<f4")
    T = _tiles(J, L, q)
    dmem, dst = dev(mem), dev(st)
    status = empty((1,), np.int32)
    _lib.call("mi3_metropolis_skew", T.data_ptr(), dst.data_ptr(), 0, dev(pos).data_ptr(), nsteps,
              dev(betas).data_ptr(), 1.0, dmem.data_ptr(), N, L, q, 0, 0, status.data_ptr(), stream())
    oracle.metropolis(J, st, pos, 0, nsteps, mem, L, q, betas=betas)
    np.testing.assert_array_equal(host(dmem, np.uint32), mem)
    np.testing.assert_array_equal(host(dst, np.uint32), st)


def test_skew_long_rows_equal_row_kernel(cuda):
    """L=512, q=21 (the large workload's shape), 256 walkers per CTA, 300
    proposals: the same walkers and RNG states as mi3_metropolis."""
    L, q, N, nsteps = 512, 21, 1024, 300
    from mi3gpu_b200.potts import synthetic_ground_truth
    J = synthetic_ground_truth(L, q, seed=1004)
    mem = oracle.pack_seqs(_seqs(L, q, N, 19))
    st = oracle.init_rng(N, 9, 2 ** 63 // (2 * N))
    pos = np.random.RandomState(4).randint(0, L, size=nsteps).astype("<u4")
    stride = int(_lib.query("mi3_jrows_stride", L, q))
    Ju = empty((L, stride), np.float32)
    _lib.call("mi3_unpack_j", dev(J).data_ptr(), Ju.data_ptr(), L, q, stream())
    T = _tiles(J, L, q)
    status = empty((1,), np.int32)
    a_mem, a_st = dev(mem), dev(st)
    _lib.call("mi3_metropolis", Ju.data_ptr(), a_st.data_ptr(), 0, dev(pos).data_ptr(), nsteps, None, 1.0,
              a_mem.data_ptr(), N, L, q, status.data_ptr(), stream())
    b_mem, b_st = dev(mem), dev(st)
    _lib.call("mi3_metropolis_skew", T.data_ptr(), b_st.data_ptr(), 0, dev(pos).data_ptr(), nsteps, None, 1.0,
              b_mem.data_ptr(), N, L, q, 0, 1, status.data_ptr(), stream())
    np.testing.assert_array_equal(host(b_mem, np.uint32), host(a_mem, np.uint32))
    np.testing.assert_array_equal(host(b_st, np.uint32), host(a_st, np.uint32))
    assert int(host(status)[0]) == 0


def test_skew_equals_row_kernel_reference_shape(cuda):
    """L=232, q=21: 1536 walkers, 600 proposals, both plans, against
    mi3_metropolis (itself bit-exact against the oracle)."""
    L, q, N, nsteps = 232, 21, 1536, 600
    from mi3gpu_b200.potts import synthetic_ground_truth
    J = synthetic_ground_truth(L, q, seed=1001)
    mem = oracle.pack_seqs(_seqs(L, q, N, 9))
    st = oracle.init_rng(N, 5, 2 ** 63 // (2 * N))
    pos = np.random.RandomState(3).randint(0, L, size=nsteps).astype("<u4")
    stride = int(_lib.query("mi3_jrows_stride", L, q))
    Ju = empty((L, stride), np.float32)
    dJ = dev(J)
    _lib.call("mi3_unpack_j", dJ.data_ptr(), Ju.data_ptr(), L, q, stream())
    T = _tiles(J, L, q)
    status = empty((1,), np.int32)
    a_mem, a_st = dev(mem), dev(st)
    _lib.call("mi3_metropolis", Ju.data_ptr(), a_st.data_ptr(), 0, dev(pos).data_ptr(), nsteps, None, 1.0,
              a_mem.data_ptr(), N, L, q, status.data_ptr(), stream())
    for wpc in (512, 768):
        b_mem, b_st = dev(mem), dev(st)
        _lib.call("mi3_metropolis_skew", T.data_ptr(), b_st.data_ptr(), 0, dev(pos).data_ptr(), nsteps, None,
                  1.0, b_mem.data_ptr(), N, L, q, wpc, 1, status.data_ptr(), stream())
        np.testing.assert_array_equal(host(b_mem, np.uint32), host(a_mem, np.uint32))
        np.testing.assert_array_equal(host(b_st, np.uint32), host(a_st, np.uint32))
    assert int(host(status)[0]) == 0


def test_skew_bad_site_reported(cuda):
    L, q, N = 16, 4, 512
    J = random_model(L, q, 6)
    T = _tiles(J, L, q)
    mem = dev(oracle.pack_seqs(_seqs(L, q, N, 7)))
    st = dev(oracle.init_rng(N, 0, 10 ** 12))
    pos = dev(np.array([3, 99, 5], dtype="<u4"))
    status = empty((1,), np.int32)
    _lib.call("mi3_metropolis_skew", T.data_ptr(), st.data_ptr(), 0, pos.data_ptr(), 3, None, 1.0,
              mem.data_ptr(), N, L, q, 0, 0, status.data_ptr(), stream())
    assert int(host(status)[0]) == 3  # MI3_STATUS_BAD_INPUT


def test_skew_rejects_unsupported_shapes(cuda):
    status = empty((1,), np.int32)
    buf = empty((16,), np.float32)
    for L, q, N, wpc in [(20, 22, 512, 0), (258, 4, 512, 512), (546, 4, 512, 0), (20, 4, 500, 0),
                         (20, 4, 1024, 640)]:
        with pytest.raises(_lib.Mi3Error):
            _lib.call("mi3_metropolis_skew", buf.data_ptr(), buf.data_ptr(), 0, buf.data_ptr(), 1, None, 1.0,
                      buf.data_ptr(), N, L, q, wpc, 1, status.data_ptr(), stream())
