"""GPU parity: every kernel of libmi3b200, called through the C ABI, against
the CPU oracle (itself pinned to the reference in test_oracle.py).

Integer/byte/index results are bit-exact; floating-point tolerances are
stated per test."""
import numpy as np
import pytest

from oracle import oracle
from mi3gpu_b200 import _lib
from tests._util import dev as _dev, host, empty, stream, random_model

_alive = []


def dev(a):
    """Device copy kept alive until the test module ends (a temporary
    passed as data_ptr() could be freed and reused before the launch)."""
    t = _dev(a)
    _alive.append(t)
    return t


@pytest.fixture(autouse=True)
def _release():
    yield
    import torch
    torch.cuda.synchronize()
    _alive.clear()

pytestmark = pytest.mark.gpu

SHAPES = [(10, 5, 512), (48, 4, 1024), (37, 21, 512), (93, 4, 512), (64, 8, 640)]


def _wmarg_ws(L, q, N):
    return empty((int(_lib.query("mi3_weighted_marg_workspace", L, q, N)) // 8 + 1,), np.int64)


def _seqs(L, q, N, seed):
    return np.random.default_rng(seed).integers(0, q, size=(N, L)).astype("<u1")


@pytest.mark.parametrize("n,off,span", [(4096, 0, 2 ** 63 // (2 * 4096)),
                                        (1024, 2 ** 62 + 12345, 987654321987),
                                        (512, 3 * (2 ** 61), 2 ** 40)])
def test_init_rng_bitexact(cuda, n, off, span):
    st = empty((n, 4), np.uint32)
    _lib.call("mi3_init_rng", st.data_ptr(), n, off, span, stream())
    np.testing.assert_array_equal(host(st, np.uint32), oracle.init_rng(n, off, span))


def test_init_rng_matches_reference_golden(cuda, golden):
    for tag in "ab":
        st = empty((64, 4), np.uint32)
        _lib.call("mi3_init_rng", st.data_ptr(), 64, int(golden[f"rng_{tag}_offset"]),
                  int(golden[f"rng_{tag}_span"]), stream())
        np.testing.assert_array_equal(host(st, np.uint32), golden[f"rng_{tag}_states"])


@pytest.mark.parametrize("L,q,N", SHAPES)
def test_unpack_j_bitexact(cuda, L, q, N):
    J = random_model(L, q, 1)
    stride = int(_lib.query("mi3_jrows_stride", L, q))
    Ju = empty((L, stride), np.float32)
    Ju.fill_(7.0)
    _lib.call("mi3_unpack_j", dev(J).data_ptr(), Ju.data_ptr(), L, q, stream())
    np.testing.assert_array_equal(host(Ju), oracle.unpack_j(J, L, q))


@pytest.mark.parametrize("L,q,N", SHAPES + [(26, 32, 512), (30, 40, 512), (2, 2, 128), (50, 21, 512)])
@pytest.mark.parametrize("nsteps", [1, 37, 300])
def test_metropolis_trajectory_bitexact(cuda, L, q, N, nsteps):
    """Same walkers, same RNG streams, same site list: identical sequences and
    RNG states after nsteps proposals (shapes with 5-bit and byte residues in
    shared memory, q=32 the largest 5-bit alphabet, q=40 above it, the
    smallest model L=2 q=2, and L=50 whose last 24-site chunk holds 2 sites,
    less than one 5-bit word)."""
    J = random_model(L, q, 2, sigma=0.5)
    seqs = _seqs(L, q, N, 3)
    mem = oracle.pack_seqs(seqs)
    st = oracle.init_rng(N, 0, 2 ** 63 // (2 * N))
    pos = np.random.RandomState(11).randint(0, L, size=nsteps + 13).astype("<u4")
    off = 13 if nsteps < 100 else 0
    stride = int(_lib.query("mi3_jrows_stride", L, q))
    Ju = empty((L, stride), np.float32)
    dJ, dmem, dst, dpos = dev(J), dev(mem), dev(st), dev(pos)
    status = empty((1,), np.int32)
    _lib.call("mi3_unpack_j", dJ.data_ptr(), Ju.data_ptr(), L, q, stream())
    _lib.call("mi3_metropolis", Ju.data_ptr(), dst.data_ptr(), off, dpos.data_ptr(), nsteps, None, 1.0,
              dmem.data_ptr(), N, L, q, status.data_ptr(), stream())
    g_mem, g_st = host(dmem, np.uint32), host(dst, np.uint32)
    assert int(host(status)[0]) == 0
    o_mem, o_st = mem.copy(), st.copy()
    oracle.metropolis(J, o_st, pos, off, nsteps, o_mem, L, q)
    np.testing.assert_array_equal(g_st, o_st)
    np.testing.assert_array_equal(g_mem, o_mem)
    assert (g_mem != mem).any()  # something was accepted


def test_metropolis_betas(cuda):
    L, q, N, nsteps = 20, 6, 512, 64
    J = random_model(L, q, 4, sigma=0.6)
    seqs = _seqs(L, q, N, 5)
    mem = oracle.pack_seqs(seqs)
    st = oracle.init_rng(N, 77, 10 ** 9)
    pos = np.random.RandomState(1).randint(0, L, size=nsteps).astype("<u4")
    betas = np.linspace(0.2, 2.0, N).astype("<f4")
    stride = int(_lib.query("mi3_jrows_stride", L, q))
    Ju = empty((L, stride), np.float32)
    dmem, dst = dev(mem), dev(st)
    status = empty((1,), np.int32)
    _lib.call("mi3_unpack_j", dev(J).data_ptr(), Ju.data_ptr(), L, q, stream())
    _lib.call("mi3_metropolis", Ju.data_ptr(), dst.data_ptr(), 0, dev(pos).data_ptr(), nsteps,
              dev(betas).data_ptr(), 1.0, dmem.data_ptr(), N, L, q, status.data_ptr(), stream())
    oracle.metropolis(J, st, pos, 0, nsteps, mem, L, q, betas=betas)
    np.testing.assert_array_equal(host(dmem, np.uint32), mem)
    np.testing.assert_array_equal(host(dst, np.uint32), st)


@pytest.mark.parametrize("L,q,N", SHAPES + [(232, 21, 512)])
def test_energies_vs_fp64(cuda, L, q, N):
    """|E - E_fp64| <= 1e-5 * max(1, |E_fp64|) (the bar); measured error is
    the float rounding of an exact-to-1e-12 sum."""
    J = random_model(L, q, 6)
    seqs = _seqs(L, q, N, 7)
    mem = oracle.pack_seqs(seqs)
    E = empty((N,), np.float32)
    ws = empty((int(_lib.query("mi3_energies_workspace", N)) // 8 + 1,), np.int64)
    _lib.call("mi3_energies", dev(J).data_ptr(), dev(mem).data_ptr(), N, N, E.data_ptr(), L, q, ws.data_ptr(),
              ws.numel() * 8, stream())
    e = host(E)
    e64 = oracle.energies_f64(J, mem, L, q)
    err = np.abs(e - e64) / np.maximum(1.0, np.abs(e64))
    assert err.max() <= 1e-5
    # deterministic: a second call gives identical bits
    E2 = empty((N,), np.float32)
    _lib.call("mi3_energies", dev(J).data_ptr(), dev(mem).data_ptr(), N, N, E2.data_ptr(), L, q, ws.data_ptr(),
              ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(E2), e)


def test_energies_golden(cuda, golden):
    for tag in "ABC":
        J, seqs = golden[f"m{tag}_J"], golden[f"m{tag}_seqs"]
        N, L = seqs.shape
        q = int(round(np.sqrt(J.shape[1])))
        E = empty((N,), np.float32)
        ws = empty((N + 1,), np.int64)
        _lib.call("mi3_energies", dev(J).data_ptr(), dev(oracle.pack_seqs(seqs)).data_ptr(), N, N, E.data_ptr(),
                  L, q, ws.data_ptr(), ws.numel() * 8, stream())
        e64 = golden[f"m{tag}_E64"]
        assert (np.abs(host(E) - e64) / np.maximum(1.0, np.abs(e64))).max() <= 1e-5


@pytest.mark.parametrize("L,q,N", SHAPES + [(232, 21, 1024)])
def test_bicounts_bitexact(cuda, L, q, N):
    seqs = _seqs(L, q, N, 8)
    mem = oracle.pack_seqs(seqs)
    out = empty((L * (L - 1) // 2, q * q), np.uint32)
    _lib.call("mi3_bicounts", dev(mem).data_ptr(), N, N, out.data_ptr(), L, q, stream())
    np.testing.assert_array_equal(host(out, np.uint32), oracle.bicounts(mem, L, q))


def test_bicounts_golden(cuda, golden):
    for tag in "ABC":
        J, seqs = golden[f"m{tag}_J"], golden[f"m{tag}_seqs"]
        N, L = seqs.shape
        q = int(round(np.sqrt(J.shape[1])))
        out = empty((L * (L - 1) // 2, q * q), np.uint32)
        _lib.call("mi3_bicounts", dev(oracle.pack_seqs(seqs)).data_ptr(), N, N, out.data_ptr(), L, q, stream())
        np.testing.assert_array_equal(host(out, np.uint32), golden[f"m{tag}_bicounts"])


def test_bicounts_partial_buffer(cuda):
    """nseq < buflen: only the first nseq columns are counted."""
    L, q, N = 30, 7, 1024
    seqs = _seqs(L, q, N, 9)
    mem = oracle.pack_seqs(seqs)
    out = empty((L * (L - 1) // 2, q * q), np.uint32)
    _lib.call("mi3_bicounts", dev(mem).data_ptr(), N, 700, out.data_ptr(), L, q, stream())
    np.testing.assert_array_equal(host(out, np.uint32), oracle.bicounts(mem, L, q, nseq=700))


@pytest.mark.parametrize("L,q,N", SHAPES)
def test_weighted_marg(cuda, L, q, N):
    """float accumulation vs double oracle: rtol 1e-5 of each pair's total."""
    seqs = _seqs(L, q, N, 10)
    mem = oracle.pack_seqs(seqs)
    w = np.random.default_rng(11).uniform(0.01, 3.0, size=N).astype("<f4")
    out = empty((L * (L - 1) // 2, q * q), np.float32)
    ws = _wmarg_ws(L, q, N)
    dw, dm = dev(w), dev(mem)
    _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, out.data_ptr(), L, q, None, ws.data_ptr(),
              ws.numel() * 8, stream())
    ref = oracle.weighted_marg_f64(w, mem, L, q)
    tot = ref.sum(axis=1, keepdims=True)
    got = host(out)
    assert (np.abs(got - ref) / tot).max() < 1e-5
    # integer (fixed-point) accumulation: a second call gives identical bits
    out2 = empty((L * (L - 1) // 2, q * q), np.float32)
    _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, out2.data_ptr(), L, q, None, ws.data_ptr(),
              ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(out2), got)


def test_weighted_marg_c1_shape_and_wide_weights(cuda):
    """L=232 q=21; weights spanning 6 decades (fixed-point shift adapts to
    the largest weight): still within 1e-5 of each pair's total."""
    L, q, N = 232, 21, 2048
    seqs = _seqs(L, q, N, 21)
    mem = oracle.pack_seqs(seqs)
    w = np.exp(np.random.default_rng(22).uniform(-14, 0, size=N)).astype("<f4")
    out = empty((L * (L - 1) // 2, q * q), np.float32)
    ws = _wmarg_ws(L, q, N)
    dw, dm = dev(w), dev(mem)
    _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, out.data_ptr(), L, q, None, ws.data_ptr(),
              ws.numel() * 8, stream())
    ref = oracle.weighted_marg_f64(w, mem, L, q)
    assert (np.abs(host(out) - ref) / ref.sum(axis=1, keepdims=True)).max() < 1e-5


def test_weighted_marg_golden(cuda, golden):
    for tag in "ABC":
        J, seqs, w = golden[f"m{tag}_J"], golden[f"m{tag}_seqs"], golden[f"m{tag}_w"]
        N, L = seqs.shape
        q = int(round(np.sqrt(J.shape[1])))
        out = empty((L * (L - 1) // 2, q * q), np.float32)
        ws = _wmarg_ws(L, q, N)
        _lib.call("mi3_weighted_marg", dev(w).data_ptr(), dev(oracle.pack_seqs(seqs)).data_ptr(), N, N,
                  out.data_ptr(), L, q, None, ws.data_ptr(), ws.numel() * 8, stream())
        ref = golden[f"m{tag}_wcounts"]
        assert (np.abs(host(out) - ref) / ref.sum(axis=1, keepdims=True)).max() < 1e-5


@pytest.mark.parametrize("q", [2, 4, 5, 8, 21])
def test_renormalize_bitexact(cuda, q):
    L = 17
    bi = np.random.default_rng(q).uniform(0, 1, size=(L * (L - 1) // 2, q * q)).astype("<f4")
    d = dev(bi)
    _lib.call("mi3_renormalize_bimarg", d.data_ptr(), L, q, stream())
    np.testing.assert_array_equal(host(d), oracle.renormalize_bimarg(bi, q))


def test_bicounts_to_bimarg(cuda):
    L, q = 12, 5
    c = np.random.default_rng(1).integers(0, 1000, size=(66, 25)).astype("<u4")
    out = empty((66, 25), np.float32)
    _lib.call("mi3_bicounts_to_bimarg", dev(c).data_ptr(), out.data_ptr(), 4096, L, q, stream())
    np.testing.assert_array_equal(host(out), oracle.bicounts_to_bimarg(c, 4096))


def test_update_j_bitexact(cuda):
    L, q = 40, 21
    rng = np.random.default_rng(12)
    n = (L * (L - 1) // 2, q * q)
    bt, bi = rng.uniform(0, 0.2, size=n).astype("<f4"), rng.uniform(0, 0.2, size=n).astype("<f4")
    Ji = rng.normal(0, 0.1, size=n).astype("<f4")
    d = dev(Ji)
    _lib.call("mi3_update_j", dev(bt).data_ptr(), dev(bi).data_ptr(), 4e-4, 1e-3, d.data_ptr(), d.data_ptr(),
              L, q, stream())
    np.testing.assert_array_equal(host(d), oracle.updatedJ(bt, bi, 4e-4, 1e-3, Ji))


@pytest.mark.parametrize("l2", [False, True])
@pytest.mark.parametrize("q", [2, 3, 4, 5, 8, 9, 11, 12, 16, 17, 21, 22, 23, 32])
def test_reg_lz_bitexact(cuda, l2, q):
    """Every cells-per-lane variant of the per-lane-tree kernel (q*q <= 512)
    and the generic kernel above it (q = 23, 32)."""
    L = 15
    rng = np.random.default_rng(13 + q)
    n = (L * (L - 1) // 2, q * q)
    bi = rng.uniform(0, 0.2, size=n).astype("<f4")
    J = rng.normal(0, 0.05, size=n).astype("<f4")
    dJ = rng.normal(0, 0.01, size=n).astype("<f4")
    d = dev(dJ)
    name = "mi3_reg_l2z" if l2 else "mi3_reg_l1z"
    _lib.call(name, dev(bi).data_ptr(), 4e-4, 1e-3, 2e-2, dev(J).data_ptr(), d.data_ptr(), L, q, stream())
    np.testing.assert_array_equal(host(d), oracle.reg_lz(bi, 4e-4, 1e-3, 2e-2, J, dJ, q, l2))


@pytest.mark.parametrize("n", [1, 1000, 262144, 1 << 20])
def test_min_weights_stats(cuda, n):
    rng = np.random.default_rng(n)
    dE = rng.normal(0, 2, size=n).astype("<f4")
    out = empty((1,), np.float32)
    _lib.call("mi3_min_floats", dev(dE).data_ptr(), n, out.data_ptr(), stream())
    assert host(out)[0] == oracle.min_floats(dE)
    w = empty((n,), np.float32)
    _lib.call("mi3_dE_to_weights", np.float32(-0.7), dev(dE).data_ptr(), w.data_ptr(), n, stream())
    wo = oracle.dE_to_weights(-0.7, dE)
    np.testing.assert_allclose(host(w), wo, rtol=3e-7)  # expf: 2 ulp
    ws = empty((int(_lib.query("mi3_weight_stats_workspace", n)) // 8 + 1,), np.int64)
    s2, s64 = empty((2,), np.float32), empty((2,), np.float64)
    _lib.call("mi3_weight_stats", w.data_ptr(), n, s2.data_ptr(), s64.data_ptr(), ws.data_ptr(), ws.numel() * 8,
              stream())
    ref64 = oracle.weight_stats_f64(host(w))
    np.testing.assert_allclose(host(s64), ref64, rtol=1e-12)
    np.testing.assert_allclose(host(s2), ref64, rtol=1e-6)
    # fused pass gives the same three results
    w2, mn = empty((n,), np.float32), empty((1,), np.float32)
    f2, f64 = empty((2,), np.float32), empty((2,), np.float64)
    _lib.call("mi3_weights_fused", np.float32(-0.7), dev(dE).data_ptr(), w2.data_ptr(), n, mn.data_ptr(),
              f2.data_ptr(), f64.data_ptr(), ws.data_ptr(), ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(w2), host(w))
    assert host(mn)[0] == oracle.min_floats(dE)
    np.testing.assert_array_equal(host(f64), host(s64))


def test_fixed_beta_and_add(cuda):
    n = 5000
    rng = np.random.default_rng(14)
    E = rng.normal(0, 5, size=n).astype("<f4")
    w = empty((n,), np.float32)
    _lib.call("mi3_fixed_beta_weights", np.float32(0.8), np.float32(-3.0), dev(E).data_ptr(), w.data_ptr(), n,
              stream())
    np.testing.assert_allclose(host(w), oracle.fixed_beta_weights(0.8, -3.0, E), rtol=3e-7)
    a, b = dev(E), dev(E * 2)
    _lib.call("mi3_add_float_bufs", a.data_ptr(), b.data_ptr(), n, stream())
    np.testing.assert_array_equal(host(a), E + E * 2)


@pytest.mark.parametrize("L,q", [(10, 5), (48, 4), (37, 21), (9, 2)])
def test_gen_indep_bitexact(cuda, L, q):
    N = 1024
    rng = np.random.default_rng(L * q)
    f = rng.uniform(0.1, 1, size=(L, q))
    f /= f.sum(axis=1, keepdims=True)
    cprob = np.cumsum(f, axis=1)
    cprob = (cprob[:, :-1] / cprob[:, -1, None]).astype("<f4")
    st = oracle.init_rng(N, 5, 10 ** 12)
    mem = np.zeros((oracle.swords(L), N), np.uint32)
    dmem, dst = dev(mem), dev(st)
    _lib.call("mi3_gen_indep", dmem.data_ptr(), N, N, dst.data_ptr(), dev(cprob).data_ptr(), L, q, stream())
    oracle.gen_indep(mem, st, cprob, L, q)
    np.testing.assert_array_equal(host(dmem, np.uint32), mem)
    np.testing.assert_array_equal(host(dst, np.uint32), st)


@pytest.mark.parametrize("L", [5, 48, 93])
def test_repack_T_bitexact(cuda, L):
    N = 1024
    seqs = _seqs(L, 21, N, L)
    mem = oracle.pack_seqs(seqs)
    out = empty((L, N // 4), np.uint32)
    _lib.call("mi3_repack_seqs_T", dev(mem).data_ptr(), N, out.data_ptr(), N // 4, L, stream())
    np.testing.assert_array_equal(host(out, np.uint32), oracle.repack_seqs_T(mem, L))
    np.testing.assert_array_equal(host(out, np.uint32).view(np.uint8), seqs.T)


REG_CASES = [("SCADJ", "mi3_reg_scadj", (0.02, 4.0)), ("X", "mi3_reg_x", (0.05,)), ("Xij", "mi3_reg_xij", ()),
             ("SCADX", "mi3_reg_scadx", (2.0, 0.05, 4.0)), ("expX", "mi3_reg_expx", (0.3,)),
             ("ddE", "mi3_reg_dde", (0.01,)), ("SCADddE", "mi3_reg_scaddde", (0.01, 0.02))]


@pytest.mark.parametrize("kind,entry,params", REG_CASES)
@pytest.mark.parametrize("q", [2, 4, 5, 21])
def test_reg_other_vs_oracle(cuda, kind, entry, params, q):
    """Bit-exact for every regularizer but expX (expf: 2 ulp -> rtol 1e-6)."""
    L = 9
    rng = np.random.default_rng(40 + q)
    n = (L * (L - 1) // 2, q * q)
    bi = rng.dirichlet(np.ones(q * q), size=n[0]).astype("<f4")
    J = rng.normal(0, 0.1, size=n).astype("<f4")
    dJ = rng.normal(0, 0.02, size=n).astype("<f4")
    lam = rng.uniform(0.01, 0.2, size=n[0]).astype("<f4")
    gamma, pc = 4e-3, 1e-2
    d = dev(dJ)
    head = [dev(bi).data_ptr()] + ([dev(lam).data_ptr()] if kind == "Xij" else [])
    if kind == "X":
        args = head + [np.float32(params[0]), gamma, pc]
    else:
        args = head + [gamma, pc] + list(params)
    _lib.call(entry, *args, dev(J).data_ptr(), d.data_ptr(), L, q, stream())
    ref = oracle.reg_other(kind, bi, gamma, pc, params, J, dJ, q, lambdas=lam if kind == "Xij" else None)
    got = host(d)
    assert not np.array_equal(ref, dJ)  # the penalty did something
    if kind == "expX":
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-9)
    else:
        np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("L,q,N", [(10, 5, 512), (48, 4, 16384), (37, 21, 1000), (93, 4, 3000), (64, 8, 640),
                                   (232, 21, 4096), (50, 32, 300), (13, 7, 130), (99, 4, 20000), (128, 8, 9000)])
def test_bicounts_tensorcore_bitexact(cuda, L, q, N):
    """FP8 one-hot GEMM counts on tcgen05 equal the integer histogram exactly
    (one chunk, or up to 19 chunks summed with atomics; partial last K
    step)."""
    seqs = _seqs(L, q, N, 50 + q)
    mem = oracle.pack_seqs(seqs)
    out = empty((L * (L - 1) // 2, q * q), np.uint32)
    out.fill_(-1)
    status = empty((1,), np.int32)
    dm = dev(mem)
    _lib.call("mi3_bicounts_tc", dm.data_ptr(), N, N, out.data_ptr(), L, q, status.data_ptr(), stream())
    assert int(host(status)[0]) == 0
    np.testing.assert_array_equal(host(out, np.uint32), oracle.bicounts(mem, L, q))


def test_bicounts_tensorcore_golden_and_partial(cuda, golden):
    for tag in "ABC":
        J, seqs = golden[f"m{tag}_J"], golden[f"m{tag}_seqs"]
        N, L = seqs.shape
        q = int(round(np.sqrt(J.shape[1])))
        out = empty((L * (L - 1) // 2, q * q), np.uint32)
        status = empty((1,), np.int32)
        dm = dev(oracle.pack_seqs(seqs))
        _lib.call("mi3_bicounts_tc", dm.data_ptr(), N, N, out.data_ptr(), L, q, status.data_ptr(), stream())
        np.testing.assert_array_equal(host(out, np.uint32), golden[f"m{tag}_bicounts"])
    # nseq < buflen: only the first nseq sequences
    L, q, N = 30, 6, 1024
    mem = oracle.pack_seqs(_seqs(L, q, N, 3))
    out = empty((L * (L - 1) // 2, q * q), np.uint32)
    status = empty((1,), np.int32)
    dm = dev(mem)
    _lib.call("mi3_bicounts_tc", dm.data_ptr(), N, 777, out.data_ptr(), L, q, status.data_ptr(), stream())
    np.testing.assert_array_equal(host(out, np.uint32), oracle.bicounts(mem, L, q, nseq=777))


@pytest.mark.parametrize("L,q", [(9, 4), (13, 21), (48, 4), (232, 21), (5, 2)])
def test_gauge_fieldless_even_vs_oracle(cuda, L, q):
    """FP64 device gauge transform vs the oracle's float64 restatement of
    fieldlessGaugeEven: equal after rounding to float up to one ulp."""
    rng = np.random.default_rng(L * q)
    npair = L * (L - 1) // 2
    J = (rng.normal(0, 0.3, size=(npair, q * q)) + rng.normal(0, 1, size=(npair, 1))).astype("<f4")
    ref = oracle.gauge_fieldless_even(J, L, q).astype("<f4")
    ws = empty((int(_lib.query("mi3_gauge_workspace", L, q)) // 8 + 1,), np.int64)
    dJ = dev(J)
    out = empty(J.shape, np.float32)
    _lib.call("mi3_gauge_fieldless_even", dJ.data_ptr(), out.data_ptr(), L, q, ws.data_ptr(), ws.numel() * 8,
              stream())
    got = host(out, np.float32)
    np.testing.assert_allclose(got, ref, rtol=2.5e-7, atol=1e-7 * np.abs(ref).max())
    # in place gives the same values
    _lib.call("mi3_gauge_fieldless_even", dJ.data_ptr(), dJ.data_ptr(), L, q, ws.data_ptr(), ws.numel() * 8,
              stream())
    np.testing.assert_array_equal(host(dJ, np.float32), got)
    # the gauge is idempotent up to rounding: zero row/column means already
    g2 = oracle.gauge_fieldless_even(got, L, q)
    np.testing.assert_allclose(g2, got, atol=1e-6 * np.abs(ref).max() + 1e-7)


@pytest.mark.parametrize("L,q", [(9, 4), (13, 21), (232, 21), (2, 3)])
@pytest.mark.parametrize("with_J", [True, False])
def test_bimarg_stats_vs_oracle(cuda, L, q, with_J):
    rng = np.random.default_rng(L + q)
    npair = L * (L - 1) // 2
    t = rng.dirichlet(np.full(q * q, 0.5), size=npair).astype("<f4")
    m = (t * rng.uniform(0.7, 1.3, size=t.shape)).astype("<f4")
    J = rng.normal(size=t.shape).astype("<f4")
    ref = oracle.bimarg_stats_f64(t, m, J if with_J else None)
    ws = empty((int(_lib.query("mi3_bimarg_stats_workspace", L)) // 8 + 1,), np.int64)
    out = empty((6,), np.float64)
    dt, dm, dj = dev(t), dev(m), dev(J)
    _lib.call("mi3_bimarg_stats", dt.data_ptr(), dm.data_ptr(), dj.data_ptr() if with_J else None, L, q,
              out.data_ptr(), ws.data_ptr(), ws.numel() * 8, stream())
    got = host(out, np.float64)
    np.testing.assert_allclose(got[[0, 2, 4, 5]], np.array(ref)[[0, 2, 4, 5]], rtol=1e-11, atol=1e-13)
    assert got[1] == ref[1] and got[3] == ref[3]
    # deterministic: a second call gives the same bits
    _lib.call("mi3_bimarg_stats", dt.data_ptr(), dm.data_ptr(), dj.data_ptr() if with_J else None, L, q,
              out.data_ptr(), ws.data_ptr(), ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(out, np.float64), got)


@pytest.mark.parametrize("L,q,N", [(20, 4, 200000), (64, 21, 300000), (232, 21, 200000)])
def test_weighted_marg_many_chunks(cuda, L, q, N):
    """Sizes whose histograms are split over many sequence chunks (the last
    one at the 65536-sequence fixed-point cap): per-chunk partial sums
    combined in fixed order, within 1e-5 of each pair's total and
    bit-identical on a second call."""
    seqs = _seqs(L, q, N, 31)
    mem = oracle.pack_seqs(seqs)
    w = np.exp(np.random.default_rng(32).normal(0, 1.0, size=N)).astype("<f4")
    out = empty((L * (L - 1) // 2, q * q), np.float32)
    ws = _wmarg_ws(L, q, N)
    dw, dm = dev(w), dev(mem)
    _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, out.data_ptr(), L, q, None, ws.data_ptr(),
              ws.numel() * 8, stream())
    got = host(out)
    ref = oracle.weighted_marg_f64(w, mem, L, q)
    assert (np.abs(got - ref) / ref.sum(axis=1, keepdims=True)).max() < 1e-5
    _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, out.data_ptr(), L, q, None, ws.data_ptr(),
              ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(out), got)
    # a workspace one byte short is rejected
    with pytest.raises(_lib.Mi3Error):
        _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, out.data_ptr(), L, q, None, ws.data_ptr(),
                  int(_lib.query("mi3_weighted_marg_workspace", L, q, N)) - 1, stream())


def _potts_like_seqs(L, q, N, seed, conc=2.0):
    """Sequences with per-site skewed residue frequencies (a frequent
    residue per site, as in equilibrated walkers)."""
    rng = np.random.default_rng(seed)
    p = rng.dirichlet(np.full(q, 1.0 / conc), size=L)
    u = rng.random((N, L))
    return (u[:, :, None] > np.cumsum(p, axis=1)[None]).sum(axis=2).clip(0, q - 1).astype("<u1")


@pytest.mark.parametrize("L,q,N", [(10, 5, 512), (37, 21, 1000), (9, 2, 3000), (232, 21, 4096)])
def test_site_consensus(cuda, L, q, N):
    seqs = _potts_like_seqs(L, q, N, L + q)
    cons = empty((L,), np.uint8)
    ws = empty((int(_lib.query("mi3_site_consensus_workspace", L, q)) // 8 + 1,), np.int64)
    _lib.call("mi3_site_consensus", dev(oracle.pack_seqs(seqs)).data_ptr(), N, N, L, q, cons.data_ptr(),
              ws.data_ptr(), ws.numel() * 8, stream())
    counts = np.stack([np.bincount(seqs[:, i], minlength=q) for i in range(L)])
    np.testing.assert_array_equal(host(cons), counts.argmax(axis=1))  # argmax: lowest index on ties


@pytest.mark.parametrize("L,q,N", [(10, 5, 512), (48, 4, 1024), (37, 21, 1000), (93, 4, 3000), (64, 8, 640),
                                   (9, 2, 3000), (20, 4, 200000), (64, 21, 300000), (29, 11, 5000)])
@pytest.mark.parametrize("which", ["consensus", "arbitrary"])
def test_weighted_marg_consensus_bitexact(cuda, L, q, N, which):
    """Skipping the consensus pairs and rebuilding their bins from site
    sums gives the same bits as the direct histogram, for the true
    consensus and for an arbitrary residue per site (including values >= q,
    which never match)."""
    seqs = _potts_like_seqs(L, q, N, 7 * L + q)
    mem = oracle.pack_seqs(seqs)
    w = np.exp(np.random.default_rng(L).normal(0, 1.5, size=N)).astype("<f4")
    if which == "consensus":
        cons = np.stack([np.bincount(seqs[:, i], minlength=q) for i in range(L)]).argmax(axis=1).astype("u1")
    else:
        cons = np.random.default_rng(q).integers(0, q + 2, size=L).astype("u1")
    ws = _wmarg_ws(L, q, N)
    dw, dm, dc = dev(w), dev(mem), dev(cons)
    a = empty((L * (L - 1) // 2, q * q), np.float32)
    b = empty((L * (L - 1) // 2, q * q), np.float32)
    _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, a.data_ptr(), L, q, None, ws.data_ptr(),
              ws.numel() * 8, stream())
    _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, b.data_ptr(), L, q, dc.data_ptr(),
              ws.data_ptr(), ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(b), host(a))
    if N * L * L < 4e9:
        ref = oracle.weighted_marg_f64(w, mem, L, q)
        assert (np.abs(host(b) - ref) / ref.sum(axis=1, keepdims=True)).max() < 1e-5


@pytest.mark.parametrize("L,q,N", [(10, 5, 512), (48, 4, 1024), (37, 21, 1000), (93, 4, 3000), (64, 8, 640),
                                   (9, 2, 3000), (232, 21, 2048), (29, 11, 5000)])
@pytest.mark.parametrize("which", ["consensus", "arbitrary"])
def test_energies_consensus_gauge(cuda, L, q, N, which):
    """Energies through the consensus gauge against the FP64 oracle, for
    the true consensus and for arbitrary reference residues.  The regauged
    couplings J' are rounded once to float (<= 2^-25 |J'| each) and summed
    in float rows of at most 16 terms (<= 2^-21 of the absolute row sum), and
    the energy is rounded once to float at the end, so
    |E - E64| <= 2^-20 * sum_pairs |J'(s_i, s_j)| + 2^-24 |E64|."""
    seqs = _potts_like_seqs(L, q, N, 3 * L + q)
    mem = oracle.pack_seqs(seqs)
    rng = np.random.default_rng(L * q)
    J = rng.normal(0, 0.3, size=(L * (L - 1) // 2, q * q)).astype("<f4")
    if which == "consensus":
        cons = np.stack([np.bincount(seqs[:, i], minlength=q) for i in range(L)]).argmax(axis=1).astype("u1")
    else:
        cons = rng.integers(0, q + 2, size=L).astype("u1")
    ws = empty((int(_lib.query("mi3_energies_cons_workspace", L, q, N)) // 8 + 1,), np.int64)
    E = empty((N,), np.float32)
    _lib.call("mi3_energies_cons", dev(J).data_ptr(), dev(mem).data_ptr(), N, N, E.data_ptr(), L, q,
              dev(cons).data_ptr(), ws.data_ptr(), ws.numel() * 8, stream())
    e64 = oracle.energies_f64(J, mem, L, q)
    got = host(E).astype(np.float64)
    # the regauged table in float64: J'(a,b) = J(a,b) - J(a,c_j) - J(c_i,b) + J(c_i,c_j)
    c = np.minimum(cons.astype(np.int64), q - 1)
    i, j = np.triu_indices(L, k=1)
    Jx = J.astype(np.float64).reshape(-1, q, q)
    P = np.arange(Jx.shape[0])
    Jg = Jx - Jx[P, :, c[j]][:, :, None] - Jx[P, c[i], :][:, None, :] + Jx[P, c[i], c[j]][:, None, None]
    eabs = oracle.energies_f64(np.abs(Jg).reshape(-1, q * q).astype("<f4"), mem, L, q)
    assert np.all(np.abs(got - e64) <= 2.0 ** -20 * eabs * 1.01 + 2.0 ** -24 * np.abs(e64) + 1e-9)
    # deterministic
    E2 = empty((N,), np.float32)
    _lib.call("mi3_energies_cons", dev(J).data_ptr(), dev(mem).data_ptr(), N, N, E2.data_ptr(), L, q,
              dev(cons).data_ptr(), ws.data_ptr(), ws.numel() * 8, stream())
    np.testing.assert_array_equal(host(E2), host(E))


@pytest.mark.parametrize("L,q,N", [(10, 5, 512), (48, 4, 1024), (37, 21, 1000), (93, 4, 3000), (64, 8, 640),
                                   (20, 4, 200000), (29, 11, 5000), (232, 21, 2048), (99, 4, 1 << 16)])
def test_weighted_marg_tensorcore_bitexact(cuda, L, q, N):
    """tcgen05 integer one-hot GEMM (three weight byte planes) gives the
    same bits as the shared-memory fixed-point histogram, and both are
    within 1e-5 of each pair's total of the FP64 oracle."""
    seqs = _potts_like_seqs(L, q, N, 11 * L + q)
    mem = oracle.pack_seqs(seqs)
    w = np.exp(np.random.default_rng(L + N).normal(0, 2.0, size=N)).astype("<f4")
    dw, dm = dev(w), dev(mem)
    a = empty((L * (L - 1) // 2, q * q), np.float32)
    b = empty((L * (L - 1) // 2, q * q), np.float32)
    ws = _wmarg_ws(L, q, N)
    _lib.call("mi3_weighted_marg", dw.data_ptr(), dm.data_ptr(), N, N, a.data_ptr(), L, q, None, ws.data_ptr(),
              ws.numel() * 8, stream())
    wst = empty((int(_lib.query("mi3_weighted_marg_tc_workspace", L, q)) // 8 + 1,), np.int64)
    status = empty((1,), np.int32)
    _lib.call("mi3_weighted_marg_tc", dw.data_ptr(), dm.data_ptr(), N, N, b.data_ptr(), L, q, wst.data_ptr(),
              wst.numel() * 8, status.data_ptr(), stream())
    assert int(host(status, np.int32)[0]) == 0
    np.testing.assert_array_equal(host(b), host(a))
    if N * L * L < 4e9:
        ref = oracle.weighted_marg_f64(w, mem, L, q)
        assert (np.abs(host(b) - ref) / ref.sum(axis=1, keepdims=True)).max() < 1e-5


def test_weighted_marg_tensorcore_rejects_bad_q(cuda):
    ws = empty((16,), np.int64)
    st = empty((1,), np.int32)
    with pytest.raises(_lib.Mi3Error):
        _lib.call("mi3_weighted_marg_tc", ws.data_ptr(), ws.data_ptr(), 512, 512, ws.data_ptr(), 10, 2,
                  ws.data_ptr(), 128, st.data_ptr(), stream())


@pytest.mark.parametrize("L,q,N", [(10, 5, 512), (48, 4, 1024), (37, 21, 1000), (93, 4, 3000), (64, 8, 640),
                                   (29, 11, 5000), (99, 4, 1 << 16), (150, 6, 4096), (33, 32, 700)])
def test_energies_tensorcore_vs_fp64(cuda, L, q, N):
    """BF16 hi/lo one-hot GEMM energies (tcgen05) against the FP64 oracle
    within the stated bound 2^-15 sum|J(s_i,s_j)| + 2^-24 |E|, and
    deterministic."""
    seqs = _potts_like_seqs(L, q, N, 13 * L + q)
    mem = oracle.pack_seqs(seqs)
    J = np.random.default_rng(L * q + 1).normal(0, 0.3, size=(L * (L - 1) // 2, q * q)).astype("<f4")
    ws = empty((N + 1,), np.int64)
    st = empty((1,), np.int32)
    E = empty((N,), np.float32)
    dJ, dm = dev(J), dev(mem)
    _lib.call("mi3_energies_tc", dJ.data_ptr(), dm.data_ptr(), N, N, E.data_ptr(), L, q, ws.data_ptr(),
              ws.numel() * 8, st.data_ptr(), stream())
    assert int(host(st, np.int32)[0]) == 0
    e64 = oracle.energies_f64(J, mem, L, q)
    eabs = oracle.energies_f64(np.abs(J), mem, L, q)
    got = host(E).astype(np.float64)
    assert np.all(np.abs(got - e64) <= 2.0 ** -15 * eabs + 2.0 ** -24 * np.abs(e64) + 1e-9)
    E2 = empty((N,), np.float32)
    _lib.call("mi3_energies_tc", dJ.data_ptr(), dm.data_ptr(), N, N, E2.data_ptr(), L, q, ws.data_ptr(),
              ws.numel() * 8, st.data_ptr(), stream())
    np.testing.assert_array_equal(host(E2), host(E))
