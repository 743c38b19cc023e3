"""The CPU oracle pinned against the reference's own code (golden vectors
from tests/golden/make_golden.py) and against invariants of the reference's
RNG test bench (mwc64x/test/test_mwc64xvec2.cl)."""
import numpy as np
import pytest

from oracle import oracle


@pytest.mark.parametrize("tag", ["a", "b"])
def test_init_rng_matches_reference_source(golden, tag):
    st = oracle.init_rng(64, int(golden[f"rng_{tag}_offset"]), int(golden[f"rng_{tag}_span"]))
    np.testing.assert_array_equal(st, golden[f"rng_{tag}_states"])


@pytest.mark.parametrize("tag", ["a", "b"])
def test_rng_draws_match_reference_source(golden, tag):
    st = golden[f"rng_{tag}_states"]
    for k, g in enumerate((0, 1, 63)):
        s = st[g].copy()
        d = oracle.rng_stream(s, 32)
        np.testing.assert_array_equal(d, golden[f"rng_{tag}_draws"][k])


@pytest.mark.parametrize("dist", [0, 1, 17, 4095, 2 ** 40 + 3])
def test_rng_skip_matches_reference_source(golden, dist):
    import ctypes
    s = golden["rng_skip_base"].copy()
    lib = oracle.lib()
    for lane in (0, 1):
        x = ctypes.c_uint32(int(s[lane]))
        c = ctypes.c_uint32(int(s[2 + lane]))
        lib.mi3o_mwc_skip(ctypes.byref(x), ctypes.byref(c), dist)
        s[lane], s[2 + lane] = x.value, c.value
    np.testing.assert_array_equal(s, golden[f"rng_skip_{dist}"])


def test_rng_skip_equals_stepping():
    """Skip(d) == d calls of NextUint2 (test_mwc64xvec2.cl:1-20)."""
    import ctypes
    base = np.array([7, 11, 13, 17], np.uint32)
    lib = oracle.lib()
    for dist in (0, 1, 2, 5, 100, 1000):
        stepped = base.copy()
        oracle.rng_stream(stepped, dist)
        s = base.copy()
        for lane in (0, 1):
            x, c = ctypes.c_uint32(int(s[lane])), ctypes.c_uint32(int(s[2 + lane]))
            lib.mi3o_mwc_skip(ctypes.byref(x), ctypes.byref(c), dist)
            s[lane], s[2 + lane] = x.value, c.value
        np.testing.assert_array_equal(s, stepped)


def test_rng_streams_partition():
    """Walker g's stream starts where walker g-1's span ends: streams seeded
    with span S equal one stream stepped S draws (dump_samples invariant,
    mwc64x/test/makefile:45-64)."""
    span = 40
    st = oracle.init_rng(3, 0, span)
    # lane v of walker g starts at distance (2g+v)*span: lane 0 of walker 0
    # stepped 2*span draws reaches lane 0 of walker 1.
    s = st[0].copy()
    d = oracle.rng_stream(s, 2 * span)
    assert s[0] == st[1][0] and s[2] == st[1][2]
    assert d.shape == (2 * span, 2)


@pytest.mark.parametrize("tag", ["A", "B", "C"])
def test_energies_match_E_potts(golden, tag):
    J, seqs = golden[f"m{tag}_J"], golden[f"m{tag}_seqs"]
    N, L = seqs.shape
    q = int(round(np.sqrt(J.shape[1])))
    mem = oracle.pack_seqs(seqs)
    e64 = oracle.energies_f64(J, mem, L, q)
    np.testing.assert_allclose(e64, golden[f"m{tag}_E64"], rtol=0, atol=1e-9)
    ek = oracle.energies_kahan(J, mem, L, q)
    scale = np.maximum(1.0, np.abs(golden[f"m{tag}_E64"]))
    assert np.max(np.abs(ek - golden[f"m{tag}_E64"]) / scale) < 1e-5


@pytest.mark.parametrize("tag", ["A", "B", "C"])
def test_bicounts_match_getMarginals(golden, tag):
    J, seqs = golden[f"m{tag}_J"], golden[f"m{tag}_seqs"]
    N, L = seqs.shape
    q = int(round(np.sqrt(J.shape[1])))
    c = oracle.bicounts(oracle.pack_seqs(seqs), L, q)
    np.testing.assert_array_equal(c, golden[f"m{tag}_bicounts"])


@pytest.mark.parametrize("tag", ["A", "B", "C"])
def test_weighted_marg_matches_getMarginals(golden, tag):
    J, seqs, w = golden[f"m{tag}_J"], golden[f"m{tag}_seqs"], golden[f"m{tag}_w"]
    N, L = seqs.shape
    q = int(round(np.sqrt(J.shape[1])))
    c = oracle.weighted_marg_f64(w, oracle.pack_seqs(seqs), L, q)
    np.testing.assert_allclose(c, golden[f"m{tag}_wcounts"], rtol=1e-12, atol=1e-12)


def test_pack_roundtrip(golden):
    seqs = golden["mA_seqs"]
    mem = oracle.pack_seqs(seqs)
    assert mem.shape == (oracle.swords(seqs.shape[1]), seqs.shape[0])
    np.testing.assert_array_equal(oracle.unpack_seqs(mem, seqs.shape[1]), seqs)


def test_unpack_j_layout(golden):
    J = golden["mA_J"]
    L, q = 10, 5
    Ju = oracle.unpack_j(J, L, q)
    stride = oracle.jrow_stride(L, q)
    assert Ju.shape == (L, stride) and stride % 4 == 0
    n = 0
    for i in range(L - 1):
        for j in range(i + 1, L):
            blk = J[n].reshape(q, q)
            np.testing.assert_array_equal(Ju[i, j * q * q:(j + 1) * q * q].reshape(q, q), blk)
            np.testing.assert_array_equal(Ju[j, i * q * q:(i + 1) * q * q].reshape(q, q), blk.T)
            n += 1
    for i in range(L):
        assert not Ju[i, i * q * q:(i + 1) * q * q].any()


def test_accept_rule():
    lib = oracle.lib()
    assert lib.mi3o_accept(0.0, 0.999999) == 1
    assert lib.mi3o_accept(-1.0, 0.5) == 0        # e^-1 = 0.37 < 0.5
    assert lib.mi3o_accept(-1.0, 0.367879) == 1
    assert lib.mi3o_accept(-1.0, 0.3679) == 0
    assert lib.mi3o_accept(-200.0, 0.0) == 0      # underflows to 0, not > 0
    assert lib.mi3o_accept(-50.0, 0.0) == 1


def test_metropolis_single_walker_by_hand():
    """Oracle sampler vs a direct Python restatement of DeltaEnergy +
    accept (mcmc.cl:360-458) for a few walkers and steps."""
    rng = np.random.default_rng(5)
    L, q, N = 7, 3, 4
    J = rng.normal(0, 0.7, size=(L * (L - 1) // 2, q * q)).astype("<f4")
    seqs = rng.integers(0, q, size=(N, L)).astype("<u1")
    st = oracle.init_rng(N, 0, 1000)
    pos = rng.integers(0, L, size=50).astype("<u4")
    mem = oracle.pack_seqs(seqs)
    st_o = st.copy()
    oracle.metropolis(J, st_o, pos, 0, 50, mem, L, q)
    out = oracle.unpack_seqs(mem, L)
    Ju = oracle.unpack_j(J, L, q)
    for g in range(N):
        s = seqs[g].copy()
        state = st[g].copy()
        for i in range(50):
            p = int(pos[i])
            r = oracle.rng_stream(state, 1)[0]
            mut = int(r[0]) % q
            cur = int(s[p])
            dE = np.float32(0)
            for m in range(L):
                if m == p:
                    continue
                a = Ju[p, m * q * q + q * mut + s[m]]
                b = Ju[p, m * q * q + q * cur + s[m]]
                dE = np.float32(dE + np.float32(a - b))
            u = np.float32((int(r[1]) >> 8) * 2.0 ** -24)
            x = np.float32(-dE)
            acc = True if x >= 0 else np.float32(np.exp(np.float64(x))) > u
            if acc:
                s[p] = mut
        np.testing.assert_array_equal(out[g], s)
        np.testing.assert_array_equal(st_o[g], state)


def test_renormalize_and_tree_sums():
    rng = np.random.default_rng(3)
    bi = rng.uniform(0, 1, size=(20, 21 * 21)).astype("<f4")
    r = oracle.renormalize_bimarg(bi, 21)
    np.testing.assert_allclose(r.sum(axis=1), 1.0, rtol=1e-5)


def test_zero_gauge_block_properties():
    rng = np.random.default_rng(4)
    for q in (2, 3, 4, 5, 21):
        Jb = rng.normal(size=q * q).astype("<f4")
        J0 = np.zeros_like(Jb)
        oracle.lib().mi3o_zero_gauge_block(Jb, J0, q)
        M = J0.reshape(q, q).astype(np.float64)
        assert np.abs(M.sum(axis=0)).max() < 1e-5 and np.abs(M.sum(axis=1)).max() < 1e-5


def test_min_weights_stats():
    rng = np.random.default_rng(6)
    x = rng.normal(0, 3, size=5000).astype("<f4")
    assert oracle.min_floats(x) == np.float32(min(0.0, x.min()))
    assert oracle.min_floats(np.abs(x)) == 0.0
    w = oracle.dE_to_weights(-1.5, x)
    arg = (-x + np.float32(-1.5)).astype(np.float64)  # the float argument of exp
    np.testing.assert_allclose(w, np.exp(arg), rtol=2.5e-7)
    s = oracle.weight_stats(w)
    s64 = oracle.weight_stats_f64(w)
    np.testing.assert_allclose(s, s64, rtol=1e-5)


def test_gauge_fieldless_even_matches_reference(golden):
    """The oracle's gauge transform against the reference's own
    fieldlessGaugeEven on the golden (h, J)."""
    h, J = golden["g_h"], golden["g_J"]
    L, q = h.shape
    out = oracle.gauge_fieldless_even(J, L, q, h=h)
    np.testing.assert_allclose(out, golden["g_fe_J"], rtol=0, atol=1e-12)


def test_bimarg_stats_f64_matches_host_formula():
    from mi3gpu_b200.potts import bimarg_stats
    rng = np.random.default_rng(11)
    L, q = 9, 5
    npair = L * (L - 1) // 2
    t = rng.dirichlet(np.ones(q * q), size=npair).astype("<f4")
    m = (t * rng.uniform(0.8, 1.2, size=t.shape)).astype("<f4")
    J = rng.normal(size=t.shape).astype("<f4")
    ssr, maxd, rel, cnt, xm, xt = oracle.bimarg_stats_f64(t, m, J)
    ferr, ssr2, maxd2 = bimarg_stats(t.astype(np.float64), m.astype(np.float64))
    assert abs(ssr - ssr2) <= 1e-14 * ssr2 and maxd == maxd2
    np.testing.assert_allclose(rel, ferr, rtol=1e-12)
    assert cnt == int(np.sum(t > np.float32(0.01)))
    # X with the pair's own marginals, summed over all pairs
    t64, m64, J64 = t.astype(np.float64), m.astype(np.float64), J.astype(np.float64)
    xm2 = sum(float(np.sum(J64[p].reshape(q, q) * (m64[p].reshape(q, q) - np.outer(m64[p].reshape(q, q).sum(1),
                                                                               m64[p].reshape(q, q).sum(0)))))
              for p in range(npair))
    np.testing.assert_allclose(xm, xm2, rtol=1e-10)


def test_validate_bimarg_matches_reference_messages():
    """potts.validate_bimarg accepts and rejects what the reference's
    validate_bimarg does (potts_common.py:50-76), with its messages
    (tests/golden/validate_vectors.npz)."""
    from pathlib import Path
    from mi3gpu_b200 import potts
    g = np.load(Path(__file__).parent / "golden" / "validate_vectors.npz")
    tags = sorted({k[:-3] for k in g.files if k.endswith("_in")})
    assert len(tags) == 5
    for tag in tags:
        want = str(g[tag + "_msg"])
        if not want:
            potts.validate_bimarg(g[tag + "_in"])
        else:
            with pytest.raises(ValueError) as e:
                potts.validate_bimarg(g[tag + "_in"])
            assert str(e.value) == want, tag


def test_check_target_rejects_what_the_reference_rejects():
    from pathlib import Path
    from mi3gpu_b200 import potts
    g = np.load(Path(__file__).parent / "golden" / "validate_vectors.npz")
    ff = g["valid_in"]
    potts.check_target(ff)
    with pytest.raises(Exception, match="'f4' format"):
        potts.check_target(ff.astype('f8'))
    z = ff.copy()
    z[3, 5] = 0
    with pytest.raises(Exception, match="0 < f < 1"):
        potts.check_target(z)


def test_gauge_change_shifts_every_energy_by_one_constant():
    """The intent of the reference's changeGauge.test_transform
    (changeGauge.py:181-201): a gauge change leaves energy differences
    unchanged.  Couplings uniform on [0, 1) (the reference test's, far from
    any gauge) moved to the fieldless-even gauge (FP64 oracle): the energies
    of random sequences, summed in FP64, all shift by one constant."""
    L, q = 9, 5
    rng = np.random.default_rng(1234)
    J = rng.random((L * (L - 1) // 2, q * q))
    Jg = oracle.gauge_fieldless_even(J, L, q)
    seqs = rng.integers(0, q, size=(200, L))
    pairs = [(i, j) for i in range(L - 1) for j in range(i + 1, L)]

    def energies(C):
        return sum(C[p, q * seqs[:, i] + seqs[:, j]] for p, (i, j) in enumerate(pairs))
    d = energies(Jg) - energies(J)
    assert abs(d.mean()) > 1.0  # the gauge did move the couplings
    assert np.ptp(d) < 1e-9 * np.abs(d).max()


def test_fp64_energies_against_32_digit_sums():
    """The intent of the reference's Mi3.getEnergiesMultiPrec (Mi3.py:79-90,
    mpmath at 32 digits): the FP64 oracle that bounds the device energies
    (1e-5 relative) is itself within 1e-12 of 32-digit sums of the same
    float32 couplings, at the reference-sized L=232, q=21."""
    mpmath = pytest.importorskip("mpmath")
    L, q, n = 232, 21, 6
    rng = np.random.default_rng(232)
    J = rng.normal(0, 0.5, size=(L * (L - 1) // 2, q * q)).astype("<f4")
    seqs = rng.integers(0, q, size=(n, L)).astype("<u1")
    E = oracle.energies_f64(J, oracle.pack_seqs(seqs), L, q)
    i, j = np.triu_indices(L, 1)
    mpmath.mp.dps = 32
    for k in range(n):
        s = seqs[k].astype(np.int64)
        terms = J[np.arange(len(i)), q * s[i] + s[j]]
        exact = mpmath.fsum(mpmath.mpf(float(t)) for t in terms)
        assert abs(E[k] - float(exact)) <= 1e-12 * max(1.0, abs(float(exact)))


def _reference_checkout():
    import os
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    cand = Path(os.environ.get("MI3_REFERENCE") or root.parent / "reference")
    return cand if (cand / "mi3gpu").is_dir() else None


@pytest.mark.parametrize("script,fixture", [("make_golden.py", "reference_vectors.npz"),
                                            ("make_msa_golden.py", "msa_vectors.npz"),
                                            ("make_validate_golden.py", "validate_vectors.npz"),
                                            ("make_hiv_fixture.py", "hiv_bimarg_pc.npz")])
def test_golden_fixtures_regenerate_from_the_reference(tmp_path, script, fixture):
    """Where the reference checkout is present, each committed fixture is
    exactly what its committed script makes from the reference's own code
    (its numpy utilities, seqload, MWC64X source compiled as C++, the HIV
    example's target).  Skipped elsewhere: every other test reads only the
    committed .npz files."""
    import subprocess
    import sys
    from pathlib import Path
    ref = _reference_checkout()
    if ref is None:
        pytest.skip("reference checkout not present")
    root = Path(__file__).resolve().parents[1]
    if script == "make_golden.py" and not (root / "oracle" / "_ref" / "libmwc64x_ref.so").exists():
        pytest.skip("oracle/_ref not built")
    out = tmp_path / fixture
    p = subprocess.run([sys.executable, str(root / "tests" / "golden" / script), "--ref", str(ref), "--out", str(out)],
                       capture_output=True, text=True, timeout=600, cwd=root)
    assert p.returncode == 0, p.stderr[-2000:]
    a, b = np.load(out), np.load(root / "tests" / "golden" / fixture)
    assert sorted(a.files) == sorted(b.files)
    for k in a.files:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_oracle_and_reference_cpu_samplers_match_exact_bimarginals():
    """The oracle's restatement of the metropolis kernel (bit-exact with the
    B200 samplers in the GPU tests) and the reference's own CPU sampler
    (extras/mcmcCPUgenThreaded.c, 16 chains) both sample the Boltzmann
    distribution: at L=8, q=3 all 3^8 states are weighted exactly; 4096
    oracle walkers after 60 sweeps, and 4096 reference samples, have
    bimarginals within the finite-sample error sum f(1 - f)/N of the exact
    ones and of each other.  The reference sampler's step adds the diagonal
    blocks of its coupling matrix, which it never writes
    (mcmcCPUgenThreaded.c:75-78, :194); MALLOC_PERTURB_ gives that memory one
    byte pattern, whose difference in dE is exactly 0, where leftover heap
    content would bias small models like this one."""
    import os
    import subprocess
    import tempfile
    from pathlib import Path
    L, q, N, sweeps = 8, 3, 4096, 60
    rng = np.random.default_rng(88)
    J = rng.normal(0, 0.45, size=(L * (L - 1) // 2, q * q)).astype("<f4")
    i, j = np.triu_indices(L, 1)
    idx = np.arange(q ** L)
    S = np.stack([(idx // q ** (L - 1 - k)) % q for k in range(L)], axis=1)
    E = sum(J[p].astype(np.float64)[S[:, i[p]] * q + S[:, j[p]]] for p in range(len(i)))
    w = np.exp(-(E - E.min()))
    w /= w.sum()
    f = np.stack([np.bincount(S[:, a] * q + S[:, b], weights=w, minlength=q * q) for a, b in zip(i, j)])

    def bimarg(seqs):
        return np.stack([np.bincount(seqs[:, a] * q + seqs[:, b], minlength=q * q) / len(seqs)
                         for a, b in zip(i, j)])

    mem = oracle.pack_seqs(rng.integers(0, q, size=(N, L)).astype("<u1"))
    st = oracle.init_rng(N, 0, 2 ** 63 // (2 * N))
    pos = rng.integers(0, L, size=sweeps * L).astype("<u4")
    oracle.metropolis(J, st, pos, 0, sweeps * L, mem, L, q)
    f_or = bimarg(oracle.unpack_seqs(mem, L).astype(np.int64))
    exp_or = float(np.sum(f * (1 - f)) / N)
    assert np.sum((f_or - f) ** 2) < 1.5 * exp_or

    exe = oracle.ref_cpu_binary()
    if exe is None:
        pytest.skip("reference CPU sampler not built (oracle/_ref)")
    alpha, burn, keep = "ABC", 4, 256
    env = dict(os.environ, MALLOC_PERTURB_="165")
    outs = []
    with tempfile.TemporaryDirectory() as td:
        jf = Path(td) / "J.dat"
        J.tofile(jf)
        for _ in range(16):
            start = "".join(alpha[k] for k in rng.integers(0, q, size=L))
            r = subprocess.run([str(exe), str(jf), str(10 * L), str(burn + keep), alpha, start], check=True,
                               capture_output=True, text=True, env=env)
            outs.append(np.array([[alpha.index(c) for c in ln] for ln in r.stdout.split()[burn:]]))
    seqs_ref = np.concatenate(outs)
    f_ref = bimarg(seqs_ref)
    exp_ref = float(np.sum(f * (1 - f)) / len(seqs_ref))
    assert np.sum((f_ref - f) ** 2) < 3.0 * exp_ref  # samples 10 sweeps apart within a chain
    assert np.sum((f_or - f_ref) ** 2) < 3.0 * exp_ref + 1.5 * exp_or
