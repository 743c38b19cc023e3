"""numpy front end of the CPU oracle (oracle/mi3_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU legs of bench.py as the checker (or the timed CPU port).  The
library in mi3gpu_b200 never imports it.

Each function restates one kernel of the reference's mi3gpu/mcmc.cl (or a
host routine of mi3gpu/mcmcGPU.py) -- the C file cites the lines -- and
takes/returns arrays in the reference's layouts.
"""
import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = HERE / "_build" / "libmi3oracle.so"
_REF_RNG = HERE / "_ref" / "libmwc64x_ref.so"
_REF_CPU = HERE / "_ref" / "mcmc_cpu"

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_c = ctypes


def _build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            _build()
        L = ctypes.CDLL(str(_LIB))
        sig = {
            "mi3o_init_rng": [_u32p, _c.c_uint32, _c.c_uint64, _c.c_uint64],
            "mi3o_vec2_next": [_u32p, _c.POINTER(_c.c_uint32), _c.POINTER(_c.c_uint32)],
            "mi3o_mwc_skip": [_c.POINTER(_c.c_uint32), _c.POINTER(_c.c_uint32), _c.c_uint64],
            "mi3o_accept": [_c.c_float, _c.c_float],
            "mi3o_unpack_j": [_f32p, _f32p, _c.c_uint32, _c.c_uint32, _c.c_uint64],
            "mi3o_metropolis": [_f32p, _c.c_uint64, _u32p, _c.c_uint32, _u32p, _c.c_uint32,
                                _c.c_void_p, _c.c_float, _u32p, _c.c_uint32, _c.c_uint32,
                                _c.c_uint32, _c.c_uint32, _c.c_uint32],
            "mi3o_energies_kahan": [_f32p, _u32p, _c.c_uint32, _c.c_uint32, _f32p, _c.c_uint32, _c.c_uint32],
            "mi3o_energies_f64": [_f32p, _u32p, _c.c_uint32, _c.c_uint32, _f64p, _c.c_uint32, _c.c_uint32],
            "mi3o_count_bivariate": [_u32p, _c.c_uint32, _c.c_uint32, _u32p, _c.c_uint32, _c.c_uint32],
            "mi3o_bicounts_to_bimarg": [_u32p, _f32p, _c.c_uint32, _c.c_uint64],
            "mi3o_min_floats": [_f32p, _c.c_uint32],
            "mi3o_weight_stats": [_f32p, _c.c_uint32, _f32p],
            "mi3o_weight_stats_f64": [_f32p, _c.c_uint32, _f64p],
            "mi3o_dE_to_weights": [_c.c_float, _f32p, _f32p, _c.c_uint32],
            "mi3o_fixed_beta_weights": [_c.c_float, _c.c_float, _f32p, _f32p, _c.c_uint32],
            "mi3o_weighted_marg_f64": [_f32p, _u32p, _c.c_uint32, _c.c_uint32, _f64p, _c.c_uint32, _c.c_uint32],
            "mi3o_renormalize_bimarg": [_f32p, _c.c_uint64, _c.c_uint32],
            "mi3o_zero_gauge_block": [_f32p, _f32p, _c.c_uint32],
            "mi3o_updatedJ": [_f32p, _f32p, _c.c_float, _c.c_float, _f32p, _f32p, _c.c_uint64],
            "mi3o_reg_lz": [_f32p, _c.c_float, _c.c_float, _c.c_float, _f32p, _f32p, _c.c_uint64,
                            _c.c_uint32, _c.c_int],
            "mi3o_reg_other": [_c.c_int, _f32p, _c.c_void_p, _c.c_float, _c.c_float, _c.c_float, _c.c_float,
                               _c.c_float, _f32p, _f32p, _c.c_uint64, _c.c_uint32],
            "mi3o_gen_indep": [_u32p, _c.c_uint32, _c.c_uint32, _u32p, _f32p, _c.c_uint32, _c.c_uint32],
            "mi3o_repack_seqs_T": [_u32p, _c.c_uint32, _u8p, _c.c_uint32, _c.c_uint32],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
        L.mi3o_accept.restype = _c.c_int
        L.mi3o_min_floats.restype = _c.c_float
        _lib = L
    return _lib


def ref_rng_lib():
    """The reference's own mwc64x .cl sources compiled as C++ (oracle/_ref),
    or None when they were not built (no reference tree)."""
    if not _REF_RNG.exists():
        try:
            _build()
        except Exception:
            return None
    if not _REF_RNG.exists():
        return None
    L = ctypes.CDLL(str(_REF_RNG))
    L.ref_init_rng2.argtypes = [_u32p, _c.c_uint32, _c.c_uint64, _c.c_uint64]
    L.ref_vec2_stream.argtypes = [_u32p, _c.c_uint32, _u32p]
    L.ref_vec2_skip.argtypes = [_u32p, _c.c_uint64]
    L.ref_scalar_seed.argtypes = [_c.c_uint64, _c.c_uint64, _c.c_uint64, _u32p]
    L.ref_scalar_stream.argtypes = [_u32p, _c.c_uint32, _u32p]
    L.ref_scalar_skip.argtypes = [_u32p, _c.c_uint64]
    return L


def ref_cpu_binary():
    """Path of the reference's CPU generator built here, or None."""
    if not _REF_CPU.exists():
        try:
            _build()
        except Exception:
            return None
    return _REF_CPU if _REF_CPU.exists() else None


# --------------------------------------------------------------- layouts
def swords(L):
    return (L - 1) // 4 + 1


def pack_seqs(seqs):
    """MCMCGPU.packSeqs_4 (mcmcGPU.py:333-347): (N, L) u1 -> (SWORDS, N) u4."""
    seqs = np.asarray(seqs, dtype=np.uint8)
    N, L = seqs.shape
    sb = np.zeros((N, 4 * swords(L)), dtype=np.uint8)
    sb[:, :L] = seqs
    return np.ascontiguousarray(sb.view("<u4").T)


def unpack_seqs(mem, L):
    """MCMCGPU.unpackSeqs_4 (mcmcGPU.py:349-354)."""
    mem = np.asarray(mem, dtype=np.uint32)
    b = np.ascontiguousarray(mem.T).view(np.uint8)
    return b[:, :L].copy()


def jrow_stride(L, q):
    n = L * q * q
    return (n + 3) & ~3


def npairs(L):
    return L * (L - 1) // 2


# ------------------------------------------------------------- kernels
def init_rng(n, offset, span):
    st = np.zeros(4 * n, np.uint32)
    lib().mi3o_init_rng(st, n, int(offset), int(span))
    return st.reshape(n, 4)


def rng_stream(state, count):
    """count vec2 draws from one walker state (modified in place)."""
    s = np.ascontiguousarray(state, dtype=np.uint32).copy()
    out = np.zeros((count, 2), np.uint32)
    r0, r1 = _c.c_uint32(), _c.c_uint32()
    for k in range(count):
        lib().mi3o_vec2_next(s, _c.byref(r0), _c.byref(r1))
        out[k] = (r0.value, r1.value)
    state[:] = s
    return out


def unpack_j(J, L, q):
    J = np.ascontiguousarray(J, dtype=np.float32)
    stride = jrow_stride(L, q)
    Ju = np.zeros(L * stride, np.float32)
    lib().mi3o_unpack_j(J, Ju, L, q, stride)
    return Ju.reshape(L, stride)


def unpack_j_tiles(J, L, q):
    """The chunk-tiled coupling layout of the skewed sampler: for each site
    pos, ceil((L + 31) / 32) chunks of [q*q cells][32 sites], holding
    unpackfV's (mcmc.cl:42-65) J_{pos,m}(a, b) at [pos][m // 32][a*q+b][m % 32]
    and zero for m == pos and m >= L.  Built from unpack_j's rows."""
    rows = unpack_j(J, L, q)[:, :L * q * q].reshape(L, L, q * q)
    nc = (L + 62) // 32
    t = np.zeros((L, nc * 32, q * q), np.float32)
    t[:, :L, :] = rows
    return np.ascontiguousarray(t.reshape(L, nc, 32, q * q).transpose(0, 1, 3, 2))


def metropolis(J, rngstates, position_list, position_offset, nsteps, seqmem, L, q,
               betas=None, beta=1.0, walkers=None):
    """Runs the sampler in place on (rngstates (N,4) u4, seqmem (SWORDS,N) u4)."""
    Ju = unpack_j(J, L, q)
    N = seqmem.shape[1]
    g0, g1 = (0, N) if walkers is None else walkers
    assert rngstates.flags.c_contiguous and seqmem.flags.c_contiguous
    bp = None
    if betas is not None:
        betas = np.ascontiguousarray(betas, dtype=np.float32)
        bp = betas.ctypes.data
    lib().mi3o_metropolis(Ju.reshape(-1), jrow_stride(L, q), rngstates.reshape(-1),
                          int(position_offset), np.ascontiguousarray(position_list, np.uint32),
                          int(nsteps), bp, float(beta), seqmem.reshape(-1), N, L, q, g0, g1)


def energies_kahan(J, seqmem, L, q, nseq=None):
    buflen = seqmem.shape[1]
    nseq = buflen if nseq is None else nseq
    E = np.zeros(nseq, np.float32)
    lib().mi3o_energies_kahan(np.ascontiguousarray(J, np.float32), np.ascontiguousarray(seqmem).reshape(-1),
                              buflen, nseq, E, L, q)
    return E


def energies_f64(J, seqmem, L, q, nseq=None):
    buflen = seqmem.shape[1]
    nseq = buflen if nseq is None else nseq
    E = np.zeros(nseq, np.float64)
    lib().mi3o_energies_f64(np.ascontiguousarray(J, np.float32), np.ascontiguousarray(seqmem).reshape(-1),
                            buflen, nseq, E, L, q)
    return E


def bicounts(seqmem, L, q, nseq=None):
    buflen = seqmem.shape[1]
    nseq = buflen if nseq is None else nseq
    out = np.zeros((npairs(L), q * q), np.uint32)
    lib().mi3o_count_bivariate(np.ascontiguousarray(seqmem).reshape(-1), buflen, nseq, out.reshape(-1), L, q)
    return out


def bicounts_to_bimarg(c, nseq):
    c = np.ascontiguousarray(c, np.uint32)
    out = np.zeros(c.shape, np.float32)
    lib().mi3o_bicounts_to_bimarg(c.reshape(-1), out.reshape(-1), nseq, c.size)
    return out


def min_floats(x):
    return float(lib().mi3o_min_floats(np.ascontiguousarray(x, np.float32), len(x)))


def weight_stats(w):
    out = np.zeros(2, np.float32)
    lib().mi3o_weight_stats(np.ascontiguousarray(w, np.float32), len(w), out)
    return out


def weight_stats_f64(w):
    out = np.zeros(2, np.float64)
    lib().mi3o_weight_stats_f64(np.ascontiguousarray(w, np.float32), len(w), out)
    return out


def dE_to_weights(ref, dE):
    dE = np.ascontiguousarray(dE, np.float32)
    w = np.zeros_like(dE)
    lib().mi3o_dE_to_weights(float(ref), dE, w, len(dE))
    return w


def fixed_beta_weights(beta, ref, E):
    E = np.ascontiguousarray(E, np.float32)
    w = np.zeros_like(E)
    lib().mi3o_fixed_beta_weights(float(beta), float(ref), E, w, len(E))
    return w


def weighted_marg_f64(w, seqmem, L, q, nseq=None):
    buflen = seqmem.shape[1]
    nseq = buflen if nseq is None else nseq
    out = np.zeros((npairs(L), q * q), np.float64)
    lib().mi3o_weighted_marg_f64(np.ascontiguousarray(w, np.float32), np.ascontiguousarray(seqmem).reshape(-1),
                                 buflen, nseq, out.reshape(-1), L, q)
    return out


def renormalize_bimarg(bi, q):
    bi = np.ascontiguousarray(bi, np.float32).copy()
    lib().mi3o_renormalize_bimarg(bi.reshape(-1), bi.shape[0], q)
    return bi


def updatedJ(bt, bi, gamma, pc, Ji):
    Jo = np.zeros_like(np.asarray(Ji, np.float32))
    lib().mi3o_updatedJ(np.ascontiguousarray(bt, np.float32).reshape(-1),
                        np.ascontiguousarray(bi, np.float32).reshape(-1), float(gamma), float(pc),
                        np.ascontiguousarray(Ji, np.float32).reshape(-1), Jo.reshape(-1), Jo.size)
    return Jo


def reg_lz(bi, gamma, pc, lJ, J, dJ, q, l2):
    dJ = np.ascontiguousarray(dJ, np.float32).copy()
    lib().mi3o_reg_lz(np.ascontiguousarray(bi, np.float32).reshape(-1), float(gamma), float(pc), float(lJ),
                      np.ascontiguousarray(J, np.float32).reshape(-1), dJ.reshape(-1), dJ.shape[0], q,
                      1 if l2 else 0)
    return dJ


REG_KINDS = {"SCADJ": 0, "X": 1, "Xij": 2, "SCADX": 3, "expX": 4, "ddE": 5, "SCADddE": 6}


def reg_other(kind, bi, gamma, pc, params, J, dJ, q, lambdas=None):
    """reg_SCADJ / X / Xij / SCADX / expX / ddE / SCADddE (mcmc.cl:904-1243)
    applied to a copy of dJ; params are the kernel's extra float arguments
    in order (SCADJ: lJ, a; X: lX; SCADX: s, r, a; expX: lam; ddE: lambda;
    SCADddE: lambda, r)."""
    dJ = np.ascontiguousarray(dJ, np.float32).copy()
    p = list(params) + [0.0] * (3 - len(params))
    lp = None
    if lambdas is not None:
        lambdas = np.ascontiguousarray(lambdas, np.float32)
        lp = lambdas.ctypes.data
    lib().mi3o_reg_other(REG_KINDS[kind], np.ascontiguousarray(bi, np.float32).reshape(-1), lp, float(gamma),
                         float(pc), float(p[0]), float(p[1]), float(p[2]),
                         np.ascontiguousarray(J, np.float32).reshape(-1), dJ.reshape(-1), dJ.shape[0], q)
    return dJ


def gen_indep(seqmem, rngstates, cprob, L, q, nseq=None):
    buflen = seqmem.shape[1]
    nseq = buflen if nseq is None else nseq
    lib().mi3o_gen_indep(seqmem.reshape(-1), buflen, nseq, rngstates.reshape(-1),
                         np.ascontiguousarray(cprob, np.float32).reshape(-1), L, q)


def repack_seqs_T(seqmem, L):
    buf4len = seqmem.shape[1]
    out = np.zeros((L, buf4len), np.uint8)
    lib().mi3o_repack_seqs_T(np.ascontiguousarray(seqmem).reshape(-1), buf4len, out.reshape(-1), buf4len, L)
    return out.view("<u4")


# ---------------------------------------------------------------------------
# Host routines of the reference's round loop, restated in float64 numpy.

def gauge_fieldless_even(J, L, q, h=None):
    """fieldlessGaugeEven(h, J) of the reference (changeGauge.py:37-155):
    zeroJGauge (row/column means of each pair moved into the fields), the
    fields centred (zeroGauge), then each field h_i(a) spread evenly over
    the L-1 couplings of site i.  Returns the float64 couplings."""
    Jx = np.asarray(J, np.float64).reshape(L * (L - 1) // 2, q, q)
    h = np.zeros((L, q)) if h is None else np.asarray(h, np.float64)
    m1, m2 = Jx.mean(axis=1), Jx.mean(axis=2)   # mean over a (per b), over b (per a)
    mJ = m1.mean(axis=1)
    J0 = Jx - m1[:, None, :] - m2[:, :, None] + mJ[:, None, None]
    h0 = h - np.sum(mJ) / L
    i, j = np.triu_indices(L, k=1)
    np.add.at(h0, j, m1)
    np.add.at(h0, i, m2)
    h0 = h0 - h0.mean(axis=1, keepdims=True)
    hd = h0 / (L - 1)
    out = J0 + hd[i][:, :, None] + hd[j][:, None, :]
    return out.reshape(-1, q * q)


def bimarg_stats_f64(target, model, J=None):
    """bimarg_stats and the X statistic of printstats (NewtonSteps.py:33-54)
    in float64: (SSR, max|t-m|, mean |t-m|/t over t > 0.01f, count,
    X_model, X_target)."""
    t32 = np.asarray(target, np.float32)
    t, m = t32.astype(np.float64), np.asarray(model, np.float32).astype(np.float64)
    d = t - m
    top = t32 > np.float32(0.01)
    cnt = int(np.sum(top))
    rel = float(np.mean(np.abs(d[top]) / t[top])) if cnt else 0.0
    xm = xt = 0.0
    if J is not None:
        npair, qq = t.shape
        q = int(round(qq ** 0.5))
        Jd = np.asarray(J, np.float32).astype(np.float64)

        def indep(f):
            fx = f.reshape(npair, q, q)
            return (fx.sum(axis=2)[:, :, None] * fx.sum(axis=1)[:, None, :]).reshape(npair, qq)
        xm = float(np.sum(Jd * (m - indep(m))))
        xt = float(np.sum(Jd * (t - indep(t))))
    return (float(np.sum(d * d)), float(np.max(np.abs(d))), rel, cnt, xm, xt)


# ---------------------------------------------------------------------------
# MSA text lines (mi3gpu/utils/seqload.py), restated in numpy.

def seqs_to_text(seqmem, L, alpha):
    """The lines writeSeqs writes for packed walkers (seqload.py:378-411,
    no id field): alpha[residue] for each site, then b'\\n'.  Returns
    (bytes as uint8 array of N*(L+1), any residue >= len(alpha)); such a
    residue is written as '?'."""
    seqs = unpack_seqs(seqmem, L)
    a = np.frombuffer(alpha.encode() if isinstance(alpha, str) else alpha, np.uint8)
    table = np.full(256, ord('?'), np.uint8)
    table[:a.size] = a
    out = np.empty((seqs.shape[0], L + 1), np.uint8)
    out[:, :L] = table[seqs]
    out[:, L] = ord('\n')
    return out.reshape(-1), bool((seqs >= a.size).any())


def text_to_seqs(text, nlines, line_len, id_len, L, alpha):
    """Lines of an MSA body back to packed walkers, as loadSeqs reads them
    (seqload.py:196-246): every line ends in b'\\n', its id field (id_len
    bytes) ends in a space, every residue is in alpha (the last index of a
    repeated letter wins, as the reference's table assignment does).
    Returns (packed (SWORDS, nlines) uint32, index of the first malformed
    line or None); malformed lines pack as zeros."""
    a = np.frombuffer(alpha.encode() if isinstance(alpha, str) else alpha, np.uint8)
    lut = np.full(256, 255, np.uint8)
    lut[a] = np.arange(a.size, dtype=np.uint8)
    rows = np.asarray(text, np.uint8)[:nlines * line_len].reshape(nlines, line_len)
    res = lut[rows[:, id_len:id_len + L]]
    bad = (rows[:, -1] != ord('\n')) | (res == 255).any(axis=1)
    if id_len:
        bad |= rows[:, id_len - 1] != ord(' ')
    res[bad] = 0
    first = int(np.argmax(bad)) if bad.any() else None
    return pack_seqs(res), first


def copy_subseq(small, seqind, marks, large, L):
    """copySubseq (mcmc.cl:99-122): every sequence of `large` (packed) takes
    the residues of small sequence `seqind` at the marked sites."""
    big = unpack_seqs(large, L)
    sub = unpack_seqs(small, L)[seqind]
    m = np.asarray(marks[:L]).astype(bool)
    big[:, m] = sub[m]
    return pack_seqs(big)


def subseq_log_frequencies(J, bseqs, sseqs, fixpos, iterbackgrounds, L, q):
    """The subsequence-frequency computation of Mi3.py:906-974 in float64
    (energies from energies_f64), with the reference's arithmetic."""
    from scipy.special import logsumexp
    large, small = (sseqs, bseqs) if iterbackgrounds else (bseqs, sseqs)
    ns = len(small)
    fixed = np.array([int(x) for x in fixpos])
    if iterbackgrounds:
        fixed = np.array([i for i in range(L) if i not in set(fixed.tolist())])
    marks = np.zeros(L, np.uint8)
    marks[fixed] = 1
    smem, lmem = pack_seqs(np.asarray(small)), pack_seqs(np.asarray(large))
    origEs = energies_f64(J, smem, L, q)
    if iterbackgrounds:
        logf = np.full(len(large), -np.inf)
        for n, eo in enumerate(origEs):
            lmem = copy_subseq(smem, n, marks, lmem, L)
            np.logaddexp(logf, eo - energies_f64(J, lmem, L, q), out=logf)
    else:
        logf = np.zeros(len(large))
        for n in range(ns):
            lmem = copy_subseq(smem, n, marks, lmem, L)
            logf[n] = logsumexp(origEs - energies_f64(J, lmem, L, q))
    return logf


# ------------------------------------------------------ equilibration test
# The reference decides equilibration with scipy.stats.spearmanr
# (NewtonSteps.py:419-428; scipy 1.18.1 here, not part of the reference
# tree).  Its published algorithm, restated: average ranks (rankdata,
# method 'average'), the Pearson correlation of the rank vectors, and the
# two-sided Student-t p-value of t = r sqrt((n-2)/((1+r)(1-r))), n-2
# degrees of freedom; a constant input gives r = NaN.

def rank_average(x):
    """1-based ranks, ties sharing the mean of their sorted positions."""
    x = np.asarray(x)
    n = x.shape[0]
    order = np.argsort(x, kind="stable")
    xs = x[order]
    start = np.ones(n, bool)
    start[1:] = xs[1:] != xs[:-1]
    end = np.ones(n, bool)
    end[:-1] = xs[1:] != xs[:-1]
    lo = np.maximum.accumulate(np.where(start, np.arange(n), 0))
    hi = np.minimum.accumulate(np.where(end, np.arange(n), n)[::-1])[::-1]
    r = np.empty(n, np.float64)
    r[order] = 0.5 * (lo + hi) + 1.0
    return r


def spearman(a, b):
    """(r, p) as scipy.stats.spearmanr(a, b) for two 1-D vectors."""
    from scipy.stats import t as student_t
    ra, rb = rank_average(a), rank_average(b)
    n = ra.shape[0]
    da, db = ra - ra.mean(), rb - rb.mean()
    saa, sbb = np.dot(da, da), np.dot(db, db)
    if saa == 0 or sbb == 0:
        return float("nan"), float("nan")
    r = float(np.dot(da, db) / np.sqrt(saa * sbb))
    r = max(-1.0, min(1.0, r))
    with np.errstate(divide="ignore"):
        tt = r * np.sqrt(max(0.0, (n - 2) / ((r + 1.0) * (1.0 - r))))
    p = float(2 * student_t.sf(abs(tt), n - 2))
    return r, p


def spearman_rcrit(n, pmin=0.02):
    """|r| below which spearmanr's p exceeds pmin (two-sided), n samples."""
    from scipy.stats import t as student_t
    tc = float(student_t.isf(pmin / 2, n - 2))
    return tc / np.sqrt(n - 2 + tc * tc)
