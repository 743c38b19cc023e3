"""Host-side Potts-model helpers used by the quasi-Newton driver.

Shapes follow the reference: couplings/bimarginals (nPairs, q*q) with pairs
(i<j) in row-major order and residue index q*a+b; fields (L, q).

Restated from the reference's utilities (numpy, FP64):
  getLq, getUnimarg, indepF, validate_bimarg  -- utils/potts_common.py:24-100
  check_target                                -- Mi3.py:1029-1034
  zeroJGauge, zeroGauge, fieldlessGaugeEven  -- utils/changeGauge.py:37-155
  mutation_pc                                -- utils/pseudocount.py:8-24
plus the synthetic ground-truth generator for the benchmark workloads.
"""
import numpy as np


def getL(size):
    return int(((1 + np.sqrt(1 + 8 * size)) // 2) + 0.5)


def getLq(J):
    return getL(J.shape[0]), int(np.sqrt(J.shape[1]) + 0.5)


def pair_indices(L):
    """(i, j) arrays of all pairs i<j in the reference's order."""
    return np.triu_indices(L, k=1)


def getUnimarg(ff):
    """Univariate marginals from bimarginals: site 0 from pair (0,1) rows,
    site j>0 from pair (0,j) columns; renormalised (potts_common.py:34-40)."""
    L, q = getLq(ff)
    ff = np.asarray(ff).reshape((L * (L - 1) // 2, q, q))
    marg = np.empty((L, q), dtype=np.result_type(ff.dtype, np.float32))
    marg[0] = ff[0].sum(axis=1)
    marg[1:] = ff[:L - 1].sum(axis=1)
    return marg / marg.sum(axis=1, keepdims=True)


def indepF(fab):
    """f_i(a) f_j(b) for every pair (potts_common.py:43-48)."""
    L, q = getLq(fab)
    fx = np.asarray(fab).reshape((fab.shape[0], q, q))
    fa, fb = fx.sum(axis=2), fx.sum(axis=1)
    return (fa[:, :, None] * fb[:, None, :]).reshape(fab.shape[0], q * q)


def validate_bimarg(ff, eps=1e-5):
    """Unimarginals implied by every bimarginal row agree and sum to 1
    (potts_common.py:50-76): the first failing check, in the reference's
    order (the sums, then pair by pair the i and j marginals), raises its
    ValueError with the reference's message."""
    L, q = getLq(ff)
    fx = np.asarray(ff).reshape((L * (L - 1) // 2, q, q))
    uni = np.empty((L, q), dtype=fx.dtype)
    uni[0] = fx[0].sum(axis=1)
    uni[1:] = fx[:L - 1].sum(axis=1)
    delta = np.abs(uni.sum(axis=1) - 1)
    if np.max(delta) > eps:
        raise ValueError("unimarg for pos {} does not sum to 1: delta {}".format(np.argmax(delta), np.max(delta)))
    i, j = pair_indices(L)
    di = np.abs(uni[i] - fx.sum(axis=2))
    dj = np.abs(uni[j] - fx.sum(axis=1))
    bad = np.flatnonzero((di.max(axis=1) > eps) | (dj.max(axis=1) > eps))
    if bad.size:
        n = int(bad[0])
        if di[n].max() > eps:
            m = int(np.argmax(di[n]))
            raise ValueError("inconsitent i unimarg {:.5f} with delta {:.5f} for bimarg {} ({},{})".format(
                uni[i[n]][m], di[n][m], n, i[n], j[n]))
        m = int(np.argmax(dj[n]))
        raise ValueError("inconsitent j unimarg {:.5f} with delta {:.5f} for bimarg {} ({},{})".format(
            uni[j[n]][m], dj[n][m], n, i[n], j[n]))


def check_target(bimarg):
    """The target checks of the reference's inference set-up
    (Mi3.py:1029-1034): float32, every entry in (0, 1], consistent
    marginals."""
    bimarg = np.asarray(bimarg)
    if bimarg.dtype != np.dtype('<f4'):
        raise Exception("Bimarg must be in 'f4' format")
    if np.any((bimarg <= 0) | (bimarg > 1)):
        raise Exception("All bimarg must be 0 < f < 1")
    validate_bimarg(bimarg)


def _impute(h, J):
    if h is None and J is None:
        raise ValueError("Must supply either h or J (or both)")
    if J is None:
        L, q = h.shape
        J = np.zeros((L * (L - 1) // 2, q * q))
    if h is None:
        L, q = getLq(J)
        h = np.zeros((L, q))
    L, q = getLq(J)
    if h.shape != (L, q):
        raise ValueError("Size of h does not match size of J")
    return L, q, np.asarray(h, dtype=np.float64), np.asarray(J, dtype=np.float64)


def zeroJGauge(h, J):
    """Couplings with zero row and column means; fields absorb the
    difference so energies are preserved (changeGauge.py:37-84)."""
    L, q, h, J = _impute(h, J)
    if np.any(np.isinf(J)) or np.any(np.isinf(h)):
        raise ValueError("Cannot convert to zero gauge because of infinities")
    Jx = J.reshape((L * (L - 1) // 2, q, q))
    mJ1, mJ2 = Jx.mean(axis=1), Jx.mean(axis=2)   # column means (over a), row means (over b)
    mJ = mJ1.mean(axis=1)
    J0 = (Jx - mJ1[:, None, :] - mJ2[:, :, None] + mJ[:, None, None]).reshape(J.shape)
    h0 = h - np.sum(mJ) / L
    i, j = pair_indices(L)
    np.add.at(h0, j, mJ1)
    np.add.at(h0, i, mJ2)
    return h0, J0


def zeroGauge(h, J):
    """Fully constrained zero gauge: zero-mean couplings and fields
    (changeGauge.py:86-114)."""
    h0, J0 = zeroJGauge(h, J)
    return h0 - h0.mean(axis=1, keepdims=True), J0


def fieldlessGaugeDistributed(h, J):
    """Fold each field h_i(a) evenly into the L-1 couplings touching site i
    (changeGauge.py:116-135)."""
    L, q, h, J = _impute(h, J)
    hd = h / (L - 1)
    i, j = pair_indices(L)
    J0 = J + np.repeat(hd[i], q, axis=1) + np.tile(hd[j], (1, q))
    return np.zeros(h.shape), J0


def fieldlessGaugeEven(h, J):
    """Zero gauge, then fields folded evenly into the couplings: the gauge in
    which the reference keeps J between rounds (changeGauge.py:137-155)."""
    return fieldlessGaugeDistributed(*zeroGauge(h, J))


def repeatseqs(seqs, n):
    """n sequences by repeating the given ones in order (Mi3.py:1206-1207):
    the seed MSA of reseed 'msa'."""
    seqs = np.asarray(seqs)
    return np.repeat(seqs, (n - 1) // seqs.shape[0] + 1, axis=0)[:n, :]


def mutation_pc(ff, N, mode='jeffreys'):
    """Covariance-preserving pseudocount (pseudocount.py:8-24): mix the
    bimarginals with uniform residues at rate mu = q/(2N+q) (Jeffreys) or
    q/(N+q) (Bayes)."""
    L, q = getLq(ff)
    mu = q / (2 * N + q) if mode == 'jeffreys' else q / (N + q)
    f = getUnimarg(ff)
    i, j = pair_indices(L)
    fsum = (f[i][:, :, None] + f[j][:, None, :]).reshape(ff.shape[0], q * q)
    out = (1 - mu) ** 2 * ff + (1 - mu) * mu * fsum / q + (mu / q) ** 2
    return out / out.sum(axis=1, keepdims=True)


def independent_couplings(unimarg):
    """Couplings of the site-independent model h = -log f (Mi3.py:1172-1179)."""
    L, q = unimarg.shape
    J = np.zeros((L * (L - 1) // 2, q * q))
    return fieldlessGaugeEven(-np.log(unimarg), J)[1].astype('<f4')


def synthetic_ground_truth(L, q, seed, contact_sigma=0.5, background_sigma=0.05):
    """Ground-truth Potts model of the benchmark workloads: fields N(0,1),
    every coupling N(0, background_sigma^2), plus N(0, contact_sigma^2) on 3L
    distinct pairs with j-i >= 4; converted to the fieldless-even gauge the
    reference works in; float32 (nPairs, q*q)."""
    rng = np.random.default_rng(seed)
    npairs = L * (L - 1) // 2
    h = rng.normal(0.0, 1.0, size=(L, q))
    J = rng.normal(0.0, background_sigma, size=(npairs, q * q))
    i, j = pair_indices(L)
    far = np.nonzero(j - i >= 4)[0]
    ncontact = min(3 * L, len(far))
    contacts = rng.choice(far, size=ncontact, replace=False)
    J[contacts] += rng.normal(0.0, contact_sigma, size=(ncontact, q * q))
    return fieldlessGaugeEven(*zeroGauge(h, J))[1].astype('<f4')


def bimarg_stats(bimarg_target, bimarg_model):
    """(rel. error of f>0.01 entries, SSR, max |diff|) (NewtonSteps.py:33-41)."""
    topbi = bimarg_target > 0.01
    with np.errstate(divide='ignore', invalid='ignore'):
        rel_err = np.abs(bimarg_target - bimarg_model) / bimarg_target
        ferr = np.mean(rel_err[topbi])
    ssr = np.sum((bimarg_target - bimarg_model) ** 2)
    maxd = np.max(np.abs(bimarg_target - bimarg_model))
    return ferr, ssr, maxd


def printsome(a, prec=4):
    return np.array2string(np.asarray(a).flatten()[:5], precision=prec, sign=' ')[1:-1]
