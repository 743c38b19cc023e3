"""End-to-end quasi-Newton inference on one device (the reference's
`Mi3.py infer` loop reduced to the hot path: NewtonSteps.newtonMCMC with
fixed-length equilibration and independent-site reseeding).

    from mi3gpu_b200.inference import make_target, infer
    target, truth = make_target(L, q, n_msa=2**16, seed=1001)
    history = infer(target, L, q, nwalkers=2**20, rounds=5)

`make_target` builds the synthetic benchmark problem: a ground-truth Potts
model (potts.synthetic_ground_truth), an "MSA" of n_msa sequences sampled
from it with the device sampler, and the target bimarginals = their counts
with the Jeffreys mutation pseudocount (the reference rejects f = 0,
Mi3.py:1032-1033).
"""
import time

import numpy as np

from . import potts
from .mcmcGPU import MCMCGPU
from .node_manager import GPU_node
from . import NewtonSteps


def sample_msa(J, L, q, n, sweeps, seed, device=0, nsteps=None):
    """n sequences sampled from the Potts model J by `sweeps` sweeps of the
    plain sampler from independent uniform starts."""
    nsteps = nsteps or 8 * L
    g = MCMCGPU((device, 0), L, q, n, 512, None, 1024, seed)
    gpus = GPU_node([g])
    gpus.initMCMC(nsteps)
    gpus.prepare_indep(np.full((L, q), 1.0 / q))
    gpus.gen_indep('main')
    gpus.setBuf('J', J)
    calls = max(1, (sweeps * L + nsteps - 1) // nsteps)
    for _ in range(calls):
        gpus.runMCMC()
    gpus.calcBicounts('main')
    counts = gpus.collect('bicount')
    seqs = gpus.collect('seq main')
    return counts, seqs


def make_target(L, q, n_msa, seed, sweeps=None, contact_sigma=0.5, device=0):
    truth = potts.synthetic_ground_truth(L, q, seed=seed, contact_sigma=contact_sigma)
    sweeps = sweeps or max(256, 4 * L)
    counts, _ = sample_msa(truth, L, q, n_msa, sweeps, seed + 1, device=device)
    f = counts.astype(np.float64) / n_msa
    target = potts.mutation_pc(f, n_msa, 'jeffreys').astype('<f4')
    return target, truth


def infer(target, L, q, nwalkers, rounds, sweeps=128, newtonsteps=1024, gamma=4e-4, damping=1e-3,
          reg=('l1z', (2e-4,)), seed=1234, device=0, log=print, fused=True, outdir=None, reseed='independent',
          sweeps_first=None, device_resident=True, tuner=None, distribute_jstep='all', alpha=None,
          equiltime=None, nsteps=None, min_equil=64, max_equil=32768, J0=None):
    """Run `rounds` quasi-Newton iterations from the independent model;
    returns the per-round history (SSR, wall seconds of MCMC and Newton
    phases) as recorded by NewtonSteps.MCMCstep.

    reseed='independent' restarts every walker from independent-site
    sequences each round (`sweeps` sweeps of equilibration); reseed='none'
    keeps the walkers from the previous round, so after a first round of
    `sweeps_first` sweeps each round only re-equilibrates to the slightly
    changed couplings.  device_resident keeps J on the device between
    rounds (gauge transform and statistics in FP64 there); False runs the
    round's host work in numpy as the reference does.  tuner: an
    autotune.Autotuner whose sampler plan and count kernel are installed
    (results do not depend on them).  distribute_jstep: 'all' runs the
    Newton steps over the walkers where they are; 'head_gpu' first gathers
    them into the device's large buffer, as the reference's option does.
    alpha: the residue letters of the run directories' MSA files (default
    seqload.default_alpha(q)).

    equiltime='auto' equilibrates as the reference's default does
    (NewtonSteps.py:395-442: rank correlation of energies between
    checkpoints, at least min_equil and at most max_equil sampler calls of
    `nsteps` steps, default 2048 as Mi3.py's --nsteps); an integer fixes the
    number of sampler calls; None derives it from `sweeps`.  sweeps_first
    may also be 'auto' (the first round only).  J0: starting
    couplings (default: the independent model of the target)."""
    potts.check_target(target)  # as the reference's set-up does (Mi3.py:1029-1034)
    unimarg = potts.getUnimarg(target)
    if J0 is None:
        J0 = potts.independent_couplings(unimarg)
    if nsteps is None:
        nsteps = 2048 if equiltime == 'auto' else 8 * L
    if equiltime is None:
        equiltime = max(1, sweeps * L // nsteps)
    p = NewtonSteps.Param()
    p.update(dict(bimarg=target, gamma0=gamma, newtonSteps=newtonsteps, pcdamping=damping, fracNeff=0.9,
                  nwalkers=nwalkers, reg=reg[0] if reg else None, regarg=reg[1] if reg else None, beta=None,
                  distribute_jstep=distribute_jstep, L=L, q=q, couplings=J0, nsteps=nsteps,
                  equiltime=equiltime, min_equil=min_equil, max_equil=max_equil, trackequil=0, outdir=outdir, mcmcsteps=rounds,
                  newton_delta=32, reseed=reseed, rngseed=seed + 1, unimarg=unimarg, fused=fused, init_indep=True,
                  device_resident=device_resident, alpha=alpha,
                  equiltime_first=(None if sweeps_first is None else 'auto' if sweeps_first == 'auto'
                                   else max(1, sweeps_first * L // nsteps))))
    g = MCMCGPU((device, 0), L, q, nwalkers, 512, outdir, 1024, seed + 1)
    gpus = GPU_node([g])
    gpus.initMCMC(nsteps)
    gpus.initJstep()
    gpus.prepare_indep(unimarg)
    if tuner is not None:
        # tune on walkers and couplings of the right kind (both are set again
        # by the round loop)
        gpus.setBuf('J', J0)
        gpus.gen_indep('main')
        tuner.tune(g)
    t0 = time.time()
    J = NewtonSteps.newtonMCMC(p, gpus, 0, 0, log)
    total = time.time() - t0
    hist = p.history or []
    return dict(history=hist, total_s=total, J=J, expected_ssr=float(np.sum(target * (1 - target)) / nwalkers))


# ---------------------------------------------------------------- other modes
def _load_seqs_into_large(g, seqs, alpha):
    """Sequences (an (N, L) uint8 array or an MSA file path) into the large
    buffer of device g, which must hold exactly that many."""
    from . import seqload
    if isinstance(seqs, np.ndarray):
        g.setBuf('seq large', seqs.astype('<u1', copy=False))
    else:
        msa = seqs if isinstance(seqs, seqload.MSAText) else seqload.read_msa(seqs, alpha)
        g.setSeqsText('large', msa)


def _count_seqs(seqs, alpha):
    from . import seqload
    if isinstance(seqs, np.ndarray):
        return seqs.shape[0], None
    msa = seqload.read_msa(seqs, alpha)
    return msa.nseq, msa


def sequence_energies(couplings, seqs, alpha=None, device=0):
    """Potts energies of a set of sequences (the reference's `energies`
    mode, Mi3.py:549-606): seqs is an (N, L) uint8 array or an MSA file in
    the reference's format.  Any N: the sequences go to the device's large
    buffer (the reference requires N to fill whole work groups)."""
    from . import seqload
    couplings = np.asarray(couplings, dtype='<f4')
    L, q = potts.getLq(couplings)
    alpha = alpha if alpha is not None else seqload.default_alpha(q)
    n, msa = _count_seqs(seqs, alpha)
    g = MCMCGPU((device, 0), L, q, 512, 512, None, 1024, 0)
    g.initLargeBufs(n)
    _load_seqs_into_large(g, seqs if msa is None else msa, alpha)
    g.setBuf('J', couplings)
    g.calcEnergies('large')
    return g.getBuf('E large').read()


def subseq_log_frequencies(couplings, backgroundseqs, subseqs, fixpos, iterbackgrounds=False, alpha=None,
                           device=0):
    """Log frequencies of subsequences at fixed sites given a sample of
    background sequences (the reference's `subseq` mode, Mi3.py:876-976):
    the marked sites of every sequence of the larger set are replaced by
    those of each sequence of the smaller set in turn (copySubseq) and the
    energies of the result are combined by log-sum-exp, with the
    reference's own arithmetic (including that its default branch needs
    both sets to be the same size).  Sequences are (N, L) uint8 arrays;
    fixpos is a list of site indices."""
    from scipy.special import logsumexp
    from . import seqload
    couplings = np.asarray(couplings, dtype='<f4')
    L, q = potts.getLq(couplings)
    alpha = alpha if alpha is not None else seqload.default_alpha(q)
    bseqs, sseqs = np.asarray(backgroundseqs, '<u1'), np.asarray(subseqs, '<u1')
    large, small = (sseqs, bseqs) if iterbackgrounds else (bseqs, sseqs)
    ns = len(small)
    if ns < 512 or ns % 512 != 0:  # whole work groups (Mi3.py:915-919)
        n_new = ns - 1 + 512 - ((ns - 1) % 512)
        small = np.concatenate([small, np.zeros((n_new - ns, L), dtype='u1')], axis=0)
    g = MCMCGPU((device, 0), L, q, small.shape[0], 512, None, 1024, 0)
    node = GPU_node([g])
    g.initLargeBufs(large.shape[0])
    g.initSubseq()
    fixedpos = np.array([int(x) for x in fixpos])
    if iterbackgrounds:
        members = set(fixedpos.tolist())
        fixedpos = np.array([i for i in range(L) if i not in members])
    marks = np.zeros(L, dtype='u1')
    marks[fixedpos] = 1
    g.setBuf('seq main', small)
    g.setBuf('seq large', large)
    g.markPos(marks)
    g.setBuf('J', couplings)
    g.calcEnergies('main')
    origEs = node.collect(['E main'])[0][:ns]
    if iterbackgrounds:
        logf = np.full(len(large), -np.inf)
        for n, eo in enumerate(origEs):
            g.copySubseq(n)
            g.calcEnergies('large')
            energies = g.getBuf('E large').read()
            np.logaddexp(logf, eo - energies, out=logf)
    else:
        logf = np.zeros(len(large))
        for n in range(ns):
            g.copySubseq(n)
            g.calcEnergies('large')
            energies = g.getBuf('E large').read()
            logf[n] = logsumexp(origEs - energies)
    return logf


def equilibrate(couplings, nwalkers, equiltime, nsteps=None, seqs=None, seedseq=None, unimarg=None, alpha=None,
                outdir=None, trackequil=0, tracked='', min_equil=64, max_equil=32768, beta=None, seed=1234,
                device=0, log=print):
    """A round of sampling from a Potts model, the reference's `gen` mode
    (Mi3.py:724-870): the walkers start from `seqs` (an (N, L) uint8 array
    or an MSA file), from one `seedseq`, or from independent-site sequences
    of `unimarg` ((L, q) marginals); they run `equiltime` sampler calls of
    `nsteps` steps ('auto': until the energies decorrelate,
    NewtonSteps.runMCMC); the result is (bimarg, bicount, energies, walkers)
    and, with outdir, the reference's files: bicounts (text), bimarg.npy,
    energies.npy and seqs (MSA text)."""
    from . import seqload
    from pathlib import Path
    couplings = np.asarray(couplings, dtype='<f4')
    L, q = potts.getLq(couplings)
    alpha = alpha if alpha is not None else seqload.default_alpha(q)
    nsteps = nsteps or L
    g = MCMCGPU((device, 0), L, q, nwalkers, 512, None, 1024, seed + 1, beta=beta)
    gpus = GPU_node([g])
    gpus.initMCMC(nsteps)
    if beta is not None:
        gpus.initJstep()
    if seedseq is not None:
        gpus.fillSeqs(np.asarray(seedseq, '<u1'))
    elif seqs is not None:
        if isinstance(seqs, np.ndarray):
            gpus.setSeqs('main', seqs.astype('<u1', copy=False))
        else:
            gpus.loadSeqs(seqs, 'main', alpha)
    elif unimarg is not None:
        gpus.prepare_indep(np.asarray(unimarg, 'f4'))
        gpus.gen_indep('main')
    else:
        raise ValueError("give seqs, seedseq or unimarg for the starting walkers")
    outdir = Path(outdir) if outdir is not None else None
    p = NewtonSteps.Param(equiltime=equiltime, trackequil=trackequil, tracked=tracked, outdir=outdir,
                          min_equil=min_equil, max_equil=max_equil, beta=beta, nsteps=nsteps, alpha=alpha, q=q,
                          device_resident=False)
    if outdir is not None:
        outdir.mkdir(parents=True, exist_ok=True)
    bimarg, bicount, energies, e_rho, _, _ = NewtonSteps.runMCMC(gpus, couplings, 'gen', p, log)
    walkers = gpus.collect('seq main')
    if outdir is not None:
        if bicount is not None:
            np.savetxt(outdir / 'bicounts', bicount, fmt='%d')
        np.save(outdir / 'bimarg', bimarg)
        np.save(outdir / 'energies', energies)
        gpus.writeSeqs(outdir / 'seqs', 'main', alpha)
    log("Mean energy:", np.mean(energies))
    return bimarg, bicount, energies, walkers


def benchmark_mcmc(couplings, nwalkers, nsteps, nloop, seqs=None, seedseq=None, device=0, log=print):
    """The reference's `benchmark` mode (Mi3.py:610-722): nloop sampler
    calls of nsteps steps after a warm-up of as many, timed by the wall
    clock; returns MC steps per second."""
    couplings = np.asarray(couplings, dtype='<f4')
    L, q = potts.getLq(couplings)
    g = MCMCGPU((device, 0), L, q, nwalkers, 512, None, 1024, 1)
    gpus = GPU_node([g])
    gpus.initMCMC(nsteps)
    if seqs is not None:
        gpus.setSeqs('main', np.asarray(seqs, '<u1'))
    elif seedseq is not None:
        gpus.fillSeqs(np.asarray(seedseq, '<u1'))
    else:
        raise Exception("'seqs' or 'seedseq' option required")
    gpus.setBuf('J', couplings)

    def run():
        for _ in range(nloop):
            gpus.runMCMC()
        gpus.wait()
    run()
    t0 = time.perf_counter()
    run()
    dt = time.perf_counter() - t0
    total = nwalkers * nloop * np.float64(nsteps)
    log(f"MC steps computed: {total}")
    log(f"MC steps per second: {total / dt:g}")
    return total / dt
