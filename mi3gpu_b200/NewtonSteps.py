"""Host quasi-Newton / MCMC driver: the reference's NewtonSteps module
(mi3gpu/NewtonSteps.py) over the B200 device group.

The control flow follows the reference function by function -- iterNewton
(:159-268), runMCMC (:385-486), MCMCstep (:610-687), newtonMCMC (:689-767),
NewtonSteps (:595-608), singleNewton (:109-124) -- and drives a GPU_node
(node_manager.py) of MCMCGPU devices.  Differences from the reference:

  * Neff comes from the FP64 weight sums ('weightstats64'), not from the
    float32 sums the reference's weight_stats kernel produces.
  * Output files are written only when param.outdir is set.
  * Parallel tempering (runMCMC_tempered) is not provided; it does not run
    in the reference either (undefined readGPUbufs / markSeqs / split).
"""
import time
from pathlib import Path

import numpy as np
from scipy.stats import spearmanr
from scipy.stats import t as student_t

from .potts import bimarg_stats, fieldlessGaugeEven, indepF, printsome


class Param(dict):
    """Attribute-style parameter dict (the reference's attrdict, Mi3.py:68-75)."""

    def __getattr__(self, attr):
        if attr.startswith('_'):
            raise AttributeError(attr)
        return self.get(attr)

    def __setattr__(self, k, v):
        self[k] = v


def getNeff(w):
    """Effective sample size (sum w)^2 / sum w^2 (NewtonSteps.py:126-130)."""
    w = np.asarray(w, dtype=np.float64)
    return (np.sum(w) ** 2) / np.sum(w ** 2)


def printstats(name, jstep, bimarg_target, bimarg_model, couplings, energies, e_rho):
    ferr, ssr, maxd = bimarg_stats(bimarg_target, bimarg_model)
    ferr, maxd = ferr * 100, maxd * 100
    C = bimarg_model - indepF(bimarg_model)
    X = np.sum(couplings * C, axis=1)
    Co = bimarg_target - indepF(bimarg_target)
    Xo = np.sum(couplings * Co, axis=1)
    X = f"{np.sum(X): 6.1f} ({np.sum(Xo): 6.1f})"
    rhostr = '(none)'
    if e_rho is not None:
        rho = [r[0] for r in e_rho]
        rhostr = np.array2string(np.array(rho), precision=2, floatmode='fixed', suppress_small=True)[1:-1]
    lowE, meanE, stdE = np.min(energies), np.mean(energies), np.std(energies)
    return (f"{name} {jstep: 6d} Error: SSR:{ssr:6.3f}   rel%:{ferr:5.2f}   max%:{maxd:5.2f}   X:{X}\n"
            f"{name} bimarg: {printsome(bimarg_model)} ...\n"
            f"{name}      J: {printsome(couplings)} ...\n"
            f"{name} min(E) = {lowE:.4f}     mean(E) = {meanE:.4f}     std(E) = {stdE:.4f}\n"
            f"{name} E Autocorr vs time: {rhostr}")


def singleNewton(bimarg, gamma, param, gpus):
    """One J update from the given bimarg (NewtonSteps.py:109-124).  As in the
    reference, the update is applied to 'dJ' and the unchanged 'J' is read
    back, so this is a no-op on J."""
    pc = param.pcdamping
    gpus.setBuf('bi', bimarg)
    gpus.updateJ(gamma, pc)
    return gpus.head_gpu.getBuf('J')[0].read()


def iterNewton(param, bimarg_model, gpus, log, fused=False):
    """Zwanzig-reweighted quasi-Newton steps until Neff < fracNeff*N
    (NewtonSteps.py:159-268).  Returns (steps, trialJ, predicted bimarg).

    fused=True replaces min_buf + dE_to_weights + weight_statistics by the
    single-pass weights_fused kernel (same values)."""
    bimarg_target = param.bimarg
    gamma = param.gamma0
    newtonSteps = param.newtonSteps
    pc = param.pcdamping
    Nfrac = param.fracNeff
    N = param.nwalkers

    log("")
    log(f"Perturbation optimization for up to {newtonSteps} steps:")
    if param.reg:
        log(f"Using regularization {param.reg} ({param.regarg})")
    s = time.time()

    seqbuf, wbufname, ebufname, etmpname = 'main', 'weights', 'E main', 'E tmp'
    allgpus = gpus
    mode = param.distribute_jstep or 'all'
    if mode != 'all':
        # the Newton phase runs on the head device (or node) over every
        # walker, gathered into its large buffer (NewtonSteps.py:181-195)
        if mode == 'head_gpu':
            gpus = allgpus.head_gpu
            log("Transferring sequences to gpu 0")
        elif mode == 'head_node':
            gpus = allgpus.head_node
            log("Transferring sequences to node 0")
        else:
            raise ValueError(f"unknown distribute_jstep {mode!r}")
        allgpus.gatherLarge(gpus)
        seqbuf, wbufname, ebufname, etmpname = 'large', 'weights large', 'E large', 'E tmp large'

    # the walkers are fixed during the Newton steps: their consensus residues
    # let the energy and weighted-bimarginal passes skip most pairs
    gpus.updateConsensus(seqbuf)
    gpus.calcEnergies(seqbuf)
    gpus.calcBicounts(seqbuf)
    gpus.bicounts_to_bimarg(seqbuf)
    gpus.merge_bimarg()
    gpus.fillBuf('dJ', 0)

    N0 = N
    ref_dE = 0.0
    if param.beta is not None:
        E = gpus.readBufs(ebufname)
        beta_mod = [(-(param.beta - 1) * x).astype('<f4') for x in E]
        dEB = np.concatenate(beta_mod)
        ref_dE = np.min(dEB)
        N0 = getNeff(np.exp(-(dEB - ref_dE)))
        gpus.setBuf(etmpname, beta_mod)
        log(f"Temperature reweight decreases Neff from {N} to {N0}")

    lastNeff = 2 * N0
    i = 0
    for i in range(newtonSteps):
        gpus.updateJ(gamma, pc)
        if param.reg is not None:
            gpus.reg(param.reg, (gamma, pc,) + tuple(param.regarg))
        gpus.calcEnergies(seqbuf, 'dJ')
        if param.beta is not None:
            gpus.addFloatBuf(ebufname, etmpname)

        if fused:
            gpus.weights_fused(ref_dE, seqbuf)
        else:
            gpus.min_buf(ebufname)
        mindE_fut = gpus.getBuf('minout')
        if not fused:
            gpus.dE_to_weights(seqbuf, ref_dE)  # ref_dE comes from the previous step
            gpus.weight_statistics(seqbuf)
        w_fut = gpus.getBuf('weightstats64')

        gpus.weightedMarg(seqbuf)
        gpus.merge_bimarg()

        wsum, wsum2 = (np.sum(x) for x in zip(*(w.read() for w in w_fut)))
        Neff = wsum ** 2 / wsum2
        if i % 64 == 0 or abs(lastNeff - Neff) / N0 > 0.05 or Neff < Nfrac * N0:
            log(f"J-step {i: 5d}   Neff: {Neff:.1f}   ({Neff / N0 * 100:.1f}% of {N0})")
            lastNeff = Neff
        if Neff < Nfrac * N0:
            log(f"Ending coupling updates because Neff/N < {Nfrac:.2f}")
            break
        ref_dE = np.min([x.read()[()] for x in mindE_fut])

    log(f"Performed {i} coupling update steps")

    if param.device_resident:
        # trial J = J + dJ formed in place on every device (the reference reads
        # bi, J, dJ back, adds them on the host and sends J down again)
        gpus.addFloatBuf('J', 'dJ')
        if gpus is not allgpus:
            allgpus.shareJ(gpus)
        st = gpus.bimargStats('bi', 'bi target', None)[0].read()
        log(f"Predicted statistics after perturbing J: SSR {st[0]:.4f}")
        if not np.isfinite(wsum) or wsum == 0:
            raise Exception("Error: Divergence. Decrease gamma or increase pc-damping")
        log(f"Total Newton-step running time: {time.time() - s:.1f} s")
        gpus.logProfile()
        return i, None, None

    bi, J, dJ = gpus.head_gpu.readBufs(['bi', 'J', 'dJ'])
    bimarg_model, trialJ = bi[0], J[0] + dJ[0]
    weights = gpus.collect(wbufname)
    gpus.setBuf('J', trialJ)
    log(f"Predicted statistics after perturbing J: SSR {bimarg_stats(bimarg_target, bimarg_model)[1]:.4f}")

    Neff = np.sum(weights)
    if not np.isfinite(Neff) or Neff == 0:
        raise Exception("Error: Divergence. Decrease gamma or increase pc-damping")
    log(f"Total Newton-step running time: {time.time() - s:.1f} s")
    gpus.logProfile()
    return i, trialJ, bimarg_model


def track_main_bufs(param, gpus, savedir=None, step=None):
    gpus.calcBicounts('main')
    gpus.calcEnergies('main')
    bicounts, energies = gpus.collect(['bicount', 'E main'])
    bimarg_model = bicounts.astype('f4') / np.float32(np.sum(bicounts[0, :]))
    if savedir is not None:
        if 'bim' in (param.tracked or '') and _writer(gpus):
            np.save(savedir / f'bimarg_{step}', bimarg_model)
        if 'E' in (param.tracked or '') and _writer(gpus):
            np.save(savedir / f'energies_{step}', energies)
        if 'seq' in (param.tracked or ''):
            gpus.writeSeqs(savedir / f'seqs_{step}', 'main', _alpha(param), zipf=True)
    return energies, bimarg_model


def _writer(gpus):
    """Whether this process writes the output files: always, except on the
    ranks other than 0 of a RankNode (each rank runs the same round loop;
    collectives run everywhere, files are written once)."""
    return getattr(gpus, 'is_writer', True)


def _alpha(param):
    from .seqload import default_alpha
    return param.alpha if param.alpha is not None else default_alpha(param.q)


def _spearman_p(r, n):
    """Two-sided p-value of a Spearman r over n samples, as
    scipy.stats.spearmanr gives it (Student t, n - 2 degrees of freedom)."""
    if not np.isfinite(r):
        return float('nan')
    r = np.float64(max(-1.0, min(1.0, float(r))))
    with np.errstate(divide='ignore'):
        t = r * np.sqrt(max(np.float64(0.0), np.float64(n - 2) / ((r + 1.0) * (1.0 - r))))  # |r| = 1: inf
    return float(2 * student_t.sf(abs(t), n - 2))


def _equilibrate_on_device(gpus, param, log):
    """runMCMC's automatic equilibration (NewtonSteps.py:395-442) with the
    rank correlation test on the device: the energies of each checkpoint are
    ranked where they are (mi3_rank_average) and only the correlations come
    back (16 bytes per checkpoint), instead of every walker's energy.  Same
    schedule (8 calls, then doubling), same rule (p > 0.02 for the last two
    lags and at least min_equil calls), same log lines."""
    n = gpus.nwalkers
    loops = 8
    for _ in range(loops):
        gpus.runMCMC()
    step = loops
    k = 0
    while True:
        for _ in range(loops):
            gpus.runMCMC()
        step += loops
        gpus.calcEnergies('main')
        gpus.rankEnergies(k)
        k += 1
        rstr = f"Step {step} <E>={gpus.energyMean():.2f}. "
        if k >= 3:
            r1, r2 = gpus.rankCorr([(k - 1, k - 2), (k - 1, k - 3)])
            p1, p2 = _spearman_p(r1, n), _spearman_p(r2, n)
            fmt = "({:.3f}, {:.2g}) ".format
            rstr += f"r={fmt(r1, p1)} prev:{fmt(r2, p2)}"
            if p1 > 0.02 and p2 > 0.02 and step >= (param.min_equil or 64):
                log(rstr + "Equilibrated.")
                break
        if step >= (param.max_equil or 32768):
            log(rstr + "Reached Max Steps. Stopping")
            break
        log(rstr + "Continuing.")
        loops = loops * 2
    rs = gpus.rankCorr([(i, k - 1) for i in range(k)])
    gpus.dropRanks()
    return step, [(float(r), _spearman_p(r, n)) for r in rs]


def runMCMC(gpus, couplings, runName, param, log):
    """Equilibrate the walkers at `couplings` and measure their bimarginals
    (NewtonSteps.py:385-486)."""
    nloop = param.equiltime
    trackequil = param.trackequil or 0
    outdir = param.outdir
    if couplings is not None:  # None: J is already resident on the devices
        gpus.setBuf('J', couplings)

    if nloop == 'auto' and trackequil == 0 and getattr(gpus, 'deviceRanks', lambda: False)():
        step, e_rho = _equilibrate_on_device(gpus, param, log)
    elif nloop == 'auto':
        equil_dir = None
        if trackequil != 0 and outdir is not None:
            equil_dir = outdir / runName / 'equilibration'
            equil_dir.mkdir(parents=True, exist_ok=True)
        loops = 8
        for _ in range(loops):
            gpus.runMCMC()
        step = loops
        equil_e = []
        while True:
            for _ in range(loops):
                gpus.runMCMC()
            step += loops
            energies, _ = track_main_bufs(param, gpus, equil_dir, step)
            equil_e.append(energies)
            rstr = f"Step {step} <E>={np.mean(energies):.2f}. "
            if len(equil_e) >= 3:
                r1, p1 = spearmanr(equil_e[-1], equil_e[-2])
                r2, p2 = spearmanr(equil_e[-1], equil_e[-3])
                fmt = "({:.3f}, {:.2g}) ".format
                rstr += f"r={fmt(r1, p1)} prev:{fmt(r2, p2)}"
                if p1 > 0.02 and p2 > 0.02 and step >= (param.min_equil or 64):
                    log(rstr + "Equilibrated.")
                    break
            if step >= (param.max_equil or 32768):
                log(rstr + "Reached Max Steps. Stopping")
                break
            log(rstr + "Continuing.")
            loops = loops * 2
        e_rho = [spearmanr(ei, equil_e[-1]) for ei in equil_e]
    elif trackequil == 0:
        for _ in range(int(nloop)):
            gpus.runMCMC()
        step = int(nloop)
        e_rho = None
    else:
        equil_dir = None
        if outdir is not None:
            equil_dir = outdir / runName / 'equilibration'
            equil_dir.mkdir(parents=True, exist_ok=True)
        equil_e = []
        for j in range(int(nloop) // trackequil):
            for _ in range(trackequil):
                gpus.runMCMC()
            energies, _ = track_main_bufs(param, gpus, equil_dir, j * trackequil)
            equil_e.append(energies)
        step = int(nloop)
        e_rho = [spearmanr(ei, equil_e[-1]) for ei in equil_e]

    if param.beta is None and param.device_resident:
        # bimarginals stay on the device ('bi'); only the energies come back
        gpus.calcBicounts('main')
        gpus.calcEnergies('main')
        gpus.bicounts_to_bimarg('main')
        if gpus.ngpus > 1:
            gpus.merge_bimarg()
        es = gpus.collect('E main')
        bimarg_model, bicount = None, None
    elif param.beta is None:
        gpus.calcBicounts('main')
        gpus.calcEnergies('main')
        bicount, es = gpus.collect(['bicount', 'E main'])
        bimarg_model = (bicount / np.sum(bicount[0, :])).astype('f4')
    else:
        log("Reweighting to account for modified temperature.")
        gpus.calcEnergies('main')
        es = gpus.collect('E main')
        gpus.fixed_beta_weights(np.min(es), 'main')
        gpus.weightedMarg('main')
        bimarg_model = gpus.collect('bi')
        bimarg_model /= np.sum(bimarg_model, axis=1, keepdims=True)
        bicount = None
    gpus.logProfile()
    return bimarg_model, bicount, es, e_rho, None, step


def NewtonSteps(runName, param, bimarg_model, gpus, log):
    outdir = param.outdir
    if param.newtonSteps != 1:
        Jsteps, newJ, bimarg_p = iterNewton(param, bimarg_model, gpus, log, fused=bool(param.fused))
        if outdir is not None and param.device_resident:
            (bimarg_p,), (newJ,) = gpus.head_gpu.readBufs(['bi', 'J'])
        if outdir is not None and _writer(gpus):
            np.save(outdir / runName / 'predictedBimarg', bimarg_p)
            np.save(outdir / runName / 'perturbedJ', newJ)
    else:
        log("Performing single newton update step")
        newJ = singleNewton(bimarg_model, param.gamma0, param, gpus)
        Jsteps = 1
    return Jsteps, newJ


def _device_stats_line(name, jstep, gpus, energies, e_rho):
    """printstats (NewtonSteps.py:43-80) from the device's FP64 statistics:
    SSR, rel% and max% of bimarg_stats, X of model and target, plus the
    first entries of the bimarginals and couplings."""
    st = gpus.bimargStats('bi', 'bi target', 'J')[0].read()
    ssr, maxd, ferr, xm, xt = float(st[0]), float(st[1]) * 100, float(st[2]) * 100, float(st[4]), float(st[5])
    head = gpus.head_gpu.gpus[0]
    rhostr = '(none)'
    if e_rho is not None:
        rho = [r[0] for r in e_rho]
        rhostr = np.array2string(np.array(rho), precision=2, floatmode='fixed', suppress_small=True)[1:-1]
    lowE, meanE, stdE = np.min(energies), np.mean(energies), np.std(energies)
    line = (f"{name} {jstep: 6d} Error: SSR:{ssr:6.3f}   rel%:{ferr:5.2f}   max%:{maxd:5.2f}   "
            f"X:{xm: 6.1f} ({xt: 6.1f})\n"
            f"{name} bimarg: {printsome(head.peekBuf('bi'))} ...\n"
            f"{name}      J: {printsome(head.peekBuf('J'))} ...\n"
            f"{name} min(E) = {lowE:.4f}     mean(E) = {meanE:.4f}     std(E) = {stdE:.4f}\n"
            f"{name} E Autocorr vs time: {rhostr}")
    return ssr, line, dict(ferr=float(st[2]), maxd=float(st[1]), X=xm, Xo=xt)


def _host_stats(bimarg_target, bimarg_model, couplings):
    """The numbers of printstats' error line (NewtonSteps.py:43-57) for the
    round history: Ferr (mean relative error of target entries > 0.01, as a
    fraction), max |diff|, and X of the model and of the target."""
    ferr, _, maxd = bimarg_stats(bimarg_target, bimarg_model)
    X = float(np.sum(couplings * (bimarg_model - indepF(bimarg_model))))
    Xo = float(np.sum(couplings * (bimarg_target - indepF(bimarg_target))))
    return dict(ferr=float(ferr), maxd=float(maxd), X=X, Xo=Xo)


def MCMCstep(runName, Jstep, couplings, param, gpus, log):
    """One round: re-gauge J, equilibrate, report, Newton-update
    (NewtonSteps.py:610-687).

    With param.device_resident the couplings never leave the devices:
    `couplings` is ignored (J is on the devices), the gauge transform and the
    statistics run there in FP64, and sequences are read back only when they
    are saved or needed for reseeding.  The returned J is then None."""
    outdir = param.outdir
    L, q = param.L, param.q
    bimarg_target = param.bimarg
    dev = bool(param.device_resident)

    log("")
    log(f"Gradient Descent step {runName}")
    if dev:
        gpus.gaugeJ('J')
        couplings = gpus.head_gpu.readBufs('J')[0] if outdir is not None else None
        run_J = None
    else:
        couplings = fieldlessGaugeEven(np.zeros((L, q)), couplings)[1].astype('<f4')
        run_J = couplings
    if outdir is not None:
        rundir = outdir / runName
        rundir.mkdir(parents=True, exist_ok=True)
        if _writer(gpus):
            np.save(rundir / 'J', couplings)
            (rundir / 'newtonsteps').write_text(str(param.newtonSteps))
            (rundir / 'jstep').write_text(str(Jstep))

    start_time = time.time()
    (bimarg_model, bicount, sampledenergies, e_rho, ptinfo,
     equilsteps) = runMCMC(gpus, run_J, runName, param, log)
    dt = time.time() - start_time
    MC_s = equilsteps * param.nsteps * np.float64(gpus.nwalkers) / dt
    log(f"Total MCMC running time: {dt:.1f} s    ({MC_s:.3g} MC/s)")

    seqs = None
    if not dev or param.reseed in ('single_random', 'single_best'):
        seqs = gpus.collect('seq main')
    if dev:
        ssr, line, extra = _device_stats_line(runName, Jstep, gpus, sampledenergies, e_rho)
        if outdir is not None:
            bimarg_model = gpus.head_gpu.collect('bi')
    else:
        line = printstats(runName, Jstep, bimarg_target, bimarg_model, couplings, sampledenergies, e_rho)
        ssr = np.sum((bimarg_target - bimarg_model) ** 2)
        extra = _host_stats(bimarg_target, bimarg_model, couplings)
    log(line)
    if outdir is not None:
        # writeStatus (NewtonSteps.py:76-94): the statistics, and the walkers
        # as a bzip2 MSA in the reference's format, formatted on the devices
        if _writer(gpus):
            (outdir / runName / 'info.txt').write_text(line)
        # compressed and written while the devices run the Newton phase
        gpus.writeSeqs(outdir / runName / 'seqs', 'main', _alpha(param), zipf=True, background=True)

    ns_delta = param.newton_delta or 32
    if param.last_ssr is not None:
        if ssr > (param.last_ssr + param.min_ssr) / 2:
            param.newtonSteps = max(ns_delta, param.newtonSteps - int(1.5 * ns_delta))
            log(f"SSR increased over min. Decreasing newtonsteps to {param.newtonSteps}")
    param.last_ssr = ssr
    param.min_ssr = min(ssr, param.min_ssr if param.min_ssr is not None else np.inf)
    param.history = (param.history or []) + [dict(run=runName, ssr=float(ssr), mcmc_s=dt, mc_per_s=MC_s,
                                                  equil_calls=int(equilsteps), jstep=int(Jstep), **extra)]

    t_newton = time.time()
    Jsteps, newJ = NewtonSteps(runName, param, bimarg_model, gpus, log)
    param.history[-1].update(newton_s=time.time() - t_newton, newton_steps=int(Jsteps),
                             round_s=time.time() - start_time)
    param.newtonSteps = min(2048, Jsteps + ns_delta)
    log(f"Increasing newtonsteps to {param.newtonSteps}")
    if outdir is not None:
        if _writer(gpus):
            (outdir / runName / 'nsteps').write_text(str(Jsteps))
    return Jstep + Jsteps, seqs, sampledenergies, newJ


def run_name_format(mcmcsteps):
    """Run directory names, run_ with ceil(log10(rounds)) digits
    (NewtonSteps.py:733)."""
    return f'run_{{:0{int(np.ceil(np.log10(mcmcsteps)))}d}}'


def last_run(outdir):
    """The last run directory of an output directory and what the
    reference's --finish reads from it (Mi3.py:377-390): (run directory,
    its round index, its newtonsteps, its jstep)."""
    runs = sorted(Path(outdir).glob('run_*'))
    if not runs:
        raise Exception(f"Did not find any runs in {outdir}")
    rundir = runs[-1]
    start = int(str(rundir).rpartition('_')[2])
    return rundir, start, int((rundir / 'newtonsteps').read_text()), int((rundir / 'jstep').read_text())


def finish(param, gpus, log):
    """Continue an interrupted run from its output directory, as the
    reference's `--finish` does (Mi3.py:373-402): the last run directory's
    round is run again from its J.npy and newtonsteps, with its jstep, and
    its walkers ('seqs', when the round got that far) loaded into the
    devices; rounds then continue up to param.mcmcsteps.  The walkers' RNG
    streams and the site list start afresh, as in the reference (a
    checkpoint, checkpoint.py, continues bit for bit instead)."""
    rundir, start, newtonsteps, jstep = last_run(param.outdir)
    log(f"Continuing from {rundir}")
    param.couplings = np.load(rundir / 'J.npy')
    param.newtonSteps = newtonsteps
    if (rundir / 'seqs').exists():
        gpus.loadSeqs(rundir / 'seqs', 'main', _alpha(param))
        param.init_indep = False  # reseed 'none' keeps the loaded walkers
    return newtonMCMC(param, gpus, start, jstep, log)


def preOpt(param, gpus, log):
    """Pre-optimisation (NewtonSteps.py:274-296): one Newton phase on the
    walkers already in the devices' main buffers (loaded sequences), before
    the first round; writes a 'preopt' status directory when param.outdir
    is set.  Returns (J after it, Newton steps taken)."""
    J = param.couplings
    log("Pre-Optimization:")
    gpus.setBuf('J', np.asarray(J, dtype='<f4'))
    gpus.calcBicounts('main')
    gpus.calcEnergies('main')
    bicount, es = gpus.collect(['bicount', 'E main'])
    bimarg = bicount.astype(np.float32) / np.float32(np.sum(bicount[0, :]))
    if param.outdir is not None:
        d = Path(param.outdir) / 'preopt'
        d.mkdir(parents=True, exist_ok=True)
        if _writer(gpus):
            (d / 'info.txt').write_text(printstats('preopt', 0, param.bimarg, bimarg, J, es, None))
        gpus.writeSeqs(d / 'seqs', 'main', _alpha(param), zipf=True)
    Jsteps, newJ = NewtonSteps('preopt', param, bimarg, gpus, log)
    if newJ is None:  # device-resident: J + dJ stays on the devices
        newJ = gpus.head_gpu.readBufs('J')[0]
    return newJ, Jsteps


def newtonMCMC(param, gpus, start_run, Jstep, log, resume=None):
    """Round loop (NewtonSteps.py:689-767) with the reseed strategies
    'independent', 'single_indep', 'single_best', 'single_random', 'none'
    and 'msa' (param.seedmsa: the seed sequences, one (n, L) uint8 array
    per device or one array for all, reset into the walkers every round;
    they are copied to the devices once and restored there), and the
    pre-optimisation of param.preopt.

    param.checkpoint (a path) writes a checkpoint after every round;
    resume (a state from checkpoint.load) continues a run from one, on the
    same trajectory as if it had not stopped."""
    from . import checkpoint
    J = param.couplings
    gpus.setBuf('bi target', param.bimarg)
    rng = np.random.RandomState(param.rngseed)
    seqs, es = None, None
    fresh = resume is None
    if fresh:
        param.max_newtonSteps = param.newtonSteps
        param.min_ssr = np.inf
    else:
        start_run, Jstep, J, seqs, es = checkpoint.restore(resume, gpus, param, rng)
        log(f"Continuing from a checkpoint before round {start_run}")
    if param.device_resident:
        gpus.setBuf('J', np.asarray(J, dtype='<f4'))
    if fresh and param.preopt:
        J, Jsteps = preOpt(param, gpus, log)
        Jstep += Jsteps
    elif fresh:
        log("No Pre-optimization")
    seed_snapshot = None
    name_fmt = run_name_format(param.mcmcsteps)
    for i in range(start_run, param.mcmcsteps):
        runname = name_fmt.format(i)
        first = fresh and i == start_run
        seed = None
        if param.seedseq is not None:
            seed, param.seedseq = param.seedseq, None
        elif param.reseed == 'single_indep':
            f = param.unimarg
            seed = np.array([rng.choice(param.q, p=f[k] / f[k].sum()) for k in range(param.L)], dtype='<u1')
        elif param.reseed == 'single_random' and seqs is not None:
            seed = seqs[rng.randint(0, seqs.shape[0])]
        elif param.reseed == 'single_best' and seqs is not None:
            seed = seqs[np.argmin(es)]
        if param.reseed == 'msa' and seed is None:
            # the seed MSA: uploaded once, then restored on the devices
            if seed_snapshot is None:
                gpus.setSeqs('main', param.seedmsa)
                seed_snapshot = gpus.snapshotSeqs()
            else:
                gpus.restoreSnapshot(seed_snapshot)
        elif seed is not None:
            if param.outdir is not None:
                rundir = Path(param.outdir) / runname
                rundir.mkdir(parents=True, exist_ok=True)
                if _writer(gpus):
                    (rundir / 'seedseq').write_text("".join(_alpha(param)[c] for c in seed))
            gpus.fillSeqs(seed)
        elif param.reseed == 'independent' or (param.reseed == 'none' and first and param.init_indep
                                                and not param.preopt):
            # 'none' keeps the walkers from round to round; they start from
            # independent-site sequences when init_indep is set (not after a
            # pre-optimisation, which ran on the loaded walkers)
            gpus.gen_indep('main')
        equil = param.equiltime
        if first and param.equiltime_first is not None:
            param.equiltime = param.equiltime_first
        Jstep, seqs, es, J = MCMCstep(runname, Jstep, J, param, gpus, log)
        param.equiltime = equil
        if param.checkpoint:
            keep = param.reseed in ('single_random', 'single_best')
            checkpoint.save(param.checkpoint, gpus, param, i + 1, Jstep, J, rng,
                            seqs if keep else None, es if keep else None)
    if param.device_resident:
        J = gpus.head_gpu.readBufs('J')[0]  # trial J of the last round, as the host path returns
    if hasattr(gpus, 'flushWrites'):
        gpus.flushWrites()
    return J
