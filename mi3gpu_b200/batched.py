"""Many independent Potts problems, one CUDA-graph launch per round.

Each problem is an ordinary MCMCGPU (its own buffers and stream).  A round --
re-gauge J, `ncalls` sampler launches, exact counts, FP64 bimarginal
statistics, the Zwanzig-reweighted quasi-Newton loop, J += dJ, statistics of
the predicted bimarginals -- is recorded once per problem by stream capture,
all problems as parallel branches of one graph; the Newton loop of each
problem is the body of a conditional WHILE node whose condition a one-thread
kernel sets from the FP64 weight sums after each step (the host loop's stop
rule, NewtonSteps.py:217-246).  A round is then one graph launch plus one
small read of the per-problem statistics.

With equil=dict(min_equil=..., max_equil=...) the sampling phase
equilibrates by itself, as runMCMC's equiltime='auto' does
(NewtonSteps.py:395-442): 8 sampler calls, then checkpoints after 8, 16,
32, ... more; at each one the walkers' energies are ranked and correlated
with the two previous checkpoints on the device (mi3_rank_average,
mi3_rank_corr), and each later checkpoint is a conditional IF node that
the previous one opens unless both correlations have p > 0.02 (after at
least min_equil calls) or max_equil calls have run (mi3_equil_control).

Kernel schedules are autotuned per shape (autotune.Autotuner): the sampler's
tile plan and the count kernel.  With the same seeds a problem follows the
same trajectory as the host-driven device-resident loop
(NewtonSteps.newtonMCMC with device_resident, reseed 'none', no consensus
energies): the graph replays the same kernels with the same arguments, and
the position list of each round is cut from the same MT19937 stream
(mcmcGPU.py:447-458) that MCMCGPU.updateRngPos would use.

No counterpart in the reference, which runs one problem per process and
drives every launch from Python.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib, potts
from .mcmcGPU import MCMCGPU, rng_buf_mul


def equil_schedule(max_equil):
    """(first call, calls) of each checkpoint of runMCMC's equilibration
    (NewtonSteps.py:395-442) after its first 8 calls: 8, 16, 32, ... more,
    until max_equil calls are reached."""
    out, calls, loops = [], 8, 8
    while True:
        out.append((calls, loops))
        calls += loops
        if calls >= max_equil:
            return out
        loops *= 2


class Problem:
    """One Potts inference problem of the batch: its target bimarginals, its
    walkers and its device buffers."""

    def __init__(self, target, L, q, nwalkers, seed, device=0, nsteps=None):
        self.L, self.q, self.N = L, q, nwalkers
        self.target = np.asarray(target, dtype='<f4')
        self.unimarg = potts.getUnimarg(self.target)
        self.J0 = potts.independent_couplings(self.unimarg)
        self.nsteps = int(nsteps or 8 * L)
        self.gpu = MCMCGPU((device, 0), L, q, nwalkers, 512, None, 1024, seed + 1)
        g = self.gpu
        g.initMCMC(self.nsteps, 0, 2 ** 63)
        g.initJstep()
        g.prepare_indep(self.unimarg)
        g.setBuf('bi target', self.target)
        g.setBuf('J', self.J0)
        dev = g.device
        # per-problem control and result words; 'randpos round' holds the
        # positions of one round's calls back to back
        self.ctl = {
            'ref': torch.zeros(1, dtype=torch.float32, device=dev),
            'count': torch.zeros(1, dtype=torch.int32, device=dev),
            'stopped': torch.zeros(1, dtype=torch.int32, device=dev),
            'stats pre': torch.zeros(6, dtype=torch.float64, device=dev),
            'stats post': torch.zeros(6, dtype=torch.float64, device=dev),
            # Newton budget and {last SSR, smallest SSR} carried across rounds
            'budget': torch.zeros(1, dtype=torch.int32, device=dev),
            'ssr state': torch.tensor([float('nan'), float('inf')], dtype=torch.float64, device=dev),
        }
        self.randpos_round = None
        # capture streams of this problem's branch and of its Newton-loop body
        self.cap_stream = _new_stream(dev)
        self.body_stream = _new_stream(dev)
        self.history = []

    def position_state(self):
        """The state of the position-list stream (for rewinding it)."""
        buf = getattr(self, '_posbuf', None)
        return (self.gpu.rngstate.get_state(), self.gpu.randpos_offset, None if buf is None else buf.copy())

    def set_position_state(self, state):
        self.gpu.rngstate.set_state(state[0])
        self.gpu.randpos_offset = state[1]
        self._posbuf = state[2]

    def round_positions(self, ncalls):
        """The sites of the next `ncalls` sampler calls, drawn exactly as
        MCMCGPU.updateRngPos draws them (a 1024-call block from the problem's
        MT19937 stream, consumed in order)."""
        g = self.gpu
        out = np.empty(ncalls * self.nsteps, dtype='<u4')
        bufsize = rng_buf_mul * self.nsteps
        host = getattr(self, '_posbuf', None)
        for c in range(ncalls):
            g.randpos_offset += self.nsteps
            if g.randpos_offset >= bufsize or host is None:
                host = g.rngstate.randint(0, self.L, size=bufsize).astype('u4')
                g.randpos_offset = 0
            out[c * self.nsteps:(c + 1) * self.nsteps] = host[g.randpos_offset:g.randpos_offset + self.nsteps]
        self._posbuf = host
        return out


def _p(t):
    return t.data_ptr()


def _new_stream(device):
    """A stream of our own (torch.cuda.Stream hands out pooled streams, which
    alias once more than 32 are in use; a capturing stream must not)."""
    with torch.cuda.device(device):
        h = ctypes.c_void_p()
        _lib.call('mi3_stream_create', ctypes.byref(h))
        return torch.cuda.ExternalStream(h.value, device=device)


class BatchedRounds:
    """Quasi-Newton rounds of many problems, one graph launch per round.

    reseed: 'none' (walkers carried between rounds, started from independent
    sequences) or 'independent' (fresh independent sequences every round).
    sweeps / sweeps_first: sweeps per round after / in the first round."""

    def __init__(self, problems, gamma=4e-4, damping=1e-3, lJ=2e-4, newton_max=1024, frac_neff=0.9,
                 sweeps=16, sweeps_first=128, reseed='none', tuner=None, device=0, ns_delta=32, equil=None):
        """equil: None (fixed sweeps per round) or dict(min_equil=64,
        max_equil=...) -- sampler calls of each problem's nsteps steps --
        for the equilibration test inside the graph."""
        if reseed not in ('none', 'independent'):
            raise ValueError("reseed must be 'none' or 'independent'")
        self.equil = None
        if equil is not None:
            self.equil = dict(min_equil=int(equil.get('min_equil', 64)), max_equil=int(equil.get('max_equil', 1024)))
            if self.equil['max_equil'] < 16:
                raise ValueError("max_equil must allow the first checkpoint (16 calls)")
        self.problems = list(problems)
        self.gamma, self.damping, self.lJ = float(gamma), float(damping), float(lJ)
        self.newton_max, self.frac, self.ns_delta = int(newton_max), float(frac_neff), int(ns_delta)
        self.reseed = reseed
        self.sweeps, self.sweeps_first = int(sweeps), int(sweeps_first)
        self.device = torch.device('cuda', device) if isinstance(device, int) else device
        self.origin = _new_stream(self.device)
        self.tuning = {}
        if tuner is not None:
            for pr in self.problems:
                self.tuning[id(pr)] = tuner.tune(pr.gpu)
        for pr in self.problems:
            pr.gpu.gen_indep('main')
            pr.ctl['budget'].fill_(self.newton_max)
            # the round's site list, sized for the longer round: graphs keep
            # its address, so it is never reallocated
            n = max(self._ncalls(pr, self.sweeps), self._ncalls(pr, self.sweeps_first), self._max_calls()) * pr.nsteps
            pr.randpos_round = torch.zeros(n, dtype=torch.int32, device=pr.gpu.device)
            if self.equil:
                self._equil_buffers(pr)
        torch.cuda.synchronize(self.device)
        self.graphs = {}
        self.rounds_done = 0

    # ------------------------------------------------------------ capture
    def _ncalls(self, pr, sweeps):
        return max(1, sweeps * pr.L // pr.nsteps)

    def _schedule(self):
        return equil_schedule(self.equil['max_equil'])

    def _max_calls(self):
        if not self.equil:
            return 0
        c0, n = self._schedule()[-1]
        return c0 + n

    def _equil_buffers(self, pr):
        from scipy.stats import t as student_t
        g, N = pr.gpu, pr.N
        J = len(self._schedule())
        dev = g.device
        pr.ctl['ranks'] = torch.zeros((J, N), dtype=torch.float32, device=dev)
        pr.ctl['rank r'] = torch.zeros((J, 2), dtype=torch.float64, device=dev)
        pr.ctl['equil out'] = torch.zeros(2, dtype=torch.int32, device=dev)
        self._ws(g, 'ws rank', 'mi3_rank_workspace', N)
        self._ws(g, 'ws corr', 'mi3_rank_corr_workspace')
        tc = float(student_t.isf(0.02 / 2, N - 2))
        pr.rcrit = tc / np.sqrt(N - 2 + tc * tc)  # |r| < rcrit  <=>  p > 0.02

    def _capture_sampling(self, pr, s, bs):
        """The equilibrating sampling phase of one problem (see the module
        docstring); `s` is the problem's capture stream, `bs` the stream its
        IF bodies are captured on."""
        g, b, c, N, L, q = pr.gpu, pr.gpu.bufs, pr.ctl, pr.N, pr.L, pr.q
        call = _lib.call
        sched = self._schedule()
        for k in range(8):
            g.sampler_call(k * pr.nsteps, _p(pr.randpos_round), pr.nsteps, _p(b['seq main']), _p(b['rngstates']),
                           _p(b['status']), s)
        handles = [None]
        for _ in range(1, len(sched)):
            h = ctypes.c_ulonglong(0)
            call('mi3_cond_handle_create', s, 0, ctypes.byref(h))
            handles.append(h.value)
        ranks, rr = c['ranks'], c['rank r']
        wr, wc = self._ws(g, 'ws rank', 'mi3_rank_workspace', N), self._ws(g, 'ws corr', 'mi3_rank_corr_workspace')
        for j, (c0, loops) in enumerate(sched):
            st = s
            if j > 0:
                call('mi3_capture_if_begin', s, bs, handles[j])
                st = bs
            for k in range(loops):
                g.sampler_call((c0 + k) * pr.nsteps, _p(pr.randpos_round), pr.nsteps, _p(b['seq main']),
                               _p(b['rngstates']), _p(b['status']), st)
            call('mi3_energies', _p(b['J']), _p(b['seq main']), N, N, _p(b['E main']), L, q, _p(b['ws energies']),
                 g._wsbytes('ws energies'), st)
            call('mi3_rank_average', _p(b['E main']), N, ranks[j].data_ptr(), *wr, st)
            test = j >= 2
            if test:
                call('mi3_rank_corr', ranks[j].data_ptr(), ranks[j - 1].data_ptr(), N, rr[j].data_ptr(), *wc, st)
                call('mi3_rank_corr', ranks[j].data_ptr(), ranks[j - 2].data_ptr(), N, rr[j].data_ptr() + 8, *wc,
                     st)
            has_next = j + 1 < len(sched)
            call('mi3_equil_control', handles[j + 1] if has_next else 0, 1 if has_next else 0,
                 rr[j].data_ptr() if test else None, rr[j].data_ptr() + 8 if test else None, pr.rcrit,
                 1 if test else 0, c0 + loops, self.equil['min_equil'], self.equil['max_equil'],
                 _p(c['equil out']), st)
            if j > 0:
                call('mi3_capture_if_end', bs)

    def _capture_problem(self, pr, ncalls):
        g, s, L, q, N = pr.gpu, pr.cap_stream.cuda_stream, pr.L, pr.q, pr.N
        npq = g.nPairs * q * q
        b = g.bufs
        c = pr.ctl
        call = _lib.call
        call('mi3_gauge_fieldless_even', _p(b['J']), _p(b['J']), L, q, *self._ws(g, 'ws gauge',
             'mi3_gauge_workspace', L, q), s)
        g.unpack_call(s)
        if self.reseed == 'independent':
            call('mi3_gen_indep', _p(b['seq main']), N, N, _p(b['rngstates']), _p(b['cprob']), L, q, s)
        if self.equil:
            self._capture_sampling(pr, s, pr.body_stream.cuda_stream)
        else:
            for k in range(ncalls):
                g.sampler_call(k * pr.nsteps, _p(pr.randpos_round), pr.nsteps, _p(b['seq main']), _p(b['rngstates']),
                               _p(b['status']), s)
        tensor = (getattr(g, 'count_kernel', None) == 'tc') if getattr(g, 'count_kernel', None) else \
            q in g.TENSOR_COUNT_Q
        if tensor:
            call('mi3_bicounts_tc', _p(b['seq main']), N, N, _p(b['bicount']), L, q, _p(b['status']), s)
        else:
            call('mi3_bicounts', _p(b['seq main']), N, N, _p(b['bicount']), L, q, s)
        call('mi3_bicounts_to_bimarg', _p(b['bicount']), _p(b['bi']), N, L, q, s)
        sws = self._ws(g, 'ws stats', 'mi3_bimarg_stats_workspace', L)
        call('mi3_bimarg_stats', _p(b['bi target']), _p(b['bi']), _p(b['J']), L, q, _p(c['stats pre']), *sws, s)
        call('mi3_newton_adapt', 0, _p(c['stats pre']), _p(c['count']), _p(c['budget']), _p(c['ssr state']),
             self.ns_delta, s)
        # Newton prologue (NewtonSteps.iterNewton): renormalised model
        # bimarginals, dJ = 0, first reference energy 0, counters 0
        call('mi3_renormalize_bimarg', _p(b['bi']), L, q, s)
        call('mi3_memset', _p(b['dJ']), 0, npq * 4, s)
        for k in ('ref', 'count', 'stopped'):
            call('mi3_memset', _p(c[k]), 0, 4, s)
        handle = ctypes.c_ulonglong(0)
        bs = pr.body_stream.cuda_stream
        call('mi3_capture_while_begin', s, bs, ctypes.byref(handle))
        call('mi3_update_j', _p(b['bi target']), _p(b['bi']), self.gamma, self.damping, _p(b['dJ']), _p(b['dJ']),
             L, q, bs)
        call('mi3_reg_l1z', _p(b['bi']), self.gamma, self.damping, self.lJ, _p(b['J']), _p(b['dJ']), L, q, bs)
        call('mi3_energies', _p(b['dJ']), _p(b['seq main']), N, N, _p(b['E main']), L, q, _p(b['ws energies']),
             g._wsbytes('ws energies'), bs)
        call('mi3_weights_fused_dev', _p(c['ref']), _p(b['E main']), _p(b['weights']), N, _p(b['minout']),
             _p(b['weightstats']), _p(b['weightstats64']), _p(b['ws reduce']), g._wsbytes('ws reduce'), bs)
        wk = getattr(g, 'wmarg_kernel', None)
        if (wk == 'tc') if wk else q in g.TENSOR_WMARG_Q:
            call('mi3_weighted_marg_tc', _p(b['weights']), _p(b['seq main']), N, N, _p(b['bi']), L, q,
                 *self._ws(g, 'ws wmarg tc', 'mi3_weighted_marg_tc_workspace', L, q), _p(b['status']), bs)
        else:
            call('mi3_weighted_marg', _p(b['weights']), _p(b['seq main']), N, N, _p(b['bi']), L, q, None,
                 _p(b['ws wmarg']), g._wsbytes('ws wmarg'), bs)
        call('mi3_renormalize_bimarg', _p(b['bi']), L, q, bs)
        call('mi3_newton_control', handle.value, _p(b['weightstats64']), _p(b['minout']), _p(c['ref']),
             _p(c['count']), _p(c['budget']), self.frac * N, _p(c['stopped']), bs)
        call('mi3_capture_while_end', bs)
        call('mi3_newton_adapt', 1, _p(c['stats pre']), _p(c['count']), _p(c['budget']), _p(c['ssr state']),
             self.ns_delta, s)
        # trial J = J + dJ, and the statistics of the predicted bimarginals
        call('mi3_add_float_bufs', _p(b['J']), _p(b['dJ']), npq, s)
        call('mi3_bimarg_stats', _p(b['bi target']), _p(b['bi']), None, L, q, _p(c['stats post']), *sws, s)

    @staticmethod
    def _ws(g, name, query, *args):
        if name not in g.bufs:
            g._setupWorkspace(name, _lib.query(query, *args))
        return _p(g.bufs[name]), g._wsbytes(name)

    def _build(self, key, sweeps):
        for pr in self.problems:
            # workspaces are created before capture (no allocation inside it)
            self._ws(pr.gpu, 'ws gauge', 'mi3_gauge_workspace', pr.L, pr.q)
            self._ws(pr.gpu, 'ws stats', 'mi3_bimarg_stats_workspace', pr.L)
            if 4 <= pr.q <= 32:
                self._ws(pr.gpu, 'ws wmarg tc', 'mi3_weighted_marg_tc_workspace', pr.L, pr.q)
        torch.cuda.synchronize(self.device)
        o = self.origin
        fork = torch.cuda.Event()
        _lib.call('mi3_capture_begin', o.cuda_stream)
        try:
            fork.record(o)
            joins = []
            for pr in self.problems:
                pr.cap_stream.wait_event(fork)
                self._capture_problem(pr, self._ncalls(pr, sweeps))
                e = torch.cuda.Event()
                e.record(pr.cap_stream)
                joins.append(e)
            for e in joins:
                o.wait_event(e)
        finally:
            graph = ctypes.c_void_p()
            rc_end = _lib.load().mi3_capture_end(o.cuda_stream, ctypes.byref(graph))
        if rc_end != 0:
            raise _lib.Mi3Error('mi3_capture_end', rc_end, _lib.load().mi3_last_error().decode())
        exec_ = ctypes.c_void_p()
        _lib.call('mi3_graph_instantiate', graph, ctypes.byref(exec_))
        self.graphs[key] = (graph, exec_)
        return exec_

    # ------------------------------------------------------------ rounds
    def run_round(self):
        """One round of every problem; returns the per-problem records."""
        first = self.rounds_done == 0
        key = 'equil' if self.equil else ('first' if first else 'next')
        sweeps = self.sweeps_first if first else self.sweeps
        exec_ = self.graphs[key][1] if key in self.graphs else self._build(key, sweeps)
        states = {}
        for pr in self.problems:
            if self.equil:
                # positions for the longest equilibration; the stream is
                # rewound to the calls actually made after the round
                states[id(pr)] = pr.position_state()
                pos = pr.round_positions(self._max_calls())
            else:
                pos = pr.round_positions(self._ncalls(pr, sweeps))
            pr.randpos_round[:pos.size].copy_(torch.from_numpy(pos.view(np.int32)))
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(self.origin)
        _lib.call('mi3_graph_launch', exec_, self.origin.cuda_stream)
        ev1.record(self.origin)
        ev1.synchronize()
        wall = time.perf_counter() - t0
        gpu_ms = ev0.elapsed_time(ev1)
        recs = []
        for pr in self.problems:
            pre = pr.ctl['stats pre'].cpu().numpy()
            post = pr.ctl['stats post'].cpu().numpy()
            count = int(pr.ctl['count'].item())
            stopped = int(pr.ctl['stopped'].item())
            pr.gpu._check_status()
            if stopped == 2:
                raise RuntimeError("Error: Divergence. Decrease gamma or increase pc-damping")
            calls = self._ncalls(pr, sweeps)
            rec = dict(run=f"run_{self.rounds_done:02d}", ssr=float(pre[0]), predicted_ssr=float(post[0]),
                       newton_steps=count - 1, mcmc_calls=calls)
            if self.equil:
                used, verdict = (int(x) for x in pr.ctl['equil out'].cpu().numpy())
                rec.update(mcmc_calls=used, equilibrated=verdict == 1)
                pr.set_position_state(states[id(pr)])
                pr.round_positions(used)
            pr.history.append(rec)
            recs.append(rec)
        self.rounds_done += 1
        return dict(gpu_ms=gpu_ms, wall_s=wall, problems=recs)

    def site_updates_per_round(self, first=False):
        """Site updates of a round (with equil: of the last round run)."""
        if self.equil:
            return sum(pr.history[-1]['mcmc_calls'] * pr.nsteps * pr.N for pr in self.problems if pr.history)
        sweeps = self.sweeps_first if first else self.sweeps
        return sum(self._ncalls(pr, sweeps) * pr.nsteps * pr.N for pr in self.problems)

    def close(self):
        for graph, exec_ in self.graphs.values():
            _lib.call('mi3_graph_destroy', graph, exec_)
        self.graphs = {}
        torch.cuda.synchronize(self.device)
        for st in [self.origin] + [x for pr in self.problems for x in (pr.cap_stream, pr.body_stream)]:
            _lib.call('mi3_stream_destroy', st.cuda_stream)
        self.origin = None
        for pr in self.problems:
            pr.cap_stream = pr.body_stream = None


def random_problems(n, seed=2000, L_range=(50, 300), qs=(4, 8, 21), walkers_log2=(14, 17), msa=1 << 14,
                    device=0, contact_sigma=0.5, sweeps=None):
    """Batch of synthetic problems: L ~ U[L_range], q from qs, walkers
    log-uniform in [2^lo, 2^hi] rounded to a multiple of 2048; each target
    from a ground truth built as potts.synthetic_ground_truth (seed + k)
    sampled by the plain sampler (`sweeps` sweeps, default max(256, 4L))."""
    from .inference import make_target
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        L = int(rng.integers(L_range[0], L_range[1] + 1))
        q = int(rng.choice(qs))
        N = int(2 ** rng.uniform(*walkers_log2))
        N = max(2048, (N // 2048) * 2048)
        target, _ = make_target(L, q, msa, seed=seed + k, sweeps=sweeps, contact_sigma=contact_sigma,
                                device=device)
        out.append(Problem(target, L, q, N, seed=seed + 1000 + k, device=device))
    return out
