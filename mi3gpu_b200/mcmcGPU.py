"""Per-device runtime: the B200 counterpart of the reference's MCMCGPU class.

This mirrors mi3gpu/mcmcGPU.py:110-1018 -- same constructor arguments,
method names, buffer names, dtypes and shapes -- so the host algorithm
(NewtonSteps.iterNewton / runMCMC, node_manager.GPU_node) drives it
unchanged.  Device buffers are PyTorch CUDA tensors used purely as memory;
all arithmetic runs in libmi3b200 (hand-written sm_100a CUDA) through the C
ABI in include/mi3b200.h.  There is no CPU fallback: without a CUDA device
or without the built library every method raises.

Ordering: the reference chains OpenCL events on an out-of-order queue so
that each command waits for the previous one (mcmcGPU.py:76-81, 211-222).
Here every MCMCGPU owns one CUDA stream and issues everything on it, which
gives the same order.  `wait_for` arguments are accepted for signature
compatibility; commands are always ordered after the previous command.
"""
import collections
import time
from pathlib import Path

import numpy as np
from numpy.random import RandomState
import torch

from . import _lib, seqload

rng_buf_mul = 1024  # position-list blocks of 1024*nsteps (mcmcGPU.py:30)


def _full_shape(buftype, bufshape):
    """numpy shape of an array of `bufshape` elements of `buftype` (a
    subarray dtype such as '<2u8' adds its own axes)."""
    dt = np.dtype(buftype)
    sub = dt.subdtype[1] if dt.subdtype is not None else ()
    return tuple(bufshape) + tuple(sub)


def _base_dtype(buftype):
    dt = np.dtype(buftype)
    return dt.subdtype[0] if dt.subdtype is not None else dt


def _spec_to_torch(buftype, bufshape, pad=0):
    """(numpy dtype string, shape) -> (torch dtype, flat element count).

    uint32 buffers are held as int32 tensors (same bits); '<2u8' (the MWC64X
    vec2 state, 16 bytes per walker) as two int64 per walker."""
    dt = np.dtype(buftype)
    if dt.subdtype is not None:
        base, sub = dt.subdtype
        n = int(np.prod(bufshape)) * int(np.prod(sub))
        dt = base
    else:
        n = int(np.prod(bufshape))
    n += int(pad or 0)
    tmap = {np.dtype('<f4'): torch.float32, np.dtype('<u4'): torch.int32, np.dtype('<i4'): torch.int32,
            np.dtype('<u8'): torch.int64, np.dtype('<f8'): torch.float64, np.dtype('<u1'): torch.uint8}
    return tmap[dt], n


class FutureBuf:
    """Result of getBuf: read() blocks until the device->host copy is done
    (mcmcGPU.py:95-108)."""

    def __init__(self, buffer, event, postprocess=None, owner=None):
        self.buffer = buffer
        self.event = event
        self.postfunc = postprocess
        self.owner = owner
        self.shape = buffer.shape
        self.dtype = buffer.dtype

    def read(self):
        self.event.synchronize()
        if self.owner is not None:
            self.owner._check_status()
        if self.postfunc is not None:
            return self.postfunc(self.buffer)
        return self.buffer


class MCMCGPU:
    def __init__(self, gpuinfo, L, q, nseq, wgsize, outdir, vsize, seed, profile=False, beta=None):
        if nseq % 512 != 0:
            raise ValueError("nwalkers/ngpus must be a multiple of 512")

        self.L = L
        self.q = q
        self.nPairs = L * (L - 1) // 2
        self.events = collections.deque()
        self.SWORDS = ((L - 1) // 4 + 1)
        self.SBYTES = (4 * self.SWORDS)
        self.nseq = {'main': nseq}
        self.nwalkers = nseq
        self.beta = 1.0 if beta is None else float(beta)

        device, gpunum = gpuinfo[0], gpuinfo[1]
        if isinstance(device, int):
            device = torch.device('cuda', device)
        if not isinstance(device, torch.device):
            device = torch.device(device)
        if device.type != 'cuda' or not torch.cuda.is_available():
            raise RuntimeError("MCMCGPU needs a CUDA device (no CPU fallback)")
        _lib.load()
        self.device = device
        self.gpunum = gpunum

        self.wgsize = wgsize
        self.nhist, self.histws = histogram_heuristic(q)
        if nseq % wgsize != 0:
            raise Exception("nseq per GPU must be a multiple of wgsize")
        if wgsize < q * q:
            raise Exception("wgsize cannot be less than q*q")

        self.logfn = None
        if outdir is not None:
            self.logfn = Path(outdir) / 'gpu-{}.log'.format(gpunum)
            with open(self.logfn, "wt") as f:
                printDevice(f.write, device)

        self.rngstate = RandomState(seed)
        self.stream = torch.cuda.Stream(device=device)
        self.profile = profile
        self._t0evt = None
        self._pending_host = collections.deque()

        self.initted = []
        self.bufs = {}
        self.buf_spec = {}
        self.seqbufs = {}
        self.Ebufs = {}
        self.largebufs = []

        nPairs, SWORDS = self.nPairs, self.SWORDS
        self._setupBuffer('J', '<f4', (nPairs, q * q))
        self._setupBuffer('Junpacked', '<f4', (L * L, q * q))
        self._setupBuffer('bi', '<f4', (nPairs, q * q))
        self._setupBuffer('bicount', '<u4', (nPairs, q * q))
        self._setupBuffer('seq main', '<u4', (SWORDS, self.nseq['main']))
        self._setupBuffer('seqL main', '<u4', (L, self.nseq['main'] // 4))
        self._setupBuffer('cprob', '<f4', (L, (q - 1)))
        self._setupBuffer('E main', '<f4', (self.nseq['main'],))
        self._setupBuffer('minout', '<f4', (1,))
        # library-side state: sampler status word and reduction/energy workspaces
        self._setupBuffer('status', '<i4', (1,))
        self._ws_nseq = 0
        self._sizeWorkspaces(nseq)
        self.fillBuf('status', 0)
        self.unpackedJ = False
        self.repackedSeqT = {'main': False}
        self.lastevt = None

    # ------------------------------------------------------------ plumbing
    def log(self, msg):
        if self.logfn is None:
            return
        with open(self.logfn, "at") as f:
            print("{: 10.3f}".format(time.process_time()), msg, file=f)

    def _ptr(self, name):
        return self.bufs[name].data_ptr()

    @property
    def _s(self):
        return self.stream.cuda_stream

    def _begin(self):
        if not self.profile:
            return None
        e = torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        if self._t0evt is None:
            self._t0evt = e
        return e

    def logevt(self, name, start=None, nbytes=None):
        """Record a command (profiling events when profile=True)."""
        evt = None
        if self.profile:
            evt = torch.cuda.Event(enable_timing=True)
            evt.record(self.stream)
            self.events.append((start, evt, name, nbytes))
        self.lastevt = evt
        return evt

    def logProfile(self):
        """Write 'EVT name start end bytes' lines (ns, relative to the first
        profiled command) for completed commands (mcmcGPU.py:224-237)."""
        if not self.profile:
            return
        out = []
        while self.events and self.events[0][1].query():
            start, end, name, nbytes = self.events.popleft()
            t0 = self._t0evt
            s = t0.elapsed_time(start) * 1e6 if start is not None else 0.0
            e = t0.elapsed_time(end) * 1e6
            out.append("EVT {} {:.0f} {:.0f} {}".format(name, s, e, nbytes if nbytes else ''))
        if self.logfn is not None and out:
            with open(self.logfn, "at") as f:
                f.write("\n".join(out) + "\n")
        return out

    def _setupBuffer(self, bufname, buftype, bufshape, pad=None):
        tdt, n = _spec_to_torch(buftype, bufshape, pad)
        if bufname == 'Junpacked':
            # padded row layout of the sampler (include/mi3b200.h)
            n = self.L * int(_lib.query('mi3_jrows_stride', self.L, self.q))
        with torch.cuda.device(self.device):
            buf = torch.empty(max(n, 1), dtype=tdt, device=self.device)
        self.bufs[bufname] = buf
        self.buf_spec[bufname] = (buftype, bufshape)
        names = bufname.split()
        if len(names) > 1:
            bufs = {'seq': self.seqbufs, 'E': self.Ebufs}
            if names[0] in bufs:
                bufs[names[0]][names[1]] = buf

    def _setupWorkspace(self, name, nbytes):
        with torch.cuda.device(self.device):
            self.bufs[name] = torch.zeros(max(int(nbytes), 16) // 8 + 2, dtype=torch.int64, device=self.device)

    def _sizeWorkspaces(self, nseq):
        """(Re)allocate the workspaces whose size grows with the number of
        sequences a call may process (main, or the large buffer)."""
        if nseq <= self._ws_nseq:
            return
        self._ws_nseq = nseq
        L, q = self.L, self.q
        self._setupWorkspace('ws energies', _lib.query('mi3_energies_workspace', nseq))
        self._setupWorkspace('ws reduce', _lib.query('mi3_weight_stats_workspace', nseq))
        self._setupWorkspace('ws wmarg', _lib.query('mi3_weighted_marg_workspace', L, q, nseq))
        if 'ws energies cons' in self.bufs:
            self._setupWorkspace('ws energies cons', _lib.query('mi3_energies_cons_workspace', L, q, nseq))

    def _span(self, seqbufname):
        """(sequences to process, row length) of a sequence buffer: all of
        'main', or the stored part of 'large' (mcmcGPU.py:504-509)."""
        if seqbufname == 'main':
            n = self.nseq['main']
            return n, n
        self.require('Large')
        return self.nstoredseqs, self.nseq[seqbufname]

    @staticmethod
    def _wbufname(seqbufname):
        return 'weights' if seqbufname == 'main' else 'weights ' + seqbufname

    def _wsbytes(self, name):
        b = self.bufs[name]
        return b.numel() * b.element_size()

    def require(self, *reqs):
        for r in reqs:
            if r not in self.initted:
                raise Exception("{} not initialized".format(r))

    def _initcomponent(self, cmp):
        if cmp in self.initted:
            raise Exception("Already initialized {}".format(cmp))
        self.initted.append(cmp)

    def _check_status(self):
        st = int(self.bufs['status'].cpu()[0])
        if st != 0:
            raise RuntimeError("libmi3b200 sampler reported status {} (a bounded wait gave up)".format(st))

    # ------------------------------------------------------------ set-up
    def initMCMC(self, nsteps, rng_offset, rng_span):
        self._initcomponent('MCMC')
        self.nsteps = nsteps
        self._setupBuffer('rngstates', '<2u8', (self.nseq['main'],))
        self._setupBuffer('Bs', '<f4', (self.nseq['main'],))
        self._setupBuffer('randpos', '<u4', (self.nsteps * rng_buf_mul,))
        self.randpos_offset = rng_buf_mul * self.nsteps
        self.setBuf('Bs', np.ones(self.nseq['main'], dtype='<f4'))
        self._initMCMC_RNG(rng_offset, rng_span)
        self.nsteps = int(nsteps)

    def initLargeBufs(self, nseq_large):
        """Sequence buffers for more sequences than this device samples
        (mcmcGPU.py:284-303): with distribute_jstep 'head_gpu' / 'head_node'
        the walkers of every device are gathered here and the Newton steps
        run over them.  Only the first nstoredseqs columns are used."""
        self._initcomponent('Large')
        nseq_large = int(nseq_large)
        if nseq_large <= 0:
            raise ValueError("the large buffer needs at least one sequence")
        self.nseq['large'] = nseq_large
        self._setupBuffer('seq large', '<u4', (self.SWORDS, nseq_large))
        self._setupBuffer('seqL large', '<u4', (self.L, nseq_large // 4))
        self._setupBuffer('E large', '<f4', (nseq_large,))
        self._setupBuffer('E tmp large', '<f4', (nseq_large,))
        self._setupBuffer('weights large', '<f4', (nseq_large,))
        self.largebufs.extend(['seq large', 'seqL large', 'E large', 'weights large'])
        self.nstoredseqs = 0
        # zeroed, as in the reference: unused columns hold residue 0
        self.fillBuf('seq large', 0)
        self.repackedSeqT['large'] = False
        self._sizeWorkspaces(nseq_large)

    def initSubseq(self):
        """The site marks of the subsequence splice (mcmcGPU.py:305-310)."""
        self.require('Large')
        self._initcomponent('Subseq')
        self._setupBuffer('markpos', '<u1', (self.SBYTES,))
        self.markPos(np.zeros(self.SBYTES, '<u1'))

    def markPos(self, marks, wait_for=None):
        """Mark the sites copySubseq replaces (mcmcGPU.py:919-925)."""
        self.require('Subseq')
        marks = np.asarray(marks).astype('<u1')
        if len(marks) == self.L:
            marks = np.concatenate([marks, np.zeros(self.SBYTES - self.L, '<u1')])
        return self.setBuf('markpos', marks)

    def copySubseq(self, seqind, wait_for=None):
        """Every sequence of the large buffer takes the residues of main
        sequence `seqind` at the marked sites (mcmcGPU.py:1001-1014)."""
        self.require('Subseq')
        if seqind >= self.nseq['main']:
            raise Exception("given index is past end of main seq buffer")
        s = self._begin()
        _lib.call('mi3_copy_subseq', self._ptr('seq main'), self.nseq['main'], int(seqind), self._ptr('markpos'),
                  self._ptr('seq large'), self.nseq['large'], self.L, self._s)
        self.repackedSeqT['large'] = False
        return self.logevt('copySubseq', s)

    def initJstep(self):
        self._initcomponent('Jstep')
        nPairs, q = self.nPairs, self.q
        self._setupBuffer('dJ', '<f4', (nPairs, q * q))
        self._setupBuffer('bi target', '<f4', (nPairs, q * q))
        self._setupBuffer('Creg', '<f4', (nPairs, q * q))
        self._setupBuffer('Xlambdas', '<f4', (nPairs,))
        self._setupBuffer('weights', '<f4', (self.nseq['main'],))
        self._setupBuffer('weightstats', '<f4', (2,))
        self._setupBuffer('weightstats64', '<f8', (2,))
        self._setupBuffer('E tmp', '<f4', (self.nseq['main'],))

    # ------------------------------------------------------------ layouts
    def packSeqs_4(self, seqs):
        """(N, L) u1 -> (SWORDS, N) u4, 4 sites per word (mcmcGPU.py:333-347)."""
        if seqs.dtype != np.dtype('<u1'):
            raise Exception("seqs must have u1 dtype")
        bseqs = np.zeros((seqs.shape[0], self.SBYTES), dtype='<u1', order='C')
        bseqs[:, :self.L] = seqs
        return np.ascontiguousarray(bseqs.view(np.uint32).T)

    def unpackSeqs_4(self, mem):
        """reverses packSeqs_4 (mcmcGPU.py:349-354)"""
        mem = np.asarray(mem).view(np.uint32).reshape(self.SWORDS, -1)
        bseqs = np.ascontiguousarray(mem.T).view(np.uint8)
        return bseqs[:, :self.L].copy()

    def repackseqs_T(self, bufname, wait_for=None):
        nseq = self.nseq[bufname]  # the whole buffer, stored or not (mcmcGPU.py:356-373)
        s = self._begin()
        _lib.call('mi3_repack_seqs_T', self._ptr('seq ' + bufname), nseq, self._ptr('seqL ' + bufname),
                  nseq // 4, self.L, self._s)
        self.repackedSeqT[bufname] = True
        return self.logevt('repackseqs_T', s)

    def prepare_indep(self, unimarg, wait_for=None):
        cprob = np.cumsum(unimarg, axis=1)
        cprob = (cprob[:, :-1] / cprob[:, -1, None]).astype('<f4')
        return self.setBuf('cprob', cprob)

    def gen_indep(self, bufname, wait_for=None):
        self.require('MCMC')
        nseq = self.nseq[bufname]
        s = self._begin()
        _lib.call('mi3_gen_indep', self._ptr('seq ' + bufname), nseq, nseq, self._ptr('rngstates'),
                  self._ptr('cprob'), self.L, self.q, self._s)
        self.repackedSeqT[bufname] = False
        return self.logevt('gen_indep', s)

    # ------------------------------------------------------------ couplings
    # Two unpacked layouts exist: the padded rows ('Junpacked') of the
    # row-streaming sampler and the chunk tiles ('Jtiles') of the skewed-lane
    # sampler; both are rebuilt lazily after J changes.
    @property
    def unpackedJ(self):
        return self._unpacked_rows

    @unpackedJ.setter
    def unpackedJ(self, v):
        self._unpacked_rows = v
        if not v:
            self._unpacked_tiles = False

    def unpackJ(self, wait_for=None, kind=None):
        kind = kind or ('tiles' if self.sampler_plan()[0] == 'skew' else 'rows')
        if kind == 'rows':
            if self._unpacked_rows:
                return wait_for
            s = self._begin()
            _lib.call('mi3_unpack_j', self._ptr('J'), self._ptr('Junpacked'), self.L, self.q, self._s)
            self._unpacked_rows = True
        else:
            if self._unpacked_tiles:
                return wait_for
            self._ensure_tiles()
            s = self._begin()
            self._unpack_tiles(self._s)
            self._unpacked_tiles = True
        return self.logevt('unpackJ', s)

    def _ensure_tiles(self):
        n = int(_lib.query('mi3_jtiles_floats', self.L, self.q))
        if 'Jtiles' not in self.bufs or self.bufs['Jtiles'].numel() != n * self.skew_replicas:
            with torch.cuda.device(self.device):
                self.bufs['Jtiles'] = torch.empty(n * self.skew_replicas, dtype=torch.float32, device=self.device)
            self._unpacked_tiles = False

    def _unpack_tiles(self, stream_ptr):
        n = int(_lib.query('mi3_jtiles_floats', self.L, self.q))
        for r in range(self.skew_replicas):
            _lib.call('mi3_unpack_j_tiles', self._ptr('J'), self._ptr('Jtiles') + 4 * n * r, self.L, self.q,
                      stream_ptr)

    def unpack_call(self, stream_ptr):
        """Launch the unpacking kernel of the current sampler plan on
        stream_ptr (for callers that record it themselves, e.g. in a CUDA
        graph, where J changes on the device)."""
        if self.sampler_plan()[0] == 'skew':
            self._ensure_tiles()
            self._unpack_tiles(stream_ptr)
        else:
            _lib.call('mi3_unpack_j', self._ptr('J'), self._ptr('Junpacked'), self.L, self.q, stream_ptr)

    # ------------------------------------------------------------ sampler plans
    # The skewed-lane sampler (mi3_metropolis_skew) gives the same
    # trajectories as the row-streaming one; it takes q <= 21 and
    # L + 31 <= 288.  Untuned, it is used from SKEW_MIN_Q on with at least
    # one CTA per SM (B200, 2048-step calls: 8.7e9 vs 6.1e9 site-updates/s at
    # L=232, q=21, 2^20 walkers; even at L=60, q=21; slower at q=4, where
    # the row kernel's gathers mostly hit the same address and broadcast).
    SKEW_DEFAULT = True
    SKEW_MIN_Q = 16
    # copies of the tiled table; CTAs read different copies, so that their
    # simultaneous reads of one coupling row spread over more L2 slices
    skew_replicas = 1

    def skew_supported(self):
        """The skewed-lane kernel takes 2 <= q <= 21 and L + 31 <= 576
        (L + 31 <= 288 with 512 or 768 walkers per CTA, else 256)."""
        return 2 <= self.q <= 21 and self.L + 31 <= 576 and self.nseq['main'] % 32 == 0

    def sampler_plan(self):
        """The plan runMCMC uses: ('skew', walkers_per_cta) or a
        (walkers_per_cta, sites_per_chunk, stages) triple of the
        row-streaming kernel ((0, 0, 0): its built-in choice).  Set by
        autotune.Autotuner.tune as metro_plan; otherwise the skewed-lane
        kernel where it applies."""
        plan = getattr(self, 'metro_plan', None)
        if plan:
            return tuple(plan)
        if (self.SKEW_DEFAULT and self.skew_supported() and self.q >= self.SKEW_MIN_Q
                and self.nseq['main'] >= 148 * 512):
            return ('skew', 512 if self.L + 31 <= 288 else 256)
        return (0, 0, 0)

    def sampler_call(self, pos_offset, pos_ptr, nsteps, seq_ptr, rng_ptr, status_ptr, stream_ptr, betas=None,
                     plan=None):
        """One sampler launch with the given plan (default: sampler_plan())
        on caller-chosen buffers; J must already be unpacked for it."""
        plan = tuple(plan) if plan else self.sampler_plan()
        N, L, q = self.nseq['main'], self.L, self.q
        if plan[0] == 'skew':
            _lib.call('mi3_metropolis_skew', self._ptr('Jtiles'), rng_ptr, int(pos_offset), pos_ptr, int(nsteps),
                      betas, self.beta, seq_ptr, N, L, q, int(plan[1]), self.skew_replicas, status_ptr, stream_ptr)
        else:
            _lib.call('mi3_metropolis_plan', self._ptr('Junpacked'), rng_ptr, int(pos_offset), pos_ptr, int(nsteps),
                      betas, self.beta, seq_ptr, N, L, q, plan[0], plan[1], plan[2], status_ptr, stream_ptr)

    # ------------------------------------------------------------ sampler
    def _initMCMC_RNG(self, rng_offset, rng_span, wait_for=None):
        self.require('MCMC')
        rng_offset = np.uint64(rng_offset)
        nwalkers = np.uint64(self.nseq['main'])
        v2 = np.uint64(2)
        walker_span = np.uint64(rng_span) // (v2 * nwalkers)
        assert walker_span * v2 * nwalkers <= np.uint64(rng_span)
        self.log("RNG offset: {}  walker-span: {}  nwalkers {}".format(rng_offset, walker_span, nwalkers))
        s = self._begin()
        _lib.call('mi3_init_rng', self._ptr('rngstates'), int(nwalkers), int(rng_offset), int(walker_span),
                  self._s)
        return self.logevt('initMCMC_RNG', s)

    def updateRngPos(self, wait_evt=None):
        """Shared site list, refilled from the host MT19937 stream every
        1024 calls (mcmcGPU.py:447-458)."""
        self.randpos_offset = self.randpos_offset + self.nsteps
        rng_evt = None
        bufsize = rng_buf_mul * self.nsteps
        if self.randpos_offset >= bufsize:
            rng = self.rngstate.randint(0, self.L, size=bufsize).astype('u4')
            rng_evt = self.setBuf('randpos', rng)
            self.randpos_offset = 0
        return np.uint32(self.randpos_offset), rng_evt

    def runMCMC(self, wait_for=None):
        """Performs a single round of mcmc sampling (nsteps MC steps)"""
        self.require('MCMC')
        self.unpackJ()
        rngoffset, _ = self.updateRngPos()
        self.repackedSeqT['main'] = False
        s = self._begin()
        betas = self._ptr('Bs') if getattr(self, 'tempering', False) else None
        self.sampler_call(rngoffset, self._ptr('randpos'), self.nsteps, self._ptr('seq main'),
                          self._ptr('rngstates'), self._ptr('status'), self._s, betas=betas)
        return self.logevt('mcmc', s)

    # ------------------------------------------------------------ statistics
    # alphabet sizes for which the tcgen05 one-hot GEMM counts beat the
    # shared-memory histogram when nothing was tuned (measured on B200 at
    # 2^18 walkers against the lanes-over-pairs histogram: 2.5x at q=4, 2.2x
    # at q=5, 1.8x at q=6, a tie at q=8 and at 2^14 walkers, slower from
    # q=12 on); both give identical integers.
    TENSOR_COUNT_Q = range(4, 7)
    # the same for the weighted bimarginals (three byte-plane integer GEMMs
    # against the shared-memory fixed-point histogram, identical results):
    # since the histogram visits pairs with lanes over pairs it is as fast at
    # q=4 (0.40 vs 0.40 ms at L=99, 2^18) and faster from q=5 on, so the
    # tensor-core form is left to the autotuner's per-shape timing
    TENSOR_WMARG_Q = range(0)

    def calcBicounts(self, seqbufname, wait_for=None, tensor=None):
        nseq, buflen = self._span(seqbufname)
        if tensor is None:
            tuned = getattr(self, 'count_kernel', None)  # set by autotune.Autotuner.tune
            tensor = (tuned == 'tc') if tuned else self.q in self.TENSOR_COUNT_Q
        s = self._begin()
        if tensor:
            _lib.call('mi3_bicounts_tc', self.seqbufs[seqbufname].data_ptr(), buflen, nseq,
                      self._ptr('bicount'), self.L, self.q, self._ptr('status'), self._s)
        else:
            _lib.call('mi3_bicounts', self.seqbufs[seqbufname].data_ptr(), buflen, nseq, self._ptr('bicount'),
                      self.L, self.q, self._s)
        return self.logevt('calcBicounts', s)

    def bicounts_to_bimarg(self, seqbufname='main', wait_for=None):
        nseq = self._span(seqbufname)[0]
        s = self._begin()
        _lib.call('mi3_bicounts_to_bimarg', self._ptr('bicount'), self._ptr('bi'), nseq, self.L, self.q,
                  self._s)
        return self.logevt('bicounts_to_bimarg', s)

    # Consensus decomposition thresholds: the fraction of site pairs at which
    # neither residue is its site's consensus, below which the consensus
    # kernels are used.  Measured at L=232 q=21 with 59% of pairs left: the
    # energy pass drops from 9.8 to 8.5 ms; the weighted histogram does not
    # gain (its masked shared-memory reductions become divergent branches,
    # which costs what the saved bank conflicts give back), so it keeps the
    # direct kernel unless nearly all pairs are skipped.
    # Since the direct pair kernels visit full slices with lanes over pairs
    # (conflict-free, tiling.cuh), the direct energy pass is faster than the
    # consensus one at every shape measured (energies of dJ on sampled
    # walkers: 5.55 vs 8.46 ms at L=232, q=21, 2^20; 0.39 vs 0.51 ms at L=99,
    # q=4, 2^18; 0.27 vs 0.28 ms at L=60, q=8, 2^18), so it is off: the
    # consensus energies are used only for alphabets up to CONS_ENERGY_MAX_Q.
    CONS_ENERGY_MAX_ACTIVE = 0.75
    CONS_ENERGY_MAX_Q = 0
    CONS_WMARG_MAX_ACTIVE = 0.2

    def updateConsensus(self, seqbufname='main'):
        """Most frequent residue of every site of the walkers -> 'cons', and
        the fraction of site pairs where neither residue is the consensus.
        When that fraction is small enough, the energies of 'dJ' (through the
        consensus gauge) and weightedMarg (bins rebuilt exactly from site
        sums) skip the other pairs; the residues only steer the work split,
        so stale ones stay correct.  No counterpart in the reference."""
        L, q = self.L, self.q
        if L * q * 4 + L > 160 * 1024 or (L * q + 1) * 8 > 200 * 1024:
            return None  # shapes the consensus kernels do not take
        if 'cons' not in self.bufs:
            self._setupBuffer('cons', '<u1', (L,))
            self._setupWorkspace('ws cons', _lib.query('mi3_site_consensus_workspace', L, q))
            self._setupWorkspace('ws energies cons', _lib.query('mi3_energies_cons_workspace', L, q,
                                                                self._ws_nseq))
        nseq, buflen = self._span(seqbufname)
        s = self._begin()
        _lib.call('mi3_site_consensus', self.seqbufs[seqbufname].data_ptr(), buflen, nseq, L, q, self._ptr('cons'),
                  self._ptr('ws cons'), self._wsbytes('ws cons'), self._s)
        evt = self.logevt('updateConsensus', s)
        # the workspace holds the per-site residue counts (uint64, L x q)
        with torch.cuda.stream(self.stream):
            counts = self.bufs['ws cons'][:L * q].to('cpu').numpy().reshape(L, q).astype(np.float64)
        off = 1.0 - counts.max(axis=1) / max(1, nseq)
        active = (off.sum() ** 2 - (off ** 2).sum()) / (L * (L - 1))
        self.consActive = float(active)
        self.consEnergies = active <= self.CONS_ENERGY_MAX_ACTIVE and self.q <= self.CONS_ENERGY_MAX_Q
        self.consWmarg = active <= self.CONS_WMARG_MAX_ACTIVE
        return evt

    def calcEnergies(self, seqbufname, Jbufname='J', wait_for=None):
        nseq, buflen = self._span(seqbufname)
        s = self._begin()
        # the consensus gauge rounds the regauged couplings (|J'| <= 4 max|J|)
        # to float once: used for the small reweighting energies of dJ, where
        # that is far below the step's statistical error; energies of J keep
        # the exact table
        if getattr(self, 'consEnergies', False) and Jbufname == 'dJ':
            _lib.call('mi3_energies_cons', self._ptr(Jbufname), self.seqbufs[seqbufname].data_ptr(), buflen, nseq,
                      self.Ebufs[seqbufname].data_ptr(), self.L, self.q, self._ptr('cons'),
                      self._ptr('ws energies cons'), self._wsbytes('ws energies cons'), self._s)
        else:
            _lib.call('mi3_energies', self._ptr(Jbufname), self.seqbufs[seqbufname].data_ptr(), buflen, nseq,
                      self.Ebufs[seqbufname].data_ptr(), self.L, self.q, self._ptr('ws energies'),
                      self._wsbytes('ws energies'), self._s)
        return self.logevt('getEnergies', s)

    def min_buf(self, buf, wait_for=None):
        self.require('Jstep')
        buflen = int(np.prod(self.buf_spec[buf][1]))
        if buf in ('E large', 'E tmp large', 'weights large'):
            # the stored part only (the reference scans the whole buffer,
            # which equals it once the buffer has been filled)
            buflen = self.nstoredseqs
        s = self._begin()
        _lib.call('mi3_min_floats', self._ptr(buf), buflen, self._ptr('minout'), self._s)
        return self.logevt('min_buf', s)

    def weight_statistics(self, buf='main', wait_for=None):
        self.require('Jstep')
        nseq = self._span(buf)[0]
        s = self._begin()
        _lib.call('mi3_weight_stats', self._ptr(self._wbufname(buf)), nseq, self._ptr('weightstats'),
                  self._ptr('weightstats64'), self._ptr('ws reduce'), self._wsbytes('ws reduce'), self._s)
        return self.logevt('weight_statistics', s)

    def dE_to_weights(self, buf='main', offset=0., wait_for=None):
        self.require('Jstep')
        nseq = self._span(buf)[0]
        s = self._begin()
        _lib.call('mi3_dE_to_weights', float(offset), self.Ebufs[buf].data_ptr(), self._ptr(self._wbufname(buf)),
                  nseq, self._s)
        return self.logevt('dE_to_weights', s)

    def weights_fused(self, offset=0., buf='main'):
        """dE -> weights, minout = min(0, min dE), weightstats in one pass
        (same results as min_buf + dE_to_weights + weight_statistics)."""
        self.require('Jstep')
        nseq = self._span(buf)[0]
        s = self._begin()
        _lib.call('mi3_weights_fused', float(offset), self.Ebufs[buf].data_ptr(), self._ptr(self._wbufname(buf)), nseq,
                  self._ptr('minout'), self._ptr('weightstats'), self._ptr('weightstats64'),
                  self._ptr('ws reduce'), self._wsbytes('ws reduce'), self._s)
        return self.logevt('weights_fused', s)

    def fixed_beta_weights(self, ref_E, seqbufname='main', wait_for=None):
        self.require('Jstep')
        nseq = self._span(seqbufname)[0]
        s = self._begin()
        _lib.call('mi3_fixed_beta_weights', float(self.beta), float(ref_E), self.Ebufs[seqbufname].data_ptr(),
                  self._ptr(self._wbufname(seqbufname)), nseq, self._s)
        return self.logevt('fixed_beta_weights', s)

    def weightedMarg(self, seqbufname='main', wait_for=None):
        self.require('Jstep')
        nseq, buflen = self._span(seqbufname)
        wbuf = self._ptr(self._wbufname(seqbufname))
        s = self._begin()
        cons = self._ptr('cons') if getattr(self, 'consWmarg', False) else None
        tuned = getattr(self, 'wmarg_kernel', None)  # set by autotune.Autotuner.tune
        tensor = (tuned == 'tc') if tuned else self.q in self.TENSOR_WMARG_Q
        if tensor and cons is None:
            if 'ws wmarg tc' not in self.bufs:
                self._setupWorkspace('ws wmarg tc', _lib.query('mi3_weighted_marg_tc_workspace', self.L, self.q))
            _lib.call('mi3_weighted_marg_tc', wbuf, self.seqbufs[seqbufname].data_ptr(), buflen,
                      nseq, self._ptr('bi'), self.L, self.q, self._ptr('ws wmarg tc'),
                      self._wsbytes('ws wmarg tc'), self._ptr('status'), self._s)
        else:
            _lib.call('mi3_weighted_marg', wbuf, self.seqbufs[seqbufname].data_ptr(), buflen,
                      nseq, self._ptr('bi'), self.L, self.q, cons, self._ptr('ws wmarg'),
                      self._wsbytes('ws wmarg'), self._s)
        return self.logevt('weightedMarg', s)

    def renormalize_bimarg(self, wait_for=None):
        s = self._begin()
        _lib.call('mi3_renormalize_bimarg', self._ptr('bi'), self.L, self.q, self._s)
        return self.logevt('renormalize_bimarg', s)

    def addFloatBuf(self, dstname, srcname, wait_for=None):
        dst, src = self.bufs[dstname], self.bufs[srcname]
        if dst.numel() != src.numel():
            raise Exception('Tried to add bufs of different sizes')
        buflen = int(np.prod(self.buf_spec[dstname][1]))
        s = self._begin()
        _lib.call('mi3_add_float_bufs', dst.data_ptr(), src.data_ptr(), buflen, self._s)
        return self.logevt('addbuf', s)

    def addBiBuffer(self, bufname, otherbuf, wait_for=None):
        selfbuf = self.bufs[bufname]
        if selfbuf.numel() != otherbuf.numel():
            raise Exception('Tried to add bufs of different sizes')
        if otherbuf.device != self.device:
            with torch.cuda.stream(self.stream):
                otherbuf = otherbuf.to(self.device, non_blocking=False)
        s = self._begin()
        _lib.call('mi3_add_float_bufs', selfbuf.data_ptr(), otherbuf.data_ptr(), self.nPairs * self.q * self.q,
                  self._s)
        return self.logevt('addbibuf', s)

    # ------------------------------------------------------------ round work on the device
    def gaugeJ(self, Jbufname='J', outbufname=None):
        """J -> fieldlessGaugeEven(0, J) (changeGauge.py:137-155) in FP64 on
        the device, in place unless outbufname is given; the reference does
        this on the host before every round (NewtonSteps.py:618)."""
        if 'ws gauge' not in self.bufs:
            self._setupWorkspace('ws gauge', _lib.query('mi3_gauge_workspace', self.L, self.q))
        out = outbufname or Jbufname
        s = self._begin()
        _lib.call('mi3_gauge_fieldless_even', self._ptr(Jbufname), self._ptr(out), self.L, self.q,
                  self._ptr('ws gauge'), self._wsbytes('ws gauge'), self._s)
        if out.split()[0] == 'J':
            self.unpackedJ = None
        return self.logevt('gaugeJ', s)

    def bimargStats(self, model='bi', target='bi target', Jbufname='J'):
        """FP64 (SSR, max|t-m|, mean rel. error over t > 0.01, its count,
        X_model, X_target) of bimarg_stats / printstats (NewtonSteps.py:33-54)
        into 'stats64'; returns the FutureBuf of that buffer."""
        if 'ws stats' not in self.bufs:
            self._setupWorkspace('ws stats', _lib.query('mi3_bimarg_stats_workspace', self.L))
            self._setupBuffer('stats64', '<f8', (6,))
        s = self._begin()
        _lib.call('mi3_bimarg_stats', self._ptr(target), self._ptr(model),
                  self._ptr(Jbufname) if Jbufname else None, self.L, self.q, self._ptr('stats64'),
                  self._ptr('ws stats'), self._wsbytes('ws stats'), self._s)
        self.logevt('bimargStats', s)
        return self.getBuf('stats64')

    def peekBuf(self, bufname, n=5):
        """First n elements of a float buffer (a few bytes read back)."""
        dev = self.bufs[bufname]
        with torch.cuda.stream(self.stream):
            host = dev[:n].to('cpu', non_blocking=False)
        return host.numpy().copy()

    # ------------------------------------------------------------ equilibration
    def rankEnergies(self, slot):
        """Average ranks of the walkers' current energies ('E main', from
        calcEnergies) into the device rank buffer `slot` -- the rank
        transform of spearmanr in runMCMC's equilibration test
        (NewtonSteps.py:419-428), done here instead of on the host."""
        n = self.nseq['main']
        name = f'Erank {slot}'
        with torch.cuda.device(self.device):
            if name not in self.bufs:
                self.bufs[name] = torch.empty(n, dtype=torch.float32, device=self.device)
            nb = int(_lib.query('mi3_rank_workspace', n))
            if 'ws rank' not in self.bufs or self.bufs['ws rank'].numel() * 8 < nb:
                self.bufs['ws rank'] = torch.empty(nb // 8 + 2, dtype=torch.int64, device=self.device)
            if 'E sums' not in self.bufs:
                self.bufs['E sums'] = torch.empty(4, dtype=torch.float64, device=self.device)
                self.bufs['E sums32'] = torch.empty(4, dtype=torch.float32, device=self.device)
        s = self._begin()
        ws = self.bufs['ws rank']
        _lib.call('mi3_rank_average', self._ptr('E main'), n, self._ptr(name), ws.data_ptr(), ws.numel() * 8,
                  self._s)
        # sum E (FP64) for the mean energy the log line reports
        _lib.call('mi3_weight_stats', self._ptr('E main'), n, self._ptr('E sums32'), self._ptr('E sums'),
                  self._ptr('ws reduce'), self._wsbytes('ws reduce'), self._s)
        return self.logevt('rankEnergies', s)

    def energyMean(self):
        """Mean of 'E main' as summed by the last rankEnergies (FP64)."""
        with torch.cuda.stream(self.stream):
            v = self.bufs['E sums'][0].to('cpu', non_blocking=False)
        return float(v) / self.nseq['main']

    def rankCorr(self, pairs):
        """Spearman r (FP64, on the device) of each (slot_a, slot_b) pair of
        rank buffers; returns a FutureBuf of the r values in pair order."""
        k = len(pairs)
        with torch.cuda.device(self.device):
            if 'rank r' not in self.bufs or self.bufs['rank r'].numel() < k:
                self.bufs['rank r'] = torch.empty(max(k, 16), dtype=torch.float64, device=self.device)
            if 'ws corr' not in self.bufs:
                nb = int(_lib.query('mi3_rank_corr_workspace'))
                self.bufs['ws corr'] = torch.empty(nb // 8 + 2, dtype=torch.float64, device=self.device)
        n = self.nseq['main']
        ws, r = self.bufs['ws corr'], self.bufs['rank r']
        for i, (a, b) in enumerate(pairs):
            _lib.call('mi3_rank_corr', self._ptr(f'Erank {a}'), self._ptr(f'Erank {b}'), n,
                      r.data_ptr() + 8 * i, ws.data_ptr(), ws.numel() * 8, self._s)
        host = torch.empty(k, dtype=torch.float64, pin_memory=True)
        with torch.cuda.stream(self.stream):
            host.copy_(r[:k], non_blocking=True)
        evt = torch.cuda.Event()
        evt.record(self.stream)
        return FutureBuf(host, evt, lambda b: b.numpy().copy(), self)

    def dropRanks(self):
        """Free the rank buffers of an equilibration run."""
        for name in [b for b in self.bufs if b.startswith('Erank ')]:
            del self.bufs[name]

    # ------------------------------------------------------------ Newton step
    def updateJ(self, gamma, pc, Jbuf='dJ', wait_for=None):
        self.require('Jstep')
        s = self._begin()
        p = self._ptr(Jbuf)
        _lib.call('mi3_update_j', self._ptr('bi target'), self._ptr('bi'), float(gamma), float(pc), p, p,
                  self.L, self.q, self._s)
        self.unpackedJ = False
        return self.logevt('updateJ', s)

    def reg_l1z(self, gamma, pc, lJ, wait_for=None):
        self.require('Jstep')
        s = self._begin()
        _lib.call('mi3_reg_l1z', self._ptr('bi'), float(gamma), float(pc), float(lJ), self._ptr('J'),
                  self._ptr('dJ'), self.L, self.q, self._s)
        self.unpackedJ = None
        return self.logevt('reg_l1z', s)

    def reg_l2z(self, gamma, pc, lJ, wait_for=None):
        self.require('Jstep')
        s = self._begin()
        _lib.call('mi3_reg_l2z', self._ptr('bi'), float(gamma), float(pc), float(lJ), self._ptr('J'),
                  self._ptr('dJ'), self.L, self.q, self._s)
        self.unpackedJ = None
        return self.logevt('reg_l2z', s)

    def _reg(self, entry, name, *args, lambdas=False):
        self.require('Jstep')
        s = self._begin()
        head = [self._ptr('bi')] + ([self._ptr('Xlambdas')] if lambdas else [])
        _lib.call(entry, *head, *[float(a) for a in args], self._ptr('J'), self._ptr('dJ'), self.L, self.q,
                  self._s)
        self.unpackedJ = None
        return self.logevt(name, s)

    def reg_SCADJ(self, gamma, pc, r, a, wait_for=None):
        """SCAD penalty on the zero-gauge couplings (mcmcGPU.py:747-759)."""
        return self._reg('mi3_reg_scadj', 'reg_SCADJ', gamma, pc, r, a)

    def reg_Xij(self, gamma, pc, wait_for=None):
        """X penalty with one lambda per pair from the 'Xlambdas' buffer, the
        semantics of the reg_Xij kernel (mcmc.cl:975-1003; the reference's
        host wrappers for X and Xij call each other's kernels,
        mcmcGPU.py:761-787)."""
        return self._reg('mi3_reg_xij', 'reg_Xij', gamma, pc, lambdas=True)

    def reg_X(self, gamma, pc, lX, wait_for=None):
        """X penalty with one global lambda (reg_X kernel, mcmc.cl:1005-1030)."""
        self.require('Jstep')
        s = self._begin()
        _lib.call('mi3_reg_x', self._ptr('bi'), float(lX), float(gamma), float(pc), self._ptr('J'),
                  self._ptr('dJ'), self.L, self.q, self._s)
        self.unpackedJ = None
        return self.logevt('reg_X', s)

    def reg_SCADX(self, gamma, pc, s, r, a, wait_for=None):
        return self._reg('mi3_reg_scadx', 'reg_SCADX', gamma, pc, s, r, a)

    def reg_expX(self, gamma, pc, lam, wait_for=None):
        return self._reg('mi3_reg_expx', 'reg_expX', gamma, pc, lam)

    def reg_ddE(self, gamma, pc, lam, wait_for=None):
        return self._reg('mi3_reg_dde', 'reg_ddE', gamma, pc, lam)

    def reg_SCADddE(self, gamma, pc, lam, r, wait_for=None):
        return self._reg('mi3_reg_scaddde', 'reg_SCADddE', gamma, pc, lam, r)

    # ------------------------------------------------------------ host I/O
    def getBuf(self, bufname, truncateLarge=True, wait_for=None):
        """Copy a device buffer to host; returns a FutureBuf
        (mcmcGPU.py:845-867)."""
        if bufname == 'Junpacked' and self._unpacked_tiles and not self._unpacked_rows:
            # the skewed-lane sampler unpacked J into the tiled layout only;
            # build the rows a reader of 'Junpacked' expects from the same J
            self.unpackJ(kind='rows')
        buftype, bufshape = self.buf_spec[bufname]
        dev = self.bufs[bufname]
        host = self._readback_buffer(bufname, dev)
        s = self._begin()
        with torch.cuda.stream(self.stream):
            host.copy_(dev, non_blocking=True)
        evt = getattr(self, '_ring_pending', None) or torch.cuda.Event()
        self._ring_pending = None
        evt.record(self.stream)
        self.logevt('getBuf', s, host.numel() * host.element_size())
        L, q = self.L, self.q

        if bufname == 'Junpacked':
            stride = int(_lib.query('mi3_jrows_stride', L, q))

            def post(b):
                a = b.numpy().reshape(L, stride)[:, :L * q * q]
                return a.reshape(L * L, q * q).copy()
            return FutureBuf(host, evt, post, self)

        shape = _full_shape(buftype, bufshape)
        # the large buffers return only their stored part unless asked
        # otherwise (mcmcGPU.py:845-867) -- those indexed by sequence: the
        # transposed 'seqL large' (sites first) is returned whole
        nret = None
        if bufname in self.largebufs and truncateLarge and bufname != 'seqL large':
            nret = self.nstoredseqs

        def post(b):
            a = b.numpy().view(_base_dtype(buftype))
            a = a[:int(np.prod(shape))].reshape(shape)
            if bufname.split()[0] == 'seq':
                return self.unpackSeqs_4(a)[:nret]
            return a[:nret].copy()
        return FutureBuf(host, evt, post, self)

    def setBuf(self, bufname, buf, wait_for=None):
        """Host (numpy) or device (tensor) -> device buffer, with the
        reference's dtype/shape checks (mcmcGPU.py:869-907)."""
        dev = self.bufs[bufname]
        if isinstance(buf, torch.Tensor):
            s = self._begin()
            with torch.cuda.stream(self.stream):
                if buf.device != self.device:
                    buf = buf.to(self.device)
                src = buf.reshape(-1).view(dev.dtype) if buf.dtype != dev.dtype else buf.reshape(-1)
                dev[:src.numel()].copy_(src, non_blocking=True)
            evt = self.logevt('setBuf', s, src.numel() * src.element_size())
            if bufname.split()[0] == 'J':
                self.unpackedJ = None
            return evt

        if bufname.split()[0] == 'seq':
            buf = self.packSeqs_4(np.asarray(buf))

        buftype, bufshape = self.buf_spec[bufname]
        if not isinstance(buf, np.ndarray):
            buf = np.array(buf, dtype=buftype)
        if np.dtype(buftype) != buf.dtype:
            raise ValueError("Buffer dtype mismatch.Expected {}, got {}".format(np.dtype(buftype), buf.dtype))
        if _full_shape(buftype, bufshape) != buf.shape and not (bufshape == (1,) or buf.size == 1):
            raise ValueError("Buffer size mismatch. Expected {}, got {}".format(bufshape, buf.shape))

        raw = np.ascontiguousarray(buf).reshape(-1).view(np.uint8)
        host = self._staging_for(bufname, raw.size)
        host.numpy()[:] = raw
        s = self._begin()
        with torch.cuda.stream(self.stream):
            dev.view(torch.uint8)[:raw.size].copy_(host, non_blocking=True)
        evt = torch.cuda.Event()
        evt.record(self.stream)
        self._staging[bufname][1] = evt
        self.logevt('setBuf', s, raw.size)
        if bufname.split()[0] == 'J':
            self.unpackedJ = None
        if bufname == 'seq large':
            self.nstoredseqs = bufshape[1]
        if bufname.split()[0] == 'seq':
            self.repackedSeqT[bufname.split()[1]] = False
        return evt

    def _readback_buffer(self, bufname, dev):
        """Pinned host buffer for a device->host read.  Small buffers (the
        per-step scalars of the Newton loop) come from a ring of 4 per name, so
        a loop does not pin fresh memory every step; a FutureBuf older than 4
        reads of the same name must have been read before it is reused."""
        nbytes = dev.numel() * dev.element_size()
        if nbytes > (1 << 20):
            return torch.empty(dev.shape, dtype=dev.dtype, pin_memory=True)
        rings = getattr(self, '_rings', None)
        if rings is None:
            rings = self._rings = {}
        ring = rings.get(bufname)
        if ring is None:
            ring = rings[bufname] = [[torch.empty(dev.shape, dtype=dev.dtype, pin_memory=True), None]
                                     for _ in range(4)] + [0]
        k = ring[4]
        ring[4] = (k + 1) % 4
        ent = ring[k]
        if ent[1] is not None:
            ent[1].synchronize()
        evt = torch.cuda.Event()
        ent[1] = evt
        self._ring_pending = evt
        return ent[0]

    def _staging_for(self, bufname, nbytes):
        """Pinned host staging buffer reused per device buffer; waits for the
        previous copy out of it before handing it back."""
        st = getattr(self, '_staging', None)
        if st is None:
            st = self._staging = {}
        ent = st.get(bufname)
        if ent is not None and ent[0].numel() >= nbytes:
            if ent[1] is not None:
                ent[1].synchronize()
            return ent[0][:nbytes]
        host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        st[bufname] = [host, None]
        return host

    def fillBuf(self, bufname, val, wait_for=None):
        dev = self.bufs[bufname]
        with torch.cuda.stream(self.stream):
            if dev.dtype in (torch.float32, torch.float64):
                dev.fill_(float(val))
            else:
                dev.fill_(int(val))
        self.logevt('fill_buffer')

    def fillSeqs(self, startseq, seqbufname='main', wait_for=None):
        nseq = self.nseq[seqbufname]
        self.setBuf('seq ' + seqbufname, np.tile(np.asarray(startseq, dtype='<u1'), (nseq, 1)))

    def packedSeqs(self, bufname='main'):
        """The device sequence buffer 'seq <bufname>' as a (SWORDS, nseq)
        int32 tensor view (4 residues per word, walker-minor)."""
        n = self.nseq[bufname]
        return self.bufs['seq ' + bufname][:self.SWORDS * n].view(self.SWORDS, n)

    def snapshotSeqs(self, bufname='main'):
        """A device copy of the walkers of 'seq <bufname>' (restoreSnapshot
        puts it back without a host round trip)."""
        with torch.cuda.stream(self.stream):
            return self.packedSeqs(bufname).clone()

    def restoreSnapshot(self, snap, bufname='main'):
        s = self._begin()
        with torch.cuda.stream(self.stream):
            self.packedSeqs(bufname).copy_(snap, non_blocking=True)
        self.repackedSeqT[bufname] = False
        return self.logevt('restoreSnapshot', s, snap.numel() * 4)

    def _largeCols(self, offset, n):
        """Columns [offset, offset+n) of 'seq large' as a (SWORDS, n) view."""
        return self.packedSeqs('large')[:, offset:offset + n]

    def storeSeqs(self, seqs=None, wait_for=None):
        """Append sequences to the large buffer after the ones stored so far
        (mcmcGPU.py:934-978): the walkers of 'seq main' when seqs is None, a
        host (n, L) uint8 array, or -- not in the reference -- a packed
        (SWORDS, n) device tensor, which may live on another device (a peer
        copy), so walkers can be gathered without passing through the host."""
        self.require('Large')
        offset = self.nstoredseqs
        if seqs is None:
            src = self.packedSeqs('main')
        elif isinstance(seqs, torch.Tensor):
            if seqs.dim() != 2 or seqs.shape[0] != self.SWORDS or seqs.element_size() != 4:
                raise ValueError(f"expected packed sequences of shape ({self.SWORDS}, n) with 4-byte words")
            src = seqs.view(torch.int32)
        else:
            seqs = np.asarray(seqs)
            if seqs.ndim != 2 or seqs.shape[1] != self.L:
                raise Exception("Sequences have wrong length: {} vs {}".format(seqs.shape[-1], self.L))
            if seqs.dtype != np.dtype('u1'):
                raise ValueError("seqs must have u1 dtype")
            src = torch.from_numpy(self.packSeqs_4(seqs).view(np.int32)).pin_memory()
        n = int(src.shape[1])
        if offset + n > self.nseq['large']:
            raise Exception("cannot store seqs past end of large buffer")
        s = self._begin()
        with torch.cuda.stream(self.stream):
            # a device tensor is read in this device's stream order: writes to
            # it from another stream must be complete (GPU_node.gatherLarge
            # waits for the source device first)
            self._largeCols(offset, n).copy_(src, non_blocking=True)
        evt = self.logevt('storeSeqs', s, 4 * self.SWORDS * n)
        if not src.is_cuda:
            # keep the pinned staging copy alive until the copy has run
            self._pending_host.append(src)
        self.nstoredseqs += n
        self.repackedSeqT['large'] = False
        return evt

    def clearLargeSeqs(self):
        """Forget the stored sequences (mcmcGPU.py:980-983)."""
        self.require('Large')
        self.nstoredseqs = 0
        self.repackedSeqT['large'] = False

    def restoreSeqs(self, offset=0, wait_for=None):
        """Copy nseq['main'] stored sequences, from column `offset` of the
        large buffer, back into 'seq main' (mcmcGPU.py:985-999, whose offset
        is not defined in the reference; here it is an argument)."""
        self.require('Large')
        nseq = self.nseq['main']
        if offset + nseq > self.nseq['large']:
            raise Exception("cannot get seqs past end of large buffer")
        if self.nstoredseqs < nseq:
            raise Exception("not enough seqs stored in large buffer")
        s = self._begin()
        with torch.cuda.stream(self.stream):
            self.packedSeqs('main').copy_(self._largeCols(offset, nseq), non_blocking=True)
        self.repackedSeqT['main'] = False
        return self.logevt('restoreSeqs', s, 4 * self.SWORDS * nseq)

    # ------------------------------------------------------------ MSA text
    def _text_scratch(self, nbytes):
        """Device byte buffer of at least nbytes (grown, never shrunk)."""
        buf = self.bufs.get('text')
        if buf is None or buf.numel() < nbytes:
            with torch.cuda.device(self.device):
                buf = torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=self.device)
            self.bufs['text'] = buf
            if 'status text' not in self.bufs:
                self._setupBuffer('status text', '<i4', (1,))
                self._setupBuffer('first bad', '<u8', (1,))
        return buf

    def getSeqsText(self, bufname='main', alpha=None):
        """The walkers of 'seq <bufname>' as the lines of an MSA file in the
        reference's format (mi3_seqs_to_text; seqload.py:378-411): a
        FutureBuf whose read() returns nseq*(L+1) uint8 bytes (for 'large',
        the stored part).  alpha defaults to seqload.default_alpha(q)."""
        alpha = seqload._as_bytes(alpha if alpha is not None else seqload.default_alpha(self.q))
        nseq, buflen = self._span(bufname)
        nbytes = nseq * (self.L + 1)
        dev = self._text_scratch(nbytes)
        self.fillBuf('status text', 0)
        s = self._begin()
        _lib.call('mi3_seqs_to_text', self.seqbufs[bufname].data_ptr(), buflen, nseq, self.L, alpha, len(alpha),
                  dev.data_ptr(), self._ptr('status text'), self._s)
        host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        st = torch.empty(1, dtype=torch.int32, pin_memory=True)
        with torch.cuda.stream(self.stream):
            host.copy_(dev[:nbytes], non_blocking=True)
            st.copy_(self.bufs['status text'], non_blocking=True)
        evt = torch.cuda.Event()
        evt.record(self.stream)
        self.logevt('getSeqsText', s, nbytes)

        def post(b):
            if int(st[0]) != 0:
                raise ValueError("a walker holds a residue outside the alphabet {!r}".format(alpha.decode()))
            return b.numpy()
        return FutureBuf(host, evt, post, self)

    def _textToSeqs(self, msa, start, n, bufname, n0):
        if msa.L != self.L:
            raise Exception("Sequences have wrong length: {} vs {}".format(msa.L, self.L))
        if msa.eof_error is not None or start + n > msa.nseq:
            seqload.check(msa)  # raises the reference's error for this file
            raise Exception("need {} sequences from line {}, the file has {}".format(n, start, msa.nseq))
        nbytes = n * msa.line_len
        dev = self._text_scratch(nbytes)
        host = self._staging_for('text', nbytes)
        host.numpy()[:] = msa.body[start * msa.line_len:(start + n) * msa.line_len]
        s = self._begin()
        with torch.cuda.stream(self.stream):
            dev[:nbytes].copy_(host, non_blocking=True)
        evt = torch.cuda.Event()
        evt.record(self.stream)
        self._staging['text'][1] = evt
        _lib.call('mi3_text_to_seqs', dev.data_ptr(), n, msa.line_len, msa.id_len, self.L, msa.alpha,
                  len(msa.alpha), self.seqbufs[bufname].data_ptr(), self.nseq[bufname], n0,
                  self._ptr('first bad'), self._s)
        self.logevt('setSeqsText', s, nbytes)
        with torch.cuda.stream(self.stream):
            first = int(self.bufs['first bad'].cpu()[0])
        if first != -1:  # UINT64_MAX: every line is well formed
            seqload.check(msa)
            raise ValueError("Sequence {} is malformed".format(start + first + 1))
        self.repackedSeqT[bufname] = False

    def setSeqsText(self, bufname, msa, start=0):
        """Lines [start, start + nseq) of a parsed MSA file (seqload.MSAText,
        from seqload.read_msa) into 'seq <bufname>', translated on the
        device (mi3_text_to_seqs).  A malformed file raises the reference's
        error for it (seqload.py:196-336).  For 'large' the lines fill the
        whole buffer and become its stored part."""
        n = self.nseq[bufname]
        self._textToSeqs(msa, start, n, bufname, 0)
        if bufname == 'large':
            self.nstoredseqs = n

    def storeSeqsText(self, msa, start=0, n=None):
        """Append lines [start, start + n) of a parsed MSA file to the large
        buffer after its stored part (storeSeqs for file input)."""
        self.require('Large')
        n = msa.nseq - start if n is None else n
        if self.nstoredseqs + n > self.nseq['large']:
            raise Exception("cannot store seqs past end of large buffer")
        self._textToSeqs(msa, start, n, 'large', self.nstoredseqs)
        self.nstoredseqs += n

    # ------------------------------------------------------------ checkpoints
    _STATE_BUFS = ('seq main', 'rngstates', 'randpos')

    def state_dict(self):
        """Host copy of the sampling state: walkers, MWC64X states, the site
        list with its read offset and the MT19937 state that refills it
        (checkpoint.py)."""
        self.stream.synchronize()
        out = {name: self.bufs[name].cpu().numpy().copy() for name in self._STATE_BUFS if name in self.bufs}
        out['randpos_offset'] = int(getattr(self, 'randpos_offset', 0))
        out['rngstate'] = self.rngstate.get_state()
        return out

    def load_state_dict(self, d):
        for name in self._STATE_BUFS:
            if name in d:
                src = torch.from_numpy(np.ascontiguousarray(d[name]))
                if src.shape != self.bufs[name].shape or src.dtype != self.bufs[name].dtype:
                    raise ValueError(f"state of {name!r} does not match this device's buffer")
                with torch.cuda.stream(self.stream):
                    self.bufs[name].copy_(src.to(self.device))
        self.stream.synchronize()
        self.randpos_offset = int(d['randpos_offset'])
        self.rngstate.set_state(d['rngstate'])
        self.repackedSeqT['main'] = False

    def wait(self):
        self.stream.synchronize()
        while self._pending_host:
            self._pending_host.popleft()
        self._check_status()


################################################################################

def printDevice(log, d):
    p = torch.cuda.get_device_properties(d)
    log("  Device '{}':\n".format(p.name))
    log("    Compute capability: {}.{}\n".format(p.major, p.minor))
    log("    Multiprocessors: {}\n".format(p.multi_processor_count))
    log("    Global Mem Size: {}\n".format(p.total_memory))


def unpackJ_CPU(couplings):
    """(nPairs, q*q) -> (L*L, q*q) with the transposed mirror
    (mcmcGPU.py:1022-1034)."""
    from .potts import getLq
    L, q = getLq(couplings)
    full = np.zeros((L * L, q * q), dtype='<f4')
    n = 0
    for i in range(L - 1):
        for j in range(i + 1, L):
            c = couplings[n, :]
            full[L * i + j, :] = c
            full[L * j + i, :] = c.reshape((q, q)).T.flatten()
            n += 1
    return full


def printGPUs(log):
    """List the visible CUDA devices (mcmcGPU.py:58-64 lists OpenCL platforms)."""
    for n in range(torch.cuda.device_count()):
        printDevice(log, torch.device('cuda', n))
        log("")


def setup_GPU_context(scriptpath, scriptfile, param, log):
    """Select the CUDA devices to use, with the reference's signature and
    return shape (mcmcGPU.py:1038-1100): (context data, devices, (info,
    build log)).  There is no run-time compilation -- the kernels are
    prebuilt for sm_100a -- so scriptpath/scriptfile are not read and the
    context data is None.  param.gpuspec: None (all visible devices) or a
    comma separated list of device indices (an OpenCL "platform:device"
    entry uses its device index)."""
    if not torch.cuda.is_available():
        raise Exception("Error: No GPUs found")
    _lib.load()
    if param.get('gpuspec') is not None:
        try:
            devs = [int(x.split(':')[-1]) for x in str(param['gpuspec']).split(',')]
        except ValueError:
            raise Exception("Error: GPU specification must be a comma separated list of devices, eg '0,1'")
        for d in devs:
            if not 0 <= d < torch.cuda.device_count():
                raise Exception("No GPU with specification {}".format(d))
    else:
        devs = list(range(torch.cuda.device_count()))
    if not devs:
        raise Exception("Error: No GPUs found")
    log("Using CUDA devices {}".format(devs))
    info = "libmi3b200 ABI {} (sm_100a)".format(_lib.load().mi3_abi_version())
    return None, [torch.device('cuda', d) for d in devs], (info, "")


def initGPU(devnum, cldat, device, nwalkers, param, log):
    """(mcmcGPU.py:1102-1119) -- cldat is setup_GPU_context's context data
    (unused)."""
    wgsize = param.get('wgsize', 512)
    if wgsize not in [1 << n for n in range(32)]:
        raise Exception("wgsize must be a power of two")
    return MCMCGPU((device, devnum), param['L'], param['q'], nwalkers, wgsize, param.get('outdir'), 1024,
                   param.get('rngseed', 0), profile=param.get('profile', False), beta=param.get('beta'))


def wgsize_heuristic(q, wgsize='auto'):
    if wgsize == 'auto':
        wgsize = 256
        while wgsize < q * q:
            wgsize *= 2
        return wgsize
    wgsize = int(wgsize)
    if wgsize < q * q:
        raise Exception("Must have wgsize >= q*q, but got {} < {}".format(wgsize, q * q))
    return wgsize


def histogram_heuristic(q):
    """(NHIST, HISTWS) of the reference (mcmcGPU.py:1135-1163); kept for
    interface parity -- the B200 kernels pick their own tiling."""
    nhist = 4096 // (q * q)
    if nhist == 0:
        raise Exception("alphabet size too large to make histogram on gpu")
    nhist = 2 ** int(np.log2(nhist))
    if q <= 12:
        hist_ws = 512
    elif q <= 16:
        hist_ws = 256
    else:
        hist_ws = 128
    if nhist > hist_ws:
        nhist = hist_ws
    return nhist, hist_ws
