"""One device per process: the reference's GPU_node over torch.distributed.

The reference spreads walkers over the GPUs of a node (node_manager.py) and
over nodes with MPI (mpi_manager.py).  Here each process drives one device
(launched one rank per GPU, as torchrun does) and RankNode stands in for the
node object that NewtonSteps talks to.  Walkers shard across ranks with
disjoint slices of the MWC64X period (node_manager.py:73-81); sampling has
no exchange.  The quasi-Newton phase has three, all collectives over the
process group (NCCL on GPUs, gloo in the CPU tests):

  * merge_bimarg: sum of the (weighted) bimarginals, then the same
    renormalisation on every rank (node_manager.py:254-304);
  * the reference energy of the next step: min over ranks of min(0, dE);
  * the weight sums behind Neff: FP64 sum over ranks.

Every rank then holds the same J, dJ and bimarginals and takes the same
number of Newton steps, because each computes the stop rule from the same
reduced numbers.  Collectives are issued on the device's own stream.

With distribute_jstep 'head_gpu' the reference gathers all walkers on its
first GPU and runs the Newton phase there while the others wait
(NewtonSteps.py:181-195).  Here every rank gathers all walkers into its own
large buffer (one broadcast per rank) and runs that same head-device phase,
with no collective inside the loop; the couplings are then broadcast from
rank 0, so all ranks continue from identical J by construction.
"""
import numpy as np
import torch
import torch.distributed as dist

from .node_manager import GPU_node


def _as_tensor(buf):
    """The device buffer as a tensor sharing its memory (numpy buffers of
    the CPU test device are wrapped without a copy)."""
    if isinstance(buf, torch.Tensor):
        return buf
    return torch.from_numpy(buf)


class RankNode(GPU_node):
    def __init__(self, gpu, group=None):
        super().__init__([gpu])
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        n = torch.tensor([gpu.nwalkers], dtype=torch.int64)
        ns = [torch.zeros_like(n) for _ in range(self.world)]
        if self._backend() == 'nccl':
            n, ns = n.to(gpu.device), [x.to(gpu.device) for x in ns]
        dist.all_gather(ns, n, group=group)
        self.walkers_per_rank = [int(x.item()) for x in ns]

    def _backend(self):
        return dist.get_backend(self.group)

    # -------------------------------------------------------- shape
    @property
    def head_gpu(self):
        return GPU_node([self.gpus[0]])

    @property
    def head_node(self):
        # the reference accepts 'head_node' only across MPI nodes (Mi3.py:452-455);
        # the ranks of one launch are one node
        raise Exception('"head_node" needs ranks on several nodes; use "head_gpu" or "all"')

    @property
    def nwalkers(self):
        return sum(self.walkers_per_rank)

    @property
    def nseq(self):
        return {'main': self.nwalkers}

    @property
    def ngpus(self):
        return self.world

    def setSeqs(self, bufname, seqs, log=None):
        """This rank's own walkers (node_manager.py:190-221 splits a global
        array across the devices of one process; here every rank passes its
        share)."""
        seqs = seqs[0] if isinstance(seqs, (list, tuple)) else seqs
        g = self.gpus[0]
        if seqs.shape[0] != g.nseq[bufname]:
            raise Exception("Expected {} sequences on rank {}, got {}".format(g.nseq[bufname], self.rank,
                                                                              seqs.shape[0]))
        g.setBuf('seq ' + bufname, seqs)

    def initMCMC(self, nsteps):
        span = np.uint64(2 ** 63) // np.uint64(self.world)
        self.gpus[0].initMCMC(nsteps, np.uint64(self.rank) * span, span)

    # -------------------------------------------------------- exchanges
    def _collective(self, fn):
        stream = getattr(self.gpus[0], 'stream', None)
        if isinstance(stream, (torch.cuda.Stream, torch.cuda.ExternalStream)):
            with torch.cuda.stream(stream):
                fn()
        else:
            fn()

    def _reduce(self, bufname, op):
        t = _as_tensor(self.gpus[0].bufs[bufname])
        self._collective(lambda: dist.all_reduce(t, op=op, group=self.group))

    def gatherLarge(self, target):
        """All ranks' walkers, in rank order, into this rank's large buffer
        (target must be this rank's head_gpu)."""
        g = self.gpus[0]
        if target.gpus != [g]:
            raise ValueError("RankNode gathers into its own device only (head_gpu)")
        total = self.nwalkers
        if 'large' not in g.nseq:
            g.initLargeBufs(total)
        if g.nseq['large'] != total:
            raise Exception("Expected {} total sequences, got {}".format(g.nseq['large'], total))
        g.wait()
        g.clearLargeSeqs()
        mine = _as_tensor(g.packedSeqs('main'))
        for r, n in enumerate(self.walkers_per_rank):
            buf = mine.contiguous() if r == self.rank else torch.empty((mine.shape[0], n), dtype=mine.dtype,
                                                                         device=mine.device)
            self._collective(lambda: dist.broadcast(buf, src=r, group=self.group))
            g.storeSeqs(buf)
        g.wait()

    @property
    def is_writer(self):
        return self.rank == 0

    def collectText(self, bufname='main', alpha=None):
        """Every rank's walkers as MSA text lines, in rank order."""
        return self._gather(self.gpus[0].getSeqsText(bufname, alpha).read())

    def loadSeqs(self, fn, bufname='main', alpha=None, zipf=None):
        """This rank's share of an MSA file: lines from the sum of the
        previous ranks' walkers on (every rank reads the file)."""
        from . import seqload
        g = self.gpus[0]
        msa = seqload.read_msa(fn, alpha if alpha is not None else seqload.default_alpha(g.q), zipf)
        if msa.nseq != self.nwalkers or msa.eof_error is not None:
            if msa.eof_error is not None:
                seqload.check(msa)
            raise Exception("Expected {} total sequences, got {}".format(self.nwalkers, msa.nseq))
        g.setSeqsText(bufname, msa, sum(self.walkers_per_rank[:self.rank]))
        return msa.headers

    def shareJ(self, head):
        """Rank 0's couplings to every rank (after the head-device phase)."""
        g = self.gpus[0]
        g.wait()
        t = _as_tensor(g.bufs['J'])
        self._collective(lambda: dist.broadcast(t, src=0, group=self.group))
        g.wait()

    def merge_bimarg(self):
        self._reduce('bi', dist.ReduceOp.SUM)
        self.gpus[0].renormalize_bimarg()

    def getBuf(self, bufname):
        if bufname == 'minout':
            self._reduce('minout', dist.ReduceOp.MIN)
        elif bufname in ('weightstats', 'weightstats64'):
            self._reduce(bufname, dist.ReduceOp.SUM)
        return super().getBuf(bufname)

    def _gather(self, arr):
        out = [None] * self.world
        dist.all_gather_object(out, arr, group=self.group)
        return out

    def collect(self, bufs):
        single = isinstance(bufs, str)
        names = [bufs] if single else list(bufs)
        local = [super(RankNode, self).collect(n) for n in names]
        ret = []
        for name, a in zip(names, local):
            kind = name.split()[0]
            if kind == 'bicount':
                t = torch.from_numpy(np.ascontiguousarray(a).astype(np.int64))
                if self._backend() == 'nccl':
                    t = t.to(self.gpus[0].device)
                dist.all_reduce(t, group=self.group)
                a = t.cpu().numpy().astype(a.dtype)
            elif kind in ('E', 'weights', 'Bs', 'seq'):
                a = np.concatenate(self._gather(np.asarray(a)), axis=0)
            elif kind == 'bi':
                a = np.mean(np.stack(self._gather(np.asarray(a))), axis=0).astype(np.asarray(a).dtype)
            ret.append(a)
        return ret[0] if single else ret
