"""Device-group facade: the reference's GPU_node (mi3gpu/node_manager.py:44-312).

The host algorithm talks to a GPU_node, which fans each call out to its
MCMCGPU devices and merges results.  The hot path of this library runs on one
device; with one device merge_bimarg is the renormalisation, exactly as in the
reference (node_manager.py:283-287).  Several devices in one process are
still accepted (walkers split across them, bimarginals summed on device 0),
for completeness rather than speed.
"""
import numpy as np

from . import seqload


def sumarr(arrlist):
    tot = arrlist[0].copy()
    for a in arrlist[1:]:
        np.add(tot, a, tot)
    return tot


def meanarr(arrlist):
    return sumarr(arrlist) / len(arrlist)


def skip_single(f):
    def skipper(x):
        if len(x) == 1:
            return x[0]
        return f(x)
    return skipper


class GPU_node:
    def __init__(self, gpus):
        self.gpus = gpus

    @property
    def head_node(self):
        return self  # one node (node_manager.py:47)

    @property
    def head_gpu(self):
        return type(self)([self.gpus[0]])

    @property
    def nwalkers(self):
        return sum(g.nwalkers for g in self.gpus)

    @property
    def nseq(self):
        ret = {'main': sum(g.nseq['main'] for g in self.gpus)}
        if 'large' in self.gpus[0].nseq:
            ret['large'] = sum(g.nseq.get('large', 0) for g in self.gpus)
        return ret

    @property
    def ngpus(self):
        return len(self.gpus)

    @property
    def gpu_list(self):
        return ["({}) {}".format(g.gpunum, g.device) for g in self.gpus]

    def initMCMC(self, nsteps):
        # the MWC64X period 2^63 split evenly across devices (node_manager.py:73-81)
        rng_span = np.uint64(2 ** 63) // np.uint64(self.ngpus)
        rng_offsets = [np.uint64(i) * rng_span for i in range(self.ngpus)]
        self._initMCMC_rng(nsteps, rng_offsets, rng_span)

    def _initMCMC_rng(self, nsteps, rng_offsets, rng_span):
        for gpu, offset in zip(self.gpus, rng_offsets):
            gpu.initMCMC(nsteps, offset, rng_span)

    def initJstep(self):
        for gpu in self.gpus:
            gpu.initJstep()

    def initLargeBufs(self, nseq):
        """Large sequence buffers on every device: one size for all, or one
        per device (node_manager.py:87-93)."""
        sizes = nseq if isinstance(nseq, (list, tuple)) else [nseq] * self.ngpus
        for n, gpu in zip(sizes, self.gpus):
            gpu.initLargeBufs(n)

    def initSubseq(self):
        for gpu in self.gpus:
            gpu.initSubseq()

    def markPos(self, marks):
        for gpu in self.gpus:
            gpu.markPos(marks)

    def copySubseq(self, seqind):
        for gpu in self.gpus:
            gpu.copySubseq(seqind)

    def storeSeqs(self, seqs=None):
        for gpu in self.gpus:
            gpu.storeSeqs(seqs)

    def clearLargeSeqs(self):
        for gpu in self.gpus:
            gpu.clearLargeSeqs()

    def gatherLarge(self, target):
        """Every device's walkers, in device order, into the large buffers of
        `target` (a GPU_node over some of these devices, e.g. head_gpu), split
        in order across its devices as np.split would.  The reference does
        this through the host, collect('seq main') then
        target.setSeqs('large', ...) (NewtonSteps.py:181-191); here the
        columns are copied device to device.  Large buffers that do not exist
        yet are created, one equal share per target device
        (Mi3.py:450-457)."""
        total = self.nwalkers
        if 'large' not in target.gpus[0].nseq:
            if total % target.ngpus:
                raise Exception("{} walkers do not split over {} devices".format(total, target.ngpus))
            target.initLargeBufs(total // target.ngpus)
        sizes = [g.nseq['large'] for g in target.gpus]
        if sum(sizes) != total:
            raise Exception("Expected {} total sequences, got {}".format(sum(sizes), total))
        self.wait()  # every device's walkers are final before they are read
        target.clearLargeSeqs()
        ti = 0
        for g in self.gpus:
            n, a = g.nseq['main'], 0
            while a < n:
                t = target.gpus[ti]
                k = min(sizes[ti] - t.nstoredseqs, n - a)
                if t is g and a == 0 and k == n:
                    t.storeSeqs(None)  # this device's own walkers
                else:
                    t.storeSeqs(g.packedSeqs('main')[:, a:a + k])
                a += k
                if t.nstoredseqs == sizes[ti]:
                    ti += 1
        target.wait()

    # ------------------------------------------------------ MSA files
    is_writer = True  # this process writes the files

    def collectText(self, bufname='main', alpha=None):
        """Every device's walkers as MSA text lines, in device order."""
        futs = [g.getSeqsText(bufname, alpha) for g in self.gpus]
        return [f.read() for f in futs]

    def writeSeqs(self, fn, bufname='main', alpha=None, zipf=None, headers=None, write_param=False,
                  background=False):
        """Write the walkers as an MSA file in the reference's format (what
        writeSeqs(fn, collect('seq main'), alpha) writes, seqload.py:353-411),
        formatting the lines on the devices.  background=True returns once
        the lines are in host memory and leaves compression and the file
        write to a background thread (overlapping the devices' next work);
        flushWrites() waits for them and raises their errors."""
        alpha = alpha if alpha is not None else seqload.default_alpha(self.gpus[0].q)
        parts = self.collectText(bufname, alpha)
        if not self.is_writer:
            return
        parts = [seqload.header_bytes(alpha, headers, write_param)] + parts
        if not background:
            seqload.write_text(fn, parts, zipf)
            return
        pending = self.__dict__.setdefault('_pending_writes', [])
        pending.append(seqload.background_writer().submit(seqload.write_text, fn, parts, zipf))

    def flushWrites(self):
        """Wait for the background file writes of writeSeqs."""
        pending = self.__dict__.get('_pending_writes') or []
        self._pending_writes = []
        for f in pending:
            f.result()

    def loadSeqs(self, fn, bufname='main', alpha=None, zipf=None):
        """Fill 'seq <bufname>' of every device, in order, from an MSA file
        (as setSeqs(bufname, loadSeqs(fn)[0]) would), parsing the lines on
        the devices; returns the file's headers."""
        msa = fn if isinstance(fn, seqload.MSAText) else seqload.read_msa(
            fn, alpha if alpha is not None else seqload.default_alpha(self.gpus[0].q), zipf)
        total = self.nseq[bufname]
        if msa.nseq != total or msa.eof_error is not None:
            if msa.eof_error is not None:
                seqload.check(msa)
            raise Exception("Expected {} total sequences, got {}".format(total, msa.nseq))
        start = 0
        for g in self.gpus:
            g.setSeqsText(bufname, msa, start)
            start += g.nseq[bufname]
        return msa.headers

    def shareJ(self, head):
        """Copy the couplings of head's first device to every other device
        (after a Newton phase that ran on `head` only)."""
        src = head.gpus[0]
        src.wait()
        for g in self.gpus:
            if g is not src:
                g.setBuf('J', src.bufs['J'])
        self.wait()

    def logProfile(self):
        for gpu in self.gpus:
            gpu.logProfile()

    def prepare_indep(self, unimarg):
        for gpu in self.gpus:
            gpu.prepare_indep(unimarg)

    def gen_indep(self, bufname):
        for gpu in self.gpus:
            gpu.gen_indep(bufname)

    def runMCMC(self):
        for gpu in self.gpus:
            gpu.runMCMC()

    def updateConsensus(self, seqbufname='main'):
        for gpu in self.gpus:
            gpu.updateConsensus(seqbufname)

    def calcEnergies(self, seqbufname, Jbufname='J'):
        for gpu in self.gpus:
            gpu.calcEnergies(seqbufname, Jbufname)

    # the device-side equilibration test ranks each device's own walkers, so
    # it stands for the reference's test over all walkers on one device only
    def deviceRanks(self):
        return self.ngpus == 1 and hasattr(self.gpus[0], 'rankEnergies')

    def rankEnergies(self, slot):
        self.gpus[0].rankEnergies(slot)

    def rankCorr(self, pairs):
        return self.gpus[0].rankCorr(pairs).read()

    def energyMean(self):
        return self.gpus[0].energyMean()

    def dropRanks(self):
        self.gpus[0].dropRanks()

    def calcBicounts(self, seqbufname):
        for gpu in self.gpus:
            gpu.calcBicounts(seqbufname)

    def bicounts_to_bimarg(self, seqbufname='main'):
        for gpu in self.gpus:
            gpu.bicounts_to_bimarg(seqbufname)

    def updateJ(self, gamma, pc, Jbuf='dJ'):
        for gpu in self.gpus:
            gpu.updateJ(gamma, pc, Jbuf)

    def reg(self, name, param):
        meth = 'reg_{}'.format(name)
        for gpu in self.gpus:
            getattr(gpu, meth)(*param)

    def min_buf(self, buf):
        for gpu in self.gpus:
            gpu.min_buf(buf)

    def weight_statistics(self, buf='main'):
        for gpu in self.gpus:
            gpu.weight_statistics(buf)

    def dE_to_weights(self, offset=0., buf='main'):
        # argument order as in the reference facade (node_manager.py:148-150)
        for gpu in self.gpus:
            gpu.dE_to_weights(offset, buf)

    def weights_fused(self, offset=0., buf='main'):
        for gpu in self.gpus:
            gpu.weights_fused(offset, buf)

    def fixed_beta_weights(self, ref_E, seqbufname='main'):
        for gpu in self.gpus:
            gpu.fixed_beta_weights(ref_E, seqbufname)

    def weightedMarg(self, seqbufname):
        for gpu in self.gpus:
            gpu.weightedMarg(seqbufname)

    def addFloatBuf(self, dstname, srcname):
        for gpu in self.gpus:
            gpu.addFloatBuf(dstname, srcname)

    def renormalize_bimarg(self):
        for gpu in self.gpus:
            gpu.renormalize_bimarg()

    def gaugeJ(self, Jbufname='J'):
        """Every device holds the same J: re-gauge each copy in place."""
        for gpu in self.gpus:
            gpu.gaugeJ(Jbufname)

    def bimargStats(self, model='bi', target='bi target', Jbufname='J'):
        """FP64 statistics of the head device's (merged) bimarginals."""
        return [self.gpus[0].bimargStats(model, target, Jbufname)]

    def getBuf(self, bufname):
        return [gpu.getBuf(bufname) for gpu in self.gpus]

    def readBufs(self, bufnames):
        if isinstance(bufnames, str):
            return [buf.read() for buf in self.getBuf(bufnames)]
        futures = [self.getBuf(bn) for bn in bufnames]
        return [[fut.read() for fut in buff] for buff in futures]

    groupfunc = {
        'weights': skip_single(np.concatenate),
        'E': skip_single(np.concatenate),
        'Bs': skip_single(np.concatenate),
        'bicount': skip_single(sumarr),
        'bi': skip_single(meanarr),
        'seq': skip_single(np.concatenate)}

    def collect(self, bufs):
        if isinstance(bufs, str):
            func = self.groupfunc.get(bufs.split()[0], lambda x: x)
            return func(self.readBufs(bufs))
        ret = []
        for bufname, arrs in zip(bufs, self.readBufs(bufs)):
            func = self.groupfunc.get(bufname.split()[0], lambda x: x)
            ret.append(func(arrs))
        return ret

    def setBuf(self, bufname, dat):
        if isinstance(dat, list):
            for gpu, buf in zip(self.gpus, dat):
                gpu.setBuf(bufname, buf)
        else:
            for gpu in self.gpus:
                gpu.setBuf(bufname, dat)

    def fillBuf(self, bufname, val):
        for gpu in self.gpus:
            gpu.fillBuf(bufname, val)

    def setSeqs(self, bufname, seqs, log=None):
        if isinstance(seqs, np.ndarray) or len(seqs) == 1:
            if not isinstance(seqs, np.ndarray):
                seqs = seqs[0]
            nbuf = self.nseq[bufname]
            if seqs.shape[0] != nbuf:
                raise Exception("Expected {} total sequences, got {}".format(nbuf, seqs.shape[0]))
            seqs = np.split(seqs, self.ngpus)
        elif len(seqs) != self.ngpus:
            raise Exception("Expected {} sequence bufs, got {}".format(self.ngpus, len(seqs)))
        if log:
            log("Transferring {} seqs to gpu's {} seq buffer...".format(str([len(s) for s in seqs]), bufname))
        for gpu, seq in zip(self.gpus, seqs):
            gpu.setBuf('seq ' + bufname, seq)

    def fillSeqs(self, seq):
        for gpu in self.gpus:
            gpu.fillSeqs(seq)

    def snapshotSeqs(self, bufname='main'):
        return [gpu.snapshotSeqs(bufname) for gpu in self.gpus]

    def restoreSnapshot(self, snaps, bufname='main'):
        for gpu, snap in zip(self.gpus, snaps):
            gpu.restoreSnapshot(snap, bufname)

    def reduce_node_bimarg(self):
        """Pairwise tree sum of 'bi' onto device 0 (node_manager.py:254-281)."""
        self.wait()
        rgpus = self.gpus
        while len(rgpus) > 1:
            h = (len(rgpus) - 1) // 2 + 1
            for even, odd in zip(rgpus[:h], rgpus[h:]):
                even.addBiBuffer('bi', odd.bufs['bi'])
            for even in rgpus[:h]:
                even.wait()
            rgpus = rgpus[:h]

    def merge_bimarg(self):
        if len(self.gpus) == 1:
            # other code expects merge_bimarg to do renormalization
            self.gpus[0].renormalize_bimarg()
            return
        self.reduce_node_bimarg()
        self.gpus[0].renormalize_bimarg()
        self.wait()
        bibuf = self.gpus[0].bufs['bi']
        for g in self.gpus[1:]:
            g.setBuf('bi', bibuf)  # device-to-device (peer) copy
        self.wait()

    def wait(self):
        for g in self.gpus:
            g.wait()
