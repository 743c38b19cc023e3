"""A CPU stand-in for MCMCGPU used only to test the host logic (GPU_node,
NewtonSteps) without a GPU.  Every method computes with the CPU oracle, so
it also documents what each device call must do."""
import numpy as np

from oracle import oracle
from mi3gpu_b200.mcmcGPU import rng_buf_mul


class _Fut:
    def __init__(self, v):
        self.v = v

    def read(self):
        return self.v


class FakeMCMCGPU:
    def __init__(self, L, q, nseq, seed, gpunum=0):
        self.L, self.q, self.nseq, self.nwalkers = L, q, {'main': nseq}, nseq
        self.nPairs = L * (L - 1) // 2
        self.gpunum = gpunum
        self.rngstate = np.random.RandomState(seed)
        self.device = 'cpu'
        self.bufs = {'J': np.zeros((self.nPairs, q * q), '<f4'), 'bi': np.zeros((self.nPairs, q * q), '<f4'),
                     'bicount': np.zeros((self.nPairs, q * q), '<u4'),
                     'seq main': np.zeros((oracle.swords(L), nseq), '<u4'), 'E main': np.zeros(nseq, '<f4'),
                     'minout': np.zeros(1, '<f4'), 'cprob': np.zeros((L, q - 1), '<f4')}
        self.calls = []
        self.largebufs = []
        self.nstoredseqs = 0

    # sequence buffers: 'main', or the stored part of 'large'
    def _seqs(self, name):
        if name == 'main':
            return self.bufs['seq main']
        return self.bufs['seq ' + name][:, :self.nstoredseqs]

    def _n(self, name):
        return self.nseq['main'] if name == 'main' else self.nstoredseqs

    @staticmethod
    def _w(name):
        return 'weights' if name == 'main' else 'weights ' + name

    def initLargeBufs(self, n):
        self.nseq['large'] = int(n)
        self.bufs.update({'seq large': np.zeros((oracle.swords(self.L), n), '<u4'), 'E large': np.zeros(n, '<f4'),
                          'E tmp large': np.zeros(n, '<f4'), 'weights large': np.zeros(n, '<f4')})
        self.largebufs = ['seq large', 'E large', 'weights large']
        self.nstoredseqs = 0

    def packedSeqs(self, name='main'):
        return self.bufs['seq ' + name].view(np.int32)

    def storeSeqs(self, seqs=None):
        if seqs is None:
            seqs = self.bufs['seq main']
        elif not isinstance(seqs, np.ndarray):  # a tensor of packed words
            seqs = seqs.cpu().numpy()
        seqs = np.asarray(seqs)
        if seqs.dtype == np.uint8:
            seqs = oracle.pack_seqs(seqs)
        seqs = seqs.view('<u4')
        n, off = seqs.shape[1], self.nstoredseqs
        if off + n > self.nseq['large']:
            raise Exception("cannot store seqs past end of large buffer")
        self.bufs['seq large'][:, off:off + n] = seqs
        self.nstoredseqs += n

    def clearLargeSeqs(self):
        self.nstoredseqs = 0

    def snapshotSeqs(self, bufname='main'):
        return self.bufs['seq ' + bufname].copy()

    def restoreSnapshot(self, snap, bufname='main'):
        self.bufs['seq ' + bufname] = snap.copy()

    def getSeqsText(self, bufname='main', alpha=None):
        from mi3gpu_b200 import seqload
        alpha = alpha if alpha is not None else seqload.default_alpha(self.q)
        text, bad = oracle.seqs_to_text(self._seqs(bufname), self.L, alpha)
        if bad:
            raise ValueError("a walker holds a residue outside the alphabet")
        return _Fut(text)

    def setSeqsText(self, bufname, msa, start=0):
        from mi3gpu_b200 import seqload
        n = self.nseq[bufname]
        if msa.eof_error is not None or start + n > msa.nseq:
            seqload.check(msa)
            raise Exception("not enough sequences")
        mem, first = oracle.text_to_seqs(msa.lines(start, start + n).reshape(-1), n, msa.line_len, msa.id_len,
                                         self.L, msa.alpha)
        if first is not None:
            seqload.check(msa)
            raise ValueError("Sequence {} is malformed".format(start + first + 1))
        self.bufs['seq ' + bufname] = mem
        if bufname == 'large':
            self.nstoredseqs = n

    def initMCMC(self, nsteps, rng_offset, rng_span):
        self.nsteps = int(nsteps)
        ws = int(rng_span) // (2 * self.nwalkers)
        self.rng_offset, self.walker_span = int(rng_offset), ws
        self.bufs['rngstates'] = oracle.init_rng(self.nwalkers, int(rng_offset), ws)
        self.bufs['randpos'] = np.zeros(self.nsteps * rng_buf_mul, '<u4')
        self.randpos_offset = rng_buf_mul * self.nsteps

    def initJstep(self):
        z = lambda: np.zeros((self.nPairs, self.q * self.q), '<f4')
        self.bufs.update({'dJ': z(), 'bi target': z(), 'weights': np.zeros(self.nwalkers, '<f4'),
                          'weightstats': np.zeros(2, '<f4'), 'weightstats64': np.zeros(2, '<f8'),
                          'E tmp': np.zeros(self.nwalkers, '<f4')})

    def updateRngPos(self):
        self.randpos_offset += self.nsteps
        if self.randpos_offset >= rng_buf_mul * self.nsteps:
            self.bufs['randpos'] = self.rngstate.randint(0, self.L, size=rng_buf_mul * self.nsteps).astype('u4')
            self.randpos_offset = 0
        return self.randpos_offset

    def runMCMC(self):
        off = self.updateRngPos()
        oracle.metropolis(self.bufs['J'], self.bufs['rngstates'], self.bufs['randpos'], off, self.nsteps,
                          self.bufs['seq main'], self.L, self.q)
        self.calls.append('runMCMC')

    def calcEnergies(self, seqbufname, Jbufname='J'):
        n = self._n(seqbufname)
        self.bufs['E ' + seqbufname][:n] = oracle.energies_f64(self.bufs[Jbufname], self._seqs(seqbufname),
                                                               self.L, self.q).astype('<f4')

    def calcBicounts(self, seqbufname):
        self.bufs['bicount'] = oracle.bicounts(self._seqs(seqbufname), self.L, self.q)

    # the device-side equilibration test (rank buffers and their correlations)
    def rankEnergies(self, slot):
        self.bufs[f'Erank {slot}'] = oracle.rank_average(self.bufs['E main']).astype('<f4')
        self.bufs['E sums'] = np.array([np.sum(self.bufs['E main'], dtype=np.float64)])

    def rankCorr(self, pairs):
        out = []
        for a, b in pairs:
            ra = self.bufs[f'Erank {a}'].astype(np.float64)
            rb = self.bufs[f'Erank {b}'].astype(np.float64)
            m = 0.5 * (len(ra) + 1)
            da, db = ra - m, rb - m
            saa, sbb = np.dot(da, da), np.dot(db, db)
            out.append(np.dot(da, db) / np.sqrt(saa * sbb) if saa > 0 and sbb > 0 else np.nan)
        return _Fut(np.array(out))

    def energyMean(self):
        return float(self.bufs['E sums'][0]) / self.nseq['main']

    def dropRanks(self):
        for k in [b for b in self.bufs if b.startswith('Erank ')]:
            del self.bufs[k]

    def bicounts_to_bimarg(self, seqbufname='main'):
        self.bufs['bi'] = oracle.bicounts_to_bimarg(self.bufs['bicount'], self._n(seqbufname))

    def updateJ(self, gamma, pc, Jbuf='dJ'):
        self.bufs[Jbuf] = oracle.updatedJ(self.bufs['bi target'], self.bufs['bi'], gamma, pc, self.bufs[Jbuf])

    def reg_l1z(self, gamma, pc, lJ):
        self.bufs['dJ'] = oracle.reg_lz(self.bufs['bi'], gamma, pc, lJ, self.bufs['J'], self.bufs['dJ'], self.q, False)

    def min_buf(self, buf):
        v = self.bufs[buf]
        if buf in self.largebufs or buf == 'E tmp large':
            v = v[:self.nstoredseqs]
        self.bufs['minout'][0] = oracle.min_floats(v)

    def dE_to_weights(self, buf='main', offset=0.):
        n = self._n(buf)
        self.bufs[self._w(buf)][:n] = oracle.dE_to_weights(offset, self.bufs['E ' + buf][:n])

    def weight_statistics(self, buf='main'):
        w = self.bufs[self._w(buf)][:self._n(buf)]
        self.bufs['weightstats'] = oracle.weight_stats(w)
        self.bufs['weightstats64'] = oracle.weight_stats_f64(w)

    def weights_fused(self, offset=0., buf='main'):
        self.min_buf('E ' + buf)
        self.dE_to_weights(buf, offset)
        self.weight_statistics(buf)

    def weightedMarg(self, seqbufname='main'):
        w = self.bufs[self._w(seqbufname)][:self._n(seqbufname)]
        self.bufs['bi'] = oracle.weighted_marg_f64(w, self._seqs(seqbufname), self.L, self.q).astype('<f4')

    def renormalize_bimarg(self):
        self.bufs['bi'] = oracle.renormalize_bimarg(self.bufs['bi'], self.q)

    def prepare_indep(self, unimarg):
        c = np.cumsum(unimarg, axis=1)
        self.bufs['cprob'] = (c[:, :-1] / c[:, -1, None]).astype('<f4')

    def gen_indep(self, bufname):
        oracle.gen_indep(self.bufs['seq main'], self.bufs['rngstates'], self.bufs['cprob'], self.L, self.q)

    def getBuf(self, name):
        v = self.bufs[name]
        if name in self.largebufs:
            v = v[..., :self.nstoredseqs]
        if name.startswith('seq'):
            return _Fut(oracle.unpack_seqs(v, self.L))
        return _Fut(np.array(v, copy=True))

    def setBuf(self, name, v):
        if name.startswith('seq'):
            v = oracle.pack_seqs(v)
        if hasattr(v, 'cpu'):  # a tensor from another device
            v = v.cpu().numpy().view(self.bufs[name].dtype).reshape(self.bufs[name].shape)
        self.bufs[name] = np.array(v, copy=True)
        if name == 'seq large':
            self.nstoredseqs = self.bufs[name].shape[1]

    def fillBuf(self, name, val):
        self.bufs[name][...] = val

    def fillSeqs(self, seq):
        self.setBuf('seq main', np.tile(np.asarray(seq, '<u1'), (self.nwalkers, 1)))

    def addFloatBuf(self, dst, src):
        self.bufs[dst] = (self.bufs[dst] + self.bufs[src]).astype('<f4')

    def updateConsensus(self, seqbufname='main'):
        pass

    def gaugeJ(self, Jbufname='J'):
        self.bufs[Jbufname] = oracle.gauge_fieldless_even(self.bufs[Jbufname], self.L, self.q).astype('<f4')

    def bimargStats(self, model='bi', target='bi target', Jbufname='J'):
        J = self.bufs[Jbufname] if Jbufname else None
        return _Fut(np.array(oracle.bimarg_stats_f64(self.bufs[target], self.bufs[model], J)))

    def peekBuf(self, name, n=5):
        return np.asarray(self.bufs[name]).reshape(-1)[:n].copy()

    def addBiBuffer(self, name, other):
        self.bufs[name] = self.bufs[name] + other

    def state_dict(self):
        out = {k: np.array(self.bufs[k], copy=True) for k in ('seq main', 'rngstates', 'randpos') if k in self.bufs}
        out['randpos_offset'] = int(self.randpos_offset)
        out['rngstate'] = self.rngstate.get_state()
        return out

    def load_state_dict(self, d):
        for k in ('seq main', 'rngstates', 'randpos'):
            if k in d:
                self.bufs[k] = np.array(d[k], copy=True)
        self.randpos_offset = int(d['randpos_offset'])
        self.rngstate.set_state(d['rngstate'])

    def logProfile(self):
        pass

    def wait(self):
        pass
