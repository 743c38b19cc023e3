"""Learned autoregressive independence proposal for the Potts sampler.

A MADE network (Germain et al., 2015: masked autoencoder for distribution
estimation) over L sites x q residues with two hidden layers of H units
models q(s) = prod_i q(s_i | s_<i).  It is trained by maximum likelihood on
sequences the MCMC itself has equilibrated at the current couplings, then
used as an independence proposal inside a Metropolis-Hastings step:

    accept s' ~ q with probability min(1, exp(-(E(s') - E(s))) q(s) / q(s'))

which leaves the Potts distribution P(s) ~ exp(-E(s)) exactly invariant, so
the sampler stays exact whatever the quality of q.  Proposal steps are
interleaved with ordinary single-site sweeps; when the acceptance rate falls
below a threshold the plain sampler carries on alone.

All arithmetic runs in libmi3b200: the forward, backward and Adam kernels
for training, the MH accept kernel and two samplers.  The tensor-core
sampler (csrc/made_tc.cu) groups the hidden units in blocks of G sites
("blocked" degrees) and runs the products between blocks as tcgen05 GEMMs,
the rest on the CUDA cores; the SIMT sampler (csrc/made.cu) walks the sites
with one forward pass per sample and takes any degrees.  PyTorch tensors
hold the parameters as device memory only.
"""
import math

import numpy as np
import torch

from . import _lib


def made_degrees(L, H, seed=0):
    """Hidden-unit degrees in [1, L-1], cycled so every degree is present."""
    rng = np.random.default_rng(seed)
    m1 = 1 + (np.arange(H) % (L - 1))
    m2 = 1 + (np.arange(H) % (L - 1))
    rng.shuffle(m1)
    rng.shuffle(m2)
    return m1, m2


def blocked_degrees(L, H, G):
    """Hidden degrees for the tensor-core sampler: block b of G sites owns
    the units of degree in (bG, bG+G]; every block gets 0, 16, 32 or 48
    units (about in proportion to its number of degrees), each cycling
    through its degrees, and the units are sorted by degree.  Raises
    ValueError when H cannot be split that way."""
    if H % 16 or G < 1:
        raise ValueError("blocked degrees need H a multiple of 16")
    nb = -(-L // G)
    degs = [list(range(b * G + 1, min(b * G + G, L - 1) + 1)) for b in range(nb)]
    nd = np.array([len(d) for d in degs], dtype=np.float64)
    groups = H // 16
    share = groups * nd / nd.sum()
    cnt = np.floor(share).astype(np.int64)
    order = np.argsort(-(share - cnt), kind="stable")
    cnt[order[:groups - int(cnt.sum())]] += 1
    if cnt.max() > 3 or np.any((cnt > 0) & (nd == 0)):
        raise ValueError(f"cannot place {H} units in blocks of {G} sites (at most 48 per block)")
    m = []
    for b in range(nb):
        m += sorted(degs[b][r % len(degs[b])] for r in range(16 * int(cnt[b])))
    return np.array(m, dtype=np.int64)


TC_TMEM_COLS, TC_MAX_UNITS = 512, 48


def tc_block_size(L, q, H):
    """The block size G (4 or 8, G q <= 32) with which the tensor-core
    sampler runs this network, or None.  The logits of all blocks
    (ceil(L/G) x roundup(G q, 16) columns), one block's layer-2
    accumulator and the walkers' sequence words (ceil(L/4) columns) must
    fit the 512 tensor-memory columns.  The larger block is preferred: at
    L=99, q=4 both run equally fast (4 sites: 32-unit blocks, twice as many
    block boundaries), and the 8-site blocking trained the better proposal
    at H=256."""
    if q not in (4, 8) or H % 16 or H > 512 or L < 2:
        return None
    for G in (8, 4):
        if G * q > 32:
            continue
        nb = -(-L // G)
        n3 = -(-G * q // 16) * 16
        if nb * n3 + TC_MAX_UNITS + -(-L // 4) > TC_TMEM_COLS:
            continue
        try:
            blocked_degrees(L, H, G)
        except ValueError:
            continue
        return G
    return None


def made_masks(L, q, H, seed=0, G=None):
    """MADE connectivity: input (site i) -> hidden-1 k iff m1[k] >= i+1;
    hidden-1 k -> hidden-2 k' iff m2[k'] >= m1[k]; hidden-2 k' -> output
    site i iff i+1 > m2[k'].  Degrees cycled and shuffled, or blocked in
    blocks of G sites when G is given.  Returned in the kernels' layouts:
    mW1T [Lq][H], mW2 [H][H] (row k'), mW3 [Lq][H]."""
    if G:
        m1 = blocked_degrees(L, H, G)
        m2 = m1.copy()
    else:
        m1, m2 = made_degrees(L, H, seed)
    din = np.repeat(np.arange(1, L + 1), q)          # degree of input / output (i, a)
    mW1T = (m1[None, :] >= din[:, None]).astype(np.float32)
    mW2 = (m2[:, None] >= m1[None, :]).astype(np.float32)
    mW3 = (din[:, None] > m2[None, :]).astype(np.float32)
    return mW1T, mW2, mW3, m1, m2


class MadeProposal:
    PARAMS = ("W1T", "b1", "W2", "b2", "W3", "b3")

    def __init__(self, L, q, H=512, device=0, seed=0, lr=1e-3, sampler="auto", G=None, gemm="tc"):
        """sampler: "tc" (tensor-core sampler, blocked degrees), "simt"
        (cycled degrees, the SIMT sampler) or "auto" (tc where it runs);
        G: the tensor-core sampler's block size (default: tc_block_size);
        gemm: the training pass's dense products as BF16 tensor-core GEMMs
        ("tc") or FP32 SIMT loops ("simt")."""
        if gemm not in ("tc", "simt"):
            raise ValueError(f"unknown gemm {gemm!r}")
        self.gemm = gemm
        self.L, self.q, self.H = L, q, H
        self.Lq = L * q
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self.lr = lr
        self.step = 0
        G = G or tc_block_size(L, q, H)
        if sampler == "auto":
            sampler = "tc" if G else "simt"
        if sampler == "tc" and not G:
            raise ValueError(f"no tensor-core sampler plan for L={L}, q={q}, H={H}")
        if sampler not in ("tc", "simt"):
            raise ValueError(f"unknown sampler {sampler!r}")
        self.sampler = sampler
        self.G = G if sampler == "tc" else None
        mW1T, mW2, mW3, m1, m2 = made_masks(L, q, H, seed, G=self.G)
        rng = np.random.default_rng(seed + 1)
        init = {
            "W1T": rng.normal(0, 1.0 / math.sqrt(L), size=(self.Lq, H)) * mW1T,
            "b1": np.zeros(H),
            "W2": rng.normal(0, 1.0 / math.sqrt(H), size=(H, H)) * mW2,
            "b2": np.zeros(H),
            "W3": rng.normal(0, 1.0 / math.sqrt(H), size=(self.Lq, H)) * mW3,
            "b3": np.zeros(self.Lq),
        }
        masks = {"W1T": mW1T, "W2": mW2, "W3": mW3}
        t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=self.device)
        self.p = {k: t(v) for k, v in init.items()}                         # float32 master
        self.pc = {k: torch.empty_like(v) for k, v in self.p.items()}       # bf16-rounded, as float
        self.ph = {k: torch.empty(v.shape, dtype=torch.bfloat16, device=self.device)
                   for k, v in self.p.items() if k.startswith("W")}          # bf16 copies (sampler)
        self.mask = {k: t(v) for k, v in masks.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.p.items()}
        # hidden-2 units grouped by degree, for the sampler
        order = np.argsort(m2, kind="stable")
        starts = np.searchsorted(m2[order], np.arange(L + 1), side="left")
        self.deg2_units = t(order, torch.int32)
        self.deg2_start = t(starts, torch.int32)
        self.m1, self.m2 = m1, m2
        self._ws = {}
        self._tc_ws = None
        self._tc_plan = np.zeros(24, dtype=np.uint64)
        self._tc_dirty = True
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.round_params()

    # ----------------------------------------------------------- plumbing
    @property
    def stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def round_params(self):
        """Refresh the bf16 copies from the float32 master parameters."""
        for k, v in self.p.items():
            _lib.call("mi3_made_round_bf16", v.data_ptr(), self.pc[k].data_ptr(),
                      self.ph[k].data_ptr() if k in self.ph else None, v.numel(), self.stream)
        self._tc_dirty = True

    def _buf(self, name, shape):
        b = self._ws.get(name)
        n = int(np.prod(shape))
        if b is None or b.numel() < n:
            b = self._ws[name] = torch.empty(n, dtype=torch.float32, device=self.device)
        return b[:n].view(*shape)

    # ----------------------------------------------------------- training
    def forward(self, seq, buflen, n0, B):
        """Teacher-forced forward of sequences n0..n0+B of a packed (SWORDS,
        buflen) buffer; returns the activations, logits and log q."""
        H, Lq = self.H, self.Lq
        a = {k: self._buf(k, (B, H)) for k in ("h1", "a1", "h2", "a2")}
        a["logits"] = self._buf("logits", (B, Lq))
        a["logq"] = self._buf("logq", (B,))
        pc = self.pc
        args = (seq.data_ptr(), buflen, n0, B, self.L, self.q, H, pc["W1T"].data_ptr(), pc["b1"].data_ptr(),
                pc["W2"].data_ptr(), pc["b2"].data_ptr(), pc["W3"].data_ptr(), pc["b3"].data_ptr(),
                a["h1"].data_ptr(), a["a1"].data_ptr(), a["h2"].data_ptr(), a["a2"].data_ptr(),
                a["logits"].data_ptr(), a["logq"].data_ptr())
        if self.gemm == "tc":
            ws, nbytes = self._gemm_ws(B)
            _lib.call("mi3_made_forward_tc", *args, ws.data_ptr(), nbytes, self.status.data_ptr(), self.stream)
        else:
            _lib.call("mi3_made_forward", *args, self.stream)
        return a

    def _gemm_ws(self, B):
        nbytes = int(_lib.query("mi3_made_gemm_workspace", B, self.L, self.q, self.H))
        ws = self._ws.get("gemm")
        if ws is None or ws.numel() < nbytes + 1024:
            ws = self._ws["gemm"] = torch.empty(nbytes + 1024, dtype=torch.uint8, device=self.device)
        off = (-ws.data_ptr()) % 1024
        return ws[off:], nbytes

    def backward(self, seq, buflen, n0, B, act):
        """Gradients of the batch-mean NLL into self.g; returns log q per sequence."""
        H, Lq = self.H, self.Lq
        dlog = self._buf("dlogits", (B, Lq))
        X = self._buf("X", (B, Lq))
        dh1, dh2 = self._buf("dh1", (B, H)), self._buf("dh2", (B, H))
        lq = self._buf("lq_bwd", (B,))
        g, pc, m = self.g, self.pc, self.mask
        args = (seq.data_ptr(), buflen, n0, B, self.L, self.q, H, pc["W2"].data_ptr(), pc["W3"].data_ptr(),
                act["h1"].data_ptr(), act["a1"].data_ptr(), act["h2"].data_ptr(), act["a2"].data_ptr(),
                act["logits"].data_ptr(), dlog.data_ptr(), X.data_ptr(), dh1.data_ptr(), dh2.data_ptr(),
                g["W1T"].data_ptr(), g["b1"].data_ptr(), g["W2"].data_ptr(), g["b2"].data_ptr(), g["W3"].data_ptr(),
                g["b3"].data_ptr(), m["W1T"].data_ptr(), m["W2"].data_ptr(), m["W3"].data_ptr(), lq.data_ptr())
        if self.gemm == "tc":
            ws, nbytes = self._gemm_ws(B)
            _lib.call("mi3_made_backward_tc", *args, ws.data_ptr(), nbytes, self.status.data_ptr(), self.stream)
        else:
            _lib.call("mi3_made_backward", *args, self.stream)
        return lq

    def adam_step(self, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        self._tc_dirty = True
        for k, v in self.p.items():
            _lib.call("mi3_made_adam", v.data_ptr(), self.pc[k].data_ptr(),
                      self.ph[k].data_ptr() if k in self.ph else None, self.g[k].data_ptr(), self.m[k].data_ptr(),
                      self.v[k].data_ptr(), self.mask[k].data_ptr() if k in self.mask else None, v.numel(),
                      float(self.lr), beta1, beta2, eps, self.step, self.stream)

    def train(self, seq, nseq, epochs=1, batch=4096, buflen=None, log=None):
        """Maximum-likelihood training on the first nseq sequences of a packed
        (SWORDS, buflen) device buffer; returns the mean NLL of each epoch."""
        buflen = buflen or nseq
        batch = min(batch, nseq)
        hist = []
        for ep in range(epochs):
            tot = torch.zeros((), dtype=torch.float64, device=self.device)
            nb = 0
            for n0 in range(0, nseq - batch + 1, batch):
                act = self.forward(seq, buflen, n0, batch)
                lq = self.backward(seq, buflen, n0, batch, act)
                self.adam_step()
                tot += lq.double().sum()
                nb += 1
            nll = -float(tot.item()) / max(1, nb * batch)
            self.check_status()
            hist.append(nll)
            if log:
                log(f"MADE epoch {ep}: mean NLL {nll:.4f} nats ({nll / self.L:.4f} per site)")
        return hist

    # ----------------------------------------------------------- sampling
    def _tc_prepare(self):
        """Weight tiles and per-block arrays of the tensor-core sampler from
        the current bf16-rounded parameters."""
        m1 = np.ascontiguousarray(self.m1, dtype=np.int32)
        m2 = np.ascontiguousarray(self.m2, dtype=np.int32)
        L, q, H, G = self.L, self.q, self.H, self.G
        nbytes = int(_lib.query("mi3_made_tc_workspace", L, q, H, G, m1.ctypes.data, m2.ctypes.data))
        if nbytes == 0:
            raise ValueError(f"no tensor-core sampler plan for L={L}, q={q}, H={H}, G={G}")
        if self._tc_ws is None or self._tc_ws.numel() < nbytes:
            self._tc_ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        pc = self.pc
        _lib.call("mi3_made_tc_prepare", L, q, H, G, m1.ctypes.data, m2.ctypes.data, pc["W1T"].data_ptr(),
                  pc["b1"].data_ptr(), pc["W2"].data_ptr(), pc["b2"].data_ptr(), pc["W3"].data_ptr(),
                  pc["b3"].data_ptr(), self._tc_ws.data_ptr(), nbytes, self._tc_plan.ctypes.data, self.stream)
        self._tc_dirty = False

    def check_status(self):
        """Raise if a tensor-core kernel (sampler or GEMM) gave up waiting."""
        st = int(self.status.item())
        if st:
            self.status.zero_()
            raise RuntimeError(f"MADE tensor-core kernel: wait timed out (status {st})")

    def sample(self, seq_out, nseq, logq_out, seed, buflen=None, given=False):
        """Draw nseq sequences into a packed buffer (given=False), or compute
        log q of the sequences already there (given=True)."""
        if self.sampler == "tc":
            if self._tc_dirty:
                self._tc_prepare()
            _lib.call("mi3_made_tc_sample", self._tc_plan.ctypes.data, seq_out.data_ptr(), buflen or nseq, nseq,
                      logq_out.data_ptr(), int(seed) & ((1 << 64) - 1), 1 if given else 0, self.status.data_ptr(),
                      self.stream)
            return
        ph, pc = self.ph, self.pc
        _lib.call("mi3_made_sample", self.L, self.q, self.H, ph["W1T"].data_ptr(), pc["b1"].data_ptr(),
                  ph["W2"].data_ptr(), pc["b2"].data_ptr(), ph["W3"].data_ptr(), pc["b3"].data_ptr(),
                  self.deg2_start.data_ptr(), self.deg2_units.data_ptr(), seq_out.data_ptr(), buflen or nseq, nseq,
                  logq_out.data_ptr(), int(seed) & ((1 << 64) - 1), 1 if given else 0, self.stream)


class LearnedSampler:
    """Interleaves independence-MH steps with an MCMCGPU's single-site
    sweeps (one proposal step every `every` sampler calls) and hands over to
    the plain sampler once the acceptance rate falls below `min_accept`."""

    def __init__(self, gpu, made, every=4, min_accept=0.01, seed=1):
        self.gpu, self.made = gpu, made
        self.every, self.min_accept = every, min_accept
        self.seed = seed
        N, sw = gpu.nseq['main'], gpu.SWORDS
        dev = gpu.device
        self.prop = torch.zeros(sw * N, dtype=torch.int32, device=dev)
        self.Ep = torch.zeros(N, dtype=torch.float32, device=dev)
        self.lq = torch.zeros(N, dtype=torch.float32, device=dev)
        self.lqp = torch.zeros(N, dtype=torch.float32, device=dev)
        self.nacc = torch.zeros(1, dtype=torch.int64, device=dev)
        self.ws = torch.zeros(int(_lib.query('mi3_energies_workspace', N)) // 8 + 2, dtype=torch.int64, device=dev)
        self.rounds = 0
        self.accepted = 0
        self.proposed = 0
        self.enabled = True

    def propose(self):
        """One independence-MH step for every walker; returns the acceptance rate."""
        g, m = self.gpu, self.made
        N, L, q = g.nseq['main'], g.L, g.q
        self.rounds += 1
        with torch.cuda.stream(g.stream):
            seq = g.bufs['seq main']
            s = g.stream.cuda_stream
            _lib.call('mi3_energies', g._ptr('J'), seq.data_ptr(), N, N, g._ptr('E main'), L, q,
                      self.ws.data_ptr(), self.ws.numel() * 8, s)
            m.sample(seq, N, self.lq, seed=0, given=True)
            m.sample(self.prop, N, self.lqp, seed=self.seed * 1000003 + self.rounds)
            _lib.call('mi3_energies', g._ptr('J'), self.prop.data_ptr(), N, N, self.Ep.data_ptr(), L, q,
                      self.ws.data_ptr(), self.ws.numel() * 8, s)
            self.nacc.zero_()
            _lib.call('mi3_mh_independence', seq.data_ptr(), self.prop.data_ptr(), N, N, L, g._ptr('E main'),
                      self.Ep.data_ptr(), self.lq.data_ptr(), self.lqp.data_ptr(),
                      self.seed * 7919 + self.rounds, self.nacc.data_ptr(), s)
            acc = int(self.nacc.item())
        m.check_status()
        return self._record(acc, N)

    def _record(self, acc, n):
        """Count one proposal step (acc of n walkers accepted); proposals stop
        for good once a step's acceptance rate is below min_accept."""
        self.accepted += acc
        self.proposed += n
        rate = acc / n
        if rate < self.min_accept:
            self.enabled = False
        return rate

    def sweeps(self, ncalls):
        """ncalls sampler calls, with a proposal step after every `every`-th
        call while proposals are enabled; returns the acceptance rates."""
        g = self.gpu
        rates = []
        for k in range(ncalls):
            g.runMCMC()
            if self.enabled and (k + 1) % self.every == 0:
                rates.append(self.propose())
        return rates
