"""Autotuner for the shape-dependent choices of the B200 kernels.

The sampler's plan (the skewed-lane kernel with 512 or 768 walkers per CTA,
or a tile plan of the row-streaming kernel: walkers per CTA, sites per
streamed coupling chunk, ring stages, which `mi3_metropolis_plans` lists;
all give the same trajectories), the bimarginal
count kernel and the weighted-bimarginal kernel (shared-memory histogram or
tcgen05 one-hot GEMM, which give the same integers) are picked per
(L, q, walkers) by timing every candidate once on the device, from the caller's own walker state copied to scratch buffers
so the chain itself is not advanced.  Results are kept in memory and, when a
cache path is given, in a JSON file keyed by device name and shape.

The reference has a heuristic work-group size for its count kernel
(mcmcGPU.py:1135-1163) and fixed launch sizes otherwise; nothing is tuned.
"""
import ctypes
import json
import os
from pathlib import Path

import torch

from . import _lib


def _events_time(stream, fn, reps):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / reps


def sampler_plans(L, q, nseq):
    """All valid plans: ('skew', walkers_per_cta) for the skewed-lane
    kernel where it applies, then the (walkers_per_cta, sites_per_chunk,
    stages) plans of the row-streaming kernel."""
    plans = []
    if 2 <= q <= 21 and L + 31 <= 576 and nseq % 32 == 0:
        plans += ([('skew', 512), ('skew', 768)] if L + 31 <= 288 else []) + [('skew', 256)]
    n = int(_lib.query('mi3_metropolis_plans', L, q, nseq, None, 0))
    buf = (ctypes.c_uint32 * (3 * max(n, 1)))()
    _lib.query('mi3_metropolis_plans', L, q, nseq, buf, n)
    return plans + [tuple(int(v) for v in buf[3 * k:3 * k + 3]) for k in range(n)]


def _plan_key(plan):
    return ",".join(map(str, plan))


def _plan_from_json(v):
    return tuple(v[:1] + [int(x) for x in v[1:]]) if v and v[0] == 'skew' else tuple(int(x) for x in v)


class Autotuner:
    def __init__(self, cache_path=None):
        self.cache_path = Path(cache_path) if cache_path else None
        self.table = {}
        if self.cache_path is not None and self.cache_path.exists():
            try:
                self.table = json.loads(self.cache_path.read_text())
            except (ValueError, OSError):
                self.table = {}  # unreadable cache: tune again

    def _key(self, kind, gpu, extra=""):
        name = torch.cuda.get_device_name(gpu.device).replace(" ", "_")
        return f"{name}/{kind}/L{gpu.L}/q{gpu.q}/N{gpu.nseq['main']}{extra}"

    def _save(self):
        """Write the table atomically; processes sharing the file (one per
        GPU) each write a private temporary and the last rename wins, so a
        reader sees some complete table."""
        if self.cache_path is None:
            return
        self.cache_path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.cache_path.with_name(f"{self.cache_path.name}.{os.getpid()}.tmp")
        tmp.write_text(json.dumps(self.table, indent=1, sort_keys=True))
        os.replace(tmp, self.cache_path)

    def sampler_plan(self, gpu, probe_steps=None, reps=2):
        """Fastest sampler plan for gpu's shape; times `reps` launches of
        probe_steps proposals per walker (default two sweeps) for every plan
        on scratch copies of the walkers and RNG states.  Returns
        (plan, {plan: ms})."""
        key = self._key("metropolis", gpu)
        if key in self.table:
            return _plan_from_json(self.table[key]["plan"]), self.table[key].get("ms", {})
        gpu.require('MCMC')
        gpu.unpackJ(kind='rows')
        if gpu.skew_supported():
            gpu.unpackJ(kind='tiles')
        L, q, N = gpu.L, gpu.q, gpu.nseq['main']
        steps = int(probe_steps or min(gpu.nsteps, 2 * L))
        with torch.cuda.stream(gpu.stream):
            seq = gpu.bufs['seq main'].clone()
            rng = gpu.bufs['rngstates'].clone()
            status = torch.zeros(1, dtype=torch.int32, device=gpu.device)
            # a scratch site list: the device's own list may not be filled yet
            gen = torch.Generator(device='cpu').manual_seed(L * 1000 + q)
            pos = torch.randint(0, L, (steps,), generator=gen, dtype=torch.int32).to(gpu.device)
        s = gpu.stream.cuda_stream
        times = {}
        for plan in sampler_plans(L, q, N):
            def run(plan=plan):
                gpu.sampler_call(0, pos.data_ptr(), steps, seq.data_ptr(), rng.data_ptr(), status.data_ptr(), s,
                                 plan=plan)
            run()
            times[plan] = _events_time(gpu.stream, run, reps)
        if int(status.item()) != 0:
            raise RuntimeError("sampler reported status {} while tuning".format(int(status.item())))
        best = min(times, key=times.get)
        self.table[key] = {"plan": list(best), "ms": {_plan_key(k): v for k, v in times.items()},
                           "probe_steps": steps}
        self._save()
        return best, self.table[key]["ms"]

    def count_kernel(self, gpu, reps=3):
        """'tc' or 'smem': the faster exact count kernel for gpu's shape
        (the tcgen05 kernel takes 4 <= q <= 32)."""
        key = self._key("counts", gpu)
        if key in self.table:
            return self.table[key]["kernel"]
        if not 4 <= gpu.q <= 32:
            self.table[key] = {"kernel": "smem"}
            self._save()
            return "smem"
        times = {}
        for kind in ("smem", "tc"):
            fn = (lambda k=kind: gpu.calcBicounts('main', tensor=(k == 'tc')))
            fn()
            times[kind] = _events_time(gpu.stream, fn, reps)
        best = min(times, key=times.get)
        self.table[key] = {"kernel": best, "ms": times}
        self._save()
        return best

    def wmarg_kernel(self, gpu, reps=3):
        """'tc' or 'smem': the faster weighted-bimarginal kernel for gpu's
        shape (identical results), timed with scratch weights."""
        key = self._key("wmarg", gpu)
        if key in self.table:
            return self.table[key]["kernel"]
        if not 4 <= gpu.q <= 32 or 'weights' not in gpu.bufs:
            self.table[key] = {"kernel": "smem"}
            self._save()
            return "smem"
        with torch.cuda.stream(gpu.stream):
            saved = gpu.bufs['weights'].clone()
            gen = torch.Generator(device='cpu').manual_seed(gpu.L)
            w = torch.exp(-0.5 * torch.rand(saved.numel(), generator=gen)).to(gpu.device)
            gpu.bufs['weights'].copy_(w)
        prev = getattr(gpu, 'wmarg_kernel', None)
        times = {}
        for kind in ("smem", "tc"):
            gpu.wmarg_kernel = kind
            fn = (lambda: gpu.weightedMarg('main'))
            fn()
            times[kind] = _events_time(gpu.stream, fn, reps)
        gpu.wmarg_kernel = prev
        with torch.cuda.stream(gpu.stream):
            gpu.bufs['weights'].copy_(saved)
        best = min(times, key=times.get)
        self.table[key] = {"kernel": best, "ms": times}
        self._save()
        return best

    def tune(self, gpu):
        """Tune every choice for gpu and install them on it."""
        plan, _ = self.sampler_plan(gpu)
        gpu.metro_plan = tuple(plan)
        gpu.count_kernel = self.count_kernel(gpu)
        gpu.wmarg_kernel = self.wmarg_kernel(gpu)
        return {"metropolis_plan": gpu.metro_plan, "count_kernel": gpu.count_kernel,
                "wmarg_kernel": gpu.wmarg_kernel}
