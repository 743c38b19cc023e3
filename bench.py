#!/usr/bin/env python3
"""Benchmark: Metropolis site-updates/s of the B200 sampler at L=232, q=21,
2^20 walkers (the reference-sized inference workload).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step is one runMCMC call: `nsteps` single-site proposals for every walker
at the shared site list (the reference's kernel call, mcmcGPU.py:460-482,
whose throughput MCMCbenchmark reports as MC steps per second, Mi3.py:706-715).
Synthetic data: a ground-truth Potts model with the workload's shape (fields
N(0,1), couplings N(0,0.05^2) plus 3L strong contacts, fieldless-even gauge)
and walkers started from independent-site sequences.

Under torchrun each rank samples its own 2^20 walkers on its own GPU with a
disjoint RNG span (walkers are independent; no collective on the data path),
so scaling is weak; the step time is the max over ranks.

--impl reference times the reference's CPU generator
(extras/mcmcCPUgenThreaded.c, built into oracle/_ref) on the host cores with
all available threads.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L_, Q_, N_ = 232, 21, 1 << 20
METRIC = "site-updates/s"

# (kernel, L, q) -> what bounds the kernel, from its ncu capture (cited)
BINDING_CITED = {
    ("k_metropolis_skew", 232, 21): {
        "resource": "instruction issue", "issue_active": 0.768, "l1tex_throughput": 0.476,
        "shared_wavefronts_per_update": 18.4, "source": "ncu --set full (profiles/metropolis_skew_L232_q21.md)"},
    ("k_metropolis", 232, 21): {
        "resource": "shared-memory pipe", "issue_active": 0.576, "l1tex_throughput": 0.914,
        "shared_wavefronts_per_update": 49.7, "source": "ncu --set full (profiles/metropolis_L232_q21.md)"},
}

# (kernel, L, q, walkers, proposals per call) -> (DRAM bytes read + written
# per launch, where the figure comes from)
TRAFFIC_CITED = {
    ("k_metropolis_skew", 232, 21, 1 << 20, 2048): (
        106627657472.0, "ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum, one full launch "
                        "(profiles/metropolis_skew_L232_q21.md)"),
    ("k_metropolis", 232, 21, 1 << 20, 2048): (
        4638818048.0, "ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum, one full launch "
                      "(profiles/metropolis_L232_q21.md)"),
}
WORKLOAD = "metropolis L=232 q=21 walkers=2^20 (plain native sampler)"


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ CPU legs
def cpu_generator_rate(J, L, q, seconds, procs, seed=0):
    """Run the reference's CPU generator (one walker per process, P
    processes) for about `seconds`; returns (updates/s, sample description)."""
    from oracle import oracle
    exe = oracle.ref_cpu_binary()
    kind = "reference"
    if exe is None:
        return None
    alpha = "ABCDEFGHIJKLMNOPQRSTUVWXYZ"[:q]
    rng = np.random.default_rng(seed)
    start = "".join(alpha[k] for k in rng.integers(0, q, size=L))
    with tempfile.TemporaryDirectory() as td:
        jf = Path(td) / "J.dat"
        np.asarray(J, dtype="<f4").tofile(jf)
        # calibrate on one process
        probe = 200_000
        t0 = time.perf_counter()
        subprocess.run([str(exe), str(jf), str(probe), "1", alpha, start], check=True, stdout=subprocess.DEVNULL)
        per = (time.perf_counter() - t0) / probe
        steps = max(1000, int(seconds / max(per, 1e-12)))
        t0 = time.perf_counter()
        ps = [subprocess.Popen([str(exe), str(jf), str(steps), "1", alpha, start], stdout=subprocess.DEVNULL)
              for _ in range(procs)]
        for p in ps:
            p.wait()
        wall = time.perf_counter() - t0
    rate = procs * steps / wall
    sample = (f"extras/mcmcCPUgenThreaded.c (oracle/_ref/mcmc_cpu), {procs} processes x {steps} "
              f"single-site updates at L={L} q={q}, {wall:.1f} s wall")
    return rate, sample, kind


# ------------------------------------------------------------ GPU arm
def run_gpu(args):
    import torch
    import torch.distributed as dist
    from mi3gpu_b200 import MCMCGPU, GPU_node, _lib
    from mi3gpu_b200.potts import synthetic_ground_truth

    rank, world, local = env_rank()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local if world > 1 else 0)

    L, q, N = args.L, args.q, args.walkers
    J = synthetic_ground_truth(L, q, seed=1001)
    gpu = MCMCGPU((dev, rank), L, q, N, 512, None, 1024, args.seed + 1)
    gpus = GPU_node([gpu])
    span = np.uint64(2 ** 63) // np.uint64(world)
    gpus._initMCMC_rng(args.nsteps, [np.uint64(rank) * span], span)
    # independent-site start (uniform marginals), generated on the device
    gpus.prepare_indep(np.full((L, q), 1.0 / q))
    gpus.gen_indep('main')
    gpus.setBuf('J', J)
    gpus.wait()
    tuned = None
    if not args.no_tune:
        # sampler tile plan and count kernel picked by timing every candidate
        # on scratch copies of the walkers (outside the timed region)
        from mi3gpu_b200.autotune import Autotuner
        t0 = time.time()
        tuned = Autotuner(ROOT / "_build" / "autotune.json").tune(gpu)
        tuned = {"metropolis_plan": list(tuned["metropolis_plan"]), "count_kernel": tuned["count_kernel"],
                 "tuning_s": round(time.time() - t0, 1)}

    s = gpu.stream
    kernel_ms = []

    def step():
        gpu.runMCMC()

    # warm-up
    for _ in range(args.warmup):
        step()
    gpus.wait()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(dev.index) as clk:
        e0.record(s)
        for k in range(args.steps):
            evs[k][0].record(s)
            step()
            evs[k][1].record(s)
        e1.record(s)
        torch.cuda.synchronize(dev)
    gpu._check_status()
    ms = e0.elapsed_time(e1)
    kernel_ms = [a.elapsed_time(b) for a, b in evs]
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())
    updates = float(N) * args.nsteps * args.steps * world
    value = updates / (ms_max / 1e3)

    # ---- end to end through the public API: J from pinned host memory each
    # step (setBuf), the sampler call, and the packed sequences read back.
    Jh = J.copy()
    e2e_steps = max(2, min(args.steps, 5))
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    ee0 = torch.cuda.Event(enable_timing=True)
    ee1 = torch.cuda.Event(enable_timing=True)
    ee0.record(s)
    for _ in range(e2e_steps):
        gpus.setBuf('J', Jh)
        gpus.runMCMC()
        fut = gpu.getBuf('seq main')
        fut.event.synchronize()
    ee1.record(s)
    torch.cuda.synchronize(dev)
    e2e_ms = ee0.elapsed_time(ee1)
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = float(N) * args.nsteps * e2e_steps * world / (float(te.item()) / 1e3)
    h2d = J.nbytes
    d2h = gpu.SWORDS * N * 4

    # ---- roofline of the sampler kernel
    per_launch_ms = statistics.mean(kernel_ms)
    upd_launch = float(N) * args.nsteps
    hbm_bytes_per_update = 4 * ((L - 1) // 4 + 1)          # sequence words per update
    onchip_bytes_per_update = 8 * (L - 1) + hbm_bytes_per_update  # 2 couplings per site + sequence words
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    achieved = upd_launch * hbm_bytes_per_update / (per_launch_ms / 1e3) / 1e9
    plan = gpu.sampler_plan()
    kernel = "k_metropolis_skew" if plan[0] == "skew" else "k_metropolis"
    # DRAM bytes of one full-size launch (2^20 walkers x 2048 proposals),
    # measured by a one-pass ncu capture of this command's own launch; a
    # cited figure, not measured in this run
    traffic, traffic_src = TRAFFIC_CITED.get((kernel, L, q, N, args.nsteps), (None, None))
    binding = BINDING_CITED.get((kernel, L, q))
    # shared-memory load roofline: 148 SMs x 128 B/clk at the sampled clock
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    smem_peak = 148 * 128 * sm_mhz * 1e6 / 1e9
    onchip = upd_launch * onchip_bytes_per_update / (per_launch_ms / 1e3) / 1e9

    newton = run_newton(args, gpu, gpus, dev, world) if args.newton_steps > 0 else None

    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "site-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (ground-truth Potts model of the workload's shape; independent-site start)",
            "config": {"workload": WORKLOAD, "L": L, "q": q, "walkers_per_gpu": N, "nsteps_per_call": args.nsteps,
                       "parallelism": f"walkers x{world} (independent RNG spans)",
                       "l2": "inputs larger than L2 (sequence buffer 243 MB); couplings stay L2-resident by design",
                       "tuned": tuned},
            "e2e": {"value": e2e_value, "unit": "site-updates/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                    "path": "GPU_node.setBuf('J') + runMCMC() + MCMCGPU.getBuf('seq main') (pinned, packed words)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic, "traffic_source": traffic_src,
                         "kernel": kernel, "plan": list(plan),
                         "algorithmic_bytes_per_update": hbm_bytes_per_update,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if pk.exists() else "fallback"},
            "roofline_onchip": {"bound": "smem", "achieved": onchip, "peak": smem_peak, "unit": "GB/s",
                                "frac": onchip / smem_peak, "bytes_per_update": onchip_bytes_per_update,
                                "peak_basis": "148 SM x 128 B/clk x sampled SM clock"},
            "binding_resource": binding,
            "kernel_ms_per_launch": per_launch_ms,
            "newton": newton,
            "gpu_launches": args.steps,
            "clocks": clocks,
        }
    return out, J


def run_newton(args, gpu, gpus, dev, world):
    """Time the Zwanzig-reweighted quasi-Newton step on the sampled walkers
    (the body of NewtonSteps.iterNewton, NewtonSteps.py:217-246): updateJ,
    reg l1z, energies of dJ, weights/min/stats, weighted bimarginals,
    renormalisation, and the per-step host read of the weight sums."""
    import torch
    from mi3gpu_b200.potts import mutation_pc
    L, q, N = args.L, args.q, args.walkers
    s = gpu.stream
    gpu.initJstep()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    # counts of the current walkers (timed separately: bimarginal-count GB/s)
    c0, c1 = ev(), ev()
    gpus.calcBicounts('main')
    c0.record(s)
    for _ in range(3):
        gpus.calcBicounts('main')
    c1.record(s)
    bicount = gpus.collect('bicount')
    count_ms = c0.elapsed_time(c1) / 3
    f = bicount.astype(np.float64) / N
    rng = np.random.default_rng(7)
    f = f * np.exp(rng.normal(0, 0.2, size=f.shape))
    f /= f.sum(axis=1, keepdims=True)
    target = mutation_pc(f, 1 << 16).astype('<f4')
    gpus.setBuf('bi target', target)
    gamma, pc, lJ = 4e-4, 1e-3, 2e-4
    gpus.updateConsensus('main')  # as iterNewton does: the walkers are fixed during the steps
    gpus.calcEnergies('main')
    gpus.calcBicounts('main')
    gpus.bicounts_to_bimarg('main')
    gpus.merge_bimarg()
    gpus.fillBuf('dJ', 0)
    ref_dE = 0.0
    names = ["updateJ+reg", "energies", "weights", "weightedMarg", "renorm"]
    per = {k: 0.0 for k in names}
    nsteps = args.newton_steps

    def one(instrument):
        nonlocal ref_dE
        evs = [ev() for _ in range(6)] if instrument else None
        if instrument:
            evs[0].record(s)
        gpus.updateJ(gamma, pc)
        gpus.reg('l1z', (gamma, pc, lJ))
        if instrument:
            evs[1].record(s)
        gpus.calcEnergies('main', 'dJ')
        if instrument:
            evs[2].record(s)
        gpus.weights_fused(ref_dE, 'main')
        mfut = gpus.getBuf('minout')
        wfut = gpus.getBuf('weightstats64')
        if instrument:
            evs[3].record(s)
        gpus.weightedMarg('main')
        if instrument:
            evs[4].record(s)
        gpus.merge_bimarg()
        if instrument:
            evs[5].record(s)
        w = wfut[0].read()
        ref_dE = float(mfut[0].read()[0])
        if instrument:
            evs[5].synchronize()
            for k in range(5):
                per[names[k]] += evs[k].elapsed_time(evs[k + 1])
        return w[0] ** 2 / w[1]

    for _ in range(3):
        one(False)
    torch.cuda.synchronize(dev)
    t0, t1 = ev(), ev()
    w0 = time.perf_counter()
    t0.record(s)
    for _ in range(nsteps):
        neff = one(False)
    t1.record(s)
    torch.cuda.synchronize(dev)
    wall = (time.perf_counter() - w0) * 1e3 / nsteps
    dev_ms = t0.elapsed_time(t1) / nsteps
    for _ in range(2):
        one(True)
    per = {k: v / 2 for k, v in per.items()}
    return {"steps": nsteps, "ms_per_newton_step": dev_ms, "wall_ms_per_newton_step": wall,
            "kernel_ms": per, "neff_frac_after": float(neff) / N,
            "bicounts_ms": count_ms, "bicounts_GBps": N * L / (count_ms / 1e3) / 1e9,
            "note": "body of iterNewton with reg l1z, fused weights pass, FP64 Neff"}


def time_call(fn, reps, stream):
    import torch
    for _ in range(2):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def run_kernels(args):
    """Per-kernel times of the pair kernels at the benchmark shapes: plain
    shared-memory counts vs tcgen05 FP8 one-hot GEMM counts, energies and
    weighted bimarginals; tensor figures use 2*N*nPairs*q^2 flops."""
    import torch
    from mi3gpu_b200 import _lib
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    fp8_peak = 2 * peaks.get("bf16_tflops", 1590.0)
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream(dev)
    s = st.cuda_stream
    rows = []
    shapes = [(232, 21, 1 << 20), (99, 4, 1 << 18), (48, 4, 16384), (512, 21, 1 << 19), (128, 8, 1 << 18),
              (150, 5, 1 << 18), (150, 6, 1 << 18), (150, 12, 1 << 18)]
    if args.shape:
        shapes = [tuple(int(x) for x in args.shape.split(","))]
    for (L, q, N) in shapes:
        g = torch.Generator(device=dev)
        g.manual_seed(L * q)
        sw = (L - 1) // 4 + 1
        seqb = torch.randint(0, q, (sw * 4, N), device=dev, dtype=torch.uint8, generator=g)
        if L % 4:
            seqb[L:] = 0
        seq = seqb.view(sw, 4, N).permute(0, 2, 1).contiguous().view(torch.int32).view(sw, N)
        npairs = L * (L - 1) // 2
        out = torch.empty(npairs * q * q, dtype=torch.int32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        J = torch.randn(npairs * q * q, device=dev) * 0.05
        E = torch.empty(N, device=dev)
        ws = torch.zeros(N + 2, dtype=torch.int64, device=dev)
        w = torch.rand(N, device=dev) + 0.5
        wws = torch.zeros(int(_lib.query("mi3_weighted_marg_workspace", L, q, N)) // 8 + 2, dtype=torch.int64, device=dev)
        bi = torch.empty(npairs * q * q, device=dev)
        reps = 5 if N * npairs > 1e10 else 20
        t_plain = time_call(lambda: _lib.call("mi3_bicounts", seq.data_ptr(), N, N, out.data_ptr(), L, q, s), reps, st)
        ref = out.clone()
        t_tc = None
        if 4 <= q <= 32:
            t_tc = time_call(lambda: _lib.call("mi3_bicounts_tc", seq.data_ptr(), N, N, out.data_ptr(), L, q,
                                               status.data_ptr(), s), reps, st)
            assert torch.equal(out, ref) and int(status.item()) == 0, "tensor-core counts differ"
        t_e = time_call(lambda: _lib.call("mi3_energies", J.data_ptr(), seq.data_ptr(), N, N, E.data_ptr(), L, q,
                                          ws.data_ptr(), ws.numel() * 8, s), reps, st)
        t_w = time_call(lambda: _lib.call("mi3_weighted_marg", w.data_ptr(), seq.data_ptr(), N, N, bi.data_ptr(), L, q, None,
                                          wws.data_ptr(), wws.numel() * 8, s), reps, st)
        t_etc = None
        if 4 <= q <= 32:
            E_tc = torch.empty_like(E)
            t_etc = time_call(lambda: _lib.call("mi3_energies_tc", J.data_ptr(), seq.data_ptr(), N, N, E_tc.data_ptr(),
                                                L, q, ws.data_ptr(), ws.numel() * 8, status.data_ptr(), s), reps, st)
            assert int(status.item()) == 0
            e_err = float(((E_tc - E).abs() / E.abs().clamp(min=1.0)).max())
            del E_tc
        t_wtc = None
        if 4 <= q <= 32:
            wst = torch.zeros(int(_lib.query("mi3_weighted_marg_tc_workspace", L, q)) // 8 + 2, dtype=torch.int64,
                              device=dev)
            bi_tc = torch.empty_like(bi)
            t_wtc = time_call(lambda: _lib.call("mi3_weighted_marg_tc", w.data_ptr(), seq.data_ptr(), N, N,
                                                bi_tc.data_ptr(), L, q, wst.data_ptr(), wst.numel() * 8,
                                                status.data_ptr(), s), reps, st)
            assert torch.equal(bi_tc, bi) and int(status.item()) == 0, "tensor-core weighted bimarginals differ"
            del wst, bi_tc
        flops = 2.0 * N * npairs * q * q
        r = {"L": L, "q": q, "N": N, "counts_smem_ms": t_plain, "counts_tc_ms": t_tc, "energies_ms": t_e,
             "weighted_ms": t_w, "weighted_tc_ms": t_wtc, "energies_tc_ms": t_etc,
             "energies_tc_max_rel_diff": e_err if t_etc else None, "counts_GBps_smem": N * L / t_plain / 1e6}
        if t_tc:
            r.update(counts_GBps_tc=N * L / t_tc / 1e6, tc_tflops=flops / t_tc / 1e9,
                     tc_frac_of_fp8=flops / t_tc / 1e9 / fp8_peak)
        if t_wtc:
            # three int8 byte planes: 3x the one-hot MACs, at the 8-bit peak
            r.update(wmarg_tc_tops=3 * flops / t_wtc / 1e9, wmarg_tc_frac_of_int8=3 * flops / t_wtc / 1e9 / fp8_peak)
        if t_etc:
            # energies: 2 N (Lq)^2 / 2 over the tile triangle, x2 for hi and lo, at the bf16 peak
            eflops = 2.0 * 2.0 * N * npairs * q * q
            r.update(energies_tc_tflops=eflops / t_etc / 1e9,
                     energies_tc_frac_of_bf16=eflops / t_etc / 1e9 / peaks.get("bf16_tflops", 1590.0))
        rows.append(r)
        del seqb, seq, out, J, E, ws, w, wws, bi
    print(json.dumps({"mode": "kernels", "fp8_peak_tflops": fp8_peak,
                      "fp8_peak_source": "2 x MEASURED_PEAKS.json bf16_tflops (of measured)",
                      "bf16_peak_tflops": peaks.get("bf16_tflops", 1590.0), "rows": rows}))


def run_msa(args):
    """The run directories' 'seqs' files at L=232 q=21 with 2^20 walkers.
    Kernels: walkers -> text lines (mi3_seqs_to_text) and back
    (mi3_text_to_seqs), timed with CUDA events, against the HBM roofline:
    per walker 4*SWORDS bytes of packed words one way and L+1 bytes of text
    the other (both buffers exceed L2).  End to end: a file written or
    loaded through GPU_node.writeSeqs / loadSeqs (device formatting,
    parallel bzip2) against the reference's route for the same file
    (collect the walkers to the host, format them in numpy, one bzip2 stream;
    loadSeqs then setSeqs), both producing the same bytes."""
    import tempfile
    import torch
    from mi3gpu_b200 import GPU_node, MCMCGPU, _lib, seqload
    L, q, N = 232, 21, 1 << 20
    sw = (L - 1) // 4 + 1
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 1)
    node = GPU_node([g])
    seqs = np.random.default_rng(0).integers(0, q, size=(N, L)).astype('u1')
    node.setSeqs('main', seqs)
    alpha = seqload.alpha21.encode()
    text = torch.empty(N * (L + 1), dtype=torch.uint8, device=g.device)
    back = torch.empty_like(g.bufs['seq main'])
    st = torch.zeros(1, dtype=torch.int32, device=g.device)
    bad = torch.zeros(1, dtype=torch.int64, device=g.device)
    s = g.stream.cuda_stream
    fmt_ms = time_call(lambda: _lib.call("mi3_seqs_to_text", g._ptr('seq main'), N, N, L, alpha, len(alpha),
                                         text.data_ptr(), st.data_ptr(), s), 20, g.stream)
    parse_ms = time_call(lambda: _lib.call("mi3_text_to_seqs", text.data_ptr(), N, L + 1, 0, L, alpha, len(alpha),
                                           back.data_ptr(), N, 0, bad.data_ptr(), s), 20, g.stream)
    assert torch.equal(back, g.bufs['seq main']) and int(st.item()) == 0 and int(bad.item()) == -1
    nbytes = N * (4 * sw + L + 1)
    out = {"mode": "msa", "config": {"workload": f"walkers <-> MSA text, L={L} q={q} walkers={N}",
                                     "l2": "buffers larger than L2"},
           "seqs_to_text_ms": fmt_ms, "text_to_seqs_ms": parse_ms,
           "seqs_to_text_GBps": nbytes / fmt_ms / 1e6, "text_to_seqs_GBps": nbytes / parse_ms / 1e6,
           "hbm_peak_GBps": hbm, "seqs_to_text_frac": nbytes / fmt_ms / 1e6 / hbm,
           "text_to_seqs_frac": nbytes / parse_ms / 1e6 / hbm, "bytes_per_walker": 4 * sw + L + 1,
           "host_cores": os.cpu_count()}
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        for zipf in (False, True):
            tag = "bz2" if zipf else "plain"
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            node.writeSeqs(d / f"dev_{tag}", zipf=zipf)
            out[f"write_{tag}_device_s"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            host = node.collect('seq main')
            seqload.write_text(d / f"host_{tag}", [seqload.format_lines(host, seqload.alpha21)], zipf, threads=1)
            out[f"write_{tag}_host_s"] = time.perf_counter() - t0
            same = (d / f"dev_{tag}").read_bytes() == (d / f"host_{tag}").read_bytes() if not zipf else None
            if zipf:
                import bz2
                same = bz2.decompress((d / "dev_bz2").read_bytes()) == bz2.decompress((d / "host_bz2").read_bytes())
            out[f"write_{tag}_same_bytes"] = bool(same)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        node.loadSeqs(d / "dev_plain")
        torch.cuda.synchronize()
        out["load_plain_device_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        host, _, _ = seqload.loadSeqs(d / "dev_plain")
        node.setSeqs('main', host)
        torch.cuda.synchronize()
        out["load_plain_host_s"] = time.perf_counter() - t0
    out["write_bz2_speedup"] = out["write_bz2_host_s"] / out["write_bz2_device_s"]
    out["write_plain_speedup"] = out["write_plain_host_s"] / out["write_plain_device_s"]
    out["load_plain_speedup"] = out["load_plain_host_s"] / out["load_plain_device_s"]
    print(json.dumps(out))


def run_streams(args):
    """The HBM-stream kernels of the quasi-Newton step and the round at
    L=232, q=21 with 2^20 walkers: CUDA-event time per launch (after a
    warm-up; every buffer is larger than L2 or read once per launch) and
    achieved GB/s = algorithmic bytes / time, against the measured HBM
    copy bandwidth.  Algorithmic bytes: each coupling-sized array (nPairs x
    q^2 floats, 47.3 MB) read or written once, per-walker arrays (4 MB)
    likewise, sequences 4*SWORDS bytes per walker."""
    import torch
    from mi3gpu_b200 import _lib
    L, q, N = args.L, args.q, args.walkers
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream(dev)
    s = st.cuda_stream
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    g = torch.Generator(device=dev).manual_seed(5)
    npairs, qq, sw = L * (L - 1) // 2, q * q, (L - 1) // 4 + 1
    nJ = npairs * qq
    rnd = lambda n, lo=0.0, hi=1.0: torch.rand(n, device=dev, generator=g) * (hi - lo) + lo
    bt, bi, J, dJ = rnd(nJ, 1e-4, 1e-2), rnd(nJ, 1e-4, 1e-2), rnd(nJ, -0.1, 0.1), rnd(nJ, -0.01, 0.01)
    Jo = torch.empty_like(J)
    cnt = torch.randint(0, N, (nJ,), device=dev, dtype=torch.int32, generator=g)
    dE = rnd(N, -2.0, 2.0)
    w = torch.empty(N, device=dev)
    out2 = torch.empty(2, device=dev)
    out2d = torch.empty(2, device=dev, dtype=torch.float64)
    minout = torch.empty(1, device=dev)
    wsr = torch.zeros(int(_lib.query("mi3_weight_stats_workspace", N)) // 8 + 2, dtype=torch.int64, device=dev)
    wsg = torch.zeros(int(_lib.query("mi3_gauge_workspace", L, q)) // 8 + 2, dtype=torch.int64, device=dev)
    wss = torch.zeros(int(_lib.query("mi3_bimarg_stats_workspace", L)) // 8 + 2, dtype=torch.int64, device=dev)
    stats = torch.empty(6, device=dev, dtype=torch.float64)
    stride = int(_lib.query("mi3_jrows_stride", L, q))
    Jrows = torch.empty(L * stride, device=dev)
    seq = torch.randint(0, q, (sw * 4, N), dtype=torch.uint8, device=dev, generator=g)
    seq[L:] = 0
    seq = seq.view(sw, 4, N).permute(0, 2, 1).contiguous().view(torch.int32).view(sw, N)
    seqL = torch.empty((L, N // 4), dtype=torch.int32, device=dev)
    rng = torch.zeros(N * 4, dtype=torch.int32, device=dev)
    cprob = torch.cumsum(torch.full((L, q), 1.0 / q, device=dev), 1)[:, :q - 1].contiguous()
    seq2 = torch.empty_like(seq)
    MB = 1e6
    Jb, Wb, Sb = nJ * 4, N * 4, sw * N * 4
    calls = [
        ("k_update_j", 4 * Jb, lambda: _lib.call("mi3_update_j", bt.data_ptr(), bi.data_ptr(), 4e-4, 1e-3,
                                                 J.data_ptr(), Jo.data_ptr(), L, q, s)),
        ("k_reg_lz (l1z)", 4 * Jb, lambda: _lib.call("mi3_reg_l1z", bi.data_ptr(), 4e-4, 1e-3, 2e-4, J.data_ptr(),
                                                    dJ.data_ptr(), L, q, s)),
        ("k_renormalize", 2 * Jb, lambda: _lib.call("mi3_renormalize_bimarg", bi.data_ptr(), L, q, s)),
        ("k_bicounts_to_bimarg", 2 * Jb, lambda: _lib.call("mi3_bicounts_to_bimarg", cnt.data_ptr(), Jo.data_ptr(),
                                                           N, L, q, s)),
        ("k_add_float_bufs", 3 * Jb, lambda: _lib.call("mi3_add_float_bufs", Jo.data_ptr(), dJ.data_ptr(), nJ, s)),
        ("gauge (fieldless even)", 2 * Jb, lambda: _lib.call("mi3_gauge_fieldless_even", J.data_ptr(),
                                                              Jo.data_ptr(), L, q, wsg.data_ptr(),
                                                              wsg.numel() * 8, s)),
        ("bimarg stats (FP64)", 3 * Jb, lambda: _lib.call("mi3_bimarg_stats", bt.data_ptr(), bi.data_ptr(),
                                                           J.data_ptr(), L, q, stats.data_ptr(), wss.data_ptr(),
                                                           wss.numel() * 8, s)),
        ("k_unpack_j", Jb + L * stride * 4, lambda: _lib.call("mi3_unpack_j", J.data_ptr(), Jrows.data_ptr(), L, q,
                                                              s)),
        ("weights fused (k_reduce)", 2 * Wb, lambda: _lib.call("mi3_weights_fused", 0.0, dE.data_ptr(),
                                                               w.data_ptr(), N, minout.data_ptr(),
                                                               out2.data_ptr(), out2d.data_ptr(), wsr.data_ptr(),
                                                               wsr.numel() * 8, s)),
        ("k_dE_to_weights", 2 * Wb, lambda: _lib.call("mi3_dE_to_weights", 0.0, dE.data_ptr(), w.data_ptr(), N,
                                                      s)),
        ("weight stats", Wb, lambda: _lib.call("mi3_weight_stats", w.data_ptr(), N, out2.data_ptr(),
                                               out2d.data_ptr(), wsr.data_ptr(), wsr.numel() * 8, s)),
        ("k_min_floats", Wb, lambda: _lib.call("mi3_min_floats", dE.data_ptr(), N, minout.data_ptr(), s)),
        ("k_repack_T", 2 * Sb, lambda: _lib.call("mi3_repack_seqs_T", seq.data_ptr(), N, seqL.data_ptr(), N // 4,
                                                 L, s)),
        ("k_init_rng", 4 * N * 4, lambda: _lib.call("mi3_init_rng", rng.data_ptr(), N, 0, (2 ** 63) // (2 * N),
                                                    s)),
        ("k_gen_indep", Sb + 2 * 4 * N * 4, lambda: _lib.call("mi3_gen_indep", seq2.data_ptr(), N, N,
                                                              rng.data_ptr(), cprob.data_ptr(), L, q, s)),
    ]
    # L2 flushed before every timed launch (a 256 MB write), the launch
    # alone between the events
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)

    def time_flushed(fn, reps=10):
        fn()
        fn()
        tot = 0.0
        for r in range(reps):
            flush.fill_(float(r))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / reps

    rows = []
    for name, nbytes, fn in calls:
        ms = time_flushed(fn)
        rows.append({"kernel": name, "ms": ms, "algorithmic_MB": nbytes / MB, "GBps": nbytes / ms / 1e6,
                     "frac_of_hbm": nbytes / ms / 1e6 / hbm})
    print(json.dumps({"mode": "streams", "config": {"workload": f"HBM-stream kernels, L={L} q={q} walkers={N}",
                                                    "l2": "flushed (256 MB write) before every timed launch"},
                      "hbm_peak_GBps": hbm, "rows": rows}))


def run_batched(args):
    """Many independent problems (L ~ U[50,300], q in {4, 8, 21}, walkers
    log-uniform in [2^14, 2^17]): quasi-Newton rounds with one CUDA-graph
    launch per round for the whole batch (walkers carried over, tuned
    kernel schedules), against the same problems driven by the host loop
    one problem at a time (inference.infer, device-resident; the consensus
    energies are off in both so that both arms compute the same numbers).
    Same seeds, same kernels: both arms give the same results."""
    import torch
    from mi3gpu_b200.autotune import Autotuner
    from mi3gpu_b200.batched import BatchedRounds, random_problems
    from mi3gpu_b200.inference import infer
    from mi3gpu_b200.mcmcGPU import MCMCGPU
    MCMCGPU.CONS_ENERGY_MAX_ACTIVE = -1.0
    t0 = time.time()
    probs = random_problems(args.problems, seed=2000, msa=1 << 14, sweeps=256)
    t_targets = time.time() - t0
    shapes = [(p.L, p.q, p.N) for p in probs]
    t0 = time.time()
    equil = dict(min_equil=64, max_equil=args.equil) if args.equil else None
    br = BatchedRounds(probs, sweeps=args.chosen_sweeps, sweeps_first=args.first_sweeps, reseed='none',
                       tuner=Autotuner(ROOT / "_build" / "autotune.json") if not args.no_tune else None, equil=equil)
    t_tune = time.time() - t0
    rounds = []
    for r in range(args.rounds):
        t0 = time.time()
        rec = br.run_round()
        if r == 0:
            rec["capture_s"] = time.time() - t0 - rec["wall_s"]
        rounds.append(rec)
    upd_first = br.site_updates_per_round(first=True)
    upd = br.site_updates_per_round(first=False)
    calls_b = [[h["mcmc_calls"] for h in p.history] for p in probs]
    steady = rounds[1:] or rounds
    gpu_s = statistics.mean(r["gpu_ms"] for r in steady) / 1e3
    batched = {
        "s_per_round": gpu_s, "s_per_round_wall": statistics.mean(r["wall_s"] for r in steady),
        "first_round_s": rounds[0]["gpu_ms"] / 1e3, "capture_s": rounds[0].get("capture_s"),
        "site_updates_per_round": upd, "sampling_site_updates_per_s_incl_newton": upd / gpu_s,
        "newton_steps_total_per_round": [sum(p["newton_steps"] for p in r["problems"]) for r in rounds],
        "tuning_s": t_tune, "graph_launches_per_round": 1}
    ssr_b = [[h["ssr"] for h in p.history] for p in probs]
    plans = {f"L{p.L}q{p.q}N{p.N}": br.tuning.get(id(p)) for p in probs[:8]}
    targets = [(p.target, p.L, p.q, p.N) for p in probs]
    br.close()
    del br, probs
    torch.cuda.empty_cache()
    # host-driven arm: the same problems (same targets and seeds) one after
    # another, same rounds
    ssr_h, calls_h = [], []
    per_round = [0.0] * args.rounds
    for k, (tgt, L, q, N) in enumerate(targets):
        kw = (dict(equiltime='auto', nsteps=8 * L, min_equil=64, max_equil=args.equil) if args.equil else
              dict(sweeps=args.chosen_sweeps, sweeps_first=args.first_sweeps))
        res = infer(tgt, L, q, N, args.rounds, newtonsteps=1024, seed=2000 + 1000 + k, log=lambda *a: None,
                    reseed='none', device_resident=True, **kw)
        for r, h in enumerate(res["history"]):
            per_round[r] += h["round_s"]
        ssr_h.append([h["ssr"] for h in res["history"]])
        calls_h.append([h["equil_calls"] for h in res["history"]])
        torch.cuda.empty_cache()
    host_s = statistics.mean(per_round[1:] or per_round)
    same = all(a == b for a, b in zip(ssr_b, ssr_h))
    same_calls = all(a == b for a, b in zip(calls_b, calls_h)) if args.equil else None
    print(json.dumps({
        "metric": "s per quasi-Newton round of a batch of independent problems, one graph launch vs host loop",
        "unit": "s/round", "value": gpu_s, "higher_is_better": False, "n_gpus": 1, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"batched {args.problems} problems, L~U[50,300], q in {{4,8,21}}, "
                               f"walkers logU[2^14,2^17], " +
                               (f"equilibration test in the graph (64 to {args.equil} calls of 8L steps)"
                                if args.equil else f"{args.chosen_sweeps} sweeps/round after a "
                                f"{args.first_sweeps}-sweep first round") + ", l1z 2e-4", "rounds": args.rounds,
                   "shapes": shapes},
        "batched": batched, "host_loop": {"s_per_round": host_s, "first_round_s": per_round[0]},
        "speedup_host_over_batched": host_s / gpu_s, "identical_ssr_histories": same,
        "identical_equilibration_calls": same_calls,
        "equilibration_calls_batched": calls_b[:8] if args.equil else None,
        "tuned_plans_sample": plans, "target_build_s": t_targets}))


def run_graph_small(args):
    """The small workload (L=48, q=4, 16384 walkers, 64 sweeps per round, a
    2^14-sequence synthetic MSA): quasi-Newton rounds driven by the host
    loop (device-resident, one launch and one sync per Newton step) against
    the same rounds recorded once as a CUDA graph (batched.BatchedRounds
    with one problem: one launch per round).  Same seeds, same kernels, same
    results; the difference is launch and synchronisation overhead.  Both
    arms are timed by the wall clock around a round (the host loop's own
    round_s), the graph's device time is reported beside it."""
    import torch
    from mi3gpu_b200.batched import BatchedRounds, Problem
    from mi3gpu_b200.inference import make_target, infer
    from mi3gpu_b200.mcmcGPU import MCMCGPU
    MCMCGPU.CONS_ENERGY_MAX_ACTIVE = -1.0  # the graph uses the direct energy kernel
    L, q, N, sweeps, rounds = 48, 4, 16384, 64, args.rounds
    target, _ = make_target(L, q, 1 << 14, seed=1000)
    res = infer(target, L, q, N, rounds, sweeps=sweeps, sweeps_first=sweeps, reseed='none', seed=77,
                device_resident=True, log=lambda *a: None)
    host = [h["round_s"] for h in res["history"]]
    pr = Problem(target, L, q, N, seed=77)
    br = BatchedRounds([pr], sweeps=sweeps, sweeps_first=sweeps, reseed='none')
    recs = [br.run_round() for _ in range(rounds)]
    graph = [r["wall_s"] for r in recs]  # wall clock, like the host loop's round_s
    graph_dev = [r["gpu_ms"] / 1e3 for r in recs]
    same = [h["ssr"] for h in pr.history] == [h["ssr"] for h in res["history"]]
    steps = [h["newton_steps"] for h in res["history"]]
    br.close()
    print(json.dumps({
        "metric": "s per quasi-Newton round, host loop vs one graph launch", "unit": "s/round",
        "value": statistics.mean(graph[1:] or graph), "higher_is_better": False, "n_gpus": 1, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"inference L={L} q={q} walkers={N}, {sweeps} sweeps/round, msa 2^14, l1z 2e-4",
                   "rounds": rounds},
        "host_loop_s_per_round": statistics.mean(host[1:] or host), "graph_s_per_round":
            statistics.mean(graph[1:] or graph), "speedup": statistics.mean(host[1:] or host) /
            statistics.mean(graph[1:] or graph), "graph_device_s_per_round": statistics.mean(graph_dev[1:] or graph_dev),
        "newton_steps_per_round": steps,
        "identical_ssr_histories": same}))


def energy_autocorr(Es):
    """Energy autocorrelation across walkers, rho(t) = corr(E_0, E_t), and
    tau_int = 1 + 2 sum_t rho(t) summed until rho first drops below 0.05."""
    E = np.asarray(Es, dtype=np.float64)  # (T, N)
    E0 = E[0] - E[0].mean()
    rho = [float(np.mean(E0 * (e - e.mean())) / (E0.std() * e.std() + 1e-300)) for e in E]
    tau = 1.0
    for r in rho[1:]:
        if r < 0.05:
            break
        tau += 2 * r
    return rho, tau


def run_learned(args, L=99, q=4, N=1 << 18, equil_sweeps=1024, track=64):
    """Learned independence proposal at L=99, q=4 with strong contacts
    (sigma 0.8): train the MADE on 2^18 equilibrated walkers, then track
    the energy autocorrelation over `track` sampler calls of one sweep each,
    plain vs. with one proposal step every `every` sweeps."""
    import torch
    from mi3gpu_b200 import MCMCGPU, GPU_node
    from mi3gpu_b200.potts import synthetic_ground_truth
    from mi3gpu_b200.learned import MadeProposal, LearnedSampler
    from mi3gpu_b200._lib import call as _lib_call, query as _lib_query
    H, epochs, every = args.hidden, args.made_epochs, args.made_every
    J = synthetic_ground_truth(L, q, seed=1003, contact_sigma=0.8)
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, args.seed + 1)
    gpus = GPU_node([g])
    gpus.initMCMC(L)  # one sweep per sampler call
    gpus.prepare_indep(np.full((L, q), 1.0 / q))
    gpus.gen_indep('main')
    gpus.setBuf('J', J)
    t0 = time.time()
    for _ in range(equil_sweeps):
        g.runMCMC()
    gpus.wait()
    t_equil = time.time() - t0
    made = MadeProposal(L, q, H=H, device=0, seed=3, lr=1e-3)
    t0 = time.time()
    hist = made.train(g.bufs['seq main'], N, epochs=epochs, batch=4096)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    start = g.bufs['seq main'].clone()
    start_rng = g.bufs['rngstates'].clone()
    # the proposal step's parts, timed with CUDA events on the sampler's stream
    parts = {}
    with torch.cuda.stream(g.stream):
        prop = torch.zeros_like(start)
        lqp = torch.zeros(N, dtype=torch.float32, device=start.device)
        ws = torch.zeros(int(_lib_query('mi3_energies_workspace', N)) // 8 + 2, dtype=torch.int64,
                         device=start.device)

        def timed(fn, reps=5):
            fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(g.stream)
            for _ in range(reps):
                fn()
            e1.record(g.stream)
            e1.synchronize()
            return e0.elapsed_time(e1) / reps

        kind = made.sampler
        for smp in ((kind, "simt") if kind != "simt" else ("simt",)):
            made.sampler = smp
            parts[f"made_sample_{smp}_ms"] = timed(lambda: made.sample(prop, N, lqp, seed=5))
            parts[f"made_logq_{smp}_ms"] = timed(lambda: made.sample(start, N, lqp, seed=0, given=True))
        made.sampler = kind
        parts["energies_ms"] = timed(lambda: _lib_call('mi3_energies', g._ptr('J'), prop.data_ptr(), N, N,
                                                       lqp.data_ptr(), L, q, ws.data_ptr(), ws.numel() * 8,
                                                       g.stream.cuda_stream))
        made.check_status()
        g.bufs['seq main'].copy_(start)
        ls_t = LearnedSampler(g, made, every=every, min_accept=0.0, seed=3)
        ls_t.propose()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(5):
            ls_t.propose()
        parts["proposal_step_ms"] = (time.perf_counter() - t1) / 5 * 1e3
        parts["sampler"] = kind
    res = {}
    for mode in ("plain", "learned"):
        g.bufs['seq main'].copy_(start)
        g.bufs['rngstates'].copy_(start_rng)
        ls = LearnedSampler(g, made, every=every, min_accept=0.005, seed=7)
        Es, rates = [], []
        gpus.calcEnergies('main')
        Es.append(gpus.collect('E main').copy())
        torch.cuda.synchronize()
        t_run = 0.0
        for k in range(track):
            t1 = time.time()
            g.runMCMC()
            if mode == "learned" and ls.enabled and (k + 1) % every == 0:
                rates.append(ls.propose())
            gpus.wait()
            t_run += time.time() - t1
            gpus.calcEnergies('main')
            Es.append(gpus.collect('E main').copy())
        rho, tau = energy_autocorr(Es)
        res[mode] = {"tau_int_sweeps": tau, "rho": [round(r, 4) for r in rho[:17]],
                     "s_per_sweep": t_run / track, "tau_int_s": tau * t_run / track,
                     "accept": rates, "mean_E": float(np.mean(Es[-1]))}
    gain = res["plain"]["tau_int_sweeps"] / res["learned"]["tau_int_sweeps"]
    print(json.dumps({"mode": "learned", "config": {"L": L, "q": q, "walkers": N, "H": H, "contact_sigma": 0.8,
                                                    "equil_sweeps": equil_sweeps, "every": every,
                                                    "train_epochs": epochs},
                      "train_nll": hist, "t_equil_s": t_equil, "t_train_s": t_train, "results": res,
                      "proposal_step": parts,
                      "tau_gain_per_sweep": gain,
                      "tau_gain_per_second": res["plain"]["tau_int_s"] / res["learned"]["tau_int_s"]}))


def run_made(args):
    """The MADE proposal's two sampler kernels alone at --L/--q/--walkers
    (default here L=99, q=4, 2^18: the learned-proposal workload): a
    network with random weights and biases, 2 + --steps draws and
    teacher-forced passes each, timed with CUDA events; the tensor-core
    sampler also repeats its own log q (same arithmetic, compared)."""
    import torch
    from mi3gpu_b200.learned import MadeProposal
    L, q, N, H = args.L, args.q, args.walkers, args.hidden
    made = MadeProposal(L, q, H=H, device=0, seed=3)
    rng = np.random.default_rng(7)
    for k in ("b1", "b2", "b3"):
        made.p[k].copy_(torch.as_tensor(rng.normal(0, 0.3, size=made.p[k].shape), dtype=torch.float32))
    made.round_params()
    sw = (L - 1) // 4 + 1
    seq = torch.zeros(sw * N, dtype=torch.int32, device="cuda")
    lq_s, lq_t = torch.zeros(N, device="cuda"), torch.zeros(N, device="cuda")
    out = {"mode": "made", "config": {"L": L, "q": q, "walkers": N, "H": H, "G": made.G}}
    kinds = ("tc", "simt") if made.sampler == "tc" else ("simt",)
    for kind in kinds:
        made.sampler = kind
        times = {}
        for given in (False, True):
            lq = lq_t if given else lq_s
            for _ in range(args.warmup):
                made.sample(seq, N, lq, seed=11, given=given)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                made.sample(seq, N, lq, seed=11, given=given)
            e1.record()
            e1.synchronize()
            times["logq_ms" if given else "sample_ms"] = e0.elapsed_time(e1) / args.steps
        made.check_status()
        times["logq_reproduced"] = bool(torch.equal(lq_s, lq_t))
        out[kind] = times
    made.sampler = kinds[0]
    print(json.dumps(out))


def headline_inference(args):
    """Seconds per quasi-Newton iteration of the plain native sampler under
    two round schedules, compact enough for the default run, on one
    synthetic target:
      reference_schedule  every round restarts the walkers from independent
                          sequences (reseed 'independent') and runs 128
                          sweeps; round host work in numpy, as in the
                          reference's NewtonSteps.py (2 rounds)
      carry_over          walkers carried over between rounds (reseed
                          'none', one of the reference's options): 128
                          sweeps in the first round and args.chosen_sweeps
                          after it; round work on the device (3 rounds)
    Both run the same sampler and the same Newton kernels; the ratio
    measures the schedule, not a tensor-core or learned-proposal form.
    s/iter of each = its last round; SSR after round 2 of each.  --mode
    inference runs the longer comparison."""
    from mi3gpu_b200.inference import make_target, infer
    from mi3gpu_b200.autotune import Autotuner
    tuner = None if args.no_tune else Autotuner(ROOT / "_build" / "autotune.json")
    target, _ = make_target(args.L, args.q, args.msa, seed=1001)
    ref = infer(target, args.L, args.q, args.walkers, 2, reseed="independent", sweeps=128,
                device_resident=False, log=lambda *a: None, tuner=tuner)["history"]
    carry = infer(target, args.L, args.q, args.walkers, 3, reseed="none", sweeps=args.chosen_sweeps,
                  sweeps_first=128, device_resident=True, log=lambda *a: None, tuner=tuner)["history"]
    r_s, c_s = ref[-1]["round_s"], carry[-1]["round_s"]
    return {"unit": "s/iter", "sampler": "the plain native sampler (same kernel and plan) in both schedules",
            "reference_schedule": r_s, "carry_over": c_s, "reference_over_carry_over": r_s / c_s,
            "ssr_round2": {"reference_schedule": ref[1]["ssr"], "carry_over": carry[1]["ssr"]},
            "reference_schedule_form": "reseed independent, 128 sweeps/round, host round work",
            "carry_over_form": f"walkers carried over, {args.chosen_sweeps} sweeps/round after a 128-sweep "
                               "first round, device-resident round work",
            "newton_steps": {"reference_schedule": ref[-1]["newton_steps"], "carry_over": carry[-1]["newton_steps"]},
            "note": "a schedule comparison of one sampler; no tensor-core or learned-proposal form is involved"}


def run_hiv(args):
    """The reference's real-data example (examples/HIV_inference/pbs.sh:
    L=93, q=4, 2^18 walkers, damping 0.01, l1z 1e-4, 64 rounds from the
    independent model; Mi3.py defaults otherwise: 2048-step sampler calls,
    automatic equilibration of at least 64 calls, 1024 initial Newton steps,
    gamma 4e-4, single_indep reseed) on its target bimarginals
    (tests/golden/hiv_bimarg_pc.npz), with the end state the reference's
    guide quotes for it (UserGuide.md:111-113).  Forms (--forms):
      recipe   the recipe as written
      carry    walkers carried over (reseed 'none'): the first round
               equilibrates automatically, later rounds run one 2048-step
               sampler call (22 sweeps)"""
    from mi3gpu_b200.inference import infer
    fx = np.load(ROOT / "tests" / "golden" / "hiv_bimarg_pc.npz")
    target = fx["bimarg"]
    L, q = 93, 4
    N = int(fx["nwalkers"]) if args.walkers == N_ else args.walkers
    rounds = int(fx["rounds"]) if args.rounds == 4 else args.rounds
    common = dict(damping=float(fx["damping"]), reg=("l1z", (float(fx["l1z"]),)), gamma=4e-4, newtonsteps=1024,
                  nsteps=2048, alpha="ABCD", device_resident=True)
    forms = {"recipe": dict(reseed="single_indep", equiltime="auto", min_equil=64),
             "carry": dict(reseed="none", equiltime=1, sweeps_first="auto", min_equil=64)}
    keep = args.forms.split(",") if args.forms else list(forms)
    out = {}
    for name in keep:
        w0 = time.time()
        res = infer(target, L, q, N, rounds, log=lambda *a: None, **common, **forms[name])
        hist = res["history"]
        last = hist[-1]
        out[name] = {"final": {"ssr": last["ssr"], "ferr": last["ferr"], "X": last["X"], "Xo": last["Xo"]},
                     "ssr": [round(h["ssr"], 4) for h in hist], "ferr": [round(h["ferr"], 5) for h in hist],
                     "X": [round(h["X"], 3) for h in hist], "equil_calls": [h["equil_calls"] for h in hist],
                     "newton_steps": [h["newton_steps"] for h in hist],
                     "round_s": [round(h["round_s"], 3) for h in hist], "wall_s": time.time() - w0,
                     "s_per_iter": statistics.mean(h["round_s"] for h in hist[1:]) if len(hist) > 1 else None}
    print(json.dumps({
        "metric": "HIV example end state after the recipe's rounds (SSR, Ferr, X)", "n_gpus": 1,
        "data": "the reference's example target (examples/HIV_inference/example_bimarg_pc.npy)",
        "config": {"workload": f"inference L=93 q=4 walkers={N} rounds={rounds} damping 0.01 l1z 1e-4"},
        "reference_end_state": {"ssr": float(fx["expect_ssr"]), "ferr": float(fx["expect_ferr"]),
                                "X": float(fx["expect_X"]), "Xo": float(fx["expect_Xo"]),
                                "source": "UserGuide.md:111-113 (run_63)"},
        "forms": out}))


def run_inference(args):
    """Quasi-Newton inference at the workload's shape on one synthetic
    target: seconds per iteration (MCMC round + Newton steps until
    Neff < 0.9 N) and the SSR of the sampled bimarginals after each round,
    for these round schedules of the plain native sampler (all use the same
    sampler and Newton kernels; they differ in how walkers are seeded, how
    long each round samples and where the round's host work runs):
      reference      every round restarts the walkers from independent
                     sequences and runs 128 sweeps; round host work (gauge
                     transform, statistics, J and sequence read-backs) in
                     numpy as in the reference's NewtonSteps.py
      reference_dev  the same sampling, with J resident on the device and
                     the round's host work done there in FP64
      carry          J resident; walkers carried over between rounds
                     (reseed 'none'): 128 sweeps in the first round,
                     args.chosen_sweeps after it
      carry_x4       as carry with four times as many sweeps per round
      carry_half     as carry with half as many sweeps per round
      carry_files    as carry, writing the reference's run directories
                     (J.npy, seqs, info.txt, ... per round) into a
                     temporary directory."""
    from mi3gpu_b200.inference import make_target, infer
    from mi3gpu_b200.autotune import Autotuner
    tuner = None if args.no_tune else Autotuner(ROOT / "_build" / "autotune.json")
    t0 = time.time()
    target, truth = make_target(args.L, args.q, args.msa, seed=1001)
    t_target = time.time() - t0
    forms = (("reference", dict(reseed="independent", sweeps=128, device_resident=False)),
             ("reference_dev", dict(reseed="independent", sweeps=128, device_resident=True)),
             ("carry", dict(reseed="none", sweeps=args.chosen_sweeps, sweeps_first=128, device_resident=True)),
             ("carry_x4", dict(reseed="none", sweeps=4 * args.chosen_sweeps, sweeps_first=128,
                               device_resident=True)),
             ("carry_half", dict(reseed="none", sweeps=max(1, args.chosen_sweeps // 2), sweeps_first=128,
                                  device_resident=True)),
             ("carry_files", dict(reseed="none", sweeps=args.chosen_sweeps, sweeps_first=128,
                                   device_resident=True, outdir="tmp")))
    if args.forms:
        keep = args.forms.split(",")
        forms = tuple(f for f in forms if f[0] in keep)
    out = {}
    for name, kw in forms:
        logs = []
        w0 = time.time()
        with tempfile.TemporaryDirectory() as tmpdir:
            run_kw = dict(kw, outdir=Path(tmpdir)) if kw.get("outdir") else kw
            res = infer(target, args.L, args.q, args.walkers, args.rounds, log=logs.append, tuner=tuner, **run_kw)
        wall = time.time() - w0
        hist = res["history"]
        cum = np.cumsum([h["round_s"] for h in hist]).tolist()
        after = [h["round_s"] for h in hist[1:]] or [hist[0]["round_s"]]
        out[name] = {"ssr": [round(h["ssr"], 5) for h in hist], "round_s": [round(h["round_s"], 3) for h in hist],
                     "mcmc_s": [round(h["mcmc_s"], 3) for h in hist],
                     "newton_s": [round(h["newton_s"], 3) for h in hist],
                     "newton_steps": [h["newton_steps"] for h in hist], "cum_s": cum,
                     "s_per_iter": statistics.mean(after), "wall_s_all_rounds": wall,
                     "final_ssr": hist[-1]["ssr"], "config": kw}
    carry = out.get("carry") or out[next(iter(out))]
    reach = {}
    bases = [b for b in ("reference", "reference_dev") if b in out]
    for base in bases:
        tgt = out[base]["final_ssr"]
        reach[base] = next((c for sv, c in zip(carry["ssr"], carry["cum_s"]) if sv <= tgt * (1 + 1e-3)), None)
    print(json.dumps({
        "metric": "s/iter (quasi-Newton round) and SSR of the plain sampler under round schedules", "unit": "s/iter",
        "value": carry["s_per_iter"], "higher_is_better": False, "n_gpus": 1, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"inference L={args.L} q={args.q} walkers={args.walkers} msa={args.msa}, l1z 2e-4",
                   "rounds": args.rounds, "s_per_iter": "mean round seconds after the first round"},
        "forms": out,
        "s_per_iter_ratio_over_carry": {b: out[b]["s_per_iter"] / carry["s_per_iter"] for b in bases},
        "carry_s_to_reach_final_ssr_of": reach,
        "expected_min_ssr": float(np.sum(target * (1 - target)) / args.walkers), "target_build_s": t_target}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nsteps", type=int, default=2048, help="MC steps per sampler call")
    ap.add_argument("--L", type=int, default=L_)
    ap.add_argument("--q", type=int, default=Q_)
    ap.add_argument("--walkers", type=int, default=N_)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--newton-steps", type=int, default=10, help="quasi-Newton steps to time (0: skip)")
    ap.add_argument("--mode", default="sampler", choices=["sampler", "inference", "kernels", "learned", "batched", "graph_small",
                                                           "msa", "streams", "hiv", "made"],
                    help="inference: run full quasi-Newton rounds and report s/iter and SSR")
    ap.add_argument("--rounds", type=int, default=4, help="inference rounds (--mode inference)")
    ap.add_argument("--msa", type=int, default=1 << 16, help="synthetic MSA size (--mode inference)")
    ap.add_argument("--chosen-sweeps", type=int, default=16, help="sweeps per round after the first (carry-over schedule)")
    ap.add_argument("--first-sweeps", type=int, default=128, help="sweeps in the first round (--mode batched)")
    ap.add_argument("--problems", type=int, default=64, help="problems in the batch (--mode batched)")
    ap.add_argument("--no-tune", action="store_true", help="built-in kernel schedules instead of autotuned ones")
    ap.add_argument("--no-inference", action="store_true", help="skip the s/iter comparison of the default run")
    ap.add_argument("--forms", default="", help="comma list of forms for --mode inference (default: all)")
    ap.add_argument("--shape", default="", help="L,q,N: one shape for --mode kernels")
    ap.add_argument("--hidden", type=int, default=512, help="MADE hidden units (--mode learned / made)")
    ap.add_argument("--made-epochs", type=int, default=48, help="MADE training epochs (--mode learned)")
    ap.add_argument("--equil", type=int, default=0,
                    help="--mode batched: equilibrate inside the graph, at most this many sampler calls")
    ap.add_argument("--made-every", type=int, default=4, help="sweeps per proposal step (--mode learned)")
    args = ap.parse_args()
    rank, world, _ = env_rank()

    if args.impl == "reference":
        if rank != 0:
            return
        from mi3gpu_b200.potts import synthetic_ground_truth
        J = synthetic_ground_truth(args.L, args.q, seed=1001)
        procs = os.cpu_count() or 1
        vals, sample, kind = [], "", "reference"
        for k in range(args.warmup + args.steps):
            r = cpu_generator_rate(J, args.L, args.q, max(1.0, args.cpu_seconds / 4), procs, seed=k)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference CPU generator not built (oracle/_ref)"}))
                return
            if k >= args.warmup:
                vals.append(r[0])
                sample, kind = r[1], r[2]
        v = statistics.mean(vals)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "site-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "L": args.L, "q": args.q},
            "cpu_baseline": {"value": v, "unit": "site-updates/s", "cores": procs, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    if args.mode == "inference":
        run_inference(args)
        return
    if args.mode == "kernels":
        run_kernels(args)
        return
    if args.mode == "learned":
        run_learned(args)
        return
    if args.mode == "batched":
        run_batched(args)
        return
    if args.mode == "graph_small":
        run_graph_small(args)
        return
    if args.mode == "msa":
        run_msa(args)
        return
    if args.mode == "streams":
        run_streams(args)
        return
    if args.mode == "hiv":
        run_hiv(args)
        return
    if args.mode == "made":
        run_made(args)
        return
    out, J = run_gpu(args)
    if rank == 0 and world == 1 and not args.no_inference:
        out["s_per_iter"] = headline_inference(args)
    if rank == 0:
        if not args.no_cpu and world == 1:  # the CPU baseline is an N=1 figure
            r = cpu_generator_rate(J, args.L, args.q, args.cpu_seconds, os.cpu_count() or 1)
            if r is not None:
                out["cpu_baseline"] = {"value": r[0], "unit": "site-updates/s", "cores": os.cpu_count() or 1,
                                       "kind": r[2], "sample": r[1]}
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
