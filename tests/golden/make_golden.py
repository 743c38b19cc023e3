"""Generate tests/golden/reference_vectors.npz from the reference itself.

Run in a container where the reference tree is available:

    python tests/golden/make_golden.py [--ref /path/to/Mi3-GPU]

It imports the reference's own numpy utilities (mi3gpu/utils/getSeqEnergies.py
E_potts, getMarginals.py getMarginals, changeGauge.py zeroGauge /
fieldlessGaugeEven, pseudocount.py mutation_pc) and the reference's MWC64X
OpenCL sources compiled as C++ (oracle/_ref/libmwc64x_ref.so, built by
oracle/Makefile), and records their outputs on seeded random inputs.  The
committed .npz pins the CPU oracle and the host helpers; tests read only the
.npz, never the reference tree.
"""
import argparse
import contextlib
import io
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None,
                    help="reference checkout (default: $MI3_REFERENCE, else ../reference beside the repository)")
    ap.add_argument("--out", default=str(HERE / "reference_vectors.npz"), help="output .npz")
    args = ap.parse_args()
    if args.ref is None:
        import os
        env = os.environ.get("MI3_REFERENCE")
        cand = Path(env) if env else Path(__file__).resolve().parents[3] / "reference"
        if not (cand / "mi3gpu").is_dir():
            ap.error("reference checkout not found: pass --ref or set MI3_REFERENCE")
        args.ref = str(cand)
    sys.path.insert(0, args.ref)
    sys.path.insert(0, str(ROOT))
    import warnings
    warnings.filterwarnings("ignore")
    from mi3gpu.utils.getSeqEnergies import E_potts
    from mi3gpu.utils.getMarginals import getMarginals
    from mi3gpu.utils.changeGauge import zeroGauge, fieldlessGaugeEven, zeroJGauge
    from mi3gpu.utils.pseudocount import mutation_pc
    from mi3gpu.utils.potts_common import getUnimarg, indepF
    from oracle import oracle

    out = {}
    rng = np.random.default_rng(20260101)

    # ---- MWC64X streams from the reference source (initRNG2 + NextUint2)
    ref = oracle.ref_rng_lib()
    assert ref is not None, "build oracle/_ref first (make -C oracle)"
    n = 64
    for tag, (off, span) in {"a": (0, (2 ** 63) // (2 * n)),
                             "b": (2 ** 62 + 12345, 987654321987)}.items():
        st = np.zeros(4 * n, np.uint32)
        ref.ref_init_rng2(st, n, off, span)
        out[f"rng_{tag}_offset"] = np.uint64(off)
        out[f"rng_{tag}_span"] = np.uint64(span)
        out[f"rng_{tag}_states"] = st.reshape(n, 4).copy()
        draws = []
        for g in (0, 1, n - 1):
            s = st[4 * g:4 * g + 4].copy()
            d = np.zeros(2 * 32, np.uint32)
            ref.ref_vec2_stream(s, 32, d)
            draws.append(d.reshape(32, 2))
        out[f"rng_{tag}_draws"] = np.stack(draws)  # walkers 0, 1, n-1
    # skip-ahead from a fixed state
    s0 = np.array([123456789, 362436069, 521288629, 88675123], np.uint32)
    for dist in (0, 1, 17, 4095, 2 ** 40 + 3):
        s = s0.copy()
        ref.ref_vec2_skip(s, dist)
        out[f"rng_skip_{dist}"] = s.copy()
    out["rng_skip_base"] = s0

    # ---- energies and bimarginal counts on random models
    models = {"A": (10, 5, 200), "B": (48, 4, 512), "C": (13, 21, 128)}
    for tag, (L, q, N) in models.items():
        npairs = L * (L - 1) // 2
        J = rng.normal(0, 0.3, size=(npairs, q * q)).astype("<f4")
        seqs = rng.integers(0, q, size=(N, L)).astype("<u1")
        w = rng.uniform(0.01, 2.0, size=N).astype("<f4")
        out[f"m{tag}_J"] = J
        out[f"m{tag}_seqs"] = seqs
        out[f"m{tag}_w"] = w
        out[f"m{tag}_E64"] = E_potts(seqs, J.astype("f8"))
        counts = getMarginals(seqs, q, nrmlz=False, uni=False)[0]
        out[f"m{tag}_bicounts"] = counts.astype("<u4")
        wc = getMarginals(seqs, q, weights=w.astype("f8"), nrmlz=False, uni=False)[0]
        out[f"m{tag}_wcounts"] = wc

    # ---- gauges and pseudocount
    L, q = 9, 4
    npairs = L * (L - 1) // 2
    h = rng.normal(0, 1, size=(L, q))
    J = rng.normal(0, 0.5, size=(npairs, q * q))
    out["g_h"], out["g_J"] = h, J
    out["g_zeroJ_h"], out["g_zeroJ_J"] = zeroJGauge(h, J)
    out["g_zero_h"], out["g_zero_J"] = zeroGauge(h, J)
    out["g_fe_h"], out["g_fe_J"] = fieldlessGaugeEven(h, J)
    seqs = rng.integers(0, q, size=(300, L)).astype("<u1")
    ff = getMarginals(seqs, q, uni=False)[0]
    out["pc_ff"] = ff
    with contextlib.redirect_stderr(io.StringIO()):
        out["pc_jeffreys"] = mutation_pc(ff, 300, "jeffreys")
        out["pc_bayes"] = mutation_pc(ff, 300, "bayes")
    out["pc_unimarg"] = getUnimarg(ff)
    out["pc_indepF"] = indepF(ff)

    dst = Path(args.out)
    np.savez_compressed(dst, **out)
    print("wrote", dst, dst.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
