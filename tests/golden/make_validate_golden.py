"""Generate tests/golden/validate_vectors.npz from the reference's bimarginal
checks (mi3gpu/utils/potts_common.py:50-76 validate_bimarg) on crafted
inputs: consistent bimarginals, rows that do not sum to 1, and rows whose
implied i or j marginals disagree.  Each case stores the input and the
message the reference raises (empty when it accepts the input).

    python tests/golden/make_validate_golden.py [--ref /path/to/Mi3-GPU]
"""
import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None,
                    help="reference checkout (default: $MI3_REFERENCE, else ../reference beside the repository)")
    ap.add_argument("--out", default=str(HERE / "validate_vectors.npz"), help="output .npz")
    args = ap.parse_args()
    if args.ref is None:
        import os
        env = os.environ.get("MI3_REFERENCE")
        cand = Path(env) if env else Path(__file__).resolve().parents[3] / "reference"
        if not (cand / "mi3gpu").is_dir():
            ap.error("reference checkout not found: pass --ref or set MI3_REFERENCE")
        args.ref = str(cand)
    sys.path.insert(0, args.ref)
    from mi3gpu.utils.potts_common import validate_bimarg

    rng = np.random.default_rng(20260303)
    L, q, n = 7, 4, 5000
    seqs = rng.integers(0, q, size=(n, L))
    npair = L * (L - 1) // 2
    ff = np.zeros((npair, q * q), np.float64)
    k = 0
    for i in range(L - 1):
        for j in range(i + 1, L):
            np.add.at(ff[k], q * seqs[:, i] + seqs[:, j], 1.0)
            k += 1
    ff = (ff / n).astype('<f4')
    cases = {"valid": ff.copy()}
    c = ff.copy()
    c[0] *= 1.01  # site 0 (and 1) no longer sum to 1
    cases["sum"] = c
    c = ff.copy()
    c[9, 1], c[9, 4] = c[9, 1] + 0.002, c[9, 4] - 0.002  # (0,1)+, (1,0)-: row sums of pair 9 move
    cases["inconsistent_i"] = c
    c = ff.copy()
    c[12, 1], c[12, 0] = c[12, 1] + 0.002, c[12, 0] - 0.002  # (0,1)+, (0,0)-: column sums of pair 12 move
    cases["inconsistent_j"] = c
    c = ff.copy()
    c[15, 0] += 3e-6  # below eps: accepted
    cases["tiny"] = c
    out = {}
    for tag, x in cases.items():
        out[f"{tag}_in"] = x
        try:
            validate_bimarg(x)
            out[f"{tag}_msg"] = np.array("")
        except ValueError as e:
            out[f"{tag}_msg"] = np.array(str(e))
    np.savez_compressed(Path(args.out), **out)
    for tag in cases:
        print(tag, repr(str(out[f"{tag}_msg"])))


if __name__ == "__main__":
    main()
