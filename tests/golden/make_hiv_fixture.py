"""Copies the reference's real-data target into a test fixture.

The reference ships one real inference problem, the HIV protease example
(examples/HIV_inference/example_bimarg_pc.npy: bivariate marginals of an
HIV dataset, L=93 sites, q=4 residue classes, pseudocounted), with its
recipe (examples/HIV_inference/pbs.sh: `Mi3.py infer --init_model
independent --alpha ABCD --nwalkers 262144 --damping 0.01 --mcsteps 64
--reg l1z:0.0001`) and the state it should reach after the 64 rounds
(UserGuide.md:111-113: "SSR: 0.010 Ferr: 0.00856 X: -10.118 (-10.878)").

This script stores that array, unchanged, with the recipe and the quoted end
state as `hiv_bimarg_pc.npz`, so the integration test and `bench.py --mode
hiv` can run without the reference tree.

    python tests/golden/make_hiv_fixture.py [--ref REFERENCE_CHECKOUT]
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
    ap.add_argument("--out", default=str(HERE / "hiv_bimarg_pc.npz"), help="output .npz")
    args = ap.parse_args()
    if args.ref is None:
        import os
        env = os.environ.get("MI3_REFERENCE")
        cand = Path(env) if env else Path(__file__).resolve().parents[3] / "reference"
        if not (cand / "mi3gpu").is_dir():
            ap.error("reference checkout not found: pass --ref or set MI3_REFERENCE")
        args.ref = str(cand)
    src = Path(args.ref) / "examples" / "HIV_inference" / "example_bimarg_pc.npy"
    bim = np.load(src)
    assert bim.shape == (93 * 92 // 2, 16) and bim.dtype == np.float32, (bim.shape, bim.dtype)
    np.savez_compressed(
        Path(args.out),
        bimarg=bim,
        alpha=np.array("ABCD"),
        # recipe of examples/HIV_inference/pbs.sh (the other options are
        # Mi3.py's defaults: nsteps 2048, equiltime auto with min_equil 64,
        # newtonsteps 1024, gamma 4e-4, fracNeff 0.9, reseed single_indep)
        nwalkers=np.int64(262144), damping=np.float64(0.01), rounds=np.int64(64), l1z=np.float64(1e-4),
        # end state quoted by UserGuide.md:111-113 for run_63
        expect_ssr=np.float64(0.010), expect_ferr=np.float64(0.00856), expect_X=np.float64(-10.118),
        expect_Xo=np.float64(-10.878),
    )
    print("wrote", args.out, bim.shape)


if __name__ == "__main__":
    sys.exit(main())
