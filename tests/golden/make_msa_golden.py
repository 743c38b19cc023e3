"""Generate tests/golden/msa_vectors.npz from the reference's MSA reader and
writer (mi3gpu/utils/seqload.py: writeSeqs, loadSeqs).

Run in a container where the reference tree is available:

    python tests/golden/make_msa_golden.py [--ref /path/to/Mi3-GPU]

Every case records the exact bytes the reference writes, or the arrays,
ids, headers or error message the reference's loader returns for a given
file, so the text format of this package (seqload.py and the device
text kernels) is pinned to the reference without the reference tree.
"""
import argparse
import bz2
import io
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None,
                    help="reference checkout (default: $MI3_REFERENCE, else ../reference beside the repository)")
    ap.add_argument("--out", default=str(HERE / "msa_vectors.npz"), help="output .npz")
    args = ap.parse_args()
    if args.ref is None:
        import os
        env = os.environ.get("MI3_REFERENCE")
        cand = Path(env) if env else Path(__file__).resolve().parents[3] / "reference"
        if not (cand / "mi3gpu").is_dir():
            ap.error("reference checkout not found: pass --ref or set MI3_REFERENCE")
        args.ref = str(cand)
    sys.path.insert(0, args.ref)
    from mi3gpu.utils import seqload
    from mi3gpu.utils.potts_common import alpha21

    out = {}
    rng = np.random.default_rng(20260202)
    tmp = Path(tempfile.mkdtemp())

    def write_case(tag, seqs, alpha, **kw):
        fn = tmp / tag
        seqload.writeSeqs(fn, seqs, alpha, **kw)
        raw = fn.read_bytes()
        if kw.get('zipf'):
            raw = bz2.decompress(raw)
        out[f"w_{tag}_seqs"] = seqs
        out[f"w_{tag}_alpha"] = np.frombuffer(alpha.encode(), np.uint8)
        out[f"w_{tag}_bytes"] = np.frombuffer(raw, np.uint8)
        if kw.get('ids') is not None:
            out[f"w_{tag}_ids"] = np.array(kw['ids'], dtype='S')
        if kw.get('headers') is not None:
            out[f"w_{tag}_headers"] = np.array(kw['headers'], dtype='U')

    # writer cases: protein alphabet, plain; with ids and PARAM; bz2;
    # a 4-letter alphabet; more sequences than one 4 MB write chunk holds
    write_case("plain", rng.integers(0, 21, size=(300, 37)).astype('u1'), alpha21)
    ids = ["seq{}".format(k) * (1 + k % 3) for k in range(57)]
    # (headers= is not written: the reference writes them as str into a
    # binary file, which raises TypeError)
    write_case("ids", rng.integers(0, 21, size=(57, 12)).astype('u1'), alpha21, ids=ids, write_param=True)
    write_case("bz2", rng.integers(0, 21, size=(128, 29)).astype('u1'), alpha21, zipf=True)
    write_case("nuc", rng.integers(0, 4, size=(64, 8)).astype('u1'), "ACGT")
    # past the reference's 4 MB write chunk (64527 lines of 65 bytes); a
    # regular pattern keeps the fixture small
    n, L = 70000, 63
    big = ((np.arange(n)[:, None] * 7 + np.arange(L)[None, :] * 3) % 4).astype('u1')
    write_case("big", big, "ACGT")

    def load_case(tag, raw, alpha=alpha21, **kw):
        fn = tmp / ("l_" + tag)
        fn.write_bytes(raw)
        out[f"l_{tag}_in"] = np.frombuffer(raw, np.uint8)
        out[f"l_{tag}_alpha"] = np.frombuffer(alpha.encode(), np.uint8)
        if 'count' in kw:
            out[f"l_{tag}_count"] = np.int64(kw['count'])
        try:
            seqs, ids, headers = seqload.loadSeqs(fn, alpha, **kw)
        except Exception as e:  # noqa: BLE001 - the message is the fixture
            out[f"l_{tag}_error"] = np.array(str(e))
            return
        out[f"l_{tag}_seqs"] = seqs
        if ids is not None:
            out[f"l_{tag}_ids"] = ids
        out[f"l_{tag}_headers"] = np.array(headers, dtype='U')

    body = b"".join(b"ACDEFGHIKL\n" for _ in range(5))
    load_case("plain", body)
    load_case("no_final_newline", body[:-1])
    load_case("extra_final_newline", body + b"\n")
    load_case("stockholm", body + b"//\n")
    load_case("stockholm_bare", body + b"//")
    load_case("headers", b"# one\n\n#PARAM {}\n  \n" + body)
    load_case("ids", b"a    ACDE\nbb   -WYV\nccc  AAAA\n")
    load_case("count", body, count=3)
    load_case("bad_length", b"ACDEF\nACDE\nACDEF\n")
    load_case("bad_residue", b"ACDEF\nACBEF\nACDEF\n")
    load_case("bad_id", b"ab ACD\nabcACD\n")
    load_case("bad_eof", b"ACDEF\nACDEF\nAC")
    nuc = rng.integers(0, 4, size=(20, 9)).astype('u1')
    load_case("nuc", b"".join(bytes(b"ACGT"[c] for c in s) + b"\n" for s in nuc), alpha="ACGT")
    load_case("bz2", bz2.compress(body))

    np.savez_compressed(Path(args.out), **out)
    print("wrote", args.out, len(out), "arrays")


if __name__ == "__main__":
    main()
