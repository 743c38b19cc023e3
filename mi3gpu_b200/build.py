"""Build recipe for libmi3b200.so (sm_100a) and the CPU oracle.

`python -m mi3gpu_b200.build` compiles every CUDA source under csrc/ into
one shared library next to this file, with the CUDA runtime linked
statically so the library only needs the NVIDIA driver at run time.
"""
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libmi3b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false",            # keep float sums in the reference's exact op order
    "-Xcompiler", "-fPIC", "-shared",
    "-cudart", "static",
    "-Xptxas", "-warn-spills",
]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (Path(c).exists() or c == "nvcc"):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(str(p) for p in CSRC.glob("*.cu"))


def build_lib(verbose=False, extra=()):
    """Compile each source to an object in parallel, then link the library."""
    from concurrent.futures import ThreadPoolExecutor
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    cflags = [f for f in NVCC_FLAGS if f not in ("-shared", "-cudart", "static")]
    objs = []

    def compile_one(src):
        obj = obj_dir / (Path(src).stem + ".o")
        cmd = [nvcc()] + cflags + list(extra) + ["-I", str(ROOT / "include"), "-c", src, "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for obj, r in ex.map(compile_one, sources()):
            if r.stdout or r.stderr:
                print(r.stdout + r.stderr, end="")
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, str(obj))
            objs.append(str(obj))
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static",
            "-Xcompiler", "-fPIC", "-o", str(LIB)] + objs
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return LIB


def reference_tree():
    """Where the reference checkout is: $MI3_REFERENCE, else a directory
    named `reference` beside this repository; None when neither exists."""
    env = os.environ.get("MI3_REFERENCE")
    cand = Path(env) if env else ROOT.parent / "reference"
    return cand if (cand / "mi3gpu").is_dir() else None


def build_oracle(verbose=False):
    cmd = ["make", "-s", "-C", str(ROOT / "oracle")]
    ref = reference_tree()
    if ref is not None:
        cmd.append("REF=" + str(ref))
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    build_lib(verbose=True, extra=[a for a in argv if a.startswith("-")])
    build_oracle(verbose=True)


if __name__ == "__main__":
    main()
