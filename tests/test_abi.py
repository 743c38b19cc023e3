"""The C ABI without a GPU: the library loads, exports every entry point
declared in include/mi3b200.h with the ctypes signature the host binds, and
rejects bad arguments with error codes before touching the device."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from mi3gpu_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    src = (ROOT / "include" / "mi3b200.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.findall(r"^\s*(?:const\s+)?[a-z0-9_]+\s*\*?\s*(mi3_[a-z0-9_A-Z]+)\s*\(", src, flags=re.M)


def test_header_declares_entry_points():
    names = declared_functions()
    assert len(names) >= 24
    assert "mi3_metropolis" in names and "mi3_energies" in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_abi_version_and_sizes():
    lib = _lib.load()
    assert lib.mi3_abi_version() == 2
    assert lib.mi3_jrows_stride(232, 21) == 232 * 441  # already a multiple of 4
    assert lib.mi3_jrows_stride(93, 21) % 4 == 0 and lib.mi3_jrows_stride(93, 21) >= 93 * 441
    assert lib.mi3_energies_workspace(1 << 20) == 8 << 20
    assert lib.mi3_weight_stats_workspace(1000) >= 16


@pytest.mark.parametrize("name,args", [
    ("mi3_metropolis", (None, None, 0, None, 10, None, 1.0, None, 512, 10, 4, None, None)),
    ("mi3_energies", (None, None, 10, 10, None, 10, 4, None, 0, None)),
    ("mi3_bicounts", (None, 10, 10, None, 10, 4, None)),
    ("mi3_weighted_marg", (None, None, 10, 10, None, 10, 4, None, None, 0, None)),
    ("mi3_update_j", (None, None, 0.1, 0.1, None, None, 10, 4, None)),
    ("mi3_reg_l1z", (None, 0.1, 0.1, 0.1, None, None, 10, 4, None)),
    ("mi3_init_rng", (None, 10, 0, 1, None)),
    ("mi3_unpack_j", (None, None, 10, 4, None)),
    ("mi3_gen_indep", (None, 10, 10, None, None, 10, 4, None)),
])
def test_null_pointers_rejected(name, args):
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call(name, *args)
    assert e.value.code == -1
    assert name in str(e.value)


def test_bad_shapes_rejected():
    # non-null dummy addresses; validation must fail before any launch
    p = 4096
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_metropolis", p, p, 0, p, 10, None, 1.0, p, 500, 10, 4, p, None)   # nseqs % 128
    assert e.value.code == -1
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_metropolis", p + 4, p, 0, p, 10, None, 1.0, p, 512, 10, 4, p, None)  # Jrows misaligned
    assert e.value.code == -3
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_energies", p, p, 10, 20, p, 10, 4, p, 1 << 20, None)  # nseq > buflen
    assert e.value.code == -1
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_energies", p, p, 100, 100, p, 10, 4, p, 8, None)  # workspace too small
    assert e.value.code == -4
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_metropolis", p, p, 0, p, 10, None, 1.0, p, 512, 10, 300, p, None)  # q > 255
    assert e.value.code == -1


@pytest.mark.parametrize("L,q,N", [(232, 21, 1 << 20), (99, 4, 1 << 18), (48, 4, 16384), (150, 8, 4096),
                                   (512, 21, 1 << 21), (2, 2, 128)])
def test_metropolis_plans_host_query(L, q, N):
    """The plan enumeration is host code: every plan respects the kernel's
    limits (walkers per CTA divide N, chunk a multiple of 4 within the row,
    2-8 stages, shared memory within 227 KB with the walkers held at 4
    residues per word, or 6 (5 bits each) when q <= 32 and the chunk is a
    multiple of 12)."""
    from mi3gpu_b200.autotune import sampler_plans
    plans = sampler_plans(L, q, N)
    assert plans, "no plan for a supported shape"
    skew = [p for p in plans if p[0] == 'skew']
    assert bool(skew) == (q <= 21 and L + 31 <= 576 and N % 32 == 0)
    for _, w in skew:  # the skewed-lane kernel: 256, 512 or 768 walkers per CTA
        assert w in (256, 512, 768) and (w == 256 or L + 31 <= 288)
    for nw, m, st in [p for p in plans if p[0] != 'skew']:
        assert nw % 32 == 0 and 64 <= nw <= 512 and N % nw == 0
        assert m % 4 == 0 and 4 <= m <= ((L + 3) // 4) * 4
        assert 2 <= st <= 8
        pk = 6 if q <= 32 and m % 12 == 0 else 4
        words = (L + pk - 1) // pk
        stage_floats = (m * q * q + 31) // 32 * 32
        smem = 128 * ((16 * st + 4 + 127) // 128) + st * stage_floats * 4 + 256 * 4 + words * nw * 4
        assert smem <= 227 * 1024


@pytest.mark.parametrize("L,q,N", [(99, 4, 1 << 18), (48, 4, 1 << 14), (232, 21, 1 << 20), (512, 21, 1 << 19),
                                   (128, 8, 1 << 18), (150, 12, 1 << 18), (2, 4, 1), (3, 32, 5000),
                                   (93, 4, 3000), (60, 4, (1 << 24) + 5), (40, 4, 1 << 27), (283, 4, 75776)])
def test_bicounts_tc_plan_host_query(L, q, N):
    """The tensor-core count kernel's launch plan is host code: the chunks
    cover the N sequences in whole 128-sequence K steps, none holds more
    than 2^24 sequences (FP32 sums of 0/1 products stay exact integers),
    and the (row tile, column tile) pairs put every site pair i < j in
    exactly one tile."""
    out = (ctypes.c_uint32 * 4)()
    assert _lib.query("mi3_bicounts_tc_plan", L, q, N, out) == 1
    ntiles, nchunks, chunk, SR = list(out)
    SC = 256 // q
    assert SR == 128 // q
    assert chunk % 128 == 0 and 0 < chunk <= 1 << 24
    assert (nchunks - 1) * chunk < N <= nchunks * chunk
    nrt, nct = -(-L // SR), -(-L // SC)
    tiles = {(r, c) for r in range(nrt) for c in range((r * SR) // SC, nct)}
    assert len(tiles) == ntiles
    i, j = np.triu_indices(L, 1)
    assert all((a, b) in tiles for a, b in set(zip((i // SR).tolist(), (j // SC).tolist())))


def test_bicounts_tc_plan_one_wave_at_L99_q4():
    """L=99, q=4, 2^18 sequences: 6 tiles x 24 chunks of 86 K steps, one
    wave of 144 CTAs on the 148 SMs."""
    out = (ctypes.c_uint32 * 4)()
    assert _lib.query("mi3_bicounts_tc_plan", 99, 4, 1 << 18, out) == 1
    assert list(out) == [6, 24, 86 * 128, 32]


def test_bicounts_tc_plan_rejects_out_of_range():
    for L, q, N in [(1, 4, 10), (10, 3, 10), (10, 33, 10), (10, 4, 0)]:
        assert _lib.query("mi3_bicounts_tc_plan", L, q, N, None) == 0


# entry points for which null is a valid argument (the default stream, an
# empty graph handle): they go on to the CUDA runtime, which needs a device
_NULL_ALLOWED = {"mi3_abi_version", "mi3_capture_begin", "mi3_capture_if_end", "mi3_capture_while_end",
                 "mi3_graph_destroy", "mi3_stream_destroy"}


def _null_args(argtypes):
    vals = []
    for a in argtypes:
        if a in (ctypes.c_void_p, ctypes.c_char_p) or (isinstance(a, type) and issubclass(a, ctypes._Pointer)):
            vals.append(None)
        elif a in (ctypes.c_float, ctypes.c_double):
            vals.append(0.5)
        else:
            vals.append(8)
    return vals


@pytest.mark.parametrize("name", sorted(n for n, (rt, _) in _lib.SIGNATURES.items()
                                        if rt is ctypes.c_int and n not in _NULL_ALLOWED))
def test_every_entry_point_rejects_null_pointers(name):
    """Every int-returning entry point checks its pointers on the host and
    returns MI3_ERR_ARG, with a message naming the call, before any device
    work (so this runs without a GPU)."""
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call(name, *_null_args(_lib.SIGNATURES[name][1]))
    assert e.value.code == -1
    msg = str(e.value).split("): ", 1)[1]  # the library's own message: "<entry point>: <reason>"
    assert name.startswith(msg.split(":")[0])


_P = 0x100000  # a stand-in device address (never dereferenced: every case fails validation first)


def _no_cuda():
    import torch
    return not torch.cuda.is_available()


@pytest.mark.skipif(not _no_cuda(), reason="host-only validation test; a device would make a launch possible")
@pytest.mark.parametrize("name,args,code", [
    ("mi3_init_rng", (_P + 8, 8, 0, 1 << 20, None), -3),
    ("mi3_unpack_j", (_P, _P + 4, 10, 4, None), -3),
    ("mi3_unpack_j_tiles", (_P, _P + 4, 10, 4, None), -3),
    ("mi3_gen_indep", (_P, 64, 64, _P + 8, _P, 10, 4, None), -3),
    ("mi3_gemm_bf16", (16, 16, 16, _P, 16, 1, _P, 16, 1, _P, 16, 1.0, 0.0, _P + 256, 1 << 30, _P, None), -3),
    ("mi3_gemm_bf16", (16, 16, 16, _P, 16, 1, _P, 16, 1, _P, 16, 1.0, 0.0, _P, 16, _P, None), -4),
])
def test_alignment_and_workspace_rejected_on_the_host(name, args, code):
    """Misaligned device pointers (MI3_ERR_ALIGN) and short workspaces
    (MI3_ERR_WORKSPACE) are rejected on the host, before any launch."""
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call(name, *args)
    assert e.value.code == code
