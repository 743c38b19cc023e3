"""mi3_energies_noalloc: the energies entry point for callers that cannot
allocate device memory (graph-capture regions, hosts whose GPU memory is
owned by a pool, bindings without a device allocator).  It keeps its
accumulators in a fixed array inside the library, so this test checks that
two calls in a row -- the second one reusing the array left dirty by the
first -- give the same energies as mi3_energies with its own workspace.
The file sorts last so that a run stopping at the first failure has already
run every other test."""
import numpy as np
import pytest

from oracle import oracle
from mi3gpu_b200 import _lib
from tests._util import dev, host, empty, stream, random_model

pytestmark = pytest.mark.gpu


def test_energies_noalloc_matches_workspace_version(cuda):
    L, q, N = 232, 21, 4096
    J = random_model(L, q, 31)
    seqs = np.random.default_rng(32).integers(0, q, size=(N, L)).astype("<u1")
    dJ, dmem = dev(J), dev(oracle.pack_seqs(seqs))
    ref = empty((N,), np.float32)
    ws = empty((int(_lib.query("mi3_energies_workspace", N)) // 8 + 1,), np.int64)
    _lib.call("mi3_energies", dJ.data_ptr(), dmem.data_ptr(), N, N, ref.data_ptr(), L, q, ws.data_ptr(),
              ws.numel() * 8, stream())
    expect = host(ref)
    for _ in range(2):  # the second call finds the first call's sums in the array
        out = empty((N,), np.float32)
        _lib.call("mi3_energies_noalloc", dJ.data_ptr(), dmem.data_ptr(), N, N, out.data_ptr(), L, q, stream())
        got = host(out)
        # same algorithm, deterministic accumulation: identical bits; the
        # parity bar of the energies (1e-5 relative to FP64) holds a fortiori
        np.testing.assert_array_equal(got, expect)
        e64 = oracle.energies_f64(J, oracle.pack_seqs(seqs), L, q)
        assert (np.abs(got - e64) / np.maximum(1.0, np.abs(e64))).max() <= 1e-5

    too_many = (1 << 20) + 1
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_energies_noalloc", dJ.data_ptr(), dmem.data_ptr(), too_many, too_many, out.data_ptr(),
                  L, q, stream())
    assert e.value.code == -1 and "capacity" in str(e.value)
