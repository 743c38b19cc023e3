"""Host side of the tensor-core MADE sampler, without a GPU: blocked hidden
degrees, the block-size choice, and the plan checks of the C ABI."""
import numpy as np
import pytest

from mi3gpu_b200 import _lib
from mi3gpu_b200.learned import blocked_degrees, made_masks, tc_block_size


@pytest.mark.parametrize("L,q,H", [(99, 4, 512), (48, 4, 512), (9, 4, 64), (40, 4, 128), (12, 4, 64),
                                   (5, 4, 32), (8, 4, 64)])
def test_blocked_degrees(L, q, H):
    G = tc_block_size(L, q, H)
    assert G in (4, 8) and G * q <= 32
    m = blocked_degrees(L, H, G)
    assert len(m) == H and m.min() >= 1 and m.max() <= L - 1
    assert np.all(np.diff(m) >= 0)
    nb = -(-L // G)
    cnt = np.bincount((m - 1) // G, minlength=nb)
    assert np.all(cnt % 16 == 0) and cnt.max() <= 48
    assert nb * (-(-G * q // 16) * 16) + 48 + -(-L // 4) <= 512
    m32 = np.ascontiguousarray(m, dtype=np.int32)
    assert _lib.query("mi3_made_tc_workspace", L, q, H, G, m32.ctypes.data, m32.ctypes.data) > 0


def test_blocked_masks_autoregressive():
    L, q, H, G = 12, 4, 64, 8
    mW1T, mW2, mW3, m1, m2 = made_masks(L, q, H, G=G)
    M = (mW3 @ mW2 @ mW1T.T > 0).reshape(L, q, L, q)
    for i in range(L):
        for j in range(L):
            assert bool(M[i, :, j, :].any()) == (j < i)


@pytest.mark.parametrize("L,q,H", [(232, 21, 512), (99, 8, 512), (99, 4, 520), (30, 3, 64)])
def test_unsupported_shapes(L, q, H):
    assert tc_block_size(L, q, H) is None


def test_plan_rejects_bad_degrees():
    L, q, H, G = 12, 4, 64, 8
    m = np.ascontiguousarray(blocked_degrees(L, H, G), dtype=np.int32)
    ok = _lib.query("mi3_made_tc_workspace", L, q, H, G, m.ctypes.data, m.ctypes.data)
    assert ok > 0
    bad = m[::-1].copy()                                   # not sorted
    assert _lib.query("mi3_made_tc_workspace", L, q, H, G, bad.ctypes.data, bad.ctypes.data) == 0
    odd = m.copy()
    odd[47] = 9                                            # 47 units in block 0, 17 in block 1
    assert _lib.query("mi3_made_tc_workspace", L, q, H, G, odd.ctypes.data, odd.ctypes.data) == 0
    assert _lib.query("mi3_made_tc_workspace", L, 5, H, G, m.ctypes.data, m.ctypes.data) == 0


def test_prepare_and_sample_reject_before_launch():
    plan = np.zeros(24, dtype=np.uint64)
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_made_tc_sample", plan.ctypes.data, 4096, 128, 128, 4096, 0, 0, 4096, None)
    assert e.value.code == -1                              # plan not prepared
    L, q, H, G = 12, 4, 64, 8
    m = np.ascontiguousarray(blocked_degrees(L, H, G), dtype=np.int32)
    p = 4096
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_made_tc_prepare", L, q, H, G, m.ctypes.data, m.ctypes.data, p, p, p, p, p, p, p, 16,
                  plan.ctypes.data, None)
    assert e.value.code == -4                              # workspace too small
    with pytest.raises(_lib.Mi3Error) as e:
        _lib.call("mi3_made_tc_prepare", L, q, H, G, m.ctypes.data, m.ctypes.data, None, p, p, p, p, p, p, 1 << 30,
                  plan.ctypes.data, None)
    assert e.value.code == -1


def test_learned_sampler_hands_over_to_plain_sweeps_below_min_accept():
    """The interleaving and hand-over of LearnedSampler.sweeps (host logic):
    one proposal step after every `every`-th sampler call, and none after a
    step whose acceptance rate fell below min_accept -- the plain sampler
    carries on alone.  The device work of a proposal step is replaced by
    scripted acceptance counts."""
    from mi3gpu_b200.learned import LearnedSampler

    class FakeGpu:
        calls = 0

        def runMCMC(self):
            FakeGpu.calls += 1

    N = 1000
    script = iter([400, 250, 5, 900])  # accepted walkers per proposal step
    ls = LearnedSampler.__new__(LearnedSampler)
    ls.gpu, ls.every, ls.min_accept = FakeGpu(), 3, 0.01
    ls.accepted = ls.proposed = 0
    ls.enabled = True
    ls.propose = lambda: ls._record(next(script), N)
    rates = ls.sweeps(20)
    assert FakeGpu.calls == 20
    assert rates == [0.4, 0.25, 0.005]  # the third step (0.5% < 1%) is the last
    assert not ls.enabled and ls.proposed == 3 * N and ls.accepted == 655
    assert ls.sweeps(6) == [] and FakeGpu.calls == 26
