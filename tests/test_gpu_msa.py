"""Walkers <-> MSA text lines on the device (mi3_seqs_to_text,
mi3_text_to_seqs) against the oracle's restatement and the bytes the
reference's writer produced, and the MCMCGPU / GPU_node file paths built on
them."""
import bz2
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle
from mi3gpu_b200 import GPU_node, MCMCGPU, _lib, seqload

pytestmark = pytest.mark.gpu
GOLD = np.load(Path(__file__).parent / "golden" / "msa_vectors.npz")


def _dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t.view(dtype) if dtype is not None else t).cuda()


def _to_text(seqmem, nseq, L, alpha):
    buflen = seqmem.shape[1]
    text = torch.zeros(nseq * (L + 1) + 64, dtype=torch.uint8, device='cuda')
    st = torch.zeros(1, dtype=torch.int32, device='cuda')
    a = alpha.encode()
    _lib.call('mi3_seqs_to_text', _dev(seqmem, torch.int32).data_ptr(), buflen, nseq, L, a, len(a),
              text.data_ptr(), st.data_ptr(), None)
    torch.cuda.synchronize()
    t = text.cpu().numpy()
    assert not t[nseq * (L + 1):].any()  # nothing written past the lines
    return t[:nseq * (L + 1)], int(st.item())


def _from_text(text, nseq, line_len, id_len, L, alpha, buflen=None, n0=0, fill=0):
    SW = oracle.swords(L)
    buflen = buflen or nseq
    mem = torch.full((SW, buflen), fill, dtype=torch.int32, device='cuda')
    bad = torch.zeros(1, dtype=torch.int64, device='cuda')
    a = alpha.encode()
    _lib.call('mi3_text_to_seqs', _dev(np.asarray(text, np.uint8)).data_ptr(), nseq, line_len, id_len, L, a,
              len(a), mem.data_ptr(), buflen, n0, bad.data_ptr(), None)
    torch.cuda.synchronize()
    b = int(bad.item())
    return mem.cpu().numpy().view(np.uint32), (None if b == -1 else b)


@pytest.mark.parametrize("L,nseq,buflen", [(1, 5, 5), (7, 100, 128), (37, 300, 300), (232, 4097, 5000),
                                           (233, 129, 129), (1500, 70, 96), (4000, 33, 33)])
def test_seqs_to_text_matches_oracle(cuda, L, nseq, buflen):
    rng = np.random.default_rng(L)
    alpha = seqload.alpha21
    seqs = rng.integers(0, 21, size=(buflen, L)).astype('u1')
    mem = oracle.pack_seqs(seqs)
    text, st = _to_text(mem, nseq, L, alpha)
    ref, bad = oracle.seqs_to_text(mem[:, :nseq], L, alpha)
    assert st == 0 and not bad
    np.testing.assert_array_equal(text, ref)


def test_seqs_to_text_reference_bytes_and_bad_residue(cuda):
    for case in ("plain", "nuc", "big"):
        p = f"w_{case}"
        seqs = GOLD[p + "_seqs"]
        text, st = _to_text(oracle.pack_seqs(seqs), seqs.shape[0], seqs.shape[1],
                            bytes(GOLD[p + "_alpha"]).decode())
        assert st == 0
        assert bytes(text) == bytes(GOLD[p + "_bytes"])
    seqs = np.zeros((40, 9), 'u1')
    seqs[17, 3] = 5  # outside a 4-letter alphabet
    text, st = _to_text(oracle.pack_seqs(seqs), 40, 9, "ACGT")
    ref, bad = oracle.seqs_to_text(oracle.pack_seqs(seqs), 9, "ACGT")
    assert st == 3 and bad  # MI3_STATUS_BAD_INPUT
    np.testing.assert_array_equal(text, ref)


@pytest.mark.parametrize("L,nseq,id_len", [(1, 3, 0), (9, 100, 0), (37, 300, 6), (232, 4097, 0), (700, 50, 12),
                                           (4000, 20, 3)])
def test_text_to_seqs_matches_oracle(cuda, L, nseq, id_len):
    rng = np.random.default_rng(L + id_len)
    alpha = "ACGT-" if L % 2 else seqload.alpha21
    seqs = rng.integers(0, len(alpha), size=(nseq, L)).astype('u1')
    ids = [f"s{k}" for k in range(nseq)] if id_len else None
    text = seqload.format_lines(seqs, alpha, ids)
    line_len = len(text) // nseq
    idl = line_len - L - 1
    mem, first = _from_text(text, nseq, line_len, idl, L, alpha, buflen=nseq + 37, n0=11, fill=-1)
    ref, rfirst = oracle.text_to_seqs(text, nseq, line_len, idl, L, alpha)
    assert first is None and rfirst is None
    np.testing.assert_array_equal(mem[:, 11:11 + nseq], ref)
    assert (mem[:, :11] == 0xffffffff).all() and (mem[:, 11 + nseq:] == 0xffffffff).all()


def test_text_to_seqs_flags_the_first_malformed_line(cuda):
    rng = np.random.default_rng(5)
    L, nseq, alpha = 50, 1000, seqload.alpha21
    seqs = rng.integers(0, 21, size=(nseq, L)).astype('u1')
    base = seqload.format_lines(seqs, alpha, [f"id{k}" for k in range(nseq)])
    line_len = len(base) // nseq
    id_len = line_len - L - 1
    for line, col, ch in ((700, id_len + 3, ord('B')), (300, line_len - 1, ord('A')), (999, id_len - 1, ord('x')),
                          (0, id_len + L - 1, ord('\n'))):
        text = base.copy()
        text[line * line_len + col] = ch
        _, first = _from_text(text, nseq, line_len, id_len, L, alpha)
        _, rfirst = oracle.text_to_seqs(text, nseq, line_len, id_len, L, alpha)
        assert first == rfirst == line
    text = base.copy()
    text[800 * line_len + id_len] = ord('J')
    text[120 * line_len + id_len + 7] = ord('O')
    assert _from_text(text, nseq, line_len, id_len, L, alpha)[1] == 120


def test_text_kernels_reject_bad_arguments(cuda):
    mem = torch.zeros((3, 64), dtype=torch.int32, device='cuda')
    text = torch.zeros(2048, dtype=torch.uint8, device='cuda')
    st = torch.zeros(1, dtype=torch.int32, device='cuda')
    bad = torch.zeros(1, dtype=torch.int64, device='cuda')
    with pytest.raises(_lib.Mi3Error):  # text not 16-byte aligned
        _lib.call('mi3_seqs_to_text', mem.data_ptr(), 64, 64, 10, b"ACGT", 4, text.data_ptr() + 1, st.data_ptr(),
                  None)
    with pytest.raises(_lib.Mi3Error):  # line length inconsistent with L and the id field
        _lib.call('mi3_text_to_seqs', text.data_ptr(), 10, 12, 0, 10, b"ACGT", 4, mem.data_ptr(), 64, 0,
                  bad.data_ptr(), None)
    with pytest.raises(_lib.Mi3Error):  # past the end of the destination buffer
        _lib.call('mi3_text_to_seqs', text.data_ptr(), 10, 11, 0, 10, b"ACGT", 4, mem.data_ptr(), 64, 60,
                  bad.data_ptr(), None)


def test_walker_text_round_trip_at_full_size(cuda):
    """2^20 walkers of L=232: device -> text -> device is the identity, the
    text equals the oracle's on a sample of lines, and both kernels read and
    write only their own buffers."""
    L, N, alpha = 232, 1 << 20, seqload.alpha21
    SW = oracle.swords(L)
    g = torch.Generator(device='cuda').manual_seed(3)
    res = torch.randint(0, 21, (N, 4 * SW), dtype=torch.int32, device='cuda', generator=g)
    res[:, L:] = 0
    b = res.to(torch.uint8).view(N, SW, 4).to(torch.int32)
    mem = (b[..., 0] | (b[..., 1] << 8) | (b[..., 2] << 16) | (b[..., 3] << 24)).t().contiguous()
    text = torch.empty(N * (L + 1), dtype=torch.uint8, device='cuda')
    st = torch.zeros(1, dtype=torch.int32, device='cuda')
    a = alpha.encode()
    _lib.call('mi3_seqs_to_text', mem.data_ptr(), N, N, L, a, len(a), text.data_ptr(), st.data_ptr(), None)
    back = torch.zeros_like(mem)
    bad = torch.zeros(1, dtype=torch.int64, device='cuda')
    _lib.call('mi3_text_to_seqs', text.data_ptr(), N, L + 1, 0, L, a, len(a), back.data_ptr(), N, 0,
              bad.data_ptr(), None)
    torch.cuda.synchronize()
    assert int(st.item()) == 0 and int(bad.item()) == -1
    assert torch.equal(back, mem)
    rows = np.random.default_rng(0).choice(N, 2000, replace=False)
    host = mem.cpu().numpy().view(np.uint32)[:, rows]
    ref, _ = oracle.seqs_to_text(host, L, alpha)
    got = text.view(N, L + 1)[torch.from_numpy(rows).cuda()].cpu().numpy().reshape(-1)
    np.testing.assert_array_equal(got, ref)


def test_mcmcgpu_text_paths(cuda, tmp_path):
    """getSeqsText / setSeqsText / storeSeqsText and GPU_node.writeSeqs /
    loadSeqs: files equal the host writer's, the reference's golden files
    load, and a malformed file raises the reference's message."""
    L, q, N = 12, 21, 512
    rng = np.random.default_rng(8)
    seqs = rng.integers(0, q, size=(N, L)).astype('u1')
    g = MCMCGPU((0, 0), L, q, N, 512, None, 1024, 1)
    node = GPU_node([g])
    node.setSeqs('main', seqs)
    assert bytes(g.getSeqsText('main').read()) == bytes(seqload.format_lines(seqs, seqload.alpha21))
    fn = tmp_path / "seqs"
    node.writeSeqs(fn, zipf=True)
    assert bz2.decompress(fn.read_bytes()) == bytes(seqload.format_lines(seqs, seqload.alpha21))
    g.fillSeqs(np.zeros(L, 'u1'))
    node.loadSeqs(fn)
    np.testing.assert_array_equal(node.collect('seq main'), seqs)
    # a file with ids and a PARAM header, written by the host writer
    ids = [f"w{k}" for k in range(N)]
    seqload.writeSeqs(fn, seqs[::-1], seqload.alpha21, ids=ids, write_param=True)
    node.loadSeqs(fn)
    np.testing.assert_array_equal(node.collect('seq main'), seqs[::-1])
    # large buffer: stored from text, read back as text
    g.initLargeBufs(2 * N)
    msa = seqload.read_msa(fn, seqload.alpha21)
    g.storeSeqsText(msa, 0, N)
    g.storeSeqsText(msa, 100, 300)
    np.testing.assert_array_equal(g.getBuf('seq large').read(), np.concatenate([seqs[::-1], seqs[::-1][100:400]]))
    assert bytes(g.getSeqsText('large').read()) == bytes(
        seqload.format_lines(np.concatenate([seqs[::-1], seqs[::-1][100:400]]), seqload.alpha21))
    # the reference's message for a malformed file
    bad = bytearray(seqload.format_lines(seqs, seqload.alpha21))
    bad[37 * (L + 1) + 4] = ord('B')
    fn.write_bytes(bytes(bad))
    with pytest.raises(ValueError, match="Invalid residue 'B' in sequence 38 position 4"):
        node.loadSeqs(fn)
    # one 4 MiB chunk with a bad end: the reference checks only line
    # lengths in its last chunk before it reports the end of the file
    fn.write_bytes(bytes(bad[:-3]))
    with pytest.raises(Exception, match="Unexpected characters at eof"):
        node.loadSeqs(fn)
    # a walker residue outside a short alphabet
    with pytest.raises(ValueError, match="outside the alphabet"):
        g.getSeqsText('main', "ACGT").read()
