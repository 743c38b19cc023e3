"""MSA text format: the host reader/writer (mi3gpu_b200.seqload) and the
oracle's restatement of the line format, against the bytes, arrays and
error messages the reference's own seqload produced
(tests/golden/make_msa_golden.py -> msa_vectors.npz)."""
import bz2
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from mi3gpu_b200 import seqload

GOLD = np.load(Path(__file__).parent / "golden" / "msa_vectors.npz")
WRITE_CASES = sorted({k.split('_')[1] for k in GOLD.files if k.startswith('w_')})
LOAD_CASES = sorted({k[2:-3] for k in GOLD.files if k.startswith('l_') and k.endswith('_in')})


def _alpha(prefix):
    return bytes(GOLD[prefix + "_alpha"]).decode()


@pytest.mark.parametrize("case", WRITE_CASES)
def test_writer_matches_reference_bytes(case, tmp_path):
    p = f"w_{case}"
    seqs, alpha = GOLD[p + "_seqs"], _alpha(p)
    ids = [x.decode() for x in GOLD[p + "_ids"]] if p + "_ids" in GOLD.files else None
    fn = tmp_path / "seqs"
    zipf = case == "bz2"
    seqload.writeSeqs(fn, seqs, alpha, ids=ids, write_param=ids is not None, zipf=zipf)
    raw = fn.read_bytes()
    if zipf:
        assert raw[:3] == b"BZh"
        raw = bz2.decompress(raw)
    assert raw == bytes(GOLD[p + "_bytes"])
    # and it reads back
    back, back_ids, headers = seqload.loadSeqs(fn, alpha)
    np.testing.assert_array_equal(back, seqs)
    if ids is not None:
        assert [x.decode() for x in back_ids] == ids


@pytest.mark.parametrize("case", LOAD_CASES)
def test_reader_matches_reference(case, tmp_path):
    p = f"l_{case}"
    fn = tmp_path / "in"
    fn.write_bytes(bytes(GOLD[p + "_in"]))
    kw = {}
    if p + "_count" in GOLD.files:
        kw['count'] = int(GOLD[p + "_count"])
    if p + "_error" in GOLD.files:
        with pytest.raises(Exception) as e:
            seqload.loadSeqs(fn, _alpha(p), **kw)
        assert str(e.value) == str(GOLD[p + "_error"])
        return
    seqs, ids, headers = seqload.loadSeqs(fn, _alpha(p), **kw)
    np.testing.assert_array_equal(seqs, GOLD[p + "_seqs"])
    if p + "_ids" in GOLD.files:
        assert list(ids) == list(GOLD[p + "_ids"])
    else:
        assert ids is None
    assert list(headers) == list(GOLD[p + "_headers"])


def test_oracle_line_format_matches_reference_writer():
    """The oracle's packed-walkers -> lines restatement gives the reference
    writer's bytes (cases without ids)."""
    for case in ("plain", "nuc", "big"):
        p = f"w_{case}"
        seqs = GOLD[p + "_seqs"]
        text, bad = oracle.seqs_to_text(oracle.pack_seqs(seqs), seqs.shape[1], _alpha(p))
        assert not bad
        assert bytes(text) == bytes(GOLD[p + "_bytes"])
        back, first = oracle.text_to_seqs(text, seqs.shape[0], seqs.shape[1] + 1, 0, seqs.shape[1], _alpha(p))
        assert first is None
        np.testing.assert_array_equal(oracle.unpack_seqs(back, seqs.shape[1]), seqs)


def test_oracle_reader_flags_the_lines_the_reference_rejects():
    for case, line in (("bad_length", 1), ("bad_residue", 1), ("bad_id", 1)):
        p = f"l_{case}"
        raw = bytes(GOLD[p + "_in"])
        msa = seqload.parse(raw, _alpha(p))
        _, first = oracle.text_to_seqs(msa.body, msa.nseq, msa.line_len, msa.id_len, msa.L, msa.alpha)
        assert first == line, case


def test_parallel_bz2_is_multistream_and_reads_back(tmp_path):
    rng = np.random.default_rng(3)
    seqs = rng.integers(0, 21, size=(150000, 120)).astype('u1')  # 18 MB of text -> 3 streams
    fn = tmp_path / "seqs"
    seqload.writeSeqs(fn, seqs, seqload.alpha21, zipf=True)
    raw = fn.read_bytes()
    assert raw.count(b"BZh9") >= 3
    with bz2.open(fn, 'rb') as f:  # the reader the reference uses
        assert f.read() == bytes(seqload.format_lines(seqs, seqload.alpha21))
    back, _, _ = seqload.loadSeqs(fn)
    np.testing.assert_array_equal(back, seqs)


def test_headers_and_param_alphabet(tmp_path):
    fn = tmp_path / "seqs"
    seqs = np.random.default_rng(1).integers(0, 4, size=(10, 6)).astype('u1')
    seqload.writeSeqs(fn, seqs, "ACGT", headers=["made here", "#second"], write_param=True)
    back, ids, headers = seqload.loadSeqs(fn, alpha=None)
    np.testing.assert_array_equal(back, seqs)
    assert headers[1:] == ["made here\n", "second\n"]
    assert headers[0].startswith("PARAM")


def test_background_writes_and_atomic_files(tmp_path):
    """GPU_node.writeSeqs(background=True): the file appears complete once
    flushWrites returns, no temporary file is left, and an error in the
    background write is raised by flushWrites."""
    from mi3gpu_b200 import GPU_node
    from tests.fake_device import FakeMCMCGPU
    L, q, N = 9, 4, 512
    g = FakeMCMCGPU(L, q, N, seed=1)
    node = GPU_node([g])
    seqs = np.random.default_rng(2).integers(0, q, size=(N, L)).astype('u1')
    node.setSeqs('main', seqs)
    node.writeSeqs(tmp_path / "a", alpha="ACGT", zipf=True, background=True)
    node.writeSeqs(tmp_path / "b", alpha="ACGT", background=True)
    node.flushWrites()
    for name in ("a", "b"):
        np.testing.assert_array_equal(seqload.loadSeqs(tmp_path / name, "ACGT")[0], seqs)
    assert sorted(p.name for p in tmp_path.iterdir()) == ["a", "b"]
    node.writeSeqs(tmp_path / "missing_dir" / "c", alpha="ACGT", background=True)
    with pytest.raises(FileNotFoundError):
        node.flushWrites()
    node.flushWrites()  # nothing pending any more


from hypothesis import given, settings, strategies as st


@st.composite
def _msa_case(draw):
    alpha = "".join(draw(st.permutations(list("ACDEFGHIKLMNPQRSTVWY-")))[:draw(st.integers(2, 21))])
    n = draw(st.integers(1, 40))
    L = draw(st.integers(1, 30))
    seqs = np.array(draw(st.lists(st.lists(st.integers(0, len(alpha) - 1), min_size=L, max_size=L),
                                  min_size=n, max_size=n)), dtype='u1').reshape(n, L)
    ids = None
    if draw(st.booleans()):
        ids = [draw(st.text(alphabet="abcxyz0123456789_", min_size=1, max_size=8)) for _ in range(n)]
    return alpha, seqs, ids


@settings(max_examples=150, deadline=None)
@given(_msa_case())
def test_round_trip_and_oracle_agree(case):
    """Any alphabet, size and id field: writer -> reader is the identity,
    and the oracle's line parser reads the same residues."""
    alpha, seqs, ids = case
    raw = bytes(seqload.header_bytes(alpha, ["x"], True)) + bytes(seqload.format_lines(seqs, alpha, ids))
    msa = seqload.parse(raw, alpha)
    back, back_ids = seqload.check(msa)
    np.testing.assert_array_equal(back, seqs)
    if ids is not None:
        assert [x.decode() for x in back_ids] == ids
    mem, first = oracle.text_to_seqs(msa.body, msa.nseq, msa.line_len, msa.id_len, msa.L, alpha)
    assert first is None
    np.testing.assert_array_equal(oracle.unpack_seqs(mem, msa.L), seqs)


@settings(max_examples=150, deadline=None)
@given(_msa_case(), st.data())
def test_one_corrupt_byte_is_flagged_on_its_line(case, data):
    """One byte of one line replaced by a character outside the alphabet
    (not a newline): the reader raises for that line and the oracle's
    parser flags the same line."""
    alpha, seqs, ids = case
    body = bytearray(seqload.format_lines(seqs, alpha, ids))
    line_len = len(body) // seqs.shape[0]
    id_len = line_len - seqs.shape[1] - 1
    line = data.draw(st.integers(0, seqs.shape[0] - 1))
    col = data.draw(st.integers(id_len, line_len - 2))  # a residue position
    body[line * line_len + col] = ord('#') if line or col else ord('!')
    msa = seqload.parse(bytes(body), alpha)
    with pytest.raises(ValueError, match=f"sequence {line + 1} position {col - id_len}"):
        seqload.check(msa)
    _, first = oracle.text_to_seqs(msa.body, msa.nseq, msa.line_len, msa.id_len, msa.L, alpha)
    assert first == line


def test_default_alphabet_beyond_21_letters(tmp_path):
    a = seqload.default_alpha(80)
    assert a[:21] == seqload.alpha21 and len(set(a)) == 80 and not set(a) & set("#/ \n")
    seqs = np.random.default_rng(0).integers(0, 80, size=(50, 11)).astype('u1')
    seqload.writeSeqs(tmp_path / "s", seqs, a)
    np.testing.assert_array_equal(seqload.loadSeqs(tmp_path / "s", a)[0], seqs)
