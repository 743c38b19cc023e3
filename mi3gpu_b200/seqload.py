"""Multiple sequence alignments as text files, in the reference's format
(mi3gpu/utils/seqload.py), so run directories written here are read by the
reference's tools and the reference's files load here.

The format (seqload.py:91-133, 196-352, 378-411):

  * optional header lines first: lines starting with '#' (kept, without
    the '#', in `headers`) and blank lines (skipped); a '#PARAM {json}'
    line may carry the alphabet;
  * then one sequence per line, every line the same length; a line may
    start with an id field, whitespace-padded to the same width for all
    lines and ending in a space (the width is one past the last space of
    the first line);
  * residues are letters of the alphabet; index i of the alphabet is
    residue value i;
  * at the end of the file a missing or one extra final newline is
    tolerated, and a Stockholm terminator '//' (with or without its
    newline) is dropped;
  * files may be bzip2-compressed (detected by the 'BZh' magic).

Errors carry the reference's messages.  The reader walks the body in the
reference's chunks (4 MiB of lines) so that, of several malformed lines,
the same one is reported.

Two deliberate differences: `headers=` is written (the reference writes
them as str into a binary file, which raises TypeError), each as one '#'
line; and a compressed file is written as several bzip2 streams
compressed in parallel threads -- a valid .bz2 that bzip2, Python's bz2
module and the reference's reader decompress to the same bytes.

Walkers that live on a device are turned into these lines there
(mi3_seqs_to_text, mi3_text_to_seqs; `MCMCGPU.getSeqsText`,
`MCMCGPU.setSeqsText`); this module handles the file around them.
"""
import bz2
import json
import os
import threading
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

alpha20 = "ACDEFGHIKLMNPQRSTVWY"
alpha21 = "-" + alpha20

_BZ2_MAGIC = b"BZh"
_CHUNK_BYTES = 4 * 1024 * 1024
_BZ2_BLOCK = 8 * 1024 * 1024  # bytes per independently compressed stream


def default_alpha(q):
    """The protein alphabet for q = 21, its first q letters for smaller q;
    for larger q it continues with the other printable ASCII characters
    except '#' (a header line marker) and '/' (the Stockholm terminator)."""
    extra = "".join(chr(c) for c in range(33, 127) if chr(c) not in alpha21 + "#/")
    full = alpha21 + extra
    if q > len(full):
        raise ValueError(f"no default alphabet for q={q}; give alpha")
    return full[:q]


def _as_bytes(alpha):
    return alpha.encode('ascii') if isinstance(alpha, str) else bytes(alpha)


# ---------------------------------------------------------------- reading
def read_file(fn, zipf=None):
    """Whole file as bytes, bzip2 decoded when compressed (zipf None:
    detect; True: require; False: never)."""
    if hasattr(fn, 'read'):
        raw = fn.read()
    else:
        raw = Path(fn).read_bytes()
    if zipf is not False and raw[:3] == _BZ2_MAGIC:
        return bz2.decompress(raw)
    if zipf is True:
        raise Exception("bz2 file expected")
    return raw


class MSAText:
    """A parsed MSA file: headers, line geometry and the body of sequence
    lines (uint8), after the end-of-file fix-ups.  `body` holds nseq lines
    of line_len = id_len + L + 1 bytes.  When the end of the file cannot be
    fixed up, `eof_error` is the exception the reference raises once its
    reader gets there, and `body` holds the whole lines before it."""

    def __init__(self, headers, alpha, body, line_len, id_len, eof_error=None):
        self.headers, self.alpha = headers, alpha
        self.body, self.line_len, self.id_len = body, line_len, id_len
        self.L = line_len - id_len - 1
        self.nseq = body.size // line_len if line_len else 0
        self.eof_error = eof_error

    def lines(self, start, stop):
        """Lines [start, stop) as a (n, line_len) uint8 array."""
        return self.body[start * self.line_len:stop * self.line_len].reshape(-1, self.line_len)


def _split_header(raw):
    """(headers, offset of the first sequence line) (seqload.py:261-270)."""
    headers, pos = [], 0
    while pos < len(raw):
        end = raw.find(b"\n", pos)
        end = len(raw) if end < 0 else end + 1
        line = raw[pos:end]
        if line.isspace():
            pos = end
        elif line.startswith(b"#"):
            headers.append(line[1:].decode('utf-8'))
            pos = end
        else:
            break
    return headers, pos


def _alpha_from_headers(headers):
    for h in headers:
        if h.startswith("PARAM"):
            a = json.loads(h[len("PARAM "):]).get('alpha')
            if a is not None:
                return a
    raise Exception("Could not determine alphabet")


def _check_lines(rows, id_len, line_len, pos):
    """Line-length and id-field checks of one chunk (seqload.py:196-215)."""
    bad = np.flatnonzero(rows[:, -1] != ord('\n'))
    if bad.size:
        raise ValueError("Sequence {} has wrong length (expected {})".format(pos + 1 + bad[0], line_len - 1))
    if id_len:
        bad = np.flatnonzero(rows[:, id_len - 1] != ord(' '))
        if bad.size:
            raise ValueError("Sequence {} has wrong id field length. Expected id length {}".format(
                pos + 1 + bad[0], id_len))


def _translate(rows, id_len, lut, pos):
    """Residue characters -> indices, with the reference's error for the
    first bad character in row-major order (seqload.py:217-241)."""
    seqs = lut[rows[:, id_len:-1]]
    bad = np.argwhere(seqs == 255)
    if bad.size:
        r, c = bad[0]
        ch = chr(rows[r, id_len + c])
        if ch == '\n':
            raise ValueError("Sequence {} has length {} (expected {})".format(r + pos + 1, c, seqs.shape[1]))
        raise ValueError("Invalid residue '{}' in sequence {} position {}".format(ch, r + pos + 1, c))
    return seqs


def _lut(alpha):
    lut = np.full(256, 255, np.uint8)
    a = np.frombuffer(alpha, np.uint8)
    lut[a] = np.arange(a.size, dtype=np.uint8)
    return lut


def _body(raw, off, line_len):
    """(body, eof error) after the end-of-file fix-ups (seqload.py:300-336):
    Stockholm terminator, one missing or one extra final newline."""
    body = np.frombuffer(raw, np.uint8)[off:]
    n = body.size
    if n > 2 and body[-2] == ord('/'):
        if body[-1] == ord('/'):
            body = body[:-2]
        elif n > 3 and body[-1] == ord('\n') and body[-3] == ord('/'):
            body = body[:-3]
    n = body.size
    if n % line_len:
        if body[-1] == ord('\n') and (n - 1) % line_len == 0:
            body = body[:-1]
        elif (n + 1) % line_len == 0:
            body = np.concatenate([body, np.array([ord('\n')], np.uint8)])
        else:
            whole = n - n % line_len
            err = Exception("Unexpected characters at eof: {}".format(repr(bytes(body[whole:]).decode('utf-8'))))
            return body[:whole], err
    return body, None


def _chunk_lines(line_len):
    return _CHUNK_BYTES // line_len


def parse(raw, alpha=None):
    """MSAText of a decoded file.  The line checks are left to the reader
    (host: loadSeqs; device: MCMCGPU.setSeqsText)."""
    headers, off = _split_header(raw)
    if alpha is None:
        alpha = _alpha_from_headers(headers)
    alpha = _as_bytes(alpha)
    end = raw.find(b"\n", off)
    first = raw[off:] if end < 0 else raw[off:end]
    line_len = len(first) + 1
    id_len = first.rfind(b" ") + 1
    if off >= len(raw):
        return MSAText(headers, alpha, np.zeros(0, np.uint8), line_len, id_len)
    body, err = _body(raw, off, line_len)
    return MSAText(headers, alpha, body, line_len, id_len, err)


def check(msa, stop=None):
    """Run the reference's checks chunk by chunk over the lines a reader
    reaches (all of them, or up to the chunk holding line `stop`) and raise
    its error for the first problem: line lengths and id fields, then
    residues, per chunk; a bad end of file once the last chunk is reached
    (whose residues the reference does not translate first).  Returns the
    translated sequences (N, L) and the ids."""
    lut = _lut(msa.alpha)
    seqs, ids = [], []
    step = _chunk_lines(msa.line_len)
    last = msa.nseq - msa.nseq % step if msa.eof_error is not None else None
    for s in range(0, max(msa.nseq, 1), step):
        rows = msa.lines(s, min(msa.nseq, s + step))
        _check_lines(rows, msa.id_len, msa.line_len, s)
        if s == last:
            raise msa.eof_error
        seqs.append(_translate(rows, msa.id_len, lut, s))
        if msa.id_len:
            raw_ids = np.ascontiguousarray(rows[:, :msa.id_len]).view(f'S{msa.id_len}').reshape(-1)
            ids.append(np.char.strip(raw_ids))
        if stop is not None and s + rows.shape[0] > stop:
            break
    else:
        if msa.eof_error is not None:
            raise msa.eof_error
    return np.concatenate(seqs), (np.concatenate(ids) if ids else None)


def read_msa(fn, alpha=None, zipf=None):
    return parse(read_file(fn, zipf), alpha)


def loadSeqs(fn, alpha=alpha21, zipf=None, count=None):
    """(seqs (N, L) uint8, ids or None, headers), as the reference's
    loadSeqs returns them (seqload.py:91-133)."""
    msa = read_msa(fn, alpha, zipf)
    if msa.nseq == 0 and msa.eof_error is None:
        raise ValueError("no sequences in file")
    seqs, ids = check(msa, count)
    if count is not None:
        seqs = seqs[:count]
        ids = ids[:count] if ids is not None else None
    return seqs, ids, msa.headers


# ---------------------------------------------------------------- writing
def format_lines(seqs, alpha=alpha21, ids=None):
    """The bytes of the sequence lines writeSeqs writes (seqload.py:378-411)."""
    alpha = np.frombuffer(_as_bytes(alpha), np.uint8)
    seqs = np.asarray(seqs)
    n, L = seqs.shape
    id_len = 0
    if ids is not None:
        ids = [x if isinstance(x, bytes) else str(x).encode('utf-8') for x in ids]
        if len(ids) != n:
            raise ValueError("need one id per sequence")
        id_len = max(len(x) for x in ids) + 1
    out = np.empty((n, id_len + L + 1), np.uint8)
    if id_len:
        out[:, :id_len] = np.array([x.ljust(id_len) for x in ids], dtype=f'S{id_len}').view(np.uint8).reshape(
            n, id_len)
    np.take(alpha, seqs, out=out[:, id_len:-1])
    out[:, -1] = ord('\n')
    return out.reshape(-1)


def header_bytes(alpha=alpha21, headers=None, write_param=False):
    out = b""
    if write_param:
        out += "#PARAM {0}\n".format(json.dumps({'alpha': _as_bytes(alpha).decode('utf-8')})).encode('utf-8')
    for h in headers or []:
        h = h if h.startswith('#') else '#' + h
        out += (h if h.endswith('\n') else h + '\n').encode('utf-8')
    return out


def write_text(fn, parts, zipf=None, threads=None):
    """Write byte blocks (bytes or uint8 arrays) in order; bzip2 (zipf True)
    compresses blocks of 8 MiB as independent streams in parallel threads
    (the compressor releases the interpreter lock).  The file appears under
    its name only when complete (written to a temporary name, then
    renamed)."""
    fn = Path(fn)
    tmp = fn.with_name(f"{fn.name}.{os.getpid()}.{threading.get_ident()}.tmp")
    try:
        _write_parts(tmp, parts, zipf, threads)
        os.replace(tmp, fn)
    finally:
        if tmp.exists():
            tmp.unlink()


def _write_parts(fn, parts, zipf, threads):
    views = [memoryview(np.ascontiguousarray(p, np.uint8) if not isinstance(p, (bytes, bytearray)) else p)
             for p in parts]
    if not zipf:
        with open(fn, 'wb') as f:
            for v in views:
                f.write(v)
        return
    blocks, cur, size = [], [], 0
    for v in views:
        for s in range(0, len(v), _BZ2_BLOCK):
            piece = v[s:s + _BZ2_BLOCK]
            cur.append(piece)
            size += len(piece)
            if size >= _BZ2_BLOCK:
                blocks.append(cur)
                cur, size = [], 0
    if cur or not blocks:
        blocks.append(cur)
    workers = threads or min(len(blocks), os.cpu_count() or 1)
    with open(fn, 'wb') as f, ThreadPoolExecutor(max_workers=max(1, workers)) as ex:
        for data in ex.map(lambda b: bz2.compress(b"".join(b)), blocks):
            f.write(data)


_writer = None


def background_writer():
    """One thread that runs file writes in submission order (each write
    compresses with its own pool of threads)."""
    global _writer
    if _writer is None:
        _writer = ThreadPoolExecutor(max_workers=1, thread_name_prefix="msa-writer")
    return _writer


def writeSeqs(fn, seqs, alpha=alpha21, ids=None, headers=None, write_param=False, zipf=None):
    """Write sequences as the reference's writeSeqs does (seqload.py:353-411)."""
    write_text(fn, [header_bytes(alpha, headers, write_param), format_lines(seqs, alpha, ids)], zipf)
