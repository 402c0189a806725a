"""FASTA / FASTQ ingest (gkc_fastx_load) against a plain Python parser with
the same record rules, on CPU: Windows line ends, multi-line FASTA records,
empty sequences, quality lines that start with '@', no final newline, and
files big enough to be cut between several threads."""
import numpy as np
import pytest

import gkc_b200 as G


def py_fastq(text):
    lines = text.split("\n")
    out, i = [], 0
    while i < len(lines):
        if lines[i].startswith("@") and i + 1 < len(lines):
            out.append(lines[i + 1].rstrip("\r"))
            i += 4
        else:
            i += 1
    return out


def py_fasta(text):
    out, cur = [], None
    for line in text.split("\n"):
        if line.startswith(">"):
            if cur is not None:
                out.append("".join(cur))
            cur = []
        elif cur is not None:
            cur.append(line.rstrip("\r"))
    if cur is not None:
        out.append("".join(cur))
    return out


def check(path, want, threads):
    reads, offs = G.load_fastx(str(path), threads=threads)
    assert len(offs) == len(want) + 1 and offs[0] == 0
    got = [reads[offs[i]:offs[i + 1]].tobytes().decode() for i in range(len(want))]
    assert got == want


def gen_reads(seed, n, lo, hi):
    r = np.random.default_rng(seed)
    al = np.array(list("ACGTNacgt"))
    return ["".join(al[r.integers(0, len(al), r.integers(lo, hi + 1))]) for _ in range(n)]


@pytest.mark.parametrize("threads", [1, 3, 8])
def test_fastq(tmp_path, threads):
    seqs = gen_reads(1, 30000, 0, 300)
    r = np.random.default_rng(2)
    parts = []
    for i, sq in enumerate(seqs):
        q = "".join(r.choice(list("@+!IJ#"), len(sq)))  # quality may start with '@' or '+'
        nl = "\r\n" if i % 7 == 0 else "\n"
        parts.append(f"@read{i} x{nl}{sq}{nl}+{nl}{q}{nl}")
    text = "".join(parts)[:-1]  # no final newline
    p = tmp_path / "r.fq"
    p.write_bytes(text.encode())
    assert py_fastq(text) == seqs
    check(p, seqs, threads)


@pytest.mark.parametrize("threads", [1, 4])
def test_fasta_multiline(tmp_path, threads):
    seqs = gen_reads(3, 20000, 0, 500)
    parts = []
    for i, sq in enumerate(seqs):
        body = "\n".join(sq[j:j + 60] for j in range(0, len(sq), 60))
        parts.append(f">s{i} desc\r\n{body}\n" if i % 5 == 0 else f">s{i}\n{body}\n")
    text = "".join(parts)
    p = tmp_path / "r.fa"
    p.write_bytes(text.encode())
    check(p, py_fasta(text), threads)


def test_rejects_other_formats(tmp_path):
    p = tmp_path / "x.txt"
    p.write_bytes(b"hello\n")
    with pytest.raises(G.GkcError):
        G.load_fastx(str(p))
    with pytest.raises(G.GkcError):
        G.load_fastx(str(tmp_path / "missing.fq"))


def test_empty_file_has_no_reads(tmp_path):
    for name, data in (("e.fq", b""), ("nl.fa", b"\n\n")):
        p = tmp_path / name
        p.write_bytes(data)
        reads, offs = G.load_fastx(str(p))
        assert len(reads) == 0 and list(offs) == [0]
