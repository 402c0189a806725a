"""FASTA / FASTQ ingest (gkc_fastx_load) on CPU: against the reference's own
loader (read_loader.hpp compiled into oracle/_ref) on the same files, and
against a plain Python parser with the same record rules: Windows line ends,
multi-line FASTA records (first line by default, joined on request), empty
sequences, quality lines that start with '@', no final newline, and files big
enough to be cut between several threads."""
import os
import subprocess
import sys

import numpy as np
import pytest

import gkc_b200 as G
import oracle_ffi as F


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


def py_fasta_first_line(text):
    out, take = [], False
    for line in text.split("\n"):
        if line.startswith(">"):
            take = True
        elif take:
            out.append(line.rstrip("\r"))
            take = False
    return out


def check(path, want, threads, flags=0):
    reads, offs = G.load_fastx(str(path), threads=threads, flags=flags)
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
    check(p, py_fasta(text), threads, flags=G.FASTX_JOIN_LINES)
    check(p, py_fasta_first_line(text), threads)  # the reference's rule: the line after the header


def test_format_from_name_or_content(tmp_path):
    p = tmp_path / "reads.txt"
    p.write_bytes(b"@r1\nACGT\n+\nIIII\n")
    with pytest.raises(G.GkcError):  # by name a FASTA file, which must start with '>'
        G.load_fastx(str(p))
    reads, offs = G.load_fastx(str(p), flags=G.FASTX_FORMAT_FROM_CONTENT)
    assert reads.tobytes() == b"ACGT" and list(offs) == [0, 4]


def write_reference_cases(d):
    """Files in the formats the reference reads: 4-line FASTQ and 2-line
    FASTA, with lower case, N, Windows line ends and quality lines that start
    with '@'; the big ones span several of the reference loader's buffers."""
    r = np.random.default_rng(7)
    cases = []
    for seed, (name, n, lo, hi) in enumerate((("small.fq", 500, 20, 300), ("big.fq", 60000, 50, 250),
                                              ("small.fa", 800, 15, 400), ("big.fa", 50000, 30, 300))):
        seqs = gen_reads(100 + seed, n, lo, hi)
        parts = []
        for i, sq in enumerate(seqs):
            nl = "\r\n" if i % 9 == 0 else "\n"
            if name.endswith("q"):
                q = "".join(r.choice(list("@+!IJ#"), len(sq)))
                parts.append(f"@read{i}{nl}{sq}{nl}+{nl}{q}{nl}")
            else:
                parts.append(f">read{i} d{nl}{sq}{nl}")
        path = os.path.join(d, name)
        with open(path, "wb") as f:
            f.write("".join(parts).encode())
        cases.append(path)
    return cases


@pytest.mark.skipif(not F.ref_loader_available(), reason="oracle/_ref was not built")
def test_matches_the_reference_loader(tmp_path):
    for path in write_reference_cases(str(tmp_path)):
        for threads in (1, 4):
            # the reference loader runs in a child process: its worker threads
            # wait on each other, so a stuck run ends with the timeout
            out = str(tmp_path / "ref.npz")
            code = ("import sys, numpy as np; sys.path.insert(0, %r); import oracle_ffi as F; "
                    "r, o = F.ref_load_reads(%r, %d); np.savez(%r, r=r, o=o)"
                    % (os.path.dirname(os.path.abspath(__file__)), path, threads, out))
            subprocess.run([sys.executable, "-c", code], check=True, timeout=120, capture_output=True)
            z = np.load(out)
            reads, offs = G.load_fastx(path, threads=threads)
            assert len(offs) == len(z["o"]), (path, threads, len(offs), len(z["o"]))
            assert np.array_equal(offs, z["o"]), (path, threads)
            assert np.array_equal(reads, z["r"]), (path, threads)


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
