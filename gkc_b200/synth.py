"""Seeded synthetic workloads (numpy mirror of csrc/synth_core.h).

The library generates the same bytes on the device (gkc_synth_* in the C ABI);
this module produces them on the host for small cases and for the CPU
baseline.  Every base is a pure function of (seed, stream, index).
"""
import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
S_IID, S_GENOME, S_SEG, S_SEGMUT, S_READPOS, S_READERR = 1, 2, 3, 4, 5, 6
ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


def _u(x):
    return np.asarray(x, dtype=np.uint64)


def mix64(z):
    z = _u(z)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def rng(seed, stream, idx):
    with np.errstate(over="ignore"):
        base = mix64(_u(seed) * np.uint64(0x9E3779B97F4A7C15) + _u(stream))
        return mix64(base + _u(idx) * np.uint64(0xD1B54A32D192ED03) + np.uint64(0x632BE59BD9B4E019))


def prob32(p):
    t = p * 4294967296.0
    return 0xFFFFFFFF if t >= 4294967295.0 else int(t)


def iid_reads(seed, n_reads, read_len, n_rate):
    """Config-1 reads: i.i.d. ACGT, each base N with probability n_rate."""
    idx = np.arange(n_reads * read_len, dtype=np.uint64)
    h = rng(seed, S_IID, idx)
    reads = ACGT[(h & np.uint64(3)).astype(np.intp)]
    reads[(h >> np.uint64(32)) < np.uint64(prob32(n_rate))] = ord("N")
    offs = np.arange(0, n_reads * read_len + 1, read_len, dtype=np.uint64)
    return reads, offs


def genome_describe(genome_len, seg_fraction=0.05):
    n = int(seg_fraction * genome_len / 3000.0 + 0.5)
    n_seg = n if (genome_len >= 4096 and n > 0) else 0
    slot = genome_len // n_seg if n_seg else 0
    return n_seg, slot


def genome(seed, genome_len, seg_fraction=0.05, divergence=0.01):
    """Genome codes (0..3): i.i.d. bases plus segment copies (1-5 kbp, 1%
    divergence) placed in disjoint slots."""
    g = (rng(seed, S_GENOME, np.arange(genome_len, dtype=np.uint64)) & np.uint64(3)).astype(np.uint8)
    n_seg, slot = genome_describe(genome_len, seg_fraction)
    thr = np.uint64(prob32(divergence))
    for s in range(n_seg):
        l = 1000 + int(rng(seed, S_SEG, 3 * s) % np.uint64(4001))
        if l + 1 >= slot:
            l = slot // 2
        room = slot - l
        dst = s * slot + int(rng(seed, S_SEG, 3 * s + 1) % np.uint64(room))
        src = int(rng(seed, S_SEG, 3 * s + 2) % np.uint64(genome_len - l))
        sp = np.arange(src, src + l, dtype=np.uint64)
        dp = np.arange(dst, dst + l, dtype=np.uint64)
        b = (rng(seed, S_GENOME, sp) & np.uint64(3)).astype(np.uint64)
        h = rng(seed, S_SEGMUT, dp)
        mut = (h >> np.uint64(32)) < thr
        b2 = (b + np.uint64(1) + (h & np.uint64(0xFFFF)) % np.uint64(3)) & np.uint64(3)
        g[dst:dst + l] = np.where(mut, b2, b).astype(np.uint8)
    return g


def short_reads(seed, genome_codes, n_reads, read_len, err_rate, first_read=0):
    """Fixed-length reads at uniform positions on both strands with i.i.d.
    substitution errors (configs 2 and 4)."""
    G = len(genome_codes)
    r = np.arange(first_read, first_read + n_reads, dtype=np.uint64)
    pos = rng(seed, S_READPOS, np.uint64(2) * r) % np.uint64(G - read_len + 1)
    strand = (rng(seed, S_READPOS, np.uint64(2) * r + np.uint64(1)) & np.uint64(1)).astype(bool)
    j = np.arange(read_len, dtype=np.uint64)
    fwd_idx = pos[:, None] + j[None, :]
    rc_idx = pos[:, None] + np.uint64(read_len - 1) - j[None, :]
    idx = np.where(strand[:, None], rc_idx, fwd_idx)
    g = genome_codes[idx.astype(np.intp)].astype(np.uint64)
    g = np.where(strand[:, None], np.uint64(3) - g, g)
    e = rng(seed, S_READERR, r[:, None] * np.uint64(read_len) + j[None, :])
    err = (e >> np.uint64(32)) < np.uint64(prob32(err_rate))
    g2 = (g + np.uint64(1) + (e & np.uint64(0xFFFF)) % np.uint64(3)) & np.uint64(3)
    g = np.where(err, g2, g)
    reads = ACGT[g.astype(np.intp)].reshape(-1)
    offs = np.arange(0, n_reads * read_len + 1, read_len, dtype=np.uint64)
    return reads, offs
