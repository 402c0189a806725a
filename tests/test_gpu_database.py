"""The database writer on the GPU: the files gkc_db_write lays out from the
count result are byte-identical to the format's restatement applied to the
oracle's merged, filtered list, and the reader finds every count."""
import numpy as np
import pytest

import db_format as D
import gkc_b200 as G
import oracle_ffi as F
from gpu_helpers import lib_counts, lib_partition

pytestmark = pytest.mark.gpu


def _reads(seed, n, lo, hi):
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    # a short alphabet run keeps counts above one; N splits superkmers
    b = np.frombuffer(b"ACGT", np.uint8)[r.integers(0, 4, int(offs[-1]))].copy()
    b[r.random(len(b)) < 0.02] = ord("N")
    return np.tile(b, 3), np.concatenate([offs[:-1] + i * offs[-1] for i in range(3)] + [[3 * offs[-1]]]).astype(np.uint64)


def _oracle_merged(reads, offs, k, p, nb, mn, mx):
    c = F.oracle_count_bins(F.oracle_partition(reads, offs, k, p, 0, nb), k, nb)
    lo = c["keys_lo"].astype(object)
    ints = lo if c["keys_hi"] is None else lo + (c["keys_hi"].astype(object) << 64)
    tot = {}
    for key, cnt in zip(ints, c["counts"]):
        tot[int(key)] = min(tot.get(int(key), 0) + int(cnt), 0xFFFFFFFF)
    ks = sorted(x for x, v in tot.items() if mn <= v <= mx)
    kw = 1 if k <= 32 else 2
    arr = np.array([[x & ((1 << 64) - 1), x >> 64][:kw] for x in ks], np.uint64).reshape(-1, kw)
    return arr, np.array([tot[x] for x in ks], np.uint32)


@pytest.mark.parametrize("k,p,nb,mn,mx,lut", [(31, 11, 64, 1, 0xFFFFFFFF, 0), (31, 11, 64, 2, 5, 6),
                                              (21, 9, 16, 1, 0xFFFFFFFF, 3), (45, 15, 32, 1, 0xFFFFFFFF, 0)])
def test_db_write_bytes_and_lookup(tmp_path, k, p, nb, mn, mx, lut):
    reads, offs = _reads(100 + k, 200, k, 400)
    keys, counts = _oracle_merged(reads, offs, k, p, nb, mn, mx)
    with G.Context(0) as c:
        lib_partition(c, reads, offs, k, p, 0, nb)
        lib_counts(c, k, nb)
        path = str(tmp_path / "db")
        c.db_write(path, mn, mx, lut)
    pre, suf = D.layout(k, keys, counts, mn, mx, lut)
    assert open(path + ".gkc_pre", "rb").read() == pre
    assert open(path + ".gkc_suf", "rb").read() == suf
    with G.Database(path) as db:
        assert db.info["n_kmers"] == len(counts)
        if len(counts):
            assert np.array_equal(db.lookup(keys), counts)
