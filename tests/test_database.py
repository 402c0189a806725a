"""The on-disk database reader of the library (host code) against files laid
out by the format's restatement in tests/db_format.py."""
import numpy as np
import pytest

import db_format as D
import gkc_b200 as G


def _sorted_keys(seed, n, k, kw):
    r = np.random.default_rng(seed)
    bits = 2 * k
    if kw == 1:
        ks = np.unique(r.integers(0, 1 << min(bits, 63), n, dtype=np.uint64) & np.uint64((1 << bits) - 1))
        return ks, ks.reshape(-1, 1)
    lo = r.integers(0, 1 << 63, n, dtype=np.uint64)
    hi = r.integers(0, 1 << (bits - 64), n, dtype=np.uint64)
    ints = sorted(set(int(a) | (int(b) << 64) for a, b in zip(lo, hi)))
    arr = np.array([[x & ((1 << 64) - 1), x >> 64] for x in ints], np.uint64)
    return ints, arr


@pytest.mark.parametrize("k,n,lut,cmax", [(31, 5000, 0, 200), (21, 3000, 4, 70000), (17, 800, 7, 3),
                                          (45, 2000, 0, 1 << 25), (63, 500, 13, 9), (31, 0, 0, 1)])
def test_reader_against_restated_layout(tmp_path, k, n, lut, cmax):
    kw = 1 if k <= 32 else 2
    _, keys = _sorted_keys(k + n, n, k, kw)
    n = len(keys)
    counts = np.random.default_rng(n).integers(1, cmax + 1, n).astype(np.uint32)
    path = str(tmp_path / "db")
    D.write(path, k, keys, counts, 2, 1000, lut)
    with G.Database(path) as db:
        info = db.info
        hdr, recs = D.parse(path)
        assert info["k"] == k and info["n_kmers"] == n and info["lut_prefix_len"] == hdr["lut_prefix_len"]
        assert info["counter_bytes"] == hdr["counter_bytes"] and info["total_count"] == int(counts.sum())
        assert (info["min_count"], info["max_count"]) == (2, 1000)
        got_k, got_c = db.read()
        assert np.array_equal(got_k, keys) and np.array_equal(got_c, counts)
        if n:
            mid_k, mid_c = db.read(n // 3, n // 2)
            assert np.array_equal(mid_k, keys[n // 3:n // 3 + n // 2])
            assert np.array_equal(db.lookup(keys), counts)
            # absent keys: neighbours of present ones that are not in the list
            present = set(D.key_ints(keys))
            probe = [x + 1 for x in D.key_ints(keys[:200]) if x + 1 not in present and x + 1 < 4 ** k]
            if probe:
                pk = np.array([[x & ((1 << 64) - 1), x >> 64][:kw] for x in probe], np.uint64)
                assert not db.lookup(pk).any()


def test_reader_rejects_damaged_files(tmp_path):
    _, keys = _sorted_keys(1, 100, 31, 1)
    path = str(tmp_path / "db")
    D.write(path, 31, keys, np.ones(len(keys), np.uint32), 1, 5)
    suf = tmp_path / "db.gkc_suf"
    data = suf.read_bytes()
    suf.write_bytes(data[:-1])  # truncated records
    with pytest.raises(G.GkcError):
        G.Database(path)
    with pytest.raises(G.GkcError):
        G.Database(str(tmp_path / "missing"))


def test_reader_single_base_kmers(tmp_path):
    """k = 1: the table has no prefix bits (two entries)."""
    keys = np.array([[0], [2], [3]], np.uint64)
    counts = np.array([4, 1, 7], np.uint32)
    path = str(tmp_path / "db")
    D.write(path, 1, keys, counts, 1, 9, 0)
    with G.Database(path) as db:
        assert db.info["lut_prefix_len"] == 0
        assert np.array_equal(db.lookup(np.array([0, 1, 2, 3], np.uint64)), [4, 0, 1, 7])
