"""The launch-shape tuner's cache and parameter checks (host only, no GPU):
entries are keyed by SM count, key width, read-length class, bin count and
bases per bin (in factors of 4);
they round-trip through the text file; out-of-range shapes are refused."""
import ctypes as C

import pytest

import gkc_b200 as G

OK, INVALID, NOT_FOUND = 0, 1, 10


def tp(target, chunk, ctas):
    return G.TuneParams(target, chunk, ctas, 0)


@pytest.fixture(autouse=True)
def clean_cache():
    G.lib().gkc_tune_cache_clear()
    yield
    G.lib().gkc_tune_cache_clear()


def lookup(sms, prm, bases, reads):
    out = G.TuneParams()
    st = G.lib().gkc_tune_cache_lookup(sms, C.byref(prm), bases, reads, C.byref(out))
    return st, out


def test_store_and_lookup_by_class():
    L = G.lib()
    short = G.params(31, 11, 256)
    assert L.gkc_tune_cache_store(148, C.byref(short), 3_000_000_000, 20_000_000, C.byref(tp(3072, 32768, 1))) == OK
    # same class: 150 bp reads, same key width and bins, bases per bin within the same factor of 4
    st, out = lookup(148, short, 4_000_000_000, 26_000_000)
    assert st == OK and out.as_dict() == {"coarse_target": 3072, "chunk_kmers": 32768, "count_ctas_per_sm": 1}
    # ten times fewer bases per bin: another size class
    assert lookup(148, short, 300_000_000, 2_000_000)[0] == NOT_FOUND
    # another class each: long reads, 128-bit keys, other bins, other SM count
    assert lookup(148, short, 2_000_000_000, 250_000)[0] == NOT_FOUND
    assert lookup(148, G.params(63, 13, 256), 3_000_000_000, 12_000_000)[0] == NOT_FOUND
    assert lookup(148, G.params(31, 11, 64), 3_000_000_000, 20_000_000)[0] == NOT_FOUND
    assert lookup(132, short, 3_000_000_000, 20_000_000)[0] == NOT_FOUND
    # k = 32 and k = 21 share the 64-bit class
    assert lookup(148, G.params(21, 11, 256), 3_000_000_000, 20_000_000)[0] == OK


def test_out_of_range_shapes_are_refused():
    L = G.lib()
    prm = G.params(31, 11, 256)
    for bad in (tp(100, 65536, 2), tp(4096, 65535, 2), tp(4096, 1 << 23, 2), tp(4096, 65536, 0),
                tp(4096, 65536, 5)):
        assert L.gkc_tune_cache_store(148, C.byref(prm), 10**9, 10**7, C.byref(bad)) == INVALID


def test_cache_file_round_trip(tmp_path):
    L = G.lib()
    a, b = G.params(31, 11, 256), G.params(25, 15, 256, True)
    assert L.gkc_tune_cache_store(148, C.byref(a), 3 * 10**9, 2 * 10**7, C.byref(tp(6144, 131072, 2))) == OK
    assert L.gkc_tune_cache_store(148, C.byref(b), 2 * 10**9, 2 * 10**5, C.byref(tp(2048, 65536, 1))) == OK
    path = str(tmp_path / "tune.txt").encode()
    assert L.gkc_tune_cache_save(path) == OK
    L.gkc_tune_cache_clear()
    assert lookup(148, a, 3 * 10**9, 2 * 10**7)[0] == NOT_FOUND
    assert L.gkc_tune_cache_load(path) == OK
    assert lookup(148, a, 3 * 10**9, 2 * 10**7)[1].as_dict()["coarse_target"] == 6144
    assert lookup(148, b, 2 * 10**9, 2 * 10**5)[1].as_dict() == {"coarse_target": 2048, "chunk_kmers": 65536,
                                                                  "count_ctas_per_sm": 1}
    # a damaged file is refused whole
    with open(path, "a") as f:
        f.write("gkc-tune 2 148 1 0 256 11 9 99 2\n")  # coarse target 9: out of range
    L.gkc_tune_cache_clear()
    assert L.gkc_tune_cache_load(path) == INVALID
    assert lookup(148, a, 3 * 10**9, 2 * 10**7)[0] == NOT_FOUND
    assert L.gkc_tune_cache_load(str(tmp_path / "missing.txt").encode()) == NOT_FOUND
