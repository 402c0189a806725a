"""Per-window minimizer / position / strand, subsampled position lists and
homopolymer compression through the C ABI, against the oracle."""
import numpy as np
import pytest

import gkc_b200 as G
import oracle_ffi as F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as T
    return T


@pytest.fixture(scope="module")
def ctx():
    c = G.Context(0)
    yield c
    c.close()


def random_reads(seed, n, lo, hi, n_rate=0.01, homopolymers=False):
    r = np.random.default_rng(seed)
    lens = r.integers(lo, hi + 1, n)
    offs = np.zeros(n + 1, np.uint64)
    offs[1:] = np.cumsum(lens)
    alphabet = np.frombuffer(b"ACGTacgtU", np.uint8)
    b = alphabet[r.integers(0, len(alphabet), int(offs[-1]))].copy()
    b[r.random(len(b)) < n_rate] = ord("N")
    if homopolymers:  # stretch random bases into runs
        rep = r.integers(1, 6, len(b))
        b = np.repeat(b, rep)[: len(b)]
    return b, offs


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


CASES = [  # seed, n, lo, hi, k, p
    (1, 300, 5, 400, 31, 11),
    (2, 200, 10, 3000, 25, 15),
    (3, 150, 60, 500, 63, 13),
    (4, 100, 1, 40, 17, 9),
]


@pytest.mark.parametrize("seed,n,lo,hi,k,p", CASES)
def test_minimizers_pos_strand_vs_oracle(torch, ctx, seed, n, lo, hi, k, p):
    reads, offs = random_reads(seed, n, lo, hi)
    nb = len(reads)
    d_reads, d_offs = to_dev(torch, reads), to_dev(torch, offs.view(np.int64))
    d_mm = torch.zeros(nb, dtype=torch.int32, device="cuda")
    d_pos = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    d_st = torch.zeros(nb, dtype=torch.int8, device="cuda")
    ctx.minimizers_device(d_reads.data_ptr(), nb, d_offs.data_ptr(), n, G.params(k, p, 1),
                          d_mm.data_ptr(), d_pos.data_ptr(), d_st.data_ptr())
    mm = d_mm.cpu().numpy().view(np.uint32)
    pos = d_pos.cpu().numpy()
    st = d_st.cpu().numpy()
    want_mm = np.full(nb, 0xFFFFFFFF, np.uint32)
    want_pos = np.full(nb, 255, np.uint8)
    want_st = np.zeros(nb, np.int8)
    for i in range(n):
        b, e = int(offs[i]), int(offs[i + 1])
        if e - b < k:
            continue
        m, ps, s = F.oracle_minimizers(reads[b:e], k, p, with_pos=True)
        want_mm[b:b + len(m)] = m
        want_pos[b:b + len(m)] = ps
        want_st[b:b + len(m)] = s
    assert np.array_equal(mm, want_mm)
    assert np.array_equal(pos, want_pos)
    assert np.array_equal(st, want_st)


class _DevBytes:
    """A raw device range, for torch.as_tensor (the CUDA array interface)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3}


def dev_bytes(torch, ptr, nbytes):
    if nbytes == 0:
        return np.zeros(0, np.uint8)
    return torch.as_tensor(_DevBytes(ptr, nbytes), device="cuda").cpu().numpy()


def subsample(torch, ctx, reads, offs, k, p, mod):
    n = len(offs) - 1
    d_reads, d_offs = to_dev(torch, reads), to_dev(torch, offs.view(np.int64))
    v = ctx.subsample_positions_device(d_reads.data_ptr(), len(reads), d_offs.data_ptr(), n,
                                       G.params(k, p, 1), mod)
    nd, npos, kw = int(v.n_distinct), int(v.n_positions), int(v.key_words)
    keys = dev_bytes(torch, v.keys, nd * kw * 8).view(np.uint64).reshape(nd, kw)
    pos_off = dev_bytes(torch, v.pos_off, (nd + 1) * 8).view(np.uint64)
    pos = dev_bytes(torch, v.positions, npos * 4).view(np.uint32)
    return nd, kw, keys, pos_off, pos


@pytest.mark.parametrize("seed,n,lo,hi,k,p,mod", [
    (5, 300, 20, 400, 31, 11, 4),
    (6, 200, 60, 500, 63, 13, 4),
    (7, 100, 25, 200, 25, 15, 1),
    (8, 50, 1, 30, 21, 7, 3),
])
def test_subsample_positions_vs_oracle(torch, ctx, seed, n, lo, hi, k, p, mod):
    reads, offs = random_reads(seed, n, lo, hi)
    reads = np.concatenate([reads, reads])  # every k-mer at least twice
    offs = np.concatenate([offs, offs[1:] + offs[-1]])
    nd, kw, keys, pos_off, pos = subsample(torch, ctx, reads, offs, k, p, mod)
    want = F.oracle_subsample(reads, offs, k, p, mod)
    assert nd == len(want["keys_lo"])
    if nd:
        assert np.array_equal(keys[:, 0], want["keys_lo"])
        if kw == 2:
            assert np.array_equal(keys[:, 1], want["keys_hi"])
    assert np.array_equal(pos_off, want["pos_off"])
    assert np.array_equal(pos, want["pos"])


def test_hpc_vs_oracle(torch, ctx):
    reads, offs = random_reads(9, 400, 0, 300, homopolymers=True)
    n, nb = len(offs) - 1, len(reads)
    d_reads, d_offs = to_dev(torch, reads), to_dev(torch, offs.view(np.int64))
    d_out = torch.zeros(max(nb, 1), dtype=torch.uint8, device="cuda")
    d_ooffs = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    d_orig = torch.zeros(max(nb, 1), dtype=torch.int32, device="cuda")
    ctx.hpc_device(d_reads.data_ptr(), nb, d_offs.data_ptr(), n, d_out.data_ptr(), d_ooffs.data_ptr(),
                   d_orig.data_ptr())
    out, ooffs, orig = d_out.cpu().numpy(), d_ooffs.cpu().numpy().view(np.uint64), d_orig.cpu().numpy()
    w_out, w_len, w_orig = F.oracle_hpc(reads, offs)
    assert np.array_equal(np.diff(ooffs).astype(np.int64), w_len.astype(np.int64))
    for r in range(n):
        b, ob, ln = int(offs[r]), int(ooffs[r]), int(w_len[r])
        assert np.array_equal(out[ob:ob + ln], w_out[b:b + ln])
        assert np.array_equal(orig[ob:ob + ln], w_orig[b:b + ln])


def test_empty_inputs(torch, ctx):
    offs = np.zeros(1, np.uint64)
    d_offs = to_dev(torch, offs.view(np.int64))
    v = ctx.subsample_positions_device(0, 0, d_offs.data_ptr(), 0, G.params(31, 11, 1), 4)
    assert v.n_distinct == 0 and v.n_positions == 0
    ctx.minimizers_device(0, 0, d_offs.data_ptr(), 0, G.params(31, 11, 1), 0, 0, 0)
