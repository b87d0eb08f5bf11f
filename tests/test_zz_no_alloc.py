"""abf_collect_ids_noalloc against abf_collect_ids, through the C ABI.

The allocation-free entry point serves callers that may not allocate device
memory while they work (a host engine that owns all device memory, a
serving thread that cannot take cudaMalloc's synchronisation, code that must
not run out of memory mid-request); its scratch is a static device array.
Two calls in a row check that the array's leftover contents from the first
call do not leak into the second. This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import adabool_b200 as ab
from adabool_b200 import Index
from adabool_b200 import _native as N

pytestmark = pytest.mark.gpu


MAX_BITS = 1 << 30  # ABF_NOALLOC_MAX_BITS


def _bitmap(rng, n_bits, density):
    n_words = (n_bits + 31) // 32
    bits = rng.random(n_words * 32) < density
    return np.packbits(bits, bitorder="little").view(np.uint32).copy()


def _sparse_words(rng, n_bits, ands):
    """Random words with each bit set with probability 2^-ands (cheap at 2^30 bits)."""
    n_words = (n_bits + 31) // 32
    w = rng.integers(0, 1 << 32, n_words, dtype=np.uint32)
    for _ in range(ands - 1):
        w &= rng.integers(0, 1 << 32, n_words, dtype=np.uint32)
    return w


def _definition(words, n_bits):
    return np.flatnonzero(np.unpackbits(words.view(np.uint8), bitorder="little")[:n_bits])


def _both(L, ix, d_bm, n_bits, cap, stream):
    import torch
    # 64 guard entries past the capacity must stay untouched
    ids_ref = torch.full((cap + 64,), -1, dtype=torch.int32, device="cuda")
    ids_na = torch.full((cap + 64,), -2, dtype=torch.int32, device="cuda")
    cnt_ref = torch.zeros(1, dtype=torch.int64, device="cuda")
    cnt_na = torch.full((1,), 12345, dtype=torch.int64, device="cuda")  # overwritten by the call
    sp = C.c_void_p(stream.cuda_stream)
    N.check(L.abf_collect_ids(ix.handle, C.c_void_p(d_bm.data_ptr()), n_bits, C.c_void_p(ids_ref.data_ptr()),
                              cap, C.c_void_p(cnt_ref.data_ptr()), sp))
    N.check(L.abf_collect_ids_noalloc(C.c_void_p(d_bm.data_ptr()), n_bits, C.c_void_p(ids_na.data_ptr()), cap,
                                      C.c_void_p(cnt_na.data_ptr()), sp))
    N.check(L.abf_collect_ids_noalloc_check(sp))  # no look-back wait gave up
    torch.cuda.synchronize()
    return ids_ref, int(cnt_ref.item()), ids_na, int(cnt_na.item())


def test_noalloc_matches_collect_ids_two_calls(dev):
    import torch
    L = ab.lib()
    rng = np.random.default_rng(2024)
    ix = Index.from_csr([0, 1], [0], 1, 64, device=0)  # the existing entry point takes an index
    stream = torch.cuda.current_stream()
    # first call large and dense, second smaller and sparse: a stale count or
    # offset from the first call would show up in the second
    for n_bits, density in ((3 * 65536 * 32 + 77, 0.7), (70_001, 0.02)):
        words = _bitmap(rng, n_bits, density)
        d_bm = torch.from_numpy(words.view(np.int32)).cuda()
        cap = int(np.unpackbits(words.view(np.uint8)).sum()) + 8
        ids_ref, n, ids_na, n_na = _both(L, ix, d_bm, n_bits, cap, stream)
        assert n_na == n
        assert np.array_equal(ids_na[:n].cpu().numpy(), ids_ref[:n].cpu().numpy())
        # and both equal the plain definition
        assert np.array_equal(ids_na[:n].cpu().numpy().astype(np.int64), _definition(words, n_bits))


def test_noalloc_largest_bitmap_and_short_capacity(dev):
    """ABF_NOALLOC_MAX_BITS bits (16,384 compaction chunks: the look-back
    crosses hundreds of 32-word windows of the static array), then the same
    bitmap with room for only part of its ids: the count stays exact and the
    ids that fit are the first ones."""
    import torch
    L = ab.lib()
    rng = np.random.default_rng(77)
    ix = Index.from_csr([0, 1], [0], 1, 64, device=0)
    stream = torch.cuda.current_stream()
    words = _sparse_words(rng, MAX_BITS, 5)  # ~3 % of the bits
    expect = _definition(words, MAX_BITS)
    d_bm = torch.from_numpy(words.view(np.int32)).cuda()
    for cap in (expect.size + 3, expect.size // 3):
        ids_ref, n, ids_na, n_na = _both(L, ix, d_bm, MAX_BITS, cap, stream)
        assert n == n_na == expect.size
        k = min(cap, n)
        got = ids_na[:k].cpu().numpy()
        assert np.array_equal(got, ids_ref[:k].cpu().numpy())
        assert np.array_equal(got.astype(np.int64), expect[:k])
        assert (ids_na[cap:] == -2).all() and (ids_ref[cap:] == -1).all()  # nothing past the capacity


def test_noalloc_refuses_oversized_bitmap(dev):
    L = ab.lib()
    st = L.abf_collect_ids_noalloc(C.c_void_p(16), MAX_BITS + 1, C.c_void_p(16), 1, C.c_void_p(16), None)
    assert st == 8  # ABF_ERR_CAPACITY, before any device work
    assert b"ABF_NOALLOC_MAX_BITS" in L.abf_last_error_string()
