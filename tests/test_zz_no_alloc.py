"""The scratch-free sort entry point, pgmpm_radix_sort_pairs_noalloc.

It exists for callers that may not allocate GPU memory while they run: a
host framework that hands this library a fixed memory budget, or a loop that
cannot pay cudaMalloc's device-wide synchronisation.  Its result must equal
the allocating entry point's, bit for bit (integer work), on consecutive
calls that reuse the shared scratch array, and it must not grow the
device's used memory.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _sort(L, fn, k, v, ko, vo, n, bits):
    """v = None passes a null value array (values = 0..n-1)."""
    rc = getattr(L, fn)(_ptr(k), _ptr(v), _ptr(ko), _ptr(vo), n, bits, None)
    return rc


def test_noalloc_sort_matches_allocating_sort_on_consecutive_calls(gpu):
    import torch

    from physgrad_b200 import _capi as C

    L = C.lib()
    cases = [(700001, 21, 11), (65537, 12, 12), (C.NOALLOC_MAX_PAIRS, 32, 13)]
    bufs = []
    for n, bits, seed in cases:
        rng = np.random.default_rng(seed)
        k = torch.from_numpy(rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32).view(np.int32)).cuda()
        v = torch.from_numpy(rng.integers(0, 1 << 31, n).astype(np.uint32).view(np.int32)).cuda()
        bufs.append((n, bits, k, v, torch.empty_like(k), torch.empty_like(v), torch.empty_like(k),
                     torch.empty_like(v)))
    torch.cuda.synchronize()
    # first call on this device: looks up the scratch array's address
    n0, b0, k0, v0, _, _, ko0, vo0 = bufs[0]
    C.check(_sort(L, "pgmpm_radix_sort_pairs_noalloc", k0, v0, ko0, vo0, n0, b0))
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for n, bits, k, v, ka, va, kn, vn in bufs:
        C.check(_sort(L, "pgmpm_radix_sort_pairs_noalloc", k, v, kn, vn, n, bits))
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before, "the no-alloc entry point changed device free memory"
        C.check(_sort(L, "pgmpm_radix_sort_pairs", k, v, ka, va, n, bits))
        torch.cuda.synchronize()
        assert torch.equal(kn, ka) and torch.equal(vn, va)
        # and it is the stable order
        kk = k.cpu().numpy().view(np.uint32)
        ref = np.argsort(kk, kind="stable")
        assert np.array_equal(kn.cpu().numpy().view(np.uint32), kk[ref])
        assert np.array_equal(vn.cpu().numpy(), v.cpu().numpy()[ref])
        free_before = torch.cuda.mem_get_info()[0]


def test_noalloc_sort_rejects_sizes_beyond_its_maximum(gpu):
    import torch

    from physgrad_b200 import _capi as C

    L = C.lib()
    k = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = _sort(L, "pgmpm_radix_sort_pairs_noalloc", k, k.clone(), torch.empty_like(k), torch.empty_like(k),
               C.NOALLOC_MAX_PAIRS + 1, 8)
    assert rc == C.PGMPM_ERR_ARG
    assert b"exceeds the maximum" in L.pgmpm_last_error()


def test_noalloc_sort_null_values_is_the_stable_permutation(gpu):
    """vals_in = NULL sorts the indices 0..n-1 along with the keys: the result
    is the stable argsort, equal to the allocating entry point's, on two calls
    in a row (the second reuses the scratch the first left behind)."""
    import torch

    from physgrad_b200 import _capi as C

    L = C.lib()
    for n, bits, seed in ((300007, 17, 21), (4099, 9, 22)):
        rng = np.random.default_rng(seed)
        kk = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        k = torch.from_numpy(kk.view(np.int32)).cuda()
        kn, vn, ka, va = (torch.empty_like(k) for _ in range(4))
        C.check(_sort(L, "pgmpm_radix_sort_pairs_noalloc", k, None, kn, vn, n, bits))
        C.check(_sort(L, "pgmpm_radix_sort_pairs", k, None, ka, va, n, bits))
        torch.cuda.synchronize()
        assert torch.equal(kn, ka) and torch.equal(vn, va)
        ref = np.argsort(kk, kind="stable").astype(np.uint32)
        assert np.array_equal(vn.cpu().numpy().view(np.uint32), ref)
        assert np.array_equal(kn.cpu().numpy().view(np.uint32), kk[ref])


def test_noalloc_sort_rejects_overlapping_outputs(gpu):
    """An output that overlaps an input (or the other output) would be written
    by the first pass while that pass still reads it: rejected before any
    work, including the cross cases (keys out over values in, a partial
    overlap) and both outputs in one array."""
    import torch

    from physgrad_b200 import _capi as C

    L = C.lib()
    n = 1024
    buf = torch.zeros(4 * n, dtype=torch.int32, device="cuda")
    k, v, ko, vo = buf[:n], buf[n:2 * n], buf[2 * n:3 * n], buf[3 * n:]
    C.check(_sort(L, "pgmpm_radix_sort_pairs_noalloc", k, v, ko, vo, n, 8))
    torch.cuda.synchronize()
    bad = [(k, v, v, vo), (k, v, ko, k), (k, v, buf[n // 2:n // 2 + n], vo), (k, v, ko, buf[2 * n + 8:3 * n + 8]),
           (k, None, ko, k)]
    for a, b, c, d in bad:
        assert _sort(L, "pgmpm_radix_sort_pairs_noalloc", a, b, c, d, n, 8) == C.PGMPM_ERR_ARG
        assert b"must not overlap" in L.pgmpm_last_error()
