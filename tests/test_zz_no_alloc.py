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


def _sort(L, fn, k, v, ko, vo, n, bits):
    rc = getattr(L, fn)(ctypes.c_void_p(k.data_ptr()), ctypes.c_void_p(v.data_ptr()), ctypes.c_void_p(ko.data_ptr()),
                        ctypes.c_void_p(vo.data_ptr()), n, bits, None)
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
