"""The allocation-free sort entry point, called through the C ABI.

mrb_radix_sort_pairs_u32_noalloc serves callers that cannot allocate device
memory (a host that owns all device memory through its own allocator, or a
latency-critical path where cudaMalloc's implicit synchronisation is not
allowed).  Its scratch is a file-scope device array shared by every call.
This test checks, on calls in a row (each runs on the array the previous
one left behind, with even and odd numbers of 8-bit passes), that it
returns exactly what the allocating entry point returns for the same input,
and that sizes over the limit are refused.  The file sorts last so that a
failure here comes after every other test has run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def _sort_with_scratch(torch, lib, keys, vals, b, e, desc):
    dk = torch.from_numpy(keys.view(np.int32).copy()).cuda()
    dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    tb = lib.mrb_radix_sort_temp_bytes(keys.shape[0], 4, b, e)
    tmp = torch.zeros(tb, dtype=torch.uint8, device="cuda")
    rc = lib.mrb_radix_sort_pairs_u32(dk.data_ptr(), dv.data_ptr(), keys.shape[0], b, e, desc,
                                      tmp.data_ptr(), tb, None)
    assert rc == 0, lib.mrb_last_error()
    torch.cuda.synchronize()
    return dk.cpu().numpy().view(np.uint32), dv.cpu().numpy().view(np.uint32)


def _sort_noalloc(torch, lib, keys, vals, b, e, desc):
    dk = torch.from_numpy(keys.view(np.int32).copy()).cuda()
    dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    rc = lib.mrb_radix_sort_pairs_u32_noalloc(dk.data_ptr(), dv.data_ptr(), keys.shape[0], b, e,
                                              desc, None)
    assert rc == 0, lib.mrb_last_error()
    torch.cuda.synchronize()
    return dk.cpu().numpy().view(np.uint32), dv.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort_twice(cuda):
    from meturay_b200._lib import lib
    torch = cuda
    rng = np.random.default_rng(99)
    # 4 and 2 passes end in the caller's buffers; 3 and 1 passes end in the
    # array's key/value copies and are copied back, so both exits run on the
    # array that the previous call left behind
    cases = [(MAX_PAIRS, 0, 32, 1), (300001, 0, 13, 1), (MAX_PAIRS - 7, 0, 24, 0),
             (65537, 8, 16, 1)]
    for n, b, e, desc in cases:  # calls in a row on the shared array
        keys = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        keys[::5] &= 0x1FFF  # repeated keys: order among equals must be kept
        vals = rng.permutation(n).astype(np.uint32)
        ek, ev = _sort_with_scratch(torch, lib, keys, vals, b, e, desc)
        gk, gv = _sort_noalloc(torch, lib, keys, vals, b, e, desc)
        assert np.array_equal(gk, ek)
        assert np.array_equal(gv, ev)


def test_noalloc_sort_rejects_oversized_input(cuda):
    from meturay_b200._lib import lib
    rc = lib.mrb_radix_sort_pairs_u32_noalloc(None, None, MAX_PAIRS + 1, 0, 32, 0, None)
    assert rc == -1
    assert b"exceed" in lib.mrb_last_error()
