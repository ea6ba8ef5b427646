"""upf_radix_sort_pairs_noalloc: the radix sort for callers that cannot call
cudaMalloc (hosts that own all device memory through their own pool, and
per-frame loops that must not pay cudaMalloc's implicit synchronisation). It
takes its scratch from a fixed array inside the library instead of from the
caller.

Checked through the C ABI against upf_radix_sort_pairs (caller scratch) on
two calls in a row with different inputs; sorting is integer work, so the
outputs must be identical. This file is collected last so that a failure here
leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sort_with_scratch(upf, torch, keys, vals, bits):
    k = torch.from_numpy(keys).cuda()
    v = torch.from_numpy(vals).cuda()
    nbytes = upf.lib().upf_radix_sort_temp_bytes(keys.size)
    tmp = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    upf.check(upf.lib().upf_radix_sort_pairs(C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), keys.size, bits,
                                             C.c_void_p(tmp.data_ptr()), nbytes, None), "upf_radix_sort_pairs")
    torch.cuda.synchronize()
    return k.cpu().numpy(), v.cpu().numpy()


def _sort_noalloc(upf, torch, keys, vals, bits):
    k = torch.from_numpy(keys).cuda()
    v = torch.from_numpy(vals).cuda()
    upf.check(upf.lib().upf_radix_sort_pairs_noalloc(C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()),
                                                     keys.size, bits, None), "upf_radix_sort_pairs_noalloc")
    torch.cuda.synchronize()
    return k.cpu().numpy(), v.cpu().numpy()


def test_noalloc_sort_matches_scratch_sort_two_calls(upf_lib):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2024)
    # calls in a row: the second smaller and with other bits, so any stale
    # contents of the shared scratch would show up; the third at exactly the
    # maximum with full 32-bit keys, where the largest tiles run and the
    # alternate buffers and digit counts end at the end of the fixed array
    for n, bits in ((1_000_003, 30), (262_147, 24), (1 << 21, 32)):
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 10] = keys[0]  # many equal keys: stability matters
        vals = np.arange(n, dtype=np.uint32)
        ref_k, ref_v = _sort_with_scratch(upf_lib, torch, keys.view(np.int32), vals.view(np.int32), bits)
        got_k, got_v = _sort_noalloc(upf_lib, torch, keys.view(np.int32), vals.view(np.int32), bits)
        assert np.array_equal(got_k, ref_k)
        assert np.array_equal(got_v, ref_v)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(got_v.view(np.uint32), order.astype(np.uint32))


def test_noalloc_sort_rejects_oversize(upf_lib):
    lib = upf_lib.lib()
    n = (1 << 21) + 1
    # rejected before any device access, so dummy pointers are never touched
    st = lib.upf_radix_sort_pairs_noalloc(C.c_void_p(16), C.c_void_p(16), n, 30, None)
    assert st == 1
    assert "maximum" in lib.upf_last_error().decode()
