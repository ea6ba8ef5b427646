"""upf_radix_sort_pairs against numpy's stable argsort, on random keys with
many duplicates.

The sort picks its tile from the input size: 512 keys up to 262,144 keys,
2048 up to 1,048,576, 8192 above. The sizes below sit on both sides of each
switch. Key widths of 8, 16, 24 and 30 bits give one to four passes; an odd
count leaves the result in the scratch buffers, so it is copied back. The
bar is bit-exact: the same keys, and the values in stable order."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [1, 31, 513, 65_536, 262_144, 262_145, 1_048_576, 1_048_577, 3_000_001]


@pytest.mark.parametrize("n", SIZES)
def test_sort_matches_stable_argsort(upf_lib, n):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(n)
    for bits in (30, 24, 16, 8):
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        keys[rng.random(n) < 0.2] = keys[0]  # a fifth of the keys equal: stability matters
        vals = rng.permutation(n).astype(np.uint32)
        k = torch.from_numpy(keys.view(np.int32)).cuda()
        v = torch.from_numpy(vals.view(np.int32)).cuda()
        nbytes = upf_lib.lib().upf_radix_sort_temp_bytes(n)
        tmp = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
        upf_lib.check(upf_lib.lib().upf_radix_sort_pairs(C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), n,
                                                         bits, C.c_void_p(tmp.data_ptr()), nbytes, None),
                      "upf_radix_sort_pairs")
        torch.cuda.synchronize()
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(k.cpu().numpy().view(np.uint32), keys[order]), (n, bits)
        assert np.array_equal(v.cpu().numpy().view(np.uint32), vals[order]), (n, bits)

