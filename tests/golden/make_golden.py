"""Generate the golden fixtures in tests/golden/ from the reference's own CPU
code (src/cpu/zIndex.cpp, src/cpu/WeightingKernel.cpp,
src/sceneConfigure/UnifiedConstants.cpp), compiled by oracle/Makefile into
oracle/_ref/libupfref.so. Run in a checkout where the reference source tree
is available:

    make -C oracle ref REF=/path/to/reference
    python tests/golden/make_golden.py

The reference has no tests, fixtures or known-answer vectors of its own;
these files pin the oracle (and through it the device path) to the
reference's tables and constants.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from oracle import pyoracle  # noqa: E402

# support radii: the reference default (2.00002 * 1/40), the two benchmark
# scenes, and two arbitrary ones
H_VALUES = [np.float32(2.5e-2 * 2.0 * 1.00001), np.float32(0.04), np.float32(0.02), np.float32(0.0123),
            np.float32(0.0375)]


def fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def main():
    if not pyoracle.ref_available():
        raise SystemExit("oracle/_ref/libupfref.so missing: make -C oracle ref")
    R = pyoracle.ref()
    out = {}
    tab = np.zeros((1024, 3), np.uint32)
    R.ref_morton_table(tab.ctypes.data_as(C.POINTER(C.c_uint32)))
    out["morton_table"] = tab
    luts = np.zeros((len(H_VALUES), 5, 301), np.float32)
    for k, h in enumerate(H_VALUES):
        R.ref_luts(C.c_float(h), fp(luts[k]))
    out["lut_h"] = np.array(H_VALUES, np.float32)
    out["luts"] = luts
    # analytic kernels at sample distances for h = 0.02
    d = np.linspace(0.0, 0.021, 97).astype(np.float32)
    kv = np.zeros((d.size, 5), np.float32)
    for i, x in enumerate(d):
        R.ref_kernels(C.c_float(x), C.c_float(0.02), fp(kv[i]))
    out["kernel_dist"] = d
    out["kernel_values_h002"] = kv
    # BoxQuery ranges for seeded boxes and block sizes
    rng = np.random.default_rng(20240601)
    boxes, sizes, firsts, lasts, counts = [], [], [], [], []
    for bs in (4, 8, 16, 32, 64):
        for _ in range(40):
            lo = rng.integers(0, 1000, 3)
            ext = rng.integers(0, 3 * bs, 3)
            hi = np.minimum(lo + ext, 1023)
            a = lo.astype(np.uint16)
            b = hi.astype(np.uint16)
            f = np.zeros(4096, np.uint32)
            l = np.zeros(4096, np.uint32)
            n = R.ref_box_query(bs, a.ctypes.data_as(C.POINTER(C.c_uint16)), b.ctypes.data_as(C.POINTER(C.c_uint16)),
                                f.ctypes.data_as(C.POINTER(C.c_uint32)), l.ctypes.data_as(C.POINTER(C.c_uint32)), 4096)
            boxes.append(np.concatenate([a, b]))
            sizes.append(bs)
            counts.append(n)
            firsts.append(f[:n])
            lasts.append(l[:n])
    out["bq_boxes"] = np.array(boxes, np.uint16)
    out["bq_block"] = np.array(sizes, np.uint32)
    out["bq_count"] = np.array(counts, np.uint32)
    out["bq_first"] = np.concatenate(firsts)
    out["bq_last"] = np.concatenate(lasts)
    # ZIndex::SetBlockSize rounding
    sz = np.arange(0, 130, dtype=np.int32)
    out["block_size_in"] = sz
    out["block_size_out"] = np.array([R.ref_block_size(int(s)) for s in sz], np.uint32)
    # UnifiedConstants defaults
    cst = np.zeros(64, np.float32)
    R.ref_default_constants(fp(cst))
    out["default_constants"] = cst[:41]
    np.savez_compressed(os.path.join(HERE, "reference_tables.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_tables.npz"))


if __name__ == "__main__":
    main()
