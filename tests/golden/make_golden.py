"""Generates tests/golden/reference_vectors.npz from the reference's OWN host code
(oracle/_ref/libamxref_host.so, compiled from the reference tree by oracle/Makefile).

Run where the reference tree is present:  python tests/golden/make_golden.py
The vectors pin the C oracle (tests/test_golden.py) on machines without the reference:
  * element accessors get_element / get_elem_nogaps / get_element_baseline
    (src/common_code.cuh:43-55,100-116) on random words with every width 1..64;
  * the bitmask accessor (src/common_code.cuh:57-63);
  * FILTER_PREDICATE_OP (src/config.cuh:107-113);
  * op_add / op_mul / op_div / op_mod / op_math / op_bool_* (src/config.cuh:5-42) at every
    output width, and the op_*_outbits rules (src/config.cuh:44-55);
  * the PCG32 stream (src/fast_prng.cuh), the input arrays, the uniform mask and the
    cluster masks generated by the reference's main() (src/main.cu:33-108,242-284).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def main():
    O.build(with_reference=True)
    ref = O.ref_host()
    assert ref is not None, "oracle/_ref/libamxref_host.so was not built (is the reference tree present?)"
    rng = np.random.default_rng(20240521)
    out = {}
    words = rng.integers(0, 2**63, size=256, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=256,
                                                                                                dtype=np.uint64)
    out["words"] = words
    for name, fn, span in [("slab", ref.amxref_get_element, lambda b: (256 // 1) * (64 // b)),
                           ("nogaps", ref.amxref_get_elem_nogaps, lambda b: (255 * 64) // b),
                           ("plain64", ref.amxref_get_element_baseline, lambda b: 256)]:
        for b in range(1, 65):
            count = min(span(b), 160)
            idx = np.sort(rng.choice(span(b), size=count, replace=False)).astype(np.uint64)
            vals = np.array([fn(b, O._p(words), int(i)) for i in idx], dtype=np.uint64)
            out[f"{name}_{b}_idx"] = idx
            out[f"{name}_{b}_val"] = vals
    out["bitmask_val"] = np.array([ref.amxref_get_bitmask_element(O._p(words), i) for i in range(256 * 64)],
                                  dtype=np.uint8)
    pv = rng.integers(0, 2**63, size=64, dtype=np.uint64)
    out["pred_in"] = pv
    out["pred_half"] = np.array([[ref.amxref_filter_predicate(b, int(v) & ((1 << b) - 1)) for v in pv]
                                 for b in range(1, 65)], dtype=np.uint8)
    l = rng.integers(1, 2**40, size=48, dtype=np.uint64)
    r = rng.integers(1, 2**40, size=48, dtype=np.uint64)
    l[:8] = rng.integers(1, 300, size=8)
    r[:8] = rng.integers(1, 300, size=8)
    out["op_l"], out["op_r"] = l, r
    for op in (0, 2, 3, 4, 10, 11, 12):
        out[f"op_{op}"] = np.array([[ref.amxref_op(op, ob, int(a), int(b)) for a, b in zip(l, r)]
                                    for ob in range(1, 65)], dtype=np.uint64)
    out["outbits_add"] = np.array([ref.amxref_op_add_outbits(b) for b in range(1, 65)], dtype=np.int32)
    out["outbits_mul"] = np.array([ref.amxref_op_mul_outbits(b) for b in range(1, 65)], dtype=np.int32)
    out["outbits_mod"] = np.array([ref.amxref_op_mod_outbits(b) for b in range(1, 65)], dtype=np.int32)
    out["binary_op_outbits"] = np.array([ref.amxref_binary_op_outbits(b) for b in range(1, 65)], dtype=np.int32)
    out["binary_op_default"] = np.array([[ref.amxref_binary_op_default(b, int(a) & ((1 << b) - 1),
                                                                       int(c) & ((1 << b) - 1))
                                          for a, c in zip(l, r)] for b in range(1, 65)], dtype=np.uint64)
    prng = np.zeros(1000, dtype=np.uint32)
    ref.amxref_prng(42, O._p(prng), 1000)
    out["pcg32_seed42"] = prng
    n = 4096
    ok, d1, d2 = O.run_reference_main(["-n", str(n), "--nv", "-r", "1"], n)
    assert ok
    out["main_data1"], out["main_data2"] = d1, d2
    for sel in ("0.01", "0.1", "0.5", "0.9"):
        for dist in ("0", "1", "2"):
            ok, _, m = O.run_reference_main(["-n", str(n), "--nv", "-m", dist, "-s", sel], n)
            assert ok
            out[f"main_mask_{dist}_{sel}"] = m.view(np.uint8)[: n // 8].copy()
    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_vectors.npz"))


if __name__ == "__main__":
    main()
