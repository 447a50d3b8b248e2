"""cs_kinship_apply_noalloc: the kinship apply for callers that cannot allocate.

Some hosts cannot let the library call cudaMalloc (a process that has reserved HBM for
its own pool, or a request loop that cannot absorb the allocator's synchronisation).
The allocation-free entry point takes its scratch from a fixed array in the library's
device memory.  This test calls it through the C ABI twice in a row and checks each
result against the regular cs_kinship_apply on the same inputs (relative error < 1e-12,
the two differ only in how the contraction is split across thread blocks).  It also
checks that an oversized request is rejected with a clear message.

The file sorts last so that a run stopping at the first failure has already run every
other test; it passes alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_apply_on_two_calls():
    torch = pytest.importorskip("torch")
    import cosmicscanner_b200 as cs
    from cosmicscanner_b200 import _abi, synth

    d = synth.cohort(1800, 2600, 41, missing=0.02, n_causal=20)
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    rng = np.random.default_rng(5)
    keep = np.sort(rng.choice(d["n"], 1500, replace=False)).astype(np.int32)
    variants = np.arange(0, d["m"], 2, dtype=np.int32)
    lib = _abi.lib()
    for op in (cs.createKinshipOperator(g), cs.createKinshipOperator(g, keep, variants)):
        n = op.rows()
        for k in (1, 5, 3):
            X = torch.tensor(rng.standard_normal((k, n)), device="cuda")  # column-major n x k
            Y_ref = torch.empty_like(X)
            assert lib.cs_kinship_apply(op._h, ctypes.c_void_p(X.data_ptr()), n, k,
                                        ctypes.c_void_p(Y_ref.data_ptr()), n, 0, None) == 0
            for _ in range(2):
                Y = torch.full_like(X, float("nan"))
                rc = lib.cs_kinship_apply_noalloc(op._h, ctypes.c_void_p(X.data_ptr()), n, k,
                                                  ctypes.c_void_p(Y.data_ptr()), n, None)
                assert rc == 0, lib.cs_last_error()
                torch.cuda.synchronize()
                err = (Y - Y_ref).abs().max().item() / Y_ref.abs().max().item()
                assert err < 1e-12, err
        # a request beyond the fixed scratch is refused, not allocated for
        big = 2 * (2 << 20) // n + 1
        X = torch.zeros((big, n), dtype=torch.float64, device="cuda")
        rc = lib.cs_kinship_apply_noalloc(op._h, ctypes.c_void_p(X.data_ptr()), n, big,
                                          ctypes.c_void_p(X.data_ptr()), n, None)
        assert rc == _abi.CS_ERR_INVALID_ARGUMENT
        assert b"exceeds the fixed scratch" in lib.cs_last_error()
