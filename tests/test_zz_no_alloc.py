"""The dot product that allocates nothing (hyb_function_dot_noalloc).

It exists for callers that cannot allocate device memory while they run, e.g. a
serving loop that admitted its work against a fixed HBM budget, or a host framework
that owns the device allocator. Its scratch is a file-scope device array instead of a
library allocation; the caller passes the two functions and a device pointer for the
result. This test calls it through the C ABI and checks it against the allocating
entry point (hyb_function_dot) on two calls in a row, so the second call also shows
that the array's leftover contents from the first call do not leak into the result.

The file is named to be collected last: if it fails, a run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dot_noalloc_matches_allocating_dot():
    import torch

    import hyb_inputs as I
    import hyteg_b200 as H

    lib = H.load()
    L = 5
    st = H.PrimitiveStorage.cuboid(2, 2, 2, L)
    a, b = H.P1Function("a", st, 0, L), H.P1Function("b", st, 0, L)
    rng = np.random.default_rng(11)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for call, (level, flag) in enumerate([(L, H.INNER | H.NEUMANN), (L - 1, H.ALL)]):
        a.set(rng.uniform(-1, 1, st.num_dofs(level)), level)
        b.set(rng.uniform(-1, 1, st.num_dofs(level)), level)
        # a different vector per call: the shared scratch still holds the previous call's partials
        code = lib.hyb_function_dot_noalloc(a.h, b.h, level, flag, ctypes.c_void_p(out.data_ptr() + 8 * call),
                                            ctypes.c_void_p(stream.cuda_stream))
        assert code == 0, lib.hyb_last_error().decode()
        torch.cuda.synchronize()
        expected = a.dot_global(b, level, flag)
        got = float(out[call].item())
        assert abs(got - expected) <= 1e-12 * max(1.0, abs(expected)), (call, got, expected)


def test_dot_noalloc_rejects_oversized_problems():
    import torch

    import hyteg_b200 as H

    lib = H.load()
    # level 7 on 96 macro-cells needs 1431 x 96 partial sums, more than the 131072 slots
    st = H.PrimitiveStorage.cuboid(4, 4, 1, 7)
    a = H.P1Function("a", st, 7, 7)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    code = lib.hyb_function_dot_noalloc(a.h, a.h, 7, H.ALL, ctypes.c_void_p(out.data_ptr()), None)
    assert code == 1  # HYB_EINVAL
    assert "too large" in lib.hyb_last_error().decode()
