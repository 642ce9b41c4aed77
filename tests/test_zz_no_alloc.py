"""trlx_g_dot_noalloc, the allocation-free projection entry point.

Some callers cannot let a library call cudaMalloc: an application-wide
device-memory budget or caching allocator owns the GPU, or the call happens
inside an operator callback or other hot loop where an allocation could
synchronize the device.  This entry point takes its reduction scratch from a
fixed array compiled into the library.  The test calls it through the C ABI
twice in a row (the shared scratch keeps the previous call's contents) and
checks both results against the allocating trlx_g_dot, within the tolerance
of the other projection tests; it also checks the size limit.  This file is
collected last so that a failure here cannot hide the other tests."""
import numpy as np
import pytest

from nutrlan_b200 import load

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MAX_COLS = 512


def test_noalloc_matches_allocating_entry_point_twice():
    lib = load()
    rng = np.random.default_rng(31)
    cases = [(70001, 37, 5, 70001, 70004), (4096, 0, 9, 4096, 4099), (999, 300, 212, 1000, 999)]
    for n, m1, m2, ld1, ld2 in cases:
        v1 = torch.as_tensor(rng.standard_normal((max(m1, 1), ld1))).cuda()
        v2 = torch.as_tensor(rng.standard_normal((max(m2, 1), ld2))).cuda()
        rr = torch.as_tensor(rng.standard_normal(n)).cuda()
        want = torch.zeros(m1 + m2, dtype=torch.float64, device="cuda")
        assert lib.trlx_g_dot(n, v1.data_ptr(), ld1, m1, v2.data_ptr(), ld2, m2, rr.data_ptr(),
                              want.data_ptr(), None) == 0
        for _ in range(2):
            got = torch.full((m1 + m2,), float("nan"), dtype=torch.float64, device="cuda")
            assert lib.trlx_g_dot_noalloc(n, v1.data_ptr(), ld1, m1, v2.data_ptr(), ld2, m2,
                                          rr.data_ptr(), got.data_ptr(), None) == 0
            torch.cuda.synchronize()
            np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=0,
                                       atol=1e-13 * np.sqrt(n) * 4)


def test_noalloc_rejects_more_columns_than_its_scratch():
    lib = load()
    n = 64
    v = torch.zeros((MAX_COLS + 1) * n, dtype=torch.float64, device="cuda")
    r = torch.zeros(n, dtype=torch.float64, device="cuda")
    w = torch.zeros(MAX_COLS + 1, dtype=torch.float64, device="cuda")
    assert lib.trlx_g_dot_noalloc(n, v.data_ptr(), n, MAX_COLS + 1, v.data_ptr(), n, 0,
                                  r.data_ptr(), w.data_ptr(), None) == -7
    assert lib.trlx_g_dot_noalloc(n, v.data_ptr(), n, MAX_COLS, v.data_ptr(), n, 0,
                                  r.data_ptr(), w.data_ptr(), None) == 0
    torch.cuda.synchronize()


def test_noalloc_zero_rows_and_no_device_allocation():
    """A rank with no local rows gets zeros; after the per-device warm-up
    (the first call loads the library's fixed array), many calls leave the
    device's free memory unchanged.  The check is coarse: free memory moves
    in the driver's allocation granules, so it catches allocations that are
    kept (a leak, a growing pool), not one that is freed within the call."""
    lib = load()
    n, m = 1 << 20, 400
    v = torch.randn(m * n, dtype=torch.float64, device="cuda")
    r = torch.randn(n, dtype=torch.float64, device="cuda")
    w = torch.full((m,), 7.0, dtype=torch.float64, device="cuda")
    assert lib.trlx_g_dot_noalloc(0, v.data_ptr(), 0, 3, v.data_ptr(), 0, 2, r.data_ptr(), w.data_ptr(),
                                  None) == 0
    torch.cuda.synchronize()
    assert torch.all(w[:5] == 0.0)
    assert lib.trlx_g_dot_noalloc(n, v.data_ptr(), n, m, v.data_ptr(), n, 0, r.data_ptr(), w.data_ptr(),
                                  None) == 0          # warm-up on this device
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(50):
        assert lib.trlx_g_dot_noalloc(n, v.data_ptr(), n, m, v.data_ptr(), n, 0, r.data_ptr(),
                                      w.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
