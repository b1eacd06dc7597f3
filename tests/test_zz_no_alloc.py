"""The allocation-free MSM entry point against the existing one.

impeller_msm_device_noalloc serves callers that cannot call cudaMalloc when
they need an MSM (device memory planned ahead of time into a fixed arena,
paths where an allocation would synchronize the device).  Its scratch is a
static device array, so this test checks, through the C ABI, that two calls
in a row give exactly the result of impeller_msm_device and of the CPU
oracle (bit-exact: integer work, tolerance zero), that an empty MSM gives
the identity, and that sizes beyond the array are refused.  This file is
collected last so that a stop-at-first-failure run has already run every
other test when it gets here; it also passes alone."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def M():
    from impeller_b200 import build
    build.build()
    from impeller_b200 import msm
    msm._lib.load()
    return msm


def test_noalloc_matches_allocating_entry_point_twice(M):
    L = M._lib.load()
    n = 1 << 14
    pts = M.gen_points_device(n, seed=3)
    ctx = M.MsmContext(pts)
    stream = torch.cuda.current_stream().cuda_stream
    for call, (m, sid) in enumerate(((n, 41), (5000, 42))):
        sc = M.gen_scalars_device(m, seed=3, stream_id=sid)
        want = ctx.msm_device(sc, n=m)
        got = torch.full((16,), -1, dtype=torch.int32, device="cuda")
        M._lib.check(L.impeller_msm_device_noalloc(pts.data_ptr(), sc.data_ptr(), m, got.data_ptr(), stream),
                     "impeller_msm_device_noalloc")
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}: n={m}"
        if m == 5000:
            pts_h = M.to_host(pts).reshape(n, 16)[:m]
            assert (M.to_host(got) == O.msm(pts_h, M.to_host(sc).reshape(m, 8))).all(), "oracle"
    ctx.close()


def test_noalloc_empty_msm_is_identity(M):
    L = M._lib.load()
    out = torch.full((16,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    M._lib.check(L.impeller_msm_device_noalloc(None, None, 0, out.data_ptr(), stream), "impeller_msm_device_noalloc")
    torch.cuda.synchronize()
    assert (M.to_host(out) == 0).all()


def test_noalloc_rejects_oversize(M):
    L = M._lib.load()
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    dummy = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = L.impeller_msm_device_noalloc(dummy.data_ptr(), dummy.data_ptr(), (1 << 14) + 1, out.data_ptr(), None)
    assert rc != 0
    assert b"IMPELLER_NOALLOC_MAX_N" in L.impeller_last_error()
