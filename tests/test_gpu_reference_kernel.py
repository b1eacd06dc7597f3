"""Parity against the reference's own GPU MSM.

The reference's core/src/msm/src/msm.cu, compiled unmodified for sm_100a
(oracle/Makefile, target ref_gpu), runs through its C ABI on the same seeded
inputs as this library; every result must be bit-identical to this library's
and, where the CPU oracle finishes in seconds, to the oracle's.  Configurations:
MsmConfig::default() (window 16, target window 16, no tables) and the
reference cost model's choice for 2^22 (window 17, target window 8, two
tables, 16 parts).  The reference's precomputed tables are also checked
against the oracle's.  Skipped where the reference library was not built
(the reference sources were absent at build time)."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_gpu as RG

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

if not (RG.available(*RG.DEFAULT_CONFIG) and RG.available(*RG.TUNED_2E22_CONFIG)):
    pytest.skip("reference GPU MSM libraries not built", allow_module_level=True)


@pytest.fixture(scope="module")
def M():
    from impeller_b200 import build
    build.build()
    from impeller_b200 import msm
    msm._lib.load()
    return msm


def _srs(M, n, seed):
    d = M.gen_points_device(n, seed=seed)
    return d, M.to_host(d).reshape(n, 16)


def test_reference_gpu_default_config_2e16(M):
    n = 1 << 16
    d, h = _srs(M, n, seed=31)
    ref = RG.RefGpuMsm(h, *RG.DEFAULT_CONFIG)
    ctx = M.MsmContext(d)
    for stream in (1, 2):
        sc = O.gen_scalars(n, seed=31, stream=stream)
        want = O.msm(h, sc)
        assert (ref.msm(sc) == want).all()
        assert (ctx.msm_host(sc) == want).all()
    ctx.close()
    ref.close()


def test_reference_gpu_tuned_config_tables_and_skew_2e20(M):
    n = 1 << 20
    d, h = _srs(M, n, seed=32)
    c, alpha = RG.TUNED_2E22_CONFIG
    ref = RG.RefGpuMsm(h, c, alpha, parts=RG.TUNED_2E22_PARTS)
    assert ref.k == 2
    tabs = ref.tables()
    want_tabs = O.precompute(h[:2048], shift=c * alpha, n_tables=2)
    assert (tabs[:, :2048] == want_tabs).all()
    assert (tabs[1, -2048:] == O.precompute(h[-2048:], shift=c * alpha, n_tables=2)[1]).all()
    ctx = M.MsmContext(d)
    ctx.precompute(M.table_window(n) or 20)
    for dist in (O.DIST_UNIFORM, O.DIST_SKEWED):
        sc = O.gen_scalars(n, seed=32, stream=3 + dist, dist=dist)
        want = O.msm(h, sc)
        assert (ref.msm(sc) == want).all(), dist
        assert (ctx.msm_host(sc) == want).all(), dist
    ctx.close()
    ref.close()


def test_reference_gpu_full_size_2e22_both_configs(M):
    n = 1 << 22
    d, h = _srs(M, n, seed=0)
    dsc = M.gen_scalars_device(n, seed=0, stream_id=1)
    sc = M.to_host(dsc).reshape(n, 8)
    ctx = M.MsmContext(d)
    ctx.precompute(M.table_window(n) or 20)
    ours = M.to_host(ctx.msm_device(dsc)).reshape(16)
    torch.cuda.synchronize()
    for (c, alpha), parts in ((RG.DEFAULT_CONFIG, 1), (RG.TUNED_2E22_CONFIG, RG.TUNED_2E22_PARTS)):
        ref = RG.RefGpuMsm(h, c, alpha, parts=parts)
        assert (ref.msm(sc) == ours).all(), (c, alpha)
        ref.close()
    ctx.close()
