"""Parity at the benchmark configurations' full sizes (seeded synthetic inputs
with the shapes of the reference's workload):

  C2  plain single MSM, n = 2^22, uniform Fr scalars -- with resident window
      tables (the benchmarked path) and with plain windows
  C3  skewed scalars, n = 2^20 (40% zeros and ones, 30% below 2^16)
  C4  64 batched MSMs, n log-uniform in [2^10, 2^20], prefixes of one SRS

every output bit-exact against the CPU oracle, plus the size-independent
properties MSM(s1 + s2) = MSM(s1) + MSM(s2) and MSM(k * s) = k * MSM(s) at
2^22.  Device-generated inputs are checked against the oracle's generator on
a prefix before the oracle consumes them."""
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


@pytest.fixture(scope="module")
def srs22(M):
    d = M.gen_points_device(1 << 22, seed=0)
    h = M.to_host(d).reshape(-1, 16)
    assert (h[:512] == O.gen_points(512, seed=0)).all()
    return d, h


def test_c2_full_size_tables_and_plain(M, srs22):
    d, h = srs22
    n = 1 << 22
    dsc = M.gen_scalars_device(n, seed=0, stream_id=1)
    sc = M.to_host(dsc).reshape(n, 8)
    assert (sc[:256] == O.gen_scalars(256, seed=0, stream=1)).all()
    want = O.msm(h, sc)
    ctx = M.MsmContext(d)
    plain = M.to_host(ctx.msm_device(dsc, c=16))
    ctx.precompute(20)
    tables = M.to_host(ctx.msm_device(dsc, c=20))
    torch.cuda.synchronize()
    assert (plain == want).all()
    assert (tables == want).all()
    ctx.close()


def test_c2_linearity_properties(M, srs22):
    d, h = srs22
    n = 1 << 22
    ctx = M.MsmContext(d)
    ctx.precompute(20)
    s1 = O.gen_scalars(n, seed=9, stream=1)
    s2 = O.gen_scalars(n, seed=9, stream=2)
    s12 = O.field_op(O.FR, O.ADD, s1, s2)
    k = O.gen_scalars(1, seed=9, stream=3)  # Montgomery form
    ks = O.field_op(O.FR, O.MUL, s1, np.repeat(k, n, 0))
    m1, m2, m12, mk = (ctx.msm_host(x) for x in (s1, s2, s12, ks))
    assert (O.point_op(O.PT_ADD, m1, m2)[0] == m12).all()
    k_plain = O.field_op(O.FR, O.FROM_MONT, k)
    assert (O.point_op(O.PT_SMUL, m1, k_plain)[0] == mk).all()
    ctx.close()


def test_c3_skewed_full_size(M):
    n = 1 << 20
    dp = M.gen_points_device(n, seed=0)
    dsc = M.gen_scalars_device(n, seed=0, stream_id=3, dist=1)
    h, sc = M.to_host(dp).reshape(n, 16), M.to_host(dsc).reshape(n, 8)
    assert (sc[:256] == O.gen_scalars(256, seed=0, stream=3, dist=O.DIST_SKEWED)).all()
    want = O.msm(h, sc)
    ctx = M.MsmContext(dp)
    assert (M.to_host(ctx.msm_device(dsc)) == want).all()
    ctx.precompute(M.table_window(n) or 20)
    assert (M.to_host(ctx.msm_device(dsc)) == want).all()
    ctx.close()


def test_many_heavy_buckets(M):
    """2^20 scalars taking 200 small values: 200 buckets of window 0 each cut
    into more than 256 slices, more heavy buckets than the fixup has blocks
    (so a block merges several, one after another), with plain windows and
    with window 8."""
    n = 1 << 20
    dp = M.gen_points_device(n, seed=5)
    h = M.to_host(dp).reshape(n, 16)
    vals = np.stack([O.int_to_limbs(O.to_mont(v, O.R_MOD)) for v in range(1, 201)])
    sc = vals[np.arange(n) % 200]
    want = O.msm(h, sc)
    ctx = M.MsmContext(dp)
    dsc = M.to_device(sc)
    for c in (0, 8):
        assert (M.to_host(ctx.msm_device(dsc, c=c)) == want).all(), c
    ctx.close()


def test_c4_batched_every_output(M):
    n = 1 << 20
    dp = M.gen_points_device(n, seed=0)
    h = M.to_host(dp).reshape(n, 16)
    ctx = M.MsmContext(dp)
    rng = np.random.default_rng(0)
    sizes = [int(round(2 ** rng.uniform(10, 20))) for _ in range(64)]
    for ct in sorted({M.table_window(s) for s in sizes} - {0}):
        ctx.precompute(ct)
    scal = [M.gen_scalars_device(s, seed=0, stream_id=1000 + i) for i, s in enumerate(sizes)]
    b = ctx.batch(sizes, graph=True)
    out = M.to_host(b.run(scal)).reshape(64, 16)
    b.close()
    for i, s in enumerate(sizes):
        want = O.msm(h[:s], M.to_host(scal[i]).reshape(s, 8))
        assert (out[i] == want).all(), (i, s)
    ctx.close()
