"""Parity of the CUDA path with the CPU oracle, bit-exact, through the C ABI.

Integer work: every comparison is exact equality of the 16-word canonical
affine result (or of the 8-word field element)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import golden_cases, h2l, kat, random_field

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def M():
    from impeller_b200 import build
    build.build()
    from impeller_b200 import msm
    msm._lib.load()
    return msm


def dev(a):
    from impeller_b200.msm import to_device
    return to_device(np.ascontiguousarray(a, dtype=np.uint32))


def host(t):
    torch.cuda.synchronize()
    from impeller_b200.msm import to_host
    return to_host(t)


def field_op_gpu(M, field, op, a, b=None):
    L = M._lib.load()
    da = dev(a)
    db = dev(b) if b is not None else None
    out = torch.zeros_like(da)
    rc = L.impeller_test_field_op(field, op, da.data_ptr(), db.data_ptr() if db is not None else None,
                                  out.data_ptr(), a.shape[0], torch.cuda.current_stream().cuda_stream)
    M._lib.check(rc)
    return host(out).reshape(-1, 8)


def point_op_gpu(M, op, p, q=None):
    L = M._lib.load()
    dp = dev(p)
    dq = dev(q) if q is not None else None
    out = torch.zeros_like(dp)
    rc = L.impeller_test_point_op(op, dp.data_ptr(), dq.data_ptr() if dq is not None else None, out.data_ptr(),
                                  p.shape[0], torch.cuda.current_stream().cuda_stream)
    M._lib.check(rc)
    return host(out).reshape(-1, 16)


# ------------------------------------------------------------------ field

@pytest.mark.parametrize("field,modulus", [(O.FQ, O.P), (O.FR, O.R_MOD)])
def test_field_ops_match_oracle(M, field, modulus):
    rng = np.random.default_rng(11 + field)
    n = 2048
    a = random_field(rng, n, modulus)
    b = random_field(rng, n, modulus)
    # edge values: 0, 1, m-1, R mod m
    edges = [0, 1, modulus - 1, (1 << 256) % modulus, modulus - 2]
    for i, v in enumerate(edges):
        a[i] = O.int_to_limbs(v)
        b[-1 - i] = O.int_to_limbs(v)
    for op in (O.ADD, O.SUB, O.MUL, O.SQR, O.NEG, O.TO_MONT, O.FROM_MONT):
        want = O.field_op(field, op, a, b)
        got = field_op_gpu(M, field, op, a, b)
        assert (got == want).all(), (field, op)
    want = O.field_op(field, O.INV, a[:64])
    assert (field_op_gpu(M, field, O.INV, a[:64]) == want).all()
    assert (field_op_gpu(M, field, 9, a[:64]) == want).all()  # binary extended Euclid
    assert (field_op_gpu(M, field, 10, a[:64]) == want).all()  # Bernstein-Yang divsteps
    want = O.field_op(field, O.POW, a[:32], b[:32])
    assert (field_op_gpu(M, field, O.POW, a[:32], b[:32]) == want).all()


@pytest.mark.parametrize("ns", ["instance1", "instance2"])
def test_fr_kat_on_gpu(M, ns):
    d = {k: h2l(v) for k, v in kat()["fr"][ns].items()}
    a, b = d["a"][None], d["b"][None]
    assert (field_op_gpu(M, O.FR, O.ADD, a, b)[0] == d["sum_mont"]).all()
    assert (field_op_gpu(M, O.FR, O.SUB, a, b)[0] == d["sub_mont"]).all()
    assert (field_op_gpu(M, O.FR, O.MUL, a, b)[0] == d["prod_mont"]).all()
    am = field_op_gpu(M, O.FR, O.TO_MONT, a)
    assert (field_op_gpu(M, O.FR, O.SQR, am)[0] == d["a_square_mont"]).all()
    assert (field_op_gpu(M, O.FR, O.POW, am, b)[0] == d["pow_mont"]).all()
    assert (field_op_gpu(M, O.FR, O.INV, am)[0] == d["a_inv_mont"]).all()


# ------------------------------------------------------------------ curve

def _kat_pt(name):
    c = kat()["curve"]
    return np.concatenate([h2l(c[name + "_x"]), h2l(c[name + "_y"])])[None]


def test_curve_kat_on_gpu(M):
    p1, p2 = _kat_pt("p1"), _kat_pt("p2")
    assert (point_op_gpu(M, 0, p1, p2) == _kat_pt("pr")).all()       # madd path
    assert (point_op_gpu(M, 2, p1, p2) == _kat_pt("pr")).all()       # XYZZ + XYZZ
    p = p1
    for _ in range(7):
        p = point_op_gpu(M, 1, p)
    assert (p == _kat_pt("p1r128")).all()
    hundred = O.int_to_limbs(100)[None]
    p2x100 = point_op_gpu(M, 3, p2, hundred)
    assert (point_op_gpu(M, 0, p1, p2x100) == _kat_pt("pr100")).all()


def test_point_ops_special_cases(M):
    pts = O.gen_points(64, seed=9)
    neg = O.point_op(O.PT_NEG, pts)
    zero = np.zeros_like(pts)
    # P + Q, P + P (doubling inside madd), P + (-P), P + O, O + P
    for q, desc in ((np.roll(pts, 1, 0), "generic"), (pts, "double"), (neg, "inverse"), (zero, "identity-rhs")):
        want = O.point_op(O.PT_ADD, pts, q)
        assert (point_op_gpu(M, 0, pts, q) == want).all(), desc
        assert (point_op_gpu(M, 2, pts, q) == want).all(), desc
    assert (point_op_gpu(M, 0, zero, pts) == pts).all()
    assert (point_op_gpu(M, 1, pts) == O.point_op(O.PT_DBL, pts)).all()
    k = O.gen_scalars(64, seed=9, stream=3, mont=False)
    assert (point_op_gpu(M, 3, pts, k) == O.point_op(O.PT_SMUL, pts, k)).all()


# ------------------------------------------------------------- generators

def test_device_generators_match_oracle(M):
    n = 3000
    for dist in (O.DIST_UNIFORM, O.DIST_SKEWED):
        for mont in (True, False):
            got = host(M.gen_scalars_device(n, seed=5, stream_id=7, dist=dist, start=123, mont=mont))
            want = O.gen_scalars(n, seed=5, stream=7, dist=dist, start=123, mont=mont)
            assert (got == want).all(), (dist, mont)
    got = host(M.gen_points_device(1024, seed=0, start=77))
    assert (got == O.gen_points(1024, seed=0, start=77)).all()


# -------------------------------------------------------------------- MSM

def _ctx(M, points):
    return M.MsmContext(points)


def test_golden_msm_cases_on_gpu(M):
    for name, pts, sc, want in golden_cases():
        ctx = _ctx(M, pts)
        for c in (0, 4, 9):
            got = host(ctx.msm_device(dev(sc), c=c))
            assert (got == want).all(), (name, c)
        assert (ctx.msm_host(sc) == want).all(), name
        ctx.close()


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 64, 257, 1000, 4096, 65536])
def test_msm_sizes_match_oracle(M, n):
    pts = O.gen_points(n, seed=0)
    sc = O.gen_scalars(n, seed=0, stream=1)
    want = O.msm(pts, sc)
    ctx = _ctx(M, pts)
    got = host(ctx.msm_device(dev(sc)))
    assert (got == want).all()
    ctx.close()


@pytest.mark.parametrize("c", [3, 5, 8, 11, 13, 16, 18, 21])
def test_msm_window_sizes(M, c):
    n = 5000
    pts = O.gen_points(n, seed=2)
    sc = O.gen_scalars(n, seed=2, stream=4)
    want = O.msm(pts, sc)
    ctx = _ctx(M, pts)
    assert (host(ctx.msm_device(dev(sc), c=c)) == want).all()
    ctx.close()


def test_msm_edge_inputs(M):
    n = 4096
    pts = O.gen_points(n, seed=4)
    ctx = _ctx(M, pts)
    one = O.int_to_limbs(O.to_mont(1, O.R_MOD))
    rm1 = O.int_to_limbs(O.to_mont(O.R_MOD - 1, O.R_MOD))
    cases = {
        "all_zero": np.zeros((n, 8), np.uint32),
        "all_one": np.repeat(one[None], n, 0),
        "all_r_minus_1": np.repeat(rm1[None], n, 0),
        "skewed": O.gen_scalars(n, seed=4, stream=5, dist=O.DIST_SKEWED),
    }
    for name, sc in cases.items():
        assert (host(ctx.msm_device(dev(sc))) == O.msm(pts, sc)).all(), name
    ctx.close()
    # repeated points: every bucket accumulation hits the doubling case
    rep = np.repeat(pts[:1], n, 0)
    sc = np.repeat(O.gen_scalars(1, seed=4, stream=6), n, 0)
    ctx = _ctx(M, rep)
    assert (host(ctx.msm_device(dev(sc), c=8)) == O.msm(rep, sc)).all()
    ctx.close()
    # P and -P interleaved with equal scalars: sum is the identity
    pm = np.empty((n, 16), np.uint32)
    pm[0::2] = pts[: n // 2]
    pm[1::2] = O.point_op(O.PT_NEG, pts[: n // 2])
    sc = np.repeat(O.gen_scalars(n // 2, seed=4, stream=7), 2, 0)
    ctx = _ctx(M, pm)
    assert (host(ctx.msm_device(dev(sc))) == 0).all()
    ctx.close()
    # identity points mixed in
    idp = pts.copy()
    idp[::3] = 0
    sc = O.gen_scalars(n, seed=4, stream=8)
    ctx = _ctx(M, idp)
    assert (host(ctx.msm_device(dev(sc))) == O.msm(idp, sc)).all()
    ctx.close()


def test_msm_prefix_of_resident_points(M):
    n = 20000
    pts = O.gen_points(n, seed=6)
    ctx = _ctx(M, pts)
    for m in (1, 999, 12345, n):
        sc = O.gen_scalars(m, seed=6, stream=m)
        assert (host(ctx.msm_device(dev(sc), n=m)) == O.msm(pts[:m], sc)).all(), m
    ctx.close()


def test_msm_device_generated_srs(M):
    # device-generated points and scalars, oracle on the same bytes
    n = 1 << 18
    dpts = M.gen_points_device(n, seed=0)
    dsc = M.gen_scalars_device(n, seed=0, stream_id=1)
    pts, sc = host(dpts).reshape(n, 16), host(dsc).reshape(n, 8)
    assert (pts[:256] == O.gen_points(256, seed=0)).all()
    ctx = M.MsmContext(dpts)
    assert (host(ctx.msm_device(dsc)) == O.msm(pts, sc)).all()
    ctx.close()


# ---------------------------------------------------------- batched MSMs

@pytest.mark.parametrize("graph", [False, True])
def test_batch_uneven_sizes(M, graph):
    srs = 1 << 15
    pts = O.gen_points(srs, seed=8)
    ctx = _ctx(M, pts)
    rng = np.random.default_rng(3)
    sizes = [int(2 ** rng.uniform(4, 15)) for _ in range(12)] + [1, srs]
    b = ctx.batch(sizes, graph=graph)
    for rep in range(2):
        scal = [O.gen_scalars(s, seed=8, stream=100 * rep + i) for i, s in enumerate(sizes)]
        out = host(b.run([dev(s) for s in scal])).reshape(-1, 16)
        for i, s in enumerate(sizes):
            assert (out[i] == O.msm(pts[:s], scal[i])).all(), (rep, i, s)
    b.close()
    ctx.close()


# ------------------------------------------------ reference ABI: msm()

def test_reference_abi_msm_default_config(M):
    n = 3000
    pts = O.gen_points(n, seed=12)
    scal = [O.gen_scalars(n, seed=12, stream=s) for s in range(3)]
    cfg = M.MsmConfig(batch_per_run=2, parts=3)
    op = M.MSM(cfg)
    sizes = op.get_buffer_size(n)
    assert len(sizes) == 1 and sizes[0] > n * 64
    buf, keep = M.alloc_gpu_buffer(sizes[0])
    res = op.run([pts], scal, [buf])
    for s, r in zip(scal, res):
        assert (r == O.msm(pts, s)).all()
    del keep


def test_reference_abi_precompute_tables(M):
    # window 13, 4 bucket sets -> 20 digit windows over 5 window tables
    n = 2000
    cfg = M.MsmConfig(window_size=13, target_window=4)
    assert cfg.get_precompute() == 5
    pts = O.gen_points(n, seed=13)
    tables = [pts.copy()] + [np.zeros_like(pts) for _ in range(4)]
    M.MSMPrecompute(cfg).get_fn()(tables, n, 1)
    want_tabs = O.precompute(pts, shift=4 * 13, n_tables=5)
    for j in range(5):
        assert (tables[j] == want_tabs[j]).all(), j
    op = M.MSM(cfg)
    buf, keep = M.alloc_gpu_buffer(op.get_buffer_size(n)[0])
    scal = [O.gen_scalars(n, seed=13, stream=1)]
    res = op.run(tables, scal, [buf])
    assert (res[0] == O.msm(pts, scal[0])).all()
    del keep


def test_reference_abi_streamed_chunks(M):
    # parts of >= 2^21 points stream their upload in chunks; uneven chunk
    # sizes, two batch groups (the second with resident points), the oracle
    # on one output and the resident-SRS path on all
    n = (1 << 21) + 4321
    d = M.gen_points_device(n, seed=14)
    pts = M.to_host(d).reshape(n, 16)
    scal = [M.to_host(M.gen_scalars_device(n, seed=14, stream_id=s)).reshape(n, 8) for s in range(3)]
    ctx = M.MsmContext(d)
    want = [ctx.msm_host(sc) for sc in scal]
    assert (want[0] == O.msm(pts, scal[0])).all()
    op = M.MSM(M.MsmConfig(batch_per_run=2, parts=1))
    buf, keep = M.alloc_gpu_buffer(op.get_buffer_size(n)[0])
    for rep in range(2):
        res = op.run([pts], scal, [buf])
        for i in range(3):
            assert (res[i] == want[i]).all(), (rep, i)
    del keep
    # two streamed parts with the partial sum carried between them
    op2 = M.MSM(M.MsmConfig(batch_per_run=1, parts=2))
    buf2, keep2 = M.alloc_gpu_buffer(op2.get_buffer_size(n)[0])
    assert (op2.run([pts], scal[:1], [buf2])[0] == want[0]).all()
    del keep2
    ctx.close()


def test_reference_abi_streamed_with_tables(M):
    # window 16 with 8 bucket sets: two window tables, both streamed
    n = (1 << 21) + 99
    cfg = M.MsmConfig(window_size=16, target_window=8)
    assert cfg.get_precompute() == 2
    d = M.gen_points_device(n, seed=15)
    pts = M.to_host(d).reshape(n, 16)
    tables = [pts.copy(), np.zeros_like(pts)]
    M.MSMPrecompute(cfg).get_fn()(tables, n, 1)
    assert (tables[1][:512] == O.precompute(pts[:512], shift=8 * 16, n_tables=2)[1]).all()
    sc = M.to_host(M.gen_scalars_device(n, seed=15, stream_id=1)).reshape(n, 8)
    ctx = M.MsmContext(d)
    want = ctx.msm_host(sc)
    op = M.MSM(cfg)
    buf, keep = M.alloc_gpu_buffer(op.get_buffer_size(n)[0])
    assert (op.run(tables, [sc], [buf])[0] == want).all()
    del keep
    # 16 parts double-buffered in two stages, two batch groups
    cfg16 = M.MsmConfig(window_size=16, target_window=8, parts=16, batch_per_run=1, stage_scalars=2, stage_points=2)
    op16 = M.MSM(cfg16)
    buf16, keep16 = M.alloc_gpu_buffer(op16.get_buffer_size(n)[0])
    sc2 = M.to_host(M.gen_scalars_device(n, seed=15, stream_id=2)).reshape(n, 8)
    res = op16.run(tables, [sc, sc2], [buf16])
    assert (res[0] == want).all()
    assert (res[1] == ctx.msm_host(sc2)).all()
    del keep16
    ctx.close()


def test_reference_abi_rejects_bad_arguments(M):
    op = M.MSM(M.MsmConfig(parts=0))
    with pytest.raises(M._lib.ImpellerError):
        op.get_buffer_size(100)


def test_resident_window_tables(M):
    n = 20000
    pts = O.gen_points(n, seed=21)
    ctx = _ctx(M, pts)
    ctx.precompute(10)
    ctx.precompute(12)  # a second table set in the same allocation
    ctx.precompute(10)  # already resident: no-op
    for m, c in ((n, 10), (n, 12), (n, 0), (777, 10), (777, 12), (n, 7), (1, 10)):
        sc = O.gen_scalars(m, seed=21, stream=m + c)
        assert (host(ctx.msm_device(dev(sc), n=m, c=c)) == O.msm(pts[:m], sc)).all(), (m, c)
    sizes = [5, 300, 9000, n, 4000]
    b = ctx.batch(sizes, windows=[10, 0, 10, 0, 12], graph=True)
    scal = [O.gen_scalars(s, seed=21, stream=500 + i) for i, s in enumerate(sizes)]
    out = host(b.run([dev(s) for s in scal])).reshape(-1, 16)
    for i, s in enumerate(sizes):
        assert (out[i] == O.msm(pts[:s], scal[i])).all(), s
    b.close()
    ctx.close()


def test_resident_host_scalars_large(M):
    # impeller_msm_host above 2^21 points: the result equals the
    # device-scalar path's, plain and with a resident table set, and the
    # oracle's
    n = (1 << 21) + 12345
    d = M.gen_points_device(n, seed=16)
    ctx = M.MsmContext(d)
    dsc = M.gen_scalars_device(n, seed=16, stream_id=1)
    sc = M.to_host(dsc).reshape(n, 8)
    got = ctx.msm_host(sc)
    assert (got == host(ctx.msm_device(dsc))).all()
    assert (got == O.msm(M.to_host(d).reshape(n, 16), sc)).all()
    ctx.precompute(20)
    for s, dist in ((2, O.DIST_UNIFORM), (3, O.DIST_SKEWED)):
        dsc = M.gen_scalars_device(n, seed=16, stream_id=s, dist=dist)
        for c in (0, 20, 16):
            assert (ctx.msm_host(M.to_host(dsc).reshape(n, 8), c=c) == host(ctx.msm_device(dsc, c=c))).all(), (s, c)
    ctx.close()
