"""BLS12-381 G1 on the CUDA path, bit-exact against the CPU oracle (and, where
it was built, the reference's own GPU MSM compiled for bls12381).

Same structure as the BN254 parity tests: field and point operations, the
device input generators, MSMs through the resident-SRS context at many sizes
and windows, the edge inputs, window tables, batched MSMs, and the
reference's msm() / msm_precompute() C ABI through the per-curve drop-in
library (lib/libmsm_bls12381_{c}_{alpha}_false.so).  Points are 24 u32
(x, y in 12-limb Montgomery form, R = 2^384), scalars 8 u32 (Montgomery Fr,
R = 2^256)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_gpu as RG

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

C = O.BLS12381
PW = 24
GOLD = os.path.join(os.path.dirname(__file__), "golden")


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


def rows(hexrows, width):
    return np.array([[int(r[8 * i:8 * i + 8], 16) for i in range(width)] for r in hexrows],
                    dtype=np.uint32).reshape(-1, width)


def field_op_gpu(M, field, op, a, b=None):
    L = M._lib.load()
    words = 12 if field == O.BLS_FQ else 8
    da = dev(a)
    db = dev(b) if b is not None else None
    out = torch.zeros_like(da)
    rc = L.impeller_test_field_op(field, op, da.data_ptr(), db.data_ptr() if db is not None else None,
                                  out.data_ptr(), a.shape[0], torch.cuda.current_stream().cuda_stream)
    M._lib.check(rc)
    return host(out).reshape(-1, words)


def point_op_gpu(M, op, p, q=None):
    L = M._lib.load()
    dp = dev(p)
    dq = dev(q) if q is not None else None
    out = torch.zeros_like(dp)
    rc = L.impeller_test_point_op_curve(C, op, dp.data_ptr(), dq.data_ptr() if dq is not None else None,
                                        out.data_ptr(), p.shape[0], torch.cuda.current_stream().cuda_stream)
    M._lib.check(rc)
    return host(out).reshape(-1, PW)


def random_elems(rng, n, modulus, words):
    return O.ints_to_array([int.from_bytes(rng.bytes(4 * words), "little") % modulus for _ in range(n)], words)


# ------------------------------------------------------------------ field

@pytest.mark.parametrize("field,modulus,words", [(O.BLS_FQ, O.P_BLS, 12), (O.BLS_FR, O.R_BLS, 8)])
def test_field_ops_match_oracle(M, field, modulus, words):
    rng = np.random.default_rng(31 + field)
    n = 2048
    a = random_elems(rng, n, modulus, words)
    b = random_elems(rng, n, modulus, words)
    mont_r = 1 << (32 * words)
    for i, v in enumerate([0, 1, modulus - 1, mont_r % modulus, modulus - 2]):
        a[i] = O.int_to_limbs(v, words)
        b[-1 - i] = O.int_to_limbs(v, words)
    for op in (O.ADD, O.SUB, O.MUL, O.SQR, O.NEG, O.TO_MONT, O.FROM_MONT):
        want = O.field_op(field, op, a, b)
        assert (field_op_gpu(M, field, op, a, b) == want).all(), (field, op)
    want = O.field_op(field, O.INV, a[:64])
    assert (field_op_gpu(M, field, O.INV, a[:64]) == want).all()
    assert (field_op_gpu(M, field, 9, a[:64]) == want).all()  # binary extended Euclid
    assert (field_op_gpu(M, field, 10, a[:64]) == want).all()  # Bernstein-Yang divsteps
    e = random_elems(rng, 32, modulus, words)
    want = O.field_op(field, O.POW, a[:32], e)
    assert (field_op_gpu(M, field, O.POW, a[:32], e) == want).all()


# ------------------------------------------------------------------ points

def test_point_ops_special_cases(M):
    pts = O.gen_points(64, seed=9, curve=C)
    neg = O.point_op(O.PT_NEG, pts, curve=C)
    zero = np.zeros_like(pts)
    for q, desc in ((np.roll(pts, 1, 0), "generic"), (pts, "double"), (neg, "inverse"), (zero, "identity-rhs")):
        want = O.point_op(O.PT_ADD, pts, q, curve=C)
        assert (point_op_gpu(M, 0, pts, q) == want).all(), desc
        assert (point_op_gpu(M, 2, pts, q) == want).all(), desc
    assert (point_op_gpu(M, 0, zero, pts) == pts).all()
    assert (point_op_gpu(M, 1, pts) == O.point_op(O.PT_DBL, pts, curve=C)).all()
    k = O.gen_scalars(64, seed=9, stream=3, mont=False, curve=C)
    assert (point_op_gpu(M, 3, pts, k) == O.point_op(O.PT_SMUL, pts, k, curve=C)).all()
    # r * P = identity
    kr = np.repeat(O.int_to_limbs(O.R_BLS)[None], 64, 0)
    assert not point_op_gpu(M, 3, pts, kr).any()


def test_device_generators_match_oracle(M):
    n = 3000
    for dist in (O.DIST_UNIFORM, O.DIST_SKEWED):
        for mont in (True, False):
            got = host(M.gen_scalars_device(n, seed=5, stream_id=7, dist=dist, start=123, mont=mont, curve=C))
            want = O.gen_scalars(n, seed=5, stream=7, dist=dist, start=123, mont=mont, curve=C)
            assert (got.reshape(n, 8) == want).all(), (dist, mont)
    got = host(M.gen_points_device(512, seed=0, start=77, curve=C)).reshape(512, PW)
    assert (got == O.gen_points(512, seed=0, start=77, curve=C)).all()


# -------------------------------------------------------------------- MSM

def _ctx(M, points):
    return M.MsmContext(points, curve=C)


def test_golden_msm_cases_on_gpu(M):
    gold = json.load(open(os.path.join(GOLD, "msm_golden_bls12381.json")))
    for case in gold["cases"]:
        pts = rows(case["points"], PW)
        sc = rows(case["scalars"], 8)
        want = rows([case["result"]], PW)[0]
        ctx = _ctx(M, pts)
        for c in (0, 4, 9):
            got = host(ctx.msm_device(dev(sc), c=c))
            assert (got == want).all(), (case["name"], c)
        assert (ctx.msm_host(sc) == want).all(), case["name"]
        ctx.close()


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 64, 257, 1000, 4096, 65536])
def test_msm_sizes_match_oracle(M, n):
    pts = O.gen_points(n, seed=0, curve=C)
    sc = O.gen_scalars(n, seed=0, stream=1, curve=C)
    want = O.msm(pts, sc, curve=C)
    ctx = _ctx(M, pts)
    assert (host(ctx.msm_device(dev(sc))) == want).all()
    ctx.close()


@pytest.mark.parametrize("c", [3, 5, 8, 11, 13, 15, 16, 17, 18, 21])
def test_msm_window_sizes(M, c):
    # c = 3, 5, 15, 17 need one more signed-digit window than ceil(255 / c)
    n = 5000
    pts = O.gen_points(n, seed=2, curve=C)
    sc = O.gen_scalars(n, seed=2, stream=4, curve=C)
    # top-of-range scalars exercise the carry out of the last window
    sc[:64] = O.ints_to_array([O.to_mont(O.R_BLS - 1 - i, O.R_BLS) for i in range(64)])
    want = O.msm(pts, sc, curve=C)
    ctx = _ctx(M, pts)
    assert (host(ctx.msm_device(dev(sc), c=c)) == want).all()
    ctx.close()


def test_msm_edge_inputs(M):
    n = 4096
    pts = O.gen_points(n, seed=4, curve=C)
    ctx = _ctx(M, pts)
    one = O.int_to_limbs(O.to_mont(1, O.R_BLS))
    rm1 = O.int_to_limbs(O.to_mont(O.R_BLS - 1, O.R_BLS))
    cases = {
        "all_zero": np.zeros((n, 8), np.uint32),
        "all_one": np.repeat(one[None], n, 0),
        "all_r_minus_1": np.repeat(rm1[None], n, 0),
        "skewed": O.gen_scalars(n, seed=4, stream=5, dist=O.DIST_SKEWED, curve=C),
    }
    for name, sc in cases.items():
        assert (host(ctx.msm_device(dev(sc))) == O.msm(pts, sc, curve=C)).all(), name
    ctx.close()
    rep = np.repeat(pts[:1], n, 0)
    sc = np.repeat(O.gen_scalars(1, seed=4, stream=6, curve=C), n, 0)
    ctx = _ctx(M, rep)
    assert (host(ctx.msm_device(dev(sc), c=8)) == O.msm(rep, sc, curve=C)).all()
    ctx.close()
    pm = np.empty((n, PW), np.uint32)
    pm[0::2] = pts[: n // 2]
    pm[1::2] = O.point_op(O.PT_NEG, pts[: n // 2], curve=C)
    sc = np.repeat(O.gen_scalars(n // 2, seed=4, stream=7, curve=C), 2, 0)
    ctx = _ctx(M, pm)
    assert (host(ctx.msm_device(dev(sc))) == 0).all()
    ctx.close()
    idp = pts.copy()
    idp[::3] = 0
    sc = O.gen_scalars(n, seed=4, stream=8, curve=C)
    ctx = _ctx(M, idp)
    assert (host(ctx.msm_device(dev(sc))) == O.msm(idp, sc, curve=C)).all()
    ctx.close()


def test_msm_prefix_and_device_srs(M):
    n = 1 << 16
    dpts = M.gen_points_device(n, seed=0, curve=C)
    dsc = M.gen_scalars_device(n, seed=0, stream_id=1, curve=C)
    pts, sc = host(dpts).reshape(n, PW), host(dsc).reshape(n, 8)
    assert (pts[:128] == O.gen_points(128, seed=0, curve=C)).all()
    ctx = M.MsmContext(dpts, curve=C)
    assert (host(ctx.msm_device(dsc)) == O.msm(pts, sc, curve=C)).all()
    for m in (1, 999, 12345):
        s = O.gen_scalars(m, seed=6, stream=m, curve=C)
        assert (host(ctx.msm_device(dev(s), n=m)) == O.msm(pts[:m], s, curve=C)).all(), m
    ctx.close()


def test_resident_window_tables_and_batch(M):
    n = 20000
    pts = O.gen_points(n, seed=21, curve=C)
    ctx = _ctx(M, pts)
    ctx.precompute(10)
    ctx.precompute(13)
    for m, c in ((n, 10), (n, 13), (n, 0), (777, 10), (777, 13), (n, 7), (1, 10)):
        sc = O.gen_scalars(m, seed=21, stream=m + c, curve=C)
        assert (host(ctx.msm_device(dev(sc), n=m, c=c)) == O.msm(pts[:m], sc, curve=C)).all(), (m, c)
    sizes = [5, 300, 9000, n, 4000]
    for graph in (False, True):
        b = ctx.batch(sizes, windows=[10, 0, 10, 0, 13], graph=graph)
        for rep in range(2):
            scal = [O.gen_scalars(s, seed=21, stream=500 + 10 * rep + i, curve=C) for i, s in enumerate(sizes)]
            out = host(b.run([dev(s) for s in scal])).reshape(-1, PW)
            for i, s in enumerate(sizes):
                assert (out[i] == O.msm(pts[:s], scal[i], curve=C)).all(), (graph, rep, s)
        b.close()
    ctx.close()


def test_server_jobs(M):
    n = 8192
    pts = O.gen_points(n, seed=22, curve=C)
    ctx = _ctx(M, pts)
    srv = M.MsmServer(ctx, max_batch=8, max_inflight=2)
    sizes = [n, 100, 4096, 1, 3000, n]
    scal = [O.gen_scalars(s, seed=22, stream=i, curve=C) for i, s in enumerate(sizes)]
    jobs = [srv.submit(s) for s in scal]
    for j, s, sc in zip(jobs, sizes, scal):
        out, _ = srv.wait(j)
        assert out.shape == (PW,)
        assert (out == O.msm(pts[:s], sc, curve=C)).all(), s
    srv.close()
    ctx.close()


# ------------------------------------------------ reference ABI: msm()

def test_reference_abi_msm_default_config(M):
    n = 3000
    pts = O.gen_points(n, seed=12, curve=C)
    scal = [O.gen_scalars(n, seed=12, stream=s, curve=C) for s in range(3)]
    cfg = M.MsmConfig(batch_per_run=2, parts=3, curve=C)
    assert cfg.bits == 255 and M.lib_name(cfg) == "msm_bls12381_16_16_false"
    op = M.MSM(cfg)
    sizes = op.get_buffer_size(n)
    assert len(sizes) == 1 and sizes[0] > n * 96
    buf, keep = M.alloc_gpu_buffer(sizes[0])
    res = op.run([pts], scal, [buf])
    for s, r in zip(scal, res):
        assert r.shape == (PW,)
        assert (r == O.msm(pts, s, curve=C)).all()
    del keep


def test_reference_abi_precompute_tables(M):
    # window 13, 4 bucket sets -> 20 digit windows over 5 window tables
    n = 2000
    cfg = M.MsmConfig(window_size=13, target_window=4, curve=C)
    assert cfg.get_precompute() == 5 == M.n_precompute(13, 4, curve=C)
    pts = O.gen_points(n, seed=13, curve=C)
    tables = [pts.copy()] + [np.zeros_like(pts) for _ in range(4)]
    M.MSMPrecompute(cfg).get_fn()(tables, n, 1)
    want_tabs = O.precompute(pts, shift=4 * 13, n_tables=5, curve=C)
    for j in range(5):
        assert (tables[j] == want_tabs[j]).all(), j
    op = M.MSM(cfg)
    buf, keep = M.alloc_gpu_buffer(op.get_buffer_size(n)[0])
    scal = [O.gen_scalars(n, seed=13, stream=1, curve=C)]
    assert (op.run(tables, scal, [buf])[0] == O.msm(pts, scal[0], curve=C)).all()
    del keep


def test_reference_abi_streamed_parts(M):
    # parts of >= 2^21 points stream their upload in chunks; 4 parts in two
    # stages with the partial sum carried between them
    n = (1 << 21) + 777
    d = M.gen_points_device(n, seed=14, curve=C)
    pts = M.to_host(d).reshape(n, PW)
    sc = M.to_host(M.gen_scalars_device(n, seed=14, stream_id=1, curve=C)).reshape(n, 8)
    ctx = M.MsmContext(d, curve=C)
    want = ctx.msm_host(sc)
    op = M.MSM(M.MsmConfig(batch_per_run=1, parts=1, curve=C))
    buf, keep = M.alloc_gpu_buffer(op.get_buffer_size(n)[0])
    assert (op.run([pts], [sc], [buf])[0] == want).all()
    del keep
    op4 = M.MSM(M.MsmConfig(batch_per_run=1, parts=4, stage_scalars=2, stage_points=2, curve=C))
    buf4, keep4 = M.alloc_gpu_buffer(op4.get_buffer_size(n)[0])
    assert (op4.run([pts], [sc], [buf4])[0] == want).all()
    del keep4
    ctx.close()
    assert (want == O.msm(pts, sc, curve=C)).all()


def test_reference_abi_rejects_incompatible_window(M):
    # c = 17 on 255-bit scalars needs 16 signed-digit windows; the reference
    # lays out ceil(255 / 17) = 15, so a 15-table layout cannot be served
    cfg = M.MsmConfig(window_size=17, target_window=5, curve=C)
    with pytest.raises(M._lib.ImpellerError):
        M.MSM(cfg).get_buffer_size(100)


# ------------------------------------- the reference's own GPU MSM (bls12381)

@pytest.mark.skipif(not RG.available(16, 16, curve=RG.BLS12381), reason="reference GPU MSM for bls12381 not built")
def test_reference_gpu_bls12381_default_config(M):
    n = 1 << 14
    d = M.gen_points_device(n, seed=33, curve=C)
    h = M.to_host(d).reshape(n, PW)
    ctx = M.MsmContext(d, curve=C)
    ref = RG.RefGpuMsm(h, 16, 16, curve=RG.BLS12381)
    for stream in (1, 2):
        sc = O.gen_scalars(n, seed=33, stream=stream, curve=C)
        want = O.msm(h, sc, curve=C)
        assert (ctx.msm_host(sc) == want).all()
        assert (ref.msm(sc) == want).all()
    ref.close()
    ctx.close()


@pytest.mark.skipif(not RG.available(16, 8, curve=RG.BLS12381), reason="reference GPU MSM (16, 8) for bls12381 not built")
def test_reference_gpu_bls12381_tables_config(M):
    # window 16 with 8 bucket sets: 16 signed-digit windows over two window tables
    n = 1 << 17
    d = M.gen_points_device(n, seed=34, curve=C)
    h = M.to_host(d).reshape(n, PW)
    ref = RG.RefGpuMsm(h, 16, 8, curve=RG.BLS12381)
    assert ref.k == 2
    tabs = ref.tables()
    assert (tabs[:, :256] == O.precompute(h[:256], shift=16 * 8, n_tables=2, curve=C)).all()
    # this library's drop-in in the same configuration, on the reference's tables
    op = M.MSM(M.MsmConfig(window_size=16, target_window=8, curve=C))
    buf, keep = M.alloc_gpu_buffer(op.get_buffer_size(n)[0])
    for stream, dist in ((1, O.DIST_UNIFORM), (2, O.DIST_SKEWED)):
        sc = O.gen_scalars(n, seed=34, stream=stream, dist=dist, curve=C)
        want = O.msm(h, sc, curve=C)
        assert (ref.msm(sc) == want).all(), dist
        assert (op.run([tabs[0], tabs[1]], [sc], [buf])[0] == want).all(), dist
    del keep
    ref.close()
