"""The NTT operator on the GPU, bit-exact against the CPU oracle and the
reference's own NTT kernels (core/src/ntt/src/ntt.cu built for sm_100a,
oracle/_ref/libref_ntt_bn254_fr.so), through the reference-named C ABI.

Integer work: every comparison is exact equality of canonical Montgomery
limbs."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

REF_NTT = os.path.join(os.path.dirname(O.__file__), "_ref", "libref_ntt_bn254_fr.so")


@pytest.fixture(scope="module")
def N():
    from impeller_b200 import build
    build.build()
    from impeller_b200 import ntt
    ntt._lib.load()
    return ntt


def dev(a):
    a = np.ascontiguousarray(a, dtype=np.uint32).reshape(-1, 8)
    return torch.from_numpy(a.view(np.int32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32).reshape(-1, 8)


def rand_field(rng, n, m):
    return O.ints_to_array([int.from_bytes(rng.bytes(32), "little") % m for _ in range(n)])


def unit_for(log_n, field=O.FR):
    return O.mont_limbs(O.root_of_unity(log_n, field), field)


def twiddles(N, log_n, field=O.FR):
    tw = np.zeros((max(1, (1 << log_n) // 2), 8), np.uint32)
    N.SsipPrecompute(field=_nf(N, field)).get_fn()(tw, unit_for(log_n, field))
    return tw


def _nf(N, field):
    return {O.FR: N.BN254_FR, O.FQ: N.BN254_FQ, O.BLS_FR: N.BLS12381_FR}[field]


@pytest.mark.parametrize("log_n", [1, 2, 3, 5, 8, 10, 11, 12, 13, 15, 17, 19, 20])
def test_ssip_ntt_matches_oracle(N, log_n):
    rng = np.random.default_rng(log_n)
    n = 1 << log_n
    x = rand_field(rng, n, O.R_MOD)
    x[0] = O.int_to_limbs(O.R_MOD - 1)  # canonical edge values
    x[-1] = 0
    tw = twiddles(N, log_n)
    assert (tw == O.ntt_roots(n // 2, unit_for(log_n))).all()
    want = O.ntt(x, unit_for(log_n))
    d = dev(x)
    N.SsipNtt().get_fn()(d, dev(tw))
    assert (host(d) == want).all()


@pytest.mark.parametrize("log_n", [1, 4, 11, 12, 16, 18])
def test_recompute_ntt_matches_oracle(N, log_n):
    rng = np.random.default_rng(100 + log_n)
    n = 1 << log_n
    x = rand_field(rng, n, O.R_MOD)
    g = N.GenPqOmegas()
    pq = np.zeros((g.get_pq_len(log_n), 8), np.uint32)
    om = np.zeros((32, 8), np.uint32)
    g.get_fn()(pq, om, n, unit_for(log_n))
    deg = (pq.shape[0] - 1).bit_length() + 1 if pq.shape[0] > 1 else 1
    want_pq, want_om = O.pq_omegas(deg, n, unit_for(log_n))
    assert (pq == want_pq).all() and (om == want_om).all()
    d = dev(x)
    N.RecomputeNtt().get_fn()(d, dev(pq), dev(om))
    assert (host(d) == O.ntt(x, unit_for(log_n))).all()


def test_rotated_and_sliced_views(N):
    rng = np.random.default_rng(7)
    log_n = 12
    n = 1 << log_n
    x = rand_field(rng, n, O.R_MOD)
    tw = dev(twiddles(N, log_n))
    f = N.SsipNtt().get_fn()
    # rotated by r: logical element i is physical (n - r + i) mod n
    for r in (1, 5, n - 1):
        d = dev(x)
        f(d, tw, rotate=r)
        logical = np.roll(x, r, axis=0)
        want = O.ntt(logical, unit_for(log_n))
        assert (np.roll(host(d), r, axis=0) == want).all(), r
    # a length-n slice of a longer array, wrapping around its end
    whole = n + 300
    big = rand_field(rng, whole, O.R_MOD)
    for off in (0, 17, 300, whole - 5):
        d = dev(big)
        f(d, tw, offset=off, whole_len=whole, length=n)
        idx = (off + np.arange(n)) % whole
        want = big.copy()
        want[idx] = O.ntt(big[idx], unit_for(log_n))
        assert (host(d) == want).all(), off


def test_distribute_powers(N):
    rng = np.random.default_rng(9)
    n = 5000
    x = rand_field(rng, n, O.R_MOD)
    pw = rand_field(rng, 7, O.R_MOD)
    f = N.DistributePowers().get_fn()
    for sl in (None, (0, n, n), (123, n, 7000), (6999, n, 7000)):
        d = dev(x)
        f(d, dev(pw), poly_slice=sl)
        begin, _, plen = sl if sl else (0, n, n)
        assert (host(d) == O.distribute_powers(x, pw, begin=begin, poly_len=plen)).all(), sl
    # powers as long as the polynomial (the coset-shift use)
    pw = rand_field(rng, n, O.R_MOD)
    d = dev(x)
    f(d, dev(pw))
    assert (host(d) == O.distribute_powers(x, pw)).all()


@pytest.mark.parametrize("log_n", [1, 6, 12, 16])
def test_other_fields(N, log_n):
    rng = np.random.default_rng(200 + log_n)
    n = 1 << log_n
    x = rand_field(rng, n, O.R_BLS)
    tw = twiddles(N, log_n, O.BLS_FR)
    d = dev(x)
    N.SsipNtt(field=N.BLS12381_FR).get_fn()(d, dev(tw))
    assert (host(d) == O.ntt(x, unit_for(log_n, O.BLS_FR), O.BLS_FR)).all()
    if log_n == 1:  # BN254 Fq: 2-adicity 1
        xq = rand_field(rng, 2, O.P)
        d = dev(xq)
        N.SsipNtt(field=N.BN254_FQ).get_fn()(d, dev(twiddles(N, 1, O.FQ)))
        assert (host(d) == O.ntt(xq, unit_for(1, O.FQ), O.FQ)).all()


def test_bad_arguments_are_errors(N):
    from impeller_b200 import lib
    L = lib.load()
    t = torch.zeros((12, 8), dtype=torch.int32, device="cuda")
    tw = torch.zeros((8, 8), dtype=torch.int32, device="cuda")
    p = lib.PolyPtr(t.data_ptr(), 12, 0, 0, 12)
    assert L.ssip_ntt(p, tw.data_ptr(), 4, None, 8, 8) != 0  # len != 2^log_len
    assert L.ssip_ntt(lib.PolyPtr(t.data_ptr() + 4, 8, 0, 0, 8), tw.data_ptr(), 3, None, 8, 8) != 0  # misaligned
    assert L.ssip_ntt(lib.PolyPtr(t.data_ptr(), 8, 0, 0, 8), tw.data_ptr(), 3, None, 11, 8) != 0
    assert L.impeller_ntt(7, lib.PolyPtr(t.data_ptr(), 8, 0, 0, 8), tw.data_ptr(), 3, None) != 0


def test_full_size_2e24_roundtrip(N):
    log_n = 24
    n = 1 << log_n
    from impeller_b200 import msm as M
    x = M.gen_scalars_device(n, seed=5, stream_id=3)  # uniform Montgomery Fr
    x0 = x.clone()
    w = O.root_of_unity(log_n)
    tw = twiddles(N, log_n)
    twi = np.zeros_like(tw)
    N.SsipPrecompute().get_fn()(twi, O.mont_limbs(pow(w, -1, O.R_MOD)))
    f = N.SsipNtt().get_fn()
    f(x, dev(tw))
    f(x, dev(twi))
    # inverse transform times n: multiply by n^-1 with distribute_powers
    ninv = dev(O.mont_limbs(pow(n, -1, O.R_MOD))[None])
    N.DistributePowers().get_fn()(x, ninv)
    assert torch.equal(x, x0)


REF_NTT_LIBS = {O.FR: REF_NTT, O.BLS_FR: os.path.join(os.path.dirname(O.__file__), "_ref", "libref_ntt_bls12381_fr.so")}


@pytest.mark.parametrize("field,log_n", [(O.FR, 10), (O.FR, 16), (O.FR, 20), (O.FR, 24),
                                         (O.BLS_FR, 12), (O.BLS_FR, 18), (O.BLS_FR, 22)])
def test_matches_reference_gpu_kernels(N, field, log_n):
    if not os.path.exists(REF_NTT_LIBS[field]):
        pytest.skip("reference NTT library for this field not built")
    from impeller_b200 import lib
    ref = ctypes.CDLL(REF_NTT_LIBS[field])
    ref.ssip_ntt.restype = ctypes.c_int
    ref.ssip_ntt.argtypes = [lib.PolyPtr, ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint,
                             ctypes.c_uint]
    ref.recompute_ntt.restype = ctypes.c_int
    ref.recompute_ntt.argtypes = [lib.PolyPtr, ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint,
                                  ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint]
    ref.ssip_precompute.restype = ctypes.c_int
    ref.ssip_precompute.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
    n = 1 << log_n
    nf = _nf(N, field)
    from impeller_b200 import msm as M
    x = M.gen_scalars_device(n, seed=6, stream_id=log_n, curve=M.BLS12381 if field == O.BLS_FR else M.BN254)
    u = np.ascontiguousarray(unit_for(log_n, field))
    tw_ref = np.zeros((n // 2, 8), np.uint32)
    assert ref.ssip_precompute(tw_ref.ctypes.data, n // 2, u.ctypes.data) == 0
    tw = twiddles(N, log_n, field)
    assert (tw == tw_ref).all()
    d_tw = dev(tw)
    ours, theirs = x.clone(), x.clone()
    N.SsipNtt(field=nf).get_fn()(ours, d_tw)
    torch.cuda.synchronize()
    assert ref.ssip_ntt(lib.PolyPtr(theirs.data_ptr(), n, 0, 0, n), d_tw.data_ptr(), log_n, None, 8, 8) == 0
    torch.cuda.synchronize()
    assert torch.equal(ours, theirs)
    # recompute variant, both libraries
    g = N.GenPqOmegas(field=nf)
    pq = np.zeros((g.get_pq_len(log_n), 8), np.uint32)
    om = np.zeros((32, 8), np.uint32)
    g.get_fn()(pq, om, n, u)
    deg = (pq.shape[0] - 1).bit_length() + 1
    d_pq, d_om = dev(pq), dev(om)
    theirs = x.clone()
    assert ref.recompute_ntt(lib.PolyPtr(theirs.data_ptr(), n, 0, 0, n), d_pq.data_ptr(), deg, d_om.data_ptr(),
                             log_n, None, 8, 8) == 0
    torch.cuda.synchronize()
    ours2 = x.clone()
    N.RecomputeNtt(field=nf).get_fn()(ours2, d_pq, d_om)
    torch.cuda.synchronize()
    assert torch.equal(theirs, ours) and torch.equal(ours2, ours)
    if log_n <= 16:
        assert (host(ours) == O.ntt(host(x), u, field)).all()
