"""The reference's multi-card split through msm() and msm_precompute(), on one GPU.

MultiGPUMSM (core/src/msm/src/msm_impl.cuh:832-845 constructor, :874-910 run
and host sum) splits the len points into cards.size() ranges of
ceil(len / cards) points, runs one MSM instance per entry of `cards` on its
own thread, and adds the per-card partial sums.  It constructs one instance
per entry, so a card id may repeat: cards = [0, 0] or [0, 0, 0] runs two or
three ranges, each with its own scratch buffer, on device 0.  That is how
this file drives the whole split on a single B200: the thread per card, the
per-card buffer carving, the carried XYZZ partials and their device-side sum
on card 0 (k_combine).

MSMPrecompute::precompute (:803-829) uses min(device count, max_cards)
devices; with one GPU and max_cards = 2 it runs on the one device.

Every output is compared bit for bit with the CPU oracle (integer work,
tolerance zero); window tables with the oracle's tables."""
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


def run_split(M, cfg, tables, scal):
    op = M.MSM(cfg)
    n = tables[0].shape[0]
    sizes = op.get_buffer_size(n)
    assert len(sizes) == len(cfg.cards)
    bufs, keep = [], []
    for s in sizes:
        b, k = M.alloc_gpu_buffer(s)
        bufs.append(b)
        keep.append(k)
    out = op.run(tables, scal, bufs)
    torch.cuda.synchronize()
    del keep
    return out


@pytest.mark.parametrize("cards", [[0, 0], [0, 0, 0]])
@pytest.mark.parametrize("parts,batch_per_run", [(1, 1), (1, 2), (3, 1), (2, 2)])
def test_card_split_plain_windows(M, cards, parts, batch_per_run):
    n = 7001  # not a multiple of 2 or 3: the last card's range is shorter
    pts = O.gen_points(n, seed=31)
    scal = [O.gen_scalars(n, seed=31, stream=s) for s in range(3)]
    cfg = M.MsmConfig(cards=cards, parts=parts, batch_per_run=batch_per_run,
                      stage_scalars=1 if parts == 1 else 2, stage_points=1 if parts == 1 else 2)
    res = run_split(M, cfg, [pts], scal)
    for i, (s, r) in enumerate(zip(scal, res)):
        assert (r == O.msm(pts, s)).all(), (cards, parts, batch_per_run, i)


@pytest.mark.parametrize("cards", [[0, 0], [0, 0, 0]])
def test_card_split_with_window_tables(M, cards):
    # window 13 with 4 bucket sets: 20 digit windows over 5 window tables,
    # the tables made by msm_precompute with max_cards = 2
    n = 6000
    cfg = M.MsmConfig(window_size=13, target_window=4, cards=cards, batch_per_run=2)
    assert cfg.get_precompute() == 5
    pts = O.gen_points(n, seed=32)
    tables = [pts.copy()] + [np.zeros_like(pts) for _ in range(4)]
    M.MSMPrecompute(cfg).get_fn()(tables, n, 2)
    want_tabs = O.precompute(pts, shift=4 * 13, n_tables=5)
    for j in range(5):
        assert (tables[j] == want_tabs[j]).all(), j
    scal = [O.gen_scalars(n, seed=32, stream=s) for s in range(3)]
    res = run_split(M, cfg, tables, scal)
    for i, (s, r) in enumerate(zip(scal, res)):
        assert (r == O.msm(pts, s)).all(), (cards, i)
    # the same tables split into parts on every card
    cfg3 = M.MsmConfig(window_size=13, target_window=4, cards=cards, parts=3, stage_scalars=2, stage_points=2)
    assert (run_split(M, cfg3, tables, scal[:1])[0] == O.msm(pts, scal[0])).all()


def test_card_split_ranges_with_nothing_left(M):
    # len = 2 over three cards: ranges of 1, 1 and 0 points; the empty range
    # contributes the identity
    pts = O.gen_points(2, seed=33)
    sc = O.gen_scalars(2, seed=33, stream=1)
    res = run_split(M, M.MsmConfig(cards=[0, 0, 0]), [pts], [sc])
    assert (res[0] == O.msm(pts, sc)).all()
    # P and -P on two cards with equal scalars: the partials cancel
    pm = np.concatenate([pts[:1], O.point_op(O.PT_NEG, pts[:1])])
    sc2 = np.repeat(sc[:1], 2, 0)
    assert (run_split(M, M.MsmConfig(cards=[0, 0]), [pm], [sc2])[0] == 0).all()


def test_card_split_streamed_ranges(M):
    # 2 x (2^21 + 6) points: each card's range streams its upload in chunks
    n = (1 << 22) + 12
    d = M.gen_points_device(n, seed=34)
    pts = M.to_host(d).reshape(n, 16)
    del d
    assert (pts[:256] == O.gen_points(256, seed=34)).all()
    sc = M.to_host(M.gen_scalars_device(n, seed=34, stream_id=1)).reshape(n, 8)
    res = run_split(M, M.MsmConfig(cards=[0, 0]), [pts], [sc])
    assert (res[0] == O.msm(pts, sc)).all()


def test_card_split_bls12381(M):
    n = 3001
    C = M.BLS12381
    pts = O.gen_points(n, seed=35, curve=O.BLS12381)
    scal = [O.gen_scalars(n, seed=35, stream=s, curve=O.BLS12381) for s in range(2)]
    cfg = M.MsmConfig(window_size=16, target_window=16, cards=[0, 0, 0], batch_per_run=2, curve=C)
    res = run_split(M, cfg, [pts], scal)
    for s, r in zip(scal, res):
        assert (r == O.msm(pts, s, curve=O.BLS12381)).all()
