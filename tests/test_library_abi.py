"""The C-ABI library builds, loads without a GPU, and exports every symbol
include/impeller_msm.h declares; the drop-in shims carry the reference's
library names and symbols.  No compute calls (no GPU needed)."""
import ctypes
import os
import subprocess

import pytest

from impeller_b200 import build, lib
from impeller_b200 import msm as M


@pytest.fixture(scope="module")
def L():
    build.build()
    return lib.load()


def test_header_declares_reference_symbols():
    names = lib.declared_symbols()
    assert names[:2] == ["msm", "msm_precompute"]
    assert set(names) == set(lib.SIGNATURES), set(names) ^ set(lib.SIGNATURES)


def test_library_exports_every_declared_symbol(L):
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    for name in lib.declared_symbols():
        assert name in exported, name
        assert getattr(L, name) is not None


def test_host_only_queries(L):
    assert L.impeller_msm_n_precompute(16, 16) == 1
    assert L.impeller_msm_n_precompute(13, 4) == 5  # ceil(254/13)=20 windows, 4 per table
    assert L.impeller_msm_n_precompute(2, 1) == 0   # invalid window size
    for n in (1 << 10, 1 << 16, 1 << 22):
        assert 3 <= L.impeller_default_window(n) <= 24
    assert b"sm_100a" in L.impeller_version()


def test_config_mirrors_reference():
    # common/src/msm_config.rs:17-25 and :52-55
    cfg = M.MsmConfig()
    assert (cfg.window_size, cfg.target_window, cfg.cards, cfg.batch_per_run, cfg.parts, cfg.bits) == \
        (16, 16, [0], 1, 1, 254)
    assert cfg.get_precompute() == 1
    assert M.MsmConfig(window_size=13, target_window=4).get_precompute() == 5
    assert M.lib_name(M.MsmConfig()) == "msm_bn254_16_16_false"
    for c in range(3, 32):
        for t in (1, 2, 5, 40):
            assert M.MsmConfig(window_size=c, target_window=t).get_precompute() == M.n_precompute(c, t)


def test_shim_has_reference_name_and_symbols(L):
    path = build.build_shim(13, 4, False)
    assert os.path.basename(path) == "libmsm_bn254_13_4_false.so"
    S = ctypes.CDLL(path)
    assert S.msm and S.msm_precompute


def test_window_table_roundtrip(L):
    M.set_window_table({10: 7, 16: 12, 22: (17, 20)})
    assert M.default_window(1 << 16) == 12
    assert M.default_window(3 << 20) == 17  # nearest log2
    assert M.table_window(1 << 22) == 20 and M.table_window(1 << 10) == 0
    M.set_window_table({})  # the cost model
    assert 3 <= M.default_window(1 << 20) <= 22 and M.table_window(1 << 20) == 0
    M.restore_default_window_table()


def test_compiled_table_matches_autotune_json(L):
    """The library's built-in window table is the committed measurement
    (impeller_b200/autotune_table.json, compiled in at build time)."""
    import json
    import os
    M.restore_default_window_table()
    path = os.path.join(os.path.dirname(M.__file__), "autotune_table.json")
    for e in json.load(open(path))["entries"]:
        n = 1 << e["log2n"]
        assert M.default_window(n) == e["plain_c"], e
        assert M.table_window(n) == (e.get("tables_c") or 0), e


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(lib.ImpellerError):
        lib.load(str(tmp_path / "libimpeller_msm.so"))


def test_ntt_library_name_and_symbols(L):
    path = build.ntt_library()
    assert os.path.basename(path) == "libntt.so"
    S = ctypes.CDLL(path)
    for sym in ("ssip_ntt", "ssip_precompute", "recompute_ntt", "gen_pq_omegas", "distribute_powers"):
        assert getattr(S, sym)
    assert L.impeller_ntt_launches(0) == 0
    assert L.impeller_ntt_launches(11) == 1   # one tile, written out reversed
    assert L.impeller_ntt_launches(20) == 3   # 9-bit pass, 11-bit pass, reorder
    assert L.impeller_ntt_launches(24) == 4


def test_bls_shim_name_and_config():
    path = build.build_shim(16, 16, False, curve=M.BLS12381)
    assert os.path.basename(path) == "libmsm_bls12381_16_16_false.so"
    cfg = M.MsmConfig(curve=M.BLS12381)
    assert cfg.bits == 255 and M.lib_name(cfg) == "msm_bls12381_16_16_false"
    assert M.n_precompute(13, 4, curve=M.BLS12381) == 5
    assert M.n_precompute(17, 5, curve=M.BLS12381) == 0  # needs a 16th window: refused
    assert M.n_precompute(17, 15, curve=M.BLS12381) == 1


def test_bls_window_avoids_carry_only_windows(L):
    for n in (1 << 10, 1 << 16, 1 << 18, 1 << 20, 1 << 22):
        c = M.default_window(n)
        cb = M.default_window(n, M.BLS12381)
        assert cb not in (3, 5, 15, 17)
        assert cb == c or (c, cb) in ((15, 16), (17, 16))
