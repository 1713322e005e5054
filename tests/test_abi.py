"""The C ABI library loads and exports every entry point include/zuikaku.h
declares (CPU only: no device work is launched here)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    src = (ROOT / "include" / "zuikaku.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(zk_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from zuikakucfd_b200 import build
    path = build.build()
    return C.CDLL(str(path))


def test_header_declares_entry_points():
    names = declared()
    for must in ("zk_create", "zk_destroy", "zk_set_mesh", "zk_set_state", "zk_get_state", "zk_step",
                 "zk_rhs", "zk_limit", "zk_max_speed", "zk_recover_primitives", "zk_load_case"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from zuikakucfd_b200 import _native
    assert set(declared()) <= set(_native.exported_symbols()) | {"zk_default_options"}


def test_default_options_and_errors_without_device(lib):
    from zuikakucfd_b200._native import zk_options
    o = zk_options()
    lib.zk_default_options(C.byref(o))
    assert (o.method, o.order, o.precision, o.limiter, o.flux, o.boundary, o.device) == (0, 2, 0, 0, 0, 0, 0)
    assert o.tvb_M == 50.0
    lib.zk_last_error.restype = C.c_char_p
    h = C.c_void_p()
    # bad options are rejected before any device work
    o.method = 7
    assert lib.zk_create(C.byref(o), C.byref(h)) == 1
    assert b"method" in lib.zk_last_error()
    assert lib.zk_create(None, C.byref(h)) == 1
    assert lib.zk_version() >= 100
    # threads per cell of the mixed DG stage: 0 (tuned), 1 or 2
    lib.zk_default_options(C.byref(o))
    o.method, o.order, o.tile_tpc = 1, 2, 4
    assert lib.zk_create(C.byref(o), C.byref(h)) == 1
    assert b"tile_tpc" in lib.zk_last_error()



def test_slab_entry_points_reject_a_null_context(lib):
    """zk_stage / zk_halo_* check their context before any device work."""
    lib.zk_last_error.restype = C.c_char_p
    n = C.c_size_t()
    lib.zk_stage.argtypes = [C.c_void_p, C.c_double, C.c_int]
    assert lib.zk_stage(None, C.c_double(1e-3), 1) == 1
    assert lib.zk_stage_limit(None, 1) == 1
    assert lib.zk_halo_bytes(None, 0, C.byref(n)) == 1
    assert lib.zk_halo_pack(None, 0, 0, None) == 1
    assert lib.zk_halo_unpack(None, 0, 1, None) == 1
    assert b"null context" in lib.zk_last_error()


def test_batch_default_options_and_bad_options(lib):
    """Batch defaults (tuned WENO tile, 10 graph steps) and option checks that
    run before any device work."""
    from zuikakucfd_b200._native import zk_batch_options
    lib.zk_last_error.restype = C.c_char_p
    o = zk_batch_options()
    lib.zk_batch_default_options(C.byref(o))
    assert (o.device, o.policy, o.graph_steps, o.autotune, o.arena_bytes) == (0, 0, 10, 1, 0)
    assert (o.weno_variant, o.dg_variant) == (-1, -1)
    h = C.c_void_p()
    for field, bad, word in (("weno_variant", 6, b"weno_variant"), ("dg_variant", 4, b"dg_variant"),
                             ("graph_steps", 0, b"graph_steps"),
                             ("autotune", 3, b"autotune"), ("policy", 9, b"policy")):
        lib.zk_batch_default_options(C.byref(o))
        setattr(o, field, bad)
        assert lib.zk_batch_create(C.byref(o), C.byref(h)) == 1
        assert word in lib.zk_last_error()
