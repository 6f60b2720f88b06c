"""The C-ABI library loads and exports every entry point include/dmap_b200.h
declares (no compute, no GPU needed)."""
import ctypes

import dmap_b200


def test_header_declares_entry_points():
    names = dmap_b200.exported_symbols()
    for n in ("dmap_create", "dmap_asset_create", "dmap_scene_create", "dmap_intersect", "dmap_intersect_host"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = dmap_b200.lib()
    missing = [n for n in dmap_b200.exported_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_defaults():
    lib = dmap_b200.lib()
    assert lib.dmap_status_string(0) == b"ok"
    o = dmap_b200._Options()
    lib.dmap_options_default(ctypes.byref(o))
    assert (o.bound, o.slab_max_level, o.leaf, o.mode) == (2, 1, 0, 0)


def test_null_context_is_rejected_without_a_device():
    lib = dmap_b200.lib()
    h = ctypes.c_void_p()
    import numpy as np
    v = np.zeros((3, 3), np.float32)
    assert lib.dmap_asset_create(None, v.ctypes.data, 0, 3, 1.0, 0.0, 0, 0, ctypes.byref(h)) != 0
