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


def test_bf16_texel_rounding():
    """to_bf16 rounds to nearest with ties to even, as torch's conversion
    does, and from_bf16 gives the patterns' values exactly."""
    import numpy as np
    import torch
    import dmap_b200 as dm
    rng = np.random.default_rng(9)
    x = np.concatenate([(rng.random(20000) * 2 - 1) * 10.0 ** rng.integers(-6, 6, 20000),
                        np.float32(1.0) + np.arange(-64, 65, dtype=np.float32) * np.float32(2.0 ** -8),
                        [0.0, -0.0, 1e-40, -1e-40, 3.0e38]]).astype(np.float32)
    bits = dm.to_bf16(x)
    ref = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(bits, ref)
    v = dm.from_bf16(bits)
    assert np.array_equal(v, torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy())
    assert np.array_equal(dm.to_bf16(v), bits)
