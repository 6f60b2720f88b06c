"""dmap_pyramid_build_noalloc: the pyramid build that allocates nothing.

Callers that cannot call cudaMalloc (a host that owns all device memory in
its own pool, or that must not allocate while frames are in flight) build
pyramids through this entry point into buffers they already hold; its FP64
working levels live in a fixed device array of the library. Its FP32
pyramid must equal the regular build's (dmap_asset_create) exactly, call
after call, since every call reuses that array.
"""
import ctypes as C

import numpy as np
import pytest

import dmap_b200 as dm

pytestmark = pytest.mark.gpu

_CODE = {np.dtype(np.float32): dm.F32, np.dtype(np.float16): dm.F16, np.dtype(np.float64): dm.F64,
         np.dtype(np.uint16): dm.BF16}


def _entry():
    fn = dm.lib().dmap_pyramid_build_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
    return fn


def _cells(n_leaf):
    return sum((n_leaf >> l) ** 2 for l in range(n_leaf.bit_length()))


def _buffers(values):
    """The caller's buffers (allocated here by the test, not by the entry
    point): a pitched node grid and the FP32 pyramid output."""
    import torch
    nodes = values.shape[0]
    per16 = 16 // values.itemsize
    pitch = (nodes + per16 - 1) // per16 * per16
    tdt = {np.float32: torch.float32, np.float16: torch.float16, np.float64: torch.float64,
           np.uint16: torch.int16}[values.dtype.type]
    src = np.ascontiguousarray(values)
    if values.dtype == np.uint16:  # bfloat16 bit patterns, moved as 16-bit words
        src = src.view(np.int16)
    grid = torch.zeros((nodes, pitch), dtype=tdt, device="cuda")
    grid[:, :nodes] = torch.from_numpy(src).cuda()
    out = torch.full((_cells(nodes - 1) * 8,), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    return grid, pitch, out


def _call(values, grid, pitch, out, scale, offset, repeat):
    return _entry()(grid.data_ptr(), _CODE[values.dtype], values.shape[0], pitch, scale, offset, int(repeat),
                    out.data_ptr(), None)


def _build_noalloc(values, scale, offset, repeat):
    grid, pitch, out = _buffers(values)
    status = _call(values, grid, pitch, out, scale, offset, repeat)
    return status, out.cpu().numpy()


def _regular(ctx, values, scale, offset, repeat):
    if values.dtype == np.uint16:
        a = dm.Asset(ctx, dm.from_bf16(values), scale, offset, repeat, texel="bf16")
    else:
        a = dm.Asset(ctx, values, scale, offset, repeat)
    return [a.level(l, "f32") for l in range(a.n_levels)]


def _compare(levels, flat):
    off = 0
    for lv in levels:
        m = lv["h0"].shape[0]
        block = flat[8 * off: 8 * (off + m * m)].reshape(m * m, 8).astype(np.float64)
        for c, ch in enumerate(dm.CHANNELS):
            assert np.array_equal(block[:, c], lv[ch].ravel()), ch
        off += m * m
    assert off * 8 == len(flat)


def test_noalloc_pyramid_equals_regular_build_call_after_call():
    ctx = dm.Context(0)
    rng = np.random.default_rng(7)
    # every texel type the entry point takes, and a small map after the
    # largest one, so that a call reuses array contents a bigger call left
    cases = [
        (rng.random((129, 129)).astype(np.float32), 1.0, 0.0, False),
        (rng.random((257, 257)).astype(np.float16), 0.7, -0.1, True),
        (rng.random((513, 513)).astype(np.float32), 0.013, 0.5, False),
        (rng.random((129, 129)).astype(np.float32), 0.3, 0.25, True),
        (dm.to_bf16(rng.random((65, 65)) - 0.5), 0.5, 0.0, False),
        (rng.random((257, 257)) * 2.0 - 1.0, 0.04, -0.02, False),
    ]
    for values, scale, offset, repeat in cases:
        status, flat = _build_noalloc(values, scale, offset, repeat)
        assert status == 0, dm.lib().dmap_status_string(status)
        _compare(_regular(ctx, values, scale, offset, repeat), flat)


def test_noalloc_second_call_takes_no_device_memory():
    """After the first call on a device (which may load the library's device
    code and commit the array), a call leaves the device's free memory as it
    was: it allocates nothing."""
    import torch
    values = np.random.default_rng(11).random((257, 257)).astype(np.float32)
    grid, pitch, out = _buffers(values)
    assert _call(values, grid, pitch, out, 0.2, 0.0, False) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert _call(values, grid, pitch, out, 0.2, 0.0, False) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_maps_beyond_its_scratch():
    import torch
    small = torch.zeros(16, dtype=torch.float32, device="cuda")
    # 1024 texels per side exceeds the fixed 512 x 512 scratch: rejected before any device work
    assert _entry()(small.data_ptr(), dm.F32, 1025, 1028, 1.0, 0.0, 0, small.data_ptr(), None) == 1
