"""Allocation-free packet query (tcg_frame_query_batch_noalloc) through the C-ABI.

The entry point serves callers that must not allocate GPU memory while they run:
a serving process whose device memory is handed out up front by its own pool
(a cudaMalloc outside it can fail or upset the pool's accounting) and
latency-critical threads (cudaMalloc/cudaFree may synchronise the device). Its
results must equal those of the allocating query, tc_frame_decode_batch with no
output planes, exactly, on two calls in a row that reuse the same static scratch.
This file is named so that pytest collects it last.
"""
import ctypes
import struct

import numpy as np
import pytest

from topos_codec_b200 import binding as B, synth

pytestmark = pytest.mark.gpu


def _bind(lib):
    fn = lib.tcg_frame_query_batch_noalloc
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.POINTER(B.BatchPacket), ctypes.c_uint32, ctypes.POINTER(B.FrameOutput)]
    return fn


def _packets(items):
    arr = (B.BatchPacket * len(items))()
    for i, (ptr, size) in enumerate(items):
        arr[i].data, arr[i].size = ptr, size
    return arr


def _raw(info):
    return ctypes.string_at(ctypes.addressof(info), ctypes.sizeof(info))


def _both(product, items):
    """(rc, infos) of the allocation-free query and of the allocating batch query."""
    fn = _bind(product._lib)
    n = len(items)
    got = (B.FrameOutput * n)()
    want = (B.FrameOutput * n)()
    rc_got = int(fn(_packets(items), n, got))
    rc_want = int(product._lib.tc_frame_decode_batch(_packets(items), n, None, None, want))
    return rc_got, got, rc_want, want


@pytest.fixture(scope="module")
def packets(product):
    import torch
    out = []
    specs = [
        (640, 360, dict(qp=6, qmatrix_id=4, features=1), dict()),
        (1920, 1080, dict(qp=8, qmatrix_id=4, features=1), dict()),
        (160, 96, dict(qp=2, bit_depth=12, pixel_format=2, profile=5, alpha_mode=1, alpha_bit_depth=16,
                       color_range=1, slice_rows=2),
         dict(bit_depth=12, pixel_format=2, limited=False, alpha=True, sigma=12)),
    ]
    for i, (w, h, ck, fk) in enumerate(specs):
        pkt = product.encode(B.make_config(w, h, **ck), synth.make_frame_np(w, h, seed=80 + i, **fk))
        dev = torch.from_numpy(np.frombuffer(pkt, dtype=np.uint8).copy()).cuda()
        out.append((pkt, dev))
    return out


def test_noalloc_query_matches_batch_query_twice(product, packets):
    import torch
    (a, da), (b, db), (c, dc) = packets
    host_c = ctypes.create_string_buffer(c, len(c))
    first = [(da.data_ptr(), len(a)), (db.data_ptr(), len(b)), (ctypes.addressof(host_c), len(c))]
    # second call: other packets in other record slots, one with a slice count
    # that the first call's records in the same slot would contradict
    second = [(dc.data_ptr(), len(c)), (da.data_ptr(), len(a))]
    torch.cuda.synchronize()
    for items in (first, second):
        rc_got, got, rc_want, want = _both(product, items)
        assert rc_got == rc_want == 0
        for x, y in zip(got, want):
            assert _raw(x) == _raw(y)
        assert got[0].slice_count > 0


def test_noalloc_query_allocates_nothing(product, packets):
    """After one warm-up call (which may look up the scratch address and load
    device code), further calls change neither the library's allocation count
    nor the device's free memory."""
    import torch
    (a, da), (b, db), (c, dc) = packets
    host_c = ctypes.create_string_buffer(c, len(c))
    items = [(da.data_ptr(), len(a)), (ctypes.addressof(host_c), len(c)), (db.data_ptr(), len(b))]
    fn = _bind(product._lib)
    count = product._lib.tcg_allocation_count
    count.restype = ctypes.c_uint64
    infos = (B.FrameOutput * len(items))()
    torch.cuda.synchronize()
    assert int(fn(_packets(items), len(items), infos)) == 0
    allocs0 = int(count())
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        assert int(fn(_packets(items), len(items), infos)) == 0
    assert int(count()) == allocs0
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_query_damaged_and_truncated(product, packets):
    import torch
    (a, _), (b, _), _ = packets
    bad = bytearray(b)
    bad[30:32] = struct.pack(">H", 0)  # zero slice count in the frame header
    cases = [a[:60], a[: len(a) // 2], bytes(bad)]
    devs = [torch.from_numpy(np.frombuffer(x, dtype=np.uint8).copy()).cuda() for x in cases]
    torch.cuda.synchronize()
    for x, d in zip(cases, devs):
        rc_got, got, rc_want, want = _both(product, [(d.data_ptr(), len(x))])
        assert rc_got == rc_want
        if rc_want == 0:
            assert _raw(got[0]) == _raw(want[0])


def test_noalloc_query_rejects_oversized_batch(product, packets):
    (a, da), _, _ = packets
    fn = _bind(product._lib)
    n = 65
    infos = (B.FrameOutput * n)()
    rc = int(fn(_packets([(da.data_ptr(), len(a))] * n), n, infos))
    assert rc == B.TC_ERR_LIMIT_EXCEEDED
    assert "64" in product.last_error()
