"""Decode delivery modes through the C-ABI against the reference library built
from its sources (oracle/_ref): tc_frame_decode_request (full, dropped alpha,
scaled to exact-half / odd / equal / 1x1 targets, reduced 1/2 1/3 1/4 1/8,
auto 2K), tc_frame_decode_scaled, tc_frame_decode_reduced,
tc_frame_decode_batch_reduced and the decoder-context calls (plane views,
batches, surfaces) on intact and damaged packets: status, frame information,
per-slice status and every delivered sample equal."""
import ctypes
import random

import numpy as np
import pytest

from test_gpu_parity import _spans
from topos_codec_b200 import binding as B, synth

pytestmark = pytest.mark.gpu


class PlaneView(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32),
                ("pixels", ctypes.c_void_p), ("stride", ctypes.c_size_t)]


class Surface(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32), ("memory_type", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("planes", PlaneView * 4)]


@pytest.fixture(scope="module")
def packets(oracle):
    """(label, packet) pairs: deblocked 4:2:2 at exact-half-friendly sizes, QPT2
    4K, odd geometry, 4:4:4 + alpha, and damaged copies."""
    out = []
    specs = [("1080p qm4 deblock", 1920, 1080, dict(qp=8, qmatrix_id=4, features=1)),
             ("640x360 deblock", 640, 360, dict(qp=20, qmatrix_id=4, features=1)),
             ("4K hq qpt2", 3840, 2160, dict(qp=4, qmatrix_id=0, features=3)),
             ("odd 203x77", 203, 77, dict(qp=12))]
    for k, (label, w, h, kw) in enumerate(specs):
        planes = synth.make_frame_np(w, h, seed=200 + k)
        out.append((label, oracle.encode(B.make_config(w, h, **kw), planes)))
    w, h = 160, 96
    planes = synth.make_frame_np(w, h, seed=210, bit_depth=12, pixel_format=2, limited=False, alpha=True, sigma=12)
    out.append(("gbr444 alpha", oracle.encode(B.make_config(w, h, qp=2, bit_depth=12, pixel_format=2, profile=5,
                                                            alpha_mode=1, alpha_bit_depth=16, color_range=1), planes)))
    rng = random.Random(9)
    for label, pkt in list(out):
        if label.startswith("4K"):
            continue
        p = bytearray(pkt)
        for _ in range(2):
            _, po, size = _spans(pkt)[rng.randrange(len(_spans(pkt)))]
            p[po + rng.randrange(size)] ^= 0x33
        out.append((label + " damaged", bytes(p)))
    return out


def _requests(w, h):
    reqs = [("full", B.make_request(0)), ("full drop alpha", B.make_request(0, flags=1)),
            ("half", B.make_request(1, target=((w + 1) // 2, (h + 1) // 2))),
            ("odd", B.make_request(1, target=(max(1, w * 2 // 3 - 1), max(1, h * 3 // 5 + 1)))),
            ("equal", B.make_request(1, target=(w, h))), ("1x1", B.make_request(1, target=(1, 1))),
            ("auto2k", B.make_request(3)), ("auto2k drop", B.make_request(3, flags=1))]
    reqs += [(f"reduced {s}", B.make_request(2, scale=s)) for s in range(1, 5)]
    return reqs


def _same(a, b, what):
    assert a.status == b.status, (what, a.status, b.status)
    assert bytes(a.info) == bytes(b.info), what
    assert len(a.planes) == len(b.planes), what
    for x, y in zip(a.planes, b.planes):
        assert np.array_equal(x, y), what


def test_decode_requests_vs_reference(product, reference, packets):
    for label, pkt in packets:
        rc, info = reference.query(pkt)
        assert rc == 0
        for rl, req in _requests(info.visible_width, info.visible_height):
            a = B.decode_request(product, pkt, req, fill=7)
            b = B.decode_request(reference, pkt, req, fill=7)
            _same(a, b, (label, rl))


def _call_planes(lib_fn, pkt, n_planes_shapes, *args):
    planes = [np.full(s, 3, dtype=np.uint16) for s in n_planes_shapes]
    ptrs = (ctypes.c_void_p * 4)(*[p.ctypes.data for p in planes])
    info = B.FrameOutput()
    buf = np.frombuffer(pkt, np.uint8)
    rc = int(lib_fn(ctypes.c_void_p(buf.ctypes.data), ctypes.c_size_t(len(pkt)), *args, ptrs, None, ctypes.byref(info)))
    return B.DecodedFrame(planes, info, rc)


def test_scaled_and_reduced_entries_vs_reference(product, reference, packets):
    for label, pkt in packets[:5]:
        rc, info = reference.query(pkt)
        w, h = info.visible_width, info.visible_height
        for tw, th in [((w + 1) // 2, (h + 1) // 2), (max(1, w // 3), max(1, h // 2)), (w, h)]:
            got = []
            for c in (product, reference):
                L = c._lib
                L.tc_frame_decode_scaled.restype = ctypes.c_int32
                i2 = B.FrameOutput()
                i2.visible_width, i2.visible_height, i2.plane_count, i2.pixel_format = tw, th, info.plane_count, \
                    info.pixel_format
                got.append(_call_planes(L.tc_frame_decode_scaled, pkt, B.ToposCodec.geometry(i2), ctypes.c_uint32(tw),
                                        ctypes.c_uint32(th)))
            _same(got[0], got[1], (label, "scaled", tw, th))
        for s in range(0, 5):
            got = []
            for c in (product, reference):
                L = c._lib
                L.tc_frame_decode_reduced.restype = ctypes.c_int32
                L.tc_decode_scale_dimensions.restype = ctypes.c_int32
                tw, th = ctypes.c_uint32(), ctypes.c_uint32()
                assert L.tc_decode_scale_dimensions(w, h, s, ctypes.byref(tw), ctypes.byref(th)) == 0
                i2 = B.FrameOutput()
                i2.visible_width, i2.visible_height, i2.plane_count, i2.pixel_format = tw.value, th.value, \
                    info.plane_count, info.pixel_format
                got.append(_call_planes(L.tc_frame_decode_reduced, pkt, B.ToposCodec.geometry(i2), ctypes.c_int32(s)))
            _same(got[0], got[1], (label, "reduced", s))


def test_batch_reduced_and_decoder_contexts_vs_reference(product, reference, packets):
    pk = [p for _, p in packets if len(p) < 4_000_000][:6]
    n = len(pk)
    bufs = [np.frombuffer(p, np.uint8) for p in pk]
    arr = (B.BatchPacket * n)()
    for i, b in enumerate(bufs):
        arr[i].data, arr[i].size = b.ctypes.data, len(pk[i])
    for scale in (1, 3, 4):
        res = []
        for c in (product, reference):
            L = c._lib
            L.tc_frame_decode_batch_reduced.restype = ctypes.c_int32
            infos = (B.FrameOutput * n)()
            assert int(L.tc_frame_decode_batch_reduced(arr, n, scale, None, None, infos)) == 0
            planes = [[np.full(s, 5, np.uint16) for s in B.ToposCodec.geometry(infos[i])] for i in range(n)]
            ptrs = (ctypes.c_void_p * (4 * n))()
            for i in range(n):
                for p, a in enumerate(planes[i]):
                    ptrs[4 * i + p] = a.ctypes.data
            infos = (B.FrameOutput * n)()
            rc = int(L.tc_frame_decode_batch_reduced(arr, n, scale, ptrs, None, infos))
            res.append((rc, [bytes(x) for x in infos], planes))
        assert res[0][0] == res[1][0] and res[0][1] == res[1][1], scale
        for x, y in zip(res[0][2], res[1][2]):
            assert all(np.array_equal(a, b) for a, b in zip(x, y)), scale
    # decoder contexts: a batch with a request, and a surface with a request
    req = B.make_request(3, flags=1)
    sreq = B.make_request(1, target=(64, 36), memory_type=1)
    for c in (product, reference):
        L = c._lib
        for f in ("tc_decoder_create", "tc_decoder_decode_batch_request", "tc_decoder_decode_surface_request",
                  "tc_decoder_prepare_request"):
            getattr(L, f).restype = ctypes.c_int32
    out = []
    for c in (product, reference):
        L = c._lib
        d = ctypes.c_void_p()
        assert L.tc_decoder_create(None, ctypes.byref(d)) == 0
        infos = (B.FrameOutput * n)()
        assert int(L.tc_decoder_decode_batch_request(d, arr, n, ctypes.byref(req), None, infos)) == 0
        planes = [[np.full(s, 9, np.uint16) for s in B.ToposCodec.geometry(infos[i])] for i in range(n)]
        views = (PlaneView * (4 * n))()
        for i in range(n):
            for p, a in enumerate(planes[i]):
                views[4 * i + p].struct_size, views[4 * i + p].abi_version = ctypes.sizeof(PlaneView), 2
                views[4 * i + p].pixels = a.ctypes.data
        infos = (B.FrameOutput * n)()
        rc = int(L.tc_decoder_decode_batch_request(d, arr, n, ctypes.byref(req), views, infos))
        pkt = pk[1]
        si = B.FrameOutput()
        assert int(L.tc_decoder_prepare_request(d, ctypes.c_void_p(bufs[1].ctypes.data), ctypes.c_size_t(len(pkt)), ctypes.byref(sreq),
                                                ctypes.byref(si))) == 0
        splanes = [np.full(s, 1, np.uint16) for s in B.ToposCodec.geometry(si)]
        surf = Surface()
        surf.struct_size, surf.abi_version, surf.memory_type = ctypes.sizeof(Surface), 2, 1
        for p, a in enumerate(splanes):
            surf.planes[p].struct_size, surf.planes[p].abi_version = ctypes.sizeof(PlaneView), 2
            surf.planes[p].pixels = a.ctypes.data
        so = B.FrameOutput()
        src = int(L.tc_decoder_decode_surface_request(d, ctypes.c_void_p(bufs[1].ctypes.data), ctypes.c_size_t(len(pkt)),
                                                      ctypes.byref(sreq), ctypes.byref(surf), ctypes.byref(so)))
        L.tc_decoder_destroy(d)
        out.append((rc, [bytes(x) for x in infos], planes, src, bytes(so), splanes))
    a, b = out
    assert a[0] == b[0] and a[1] == b[1] and a[3] == b[3] and a[4] == b[4]
    for x, y in zip(a[2], b[2]):
        assert all(np.array_equal(p, q) for p, q in zip(x, y))
    assert all(np.array_equal(p, q) for p, q in zip(a[5], b[5]))


def test_exact_half_edge_blocks_vs_reference(product, reference):
    """Exact-half delivery of planes whose last block column is narrower than 8
    pixels (the reference's 4x4 block store reads entries past the block's
    computed prefix): wide planes, planes one block wide with the partial last
    block row in its own slice band or sharing one, 10/12/16-bit, deblocked."""
    cases = [(115, 58, dict(qp=30, qmatrix_id=3, features=2, qp_delta_chroma=3), {}),
             (12, 40, dict(qp=8), {}), (12, 40, dict(qp=8, slice_rows=1), {}),
             (6, 44, dict(qp=8, slice_rows=2), {}), (6, 44, dict(qp=8, slice_rows=1), {}),
             (4, 28, dict(qp=8, slice_rows=3), {}), (6, 12, dict(qp=8), {}), (2, 6, dict(qp=8), {}),
             (44, 30, dict(qp=6, features=1, qmatrix_id=4), {}),
             (90, 22, dict(qp=10, bit_depth=12, qmatrix_id=1), dict(bit_depth=12)),
             (38, 26, dict(qp=40, bit_depth=16), dict(bit_depth=16, limited=False)),
             (30, 14, dict(qp=3, bit_depth=12, pixel_format=2, profile=5, color_range=1),
              dict(bit_depth=12, pixel_format=2, limited=False))]
    for k, (w, h, ck, kw) in enumerate(cases):
        planes = synth.make_frame_np(w, h, seed=300 + k, **kw)
        pkt = reference.encode(B.make_config(w, h, **ck), planes)
        for rl, req in [("half", B.make_request(1, target=((w + 1) // 2, (h + 1) // 2))),
                        ("reduced half", B.make_request(2, scale=1))]:
            a = B.decode_request(product, pkt, req, fill=7)
            b = B.decode_request(reference, pkt, req, fill=7)
            _same(a, b, (w, h, ck, rl))
