"""V8 segmented multi-chain rANS (reserved[0] = 9) on the GPU through the C ABI:
packets, statistics and statuses against the reference library and the
oracle, at random geometry and formats, at full size, and batched beside
V7-R2 frames. The bar is byte-identical packets."""
import random

import numpy as np
import pytest

from topos_codec_b200 import binding as B, synth
from test_oracle import _random_v8_config, _v8

pytestmark = pytest.mark.gpu


def test_v8_encode_random_vs_reference(product, reference, oracle):
    rng = random.Random(9090)
    coded = 0
    for i in range(60):
        w, h, kw, ck, sb, tl = _random_v8_config(rng)
        planes = synth.make_frame_np(w, h, seed=300 + i, **kw)
        cfg = _v8(B.make_config(w, h, **ck), sb, tl)
        ra, pa, sa = reference.encode_status(cfg, planes)
        rg, pg, sg = product.encode_status(cfg, planes)
        assert rg == ra, (w, h, ck, sb, tl, product.last_error())
        if ra != 0:
            continue
        coded += 1
        assert pg == pa, (w, h, ck, sb, tl)
        assert sg.as_dict() == sa.as_dict()
        assert oracle.encode(cfg, planes) == pa
    assert coded >= 40


@pytest.mark.parametrize("size,ck", [((1920, 1080), dict(qp=8, qmatrix_id=4)),
                                     ((3840, 2160), dict(qp=4, qmatrix_id=0))])
def test_v8_encode_full_size_vs_reference(product, reference, size, ck):
    w, h = size
    planes = synth.make_frame_np(w, h, seed=0, frame=2)
    cfg = _v8(B.make_config(w, h, **ck), 0, 0)
    pa = reference.encode(cfg, planes)
    assert product.encode(cfg, planes) == pa


def test_v8_batch_beside_v7_equals_single_calls(product):
    """A batch mixing V8 frames (several segment and tile sizes) and V7-R2
    frames: every packet equals the single call's."""
    specs = [(320, 180, 9, 4, 5), (256, 144, 8, 0, 0), (640, 360, 9, 3, 0), (200, 120, 9, 5, 6), (1280, 720, 8, 0, 0)]
    cfgs, frames = [], []
    for i, (w, h, em, sb, tl) in enumerate(specs):
        cfg = B.make_config(w, h, qp=6 + i, qmatrix_id=4)
        if em == 9:
            cfg = _v8(cfg, sb, tl)
        cfgs.append(cfg)
        frames.append(synth.make_frame_np(w, h, seed=40 + i))
    rc, pk, rcs, st = product.encode_batch(cfgs, frames)
    assert rc == 0 and rcs == [0] * len(specs)
    for cfg, planes, p in zip(cfgs, frames, pk):
        assert product.encode(cfg, planes) == p


def _same_decode(a, b):
    return (a.status == b.status and a.slice_status == b.slice_status
            and a.info.concealed_slices == b.info.concealed_slices
            and all(np.array_equal(x, y) for x, y in zip(a.planes, b.planes)))


def test_v8_decode_random_vs_reference(product, reference):
    """Reference V8 packets of random configurations decode to the same
    planes, statuses and frame information on the GPU."""
    rng = random.Random(4242)
    n = 0
    for i in range(60):
        w, h, kw, ck, sb, tl = _random_v8_config(rng)
        cfg = _v8(B.make_config(w, h, **ck), sb, tl)
        rc, pkt, _ = reference.encode_status(cfg, synth.make_frame_np(w, h, seed=500 + i, **kw))
        if rc != 0:
            continue
        n += 1
        a, b = reference.decode_status(pkt), product.decode_status(pkt)
        assert _same_decode(a, b), (w, h, ck, sb, tl)
        qa, qb = reference.query(pkt), product.query(pkt)
        assert qa[0] == qb[0] and bytes(qa[1]) == bytes(qb[1])
    assert n >= 40


def test_v8_decode_damaged_vs_reference(product, reference):
    """Segment streams changed with the tile CRC re-sealed (that segment alone
    is concealed), with the CRC stale (the tile is concealed), and bytes
    changed anywhere (structural rejects, bad tables, concealment)."""
    from v8_packets import layout, plane_blocks, reseal_tile
    rng = random.Random(77)
    for (w, h, sb, tl) in [(320, 180, 3, 4), (256, 144, 5, 0), (1920, 1080, 0, 0)]:
        cfg = _v8(B.make_config(w, h, qp=6, qmatrix_id=4), sb, tl)
        pkt = reference.encode(cfg, synth.make_frame_np(w, h, seed=12))
        lay = layout(pkt, plane_blocks(w, h, 0))
        for trial in range(30):
            p = bytearray(pkt)
            pl = lay[rng.randrange(3)]
            kind = trial % 3
            if kind < 2:
                t = rng.randrange(len(pl["tiles"]))
                sf, sn = pl["tiles"][t]
                if sn == sf:
                    continue
                for _ in range(rng.randint(1, 2)):
                    so, ln = pl["segs"][rng.randrange(sf, sn)]
                    p[pl["streams"] + so + rng.randrange(ln)] ^= 1 + rng.randrange(255)
                if kind == 0:
                    reseal_tile(p, pl, t)
            else:
                p[rng.randrange(53, len(p))] ^= 1 + rng.randrange(255)
            p = bytes(p)
            assert _same_decode(reference.decode_status(p), product.decode_status(p)), (w, h, trial)


def test_v8_decode_full_size_and_device_resident(product, reference):
    """3840x2160 HQ-like V8 frame: host packet and device-resident packet and
    planes decode like the reference."""
    import torch
    w, h = 3840, 2160
    cfg = _v8(B.make_config(w, h, qp=4, qmatrix_id=0), 0, 0)
    pkt = reference.encode(cfg, synth.make_frame_np(w, h, seed=3, frame=1))
    a, b = reference.decode_status(pkt), product.decode_status(pkt)
    assert _same_decode(a, b)
    dpkt = torch.from_numpy(np.frombuffer(pkt, dtype=np.uint8).copy()).cuda()
    planes = [torch.zeros(s, dtype=torch.int16, device="cuda") for s in B.plane_shapes(cfg)]
    import ctypes
    ptrs = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in planes], None)
    info = B.FrameOutput()
    rc = product._lib.tc_frame_decode(ctypes.c_void_p(dpkt.data_ptr()), len(pkt), ptrs, None, ctypes.byref(info))
    assert rc == 0 and info.concealed_slices == 0
    for x, y in zip(a.planes, planes):
        assert np.array_equal(x, y.cpu().numpy().view(np.uint16))


def test_v8_in_batch_decode_is_rejected_like_reference(product, reference):
    """tc_frame_decode_batch takes V7 packets only; a V8 packet fails the batch
    with the reference's status (its V7 scanner rejects major 8)."""
    cfg = _v8(B.make_config(128, 64, qp=8), 0, 0)
    pkt = reference.encode(cfg, synth.make_frame_np(128, 64, seed=1))
    ra, _ = reference.decode_batch([pkt])
    rb, _ = product.decode_batch([pkt])
    assert ra == rb == B.TC_ERR_UNSUPPORTED_VERSION


def test_v8_batch_decode_equals_single_calls(product, reference):
    """tcg_frame_decode_v8_batch: frames of several sizes and segment / tile
    layouts, one of them damaged, decode in one launch sequence exactly as
    tc_frame_decode (and the reference) decodes each alone; a V7 packet in the
    batch fails the call."""
    import ctypes
    from v8_packets import layout, plane_blocks
    specs = [(320, 180, 3, 4), (640, 360, 4, 5), (257, 131, 5, 0), (1920, 1080, 0, 0)]
    pkts = []
    for i, (w, h, sb, tl) in enumerate(specs):
        cfg = _v8(B.make_config(w, h, qp=5 + i, qmatrix_id=4), sb, tl)
        rc, pkt, _ = reference.encode_status(cfg, synth.make_frame_np(w, h, seed=900 + i))
        assert rc == 0
        pkts.append(pkt)
    bad = bytearray(pkts[1])
    pl = layout(pkts[1], plane_blocks(640, 360, 0))[0]
    so, ln = pl["segs"][3]
    bad[pl["streams"] + so + ln // 2] ^= 0x5A
    pkts[1] = bytes(bad)
    want = [reference.decode_status(p) for p in pkts]
    fn = product._lib.tcg_frame_decode_v8_batch
    fn.restype = ctypes.c_int32
    n = len(pkts)
    bufs = [np.frombuffer(p, dtype=np.uint8) for p in pkts]
    arr = (B.BatchPacket * n)()
    for i, b in enumerate(bufs):
        arr[i].data, arr[i].size = b.ctypes.data, b.size
    planes = [[np.zeros(x.shape, dtype=np.uint16) for x in wd.planes] for wd in want]
    ptrs = (ctypes.c_void_p * (4 * n))()
    for i in range(n):
        for p, a in enumerate(planes[i]):
            ptrs[4 * i + p] = a.ctypes.data
    infos = (B.FrameOutput * n)()
    assert fn(arr, n, ptrs, None, infos) == 0
    for i in range(n):
        assert infos[i].concealed_slices == want[i].info.concealed_slices
        assert list(infos[i].slice_status[:infos[i].slice_count]) == want[i].slice_status
        for a, b in zip(planes[i], want[i].planes):
            assert np.array_equal(a, b)
    assert want[1].info.concealed_slices > 0
    v7 = product.encode(B.make_config(64, 48, qp=8), synth.make_frame_np(64, 48, seed=1))
    b7 = np.frombuffer(v7, dtype=np.uint8)
    arr[0].data, arr[0].size = b7.ctypes.data, b7.size
    assert fn(arr, n, None, None, infos) == B.TC_ERR_UNSUPPORTED_VERSION


def test_v8_request_scaled_and_reduced_entries_vs_reference(product, reference):
    """A V8 packet through tc_frame_decode_request (every mode),
    tc_frame_decode_scaled and tc_frame_decode_reduced: the full decode where
    the reference has one, and otherwise its status and frame information."""
    import ctypes
    from test_gpu_decode_modes import _call_planes, _requests, _same
    cfg = _v8(B.make_config(320, 180, qp=7, qmatrix_id=4), 4, 5)
    pkt = reference.encode(cfg, synth.make_frame_np(320, 180, seed=77))
    rc, info = reference.query(pkt)
    assert rc == 0
    w, h = info.visible_width, info.visible_height
    for rl, req in _requests(w, h):
        _same(B.decode_request(product, pkt, req, fill=7), B.decode_request(reference, pkt, req, fill=7), rl)
    for tw, th in [((w + 1) // 2, (h + 1) // 2), (w, h)]:
        got = []
        for c in (product, reference):
            c._lib.tc_frame_decode_scaled.restype = ctypes.c_int32
            i2 = B.FrameOutput()
            i2.visible_width, i2.visible_height, i2.plane_count, i2.pixel_format = tw, th, info.plane_count, \
                info.pixel_format
            got.append(_call_planes(c._lib.tc_frame_decode_scaled, pkt, B.ToposCodec.geometry(i2),
                                    ctypes.c_uint32(tw), ctypes.c_uint32(th)))
        _same(got[0], got[1], ("scaled", tw, th))
        assert got[0].status == B.TC_ERR_NOT_IMPLEMENTED
    for s in range(0, 5):
        got = []
        for c in (product, reference):
            c._lib.tc_frame_decode_reduced.restype = ctypes.c_int32
            got.append(_call_planes(c._lib.tc_frame_decode_reduced, pkt, B.ToposCodec.geometry(info),
                                    ctypes.c_int32(s)))
        _same(got[0], got[1], ("reduced", s))
