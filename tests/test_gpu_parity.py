"""GPU parity through the C-ABI: packets byte-identical to the oracle and to the
reference fixtures, decoded pixels and per-slice concealment identical."""
import json
import os
import random
import struct
import zlib

import numpy as np
import pytest

from conftest import GOLDEN
from test_oracle import _random_config
from topos_codec_b200 import binding as B, synth

pytestmark = pytest.mark.gpu


def _cases():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", [c["name"] for c in _cases()])
def test_fixture_encode_decode(product, case):
    meta = next(c for c in _cases() if c["name"] == case)
    z = np.load(os.path.join(GOLDEN, f"{case}.npz"))
    planes = [z[f"in{p}"] for p in range(meta["planes"])]
    cfg = B.make_config(meta["width"], meta["height"], **meta["config"])
    pkt, stats = product.encode_frame(cfg, planes)
    assert pkt == z["packet"].tobytes()
    assert stats == meta["stats"]
    dec = product.decode(z["packet"].tobytes())
    assert dec.status == 0
    for p, a in enumerate(dec.planes):
        assert np.array_equal(a, z[f"dec{p}"]), p
    bad = product.decode_status(z["damaged"].tobytes(), fill=0)
    assert bad.status == meta["damaged_rc"]
    assert bad.slice_status == list(z["bad_status"])
    for p, a in enumerate(bad.planes):
        assert np.array_equal(a, z[f"bad{p}"]), p


def test_random_configs_vs_oracle(product, oracle):
    rng = random.Random(99)
    for i in range(60):
        w, h, kw, ck = _random_config(rng)
        planes = synth.make_frame_np(w, h, seed=500 + i, **kw)
        cfg = B.make_config(w, h, **ck)
        ra, pa, sa = oracle.encode_status(cfg, planes)
        rb, pb, sb = product.encode_status(cfg, planes)
        assert ra == rb, (i, w, h, ck, product.last_error())
        if ra != 0:
            continue
        assert pa == pb, (i, w, h, ck)
        assert sa.as_dict() == sb.as_dict()
        da, db = oracle.decode(pa), product.decode(pa)
        assert da.status == db.status
        for x, y in zip(da.planes, db.planes):
            assert np.array_equal(x, y), (i, w, h, ck)


def _spans(pkt):
    off, out = 53, []
    while off < len(pkt):
        size = struct.unpack(">I", pkt[off:off + 4])[0]
        out.append((off, off + 17, size))
        off += 17 + size
    return out


def test_damaged_packets_vs_oracle(product, oracle):
    rng = random.Random(3)
    for case in range(2):
        if case == 0:
            w, h = 160, 96
            planes = synth.make_frame_np(w, h, seed=31, bit_depth=12, pixel_format=2, limited=False, alpha=True, sigma=12)
            cfg = B.make_config(w, h, qp=2, bit_depth=12, pixel_format=2, profile=5, alpha_mode=1, alpha_bit_depth=16,
                                color_range=1, slice_rows=2)
        else:
            w, h = 256, 128
            planes = synth.make_frame_np(w, h, seed=32)
            cfg = B.make_config(w, h, qp=8, qmatrix_id=4, features=1, slice_rows=2)
        pkt = oracle.encode(cfg, planes)
        spans = _spans(pkt)
        for trial in range(80):
            p = bytearray(pkt)
            ho, po, size = spans[rng.randrange(len(spans))]
            for _ in range(rng.randint(1, 3)):
                p[po + rng.randrange(size)] = rng.randrange(256)
            if trial % 2 == 0:
                p[ho + 13:ho + 17] = struct.pack(">I", zlib.crc32(bytes(p[po:po + size])) & 0xFFFFFFFF)
            p = bytes(p)
            da, db = oracle.decode_status(p), product.decode_status(p)
            assert da.status == db.status, trial
            assert da.slice_status == db.slice_status, trial
            for x, y in zip(da.planes, db.planes):
                assert np.array_equal(x, y), trial


def test_1080p_422_deblock_roundtrip(product, oracle):
    """1920x1080 10-bit 4:2:2, qp 8, edge-balanced matrix, deblock."""
    planes = synth.make_frame_np(1920, 1080, seed=0)
    cfg = B.make_config(1920, 1080, qp=8, qmatrix_id=4, features=1)
    pa = oracle.encode(cfg, planes)
    pb = product.encode(cfg, planes)
    assert pa == pb
    da, db = oracle.decode(pa), product.decode(pa)
    for x, y in zip(da.planes, db.planes):
        assert np.array_equal(x, y)


def test_4k_422_hq_full_size(product, oracle):
    """3840x2160 10-bit 4:2:2 HQ (qp 4, flat matrix, deblock + refined table)."""
    planes = synth.make_frame_np(3840, 2160, seed=1, frame=7)
    cfg = B.make_config(3840, 2160, qp=4, qmatrix_id=0, features=3)
    pa = oracle.encode(cfg, planes)
    pb = product.encode(cfg, planes)
    assert pa == pb
    da, db = oracle.decode(pa), product.decode(pa)
    for x, y in zip(da.planes, db.planes):
        assert np.array_equal(x, y)


def test_batch_encode_equals_single(product):
    sizes = [(1280, 720), (64, 48), (1920, 1080), (333, 77)]
    cfgs, frames = [], []
    for i, (w, h) in enumerate(sizes):
        frames.append(synth.make_frame_np(w, h, seed=60 + i))
        cfgs.append(B.make_config(w, h, qp=2 + 4 * i, qmatrix_id=4 if i % 2 else 0, features=1 + (i % 2)))
    rc, pkts, rcs, stats = product.encode_batch(cfgs, frames)
    assert rc == 0 and rcs == [0] * len(sizes)
    for c, f, p in zip(cfgs, frames, pkts):
        assert p == product.encode(c, f)


def test_batch_decode_equals_single(product):
    pkts = []
    for i, (w, h) in enumerate([(640, 360), (96, 64), (1920, 1080)]):
        pkts.append(product.encode(B.make_config(w, h, qp=6, qmatrix_id=4, features=1), synth.make_frame_np(w, h, seed=70 + i)))
    rc, frames = product.decode_batch(pkts)
    assert rc == 0
    for p, f in zip(pkts, frames):
        d = product.decode(p)
        for x, y in zip(d.planes, f.planes):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("chunks", ["2", "3", "4"])
def test_pipelined_host_batches_vs_oracle(product, oracle, monkeypatch, chunks):
    """Host-memory batches split into chunks on separate contexts and streams
    (TCG_PIPELINE forces the split that large batches get by size): packets
    byte-identical to the oracle, pixels and per-slice concealment of a batch
    holding damaged packets identical to the oracle's."""
    sizes = [(1280, 720), (64, 48), (1920, 1080), (333, 77), (640, 360), (256, 128)]
    cfgs, frames = [], []
    for i, (w, h) in enumerate(sizes):
        frames.append(synth.make_frame_np(w, h, seed=80 + i))
        cfgs.append(B.make_config(w, h, qp=2 + 3 * i, qmatrix_id=4 if i % 2 else 0, features=1 + (i % 2), slice_rows=2))
    monkeypatch.setenv("TCG_PIPELINE", chunks)
    rc, pkts, rcs, _ = product.encode_batch(cfgs, frames)
    assert rc == 0 and rcs == [0] * len(sizes)
    for c, f, p in zip(cfgs, frames, pkts):
        assert p == oracle.encode(c, f)
    rng = random.Random(int(chunks))
    batch = list(pkts)
    for k in (1, 4):  # one damaged payload byte in two of the packets
        p = bytearray(batch[k])
        _, po, size = _spans(batch[k])[rng.randrange(len(_spans(batch[k])))]
        p[po + rng.randrange(size)] ^= 0x5A
        batch[k] = bytes(p)
    rc, got = product.decode_batch(batch)
    assert rc in (B.TC_OK, B.TC_WARN_CONCEALED)
    for p, f in zip(batch, got):
        want = oracle.decode_status(p)
        assert want.status in (B.TC_OK, B.TC_WARN_CONCEALED)
        assert f.info.concealed_slices == sum(1 for s in want.slice_status if s != 0)
        for x, y in zip(want.planes, f.planes):
            assert np.array_equal(x, y)


def test_device_resident_encode_decode(product):
    """Device pointers for samples, packets and output planes (no host staging):
    same packet and pixels as the host-memory path, including a damaged packet
    parsed from its device-walked headers."""
    import ctypes

    import torch
    w, h = 640, 360
    planes = synth.make_frame_np(w, h, seed=9)
    cfg = B.make_config(w, h, qp=6, qmatrix_id=4, features=1)
    host_pkt = product.encode(cfg, planes)
    dev = [torch.from_numpy(p.astype(np.int32)).cuda().to(torch.uint16) for p in planes]
    fi = B.FrameInput()
    fi.struct_size, fi.abi_version = ctypes.sizeof(B.FrameInput), 2
    for i, t in enumerate(dev):
        fi.planes[i], fi.strides[i] = t.data_ptr(), t.shape[1]
    out = torch.zeros(2 * len(host_pkt), dtype=torch.uint8, device="cuda")
    st = B.FrameStats()
    rc = product._lib.tc_frame_encode(ctypes.byref(cfg), ctypes.byref(fi), ctypes.c_void_p(out.data_ptr()),
                                      out.numel(), ctypes.byref(st))
    assert rc == 0 and out[: st.packet_size].cpu().numpy().tobytes() == host_pkt
    ref = product.decode(host_pkt)
    for pkt_bytes, want_status in ((host_pkt, 0), (host_pkt[:-1], B.TC_ERR_MALFORMED)):
        dpkt = torch.from_numpy(np.frombuffer(pkt_bytes, dtype=np.uint8).copy()).cuda()
        outs = [torch.zeros(p.shape, dtype=torch.uint16, device="cuda") for p in ref.planes]
        ptrs = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in outs], None)
        info = B.FrameOutput()
        rc = product._lib.tc_frame_decode(ctypes.c_void_p(dpkt.data_ptr()), len(pkt_bytes), ptrs, None,
                                          ctypes.byref(info))
        hrc, _ = product.query(pkt_bytes)
        assert rc == (0 if hrc == 0 else hrc)
        if want_status == 0:
            for a, b in zip(outs, ref.planes):
                assert np.array_equal(a.cpu().numpy(), b)


def test_strided_io_and_buffer_too_small(product):
    w, h = 200, 120
    planes = synth.make_frame_np(w, h, seed=5)
    cfg = B.make_config(w, h, qp=8, qmatrix_id=4, features=1)
    tight = product.encode(cfg, planes)
    padded = []
    for a in planes:
        big = np.full((a.shape[0], a.shape[1] + 37), 7, dtype=np.uint16)
        big[:, : a.shape[1]] = a
        padded.append(big[:, : a.shape[1]])
    assert product.encode(cfg, padded) == tight
    rc, pkt, st = product.encode_status(cfg, planes, out_cap=len(tight) - 1)
    assert rc == B.TC_ERR_BUFFER_TOO_SMALL and st.packet_size == len(tight)


@pytest.mark.parametrize("tiling", ["lane", "lane4", "lane2", "lane1", "warp", "split"])
def test_decode_tilings_vs_oracle(product, oracle, monkeypatch, tiling):
    """Every decode-chain tiling (lane per slice with 8/4/2/1 slices per warp,
    warp per slice, the two-stream split) decodes random configurations and
    damaged packets exactly like the oracle."""
    monkeypatch.setenv("TCG_DCHAIN", tiling)
    rng = random.Random(123)
    pkts = []
    for i in range(16):
        w, h, kw, ck = _random_config(rng)
        rc, pkt, _ = oracle.encode_status(B.make_config(w, h, **ck), synth.make_frame_np(w, h, seed=700 + i, **kw))
        if rc == 0:
            pkts.append(pkt)
    for pkt in list(pkts[:8]):
        spans = _spans(pkt)
        for _ in range(4):
            p = bytearray(pkt)
            ho, po, size = spans[rng.randrange(len(spans))]
            p[po + rng.randrange(size)] ^= 1 + rng.randrange(255)
            p[ho + 13:ho + 17] = struct.pack(">I", zlib.crc32(bytes(p[po:po + size])) & 0xFFFFFFFF)
            pkts.append(bytes(p))
    for pkt in pkts:
        da, db = oracle.decode_status(pkt), product.decode_status(pkt)
        assert da.status == db.status
        assert da.slice_status == db.slice_status
        for x, y in zip(da.planes, db.planes):
            assert np.array_equal(x, y)
    rc, frames = product.decode_batch(pkts[:16])
    for pkt, f in zip(pkts[:16], frames):
        d = oracle.decode_status(pkt)
        for x, y in zip(d.planes, f.planes):
            assert np.array_equal(x, y)


def test_mixed_tier_batch_vs_oracle(product, oracle):
    """A batch mixing resolutions, tiers (the product's tier mapping) and QPs
    encodes and decodes exactly like the oracle, frame by frame."""
    from topos_codec_b200 import workloads as WL
    specs = [(1280, 720, "proxy", 16), (1920, 1080, "hq", 2), (3840, 2160, "422", 9), (1280, 720, "lt", 5),
             (3840, 2160, "hq", 4)]
    cfgs = [WL.mixed_config(*s) for s in specs]
    frames = [synth.make_frame_np(w, h, seed=90 + i) for i, (w, h, _, _) in enumerate(specs)]
    rc, pkts, rcs, _ = product.encode_batch(cfgs, frames)
    assert rc == 0 and rcs == [0] * len(specs)
    for c, f, p in zip(cfgs, frames, pkts):
        assert p == oracle.encode(c, f)
    rc, dec = product.decode_batch(pkts)
    assert rc == 0
    for p, d in zip(pkts, dec):
        o = oracle.decode(p)
        for x, y in zip(o.planes, d.planes):
            assert np.array_equal(x, y)


def test_gbr4444_alpha_full_size_damaged_vs_oracle(product, oracle):
    """4096x2160 12-bit GBR 4:4:4 with a 16-bit alpha plane at qp 2: identical
    packet, then damaged copies (1 % of the slices, one payload byte each)
    decode with the oracle's per-slice concealment status and pixels."""
    from topos_codec_b200 import workloads as WL
    cfg = WL.gbr_config()
    planes = synth.make_frame_np(4096, 2160, seed=21, bit_depth=12, pixel_format=2, limited=False, alpha=True,
                                 sigma=12)
    pkt = product.encode(cfg, planes)
    assert pkt == oracle.encode(cfg, planes)
    for seed in range(3):
        bad = WL.corrupt_slices([pkt], 0.01, seed=seed)[0]
        d, o = product.decode_status(bad), oracle.decode_status(bad)
        assert d.status == o.status and d.slice_status == o.slice_status
        assert any(s != 0 for s in o.slice_status)
        for x, y in zip(o.planes, d.planes):
            assert np.array_equal(x, y)
