"""The oracle is the checker, so it is pinned first: against the reference's
own golden conformance set, against fixtures produced by the reference
library, and by seeded differential runs against the reference library."""
import glob
import json
import os
import random
import struct
import subprocess
import zlib

import numpy as np
import pytest

from conftest import GOLDEN, REF_DIR, ROOT, reference_path
from topos_codec_b200 import binding as B, synth

REF_GOLDEN = reference_path("native", "tests", "conformance", "golden_codec_v7r2_intra.bin")


def _cases():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def _load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def test_reference_golden_set_on_oracle(built, tmp_path):
    """The reference's golden driver (golden_codec.c, intra-r2 set: 10/12-bit,
    4:2:2/4:4:4/GBR, alpha modes 1/2, 1x1) linked against the oracle."""
    objs = os.path.join(REF_DIR, "obj", "golden_codec.o")
    if not (os.path.exists(objs) and os.path.exists(REF_GOLDEN)):
        pytest.skip("reference golden driver or golden file not available")
    exe = str(tmp_path / "golden_on_oracle")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "golden-on",
                    f"LIB={os.path.join(ROOT, 'oracle', 'liboracle_tc.so')}", f"OUT={exe}"], check=True)
    r = subprocess.run([exe, "check", REF_GOLDEN, "intra-r2"], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "16 records byte-exact" in r.stdout


@pytest.mark.parametrize("case", [c["name"] for c in _cases()])
def test_oracle_matches_reference_fixture(oracle, case):
    meta = next(c for c in _cases() if c["name"] == case)
    z = _load(case)
    planes = [z[f"in{p}"] for p in range(meta["planes"])]
    cfg = B.make_config(meta["width"], meta["height"], **meta["config"])
    pkt, stats = oracle.encode_frame(cfg, planes)
    assert pkt == z["packet"].tobytes()
    assert stats == meta["stats"]
    dec = oracle.decode(z["packet"].tobytes())
    for p, a in enumerate(dec.planes):
        assert np.array_equal(a, z[f"dec{p}"])
    bad = oracle.decode_status(z["damaged"].tobytes(), fill=0)
    assert bad.status == meta["damaged_rc"]
    assert bad.slice_status == list(z["bad_status"])
    for p, a in enumerate(bad.planes):
        assert np.array_equal(a, z[f"bad{p}"])


def _random_config(rng):
    kind = rng.choice(["422", "422", "444", "gbr", "422_12", "422_16", "alpha"])
    w, h = rng.randint(1, 150), rng.randint(1, 90)
    kw, ck = {}, dict(qp=rng.choice([0, 2, 4, 8, 16, 30, 51, 63]), slice_rows=rng.choice([0, 1, 2, 3, 16]))
    if kind == "422":
        ck.update(qmatrix_id=rng.choice([0, 1, 3, 4]), features=rng.choice([0, 1, 2, 3]),
                  qp_delta_chroma=rng.choice([0, -2, 3]), qp_delta_luma=rng.choice([0, 1]))
    elif kind == "444":
        kw = {"pixel_format": 1}
        ck.update(pixel_format=1, qmatrix_id=rng.choice([0, 1]))
    elif kind == "gbr":
        kw = {"pixel_format": 2, "bit_depth": 12, "limited": False}
        ck.update(pixel_format=2, bit_depth=12, profile=5, qmatrix_id=rng.choice([0, 1, 2]), color_range=1)
    elif kind == "422_12":
        kw = {"bit_depth": 12}
        ck.update(bit_depth=12, qmatrix_id=1)
    elif kind == "422_16":
        kw = {"bit_depth": 16, "limited": False}
        ck.update(bit_depth=16, qp=rng.choice([20, 30, 60, 80]))
    else:
        am = rng.choice([1, 2])
        kw = {"alpha": True}
        ck.update(alpha_mode=am, alpha_bit_depth=16 if am == 1 else rng.choice([8, 10, 12]))
    return w, h, kw, ck


def test_oracle_differential_vs_reference(oracle, reference):
    rng = random.Random(20261203)
    for i in range(40):
        w, h, kw, ck = _random_config(rng)
        planes = synth.make_frame_np(w, h, seed=i, **kw)
        cfg = B.make_config(w, h, **ck)
        ra, pa, sa = reference.encode_status(cfg, planes)
        rb, pb, sb = oracle.encode_status(cfg, planes)
        assert ra == rb, (w, h, ck)
        if ra != 0:
            continue
        assert pa == pb, (w, h, ck)
        assert sa.as_dict() == sb.as_dict()
        da, db = reference.decode(pa), oracle.decode(pa)
        assert da.status == db.status
        assert all(np.array_equal(x, y) for x, y in zip(da.planes, db.planes))


def test_oracle_concealment_vs_reference(oracle, reference):
    rng = random.Random(7)
    w, h = 120, 64
    planes = synth.make_frame_np(w, h, seed=3, bit_depth=12, pixel_format=2, limited=False, alpha=True, sigma=12)
    cfg = B.make_config(w, h, qp=2, bit_depth=12, pixel_format=2, profile=5, alpha_mode=1, alpha_bit_depth=16,
                        color_range=1, slice_rows=2)
    pkt = reference.encode(cfg, planes)
    spans = []
    off = 53
    while off < len(pkt):
        size = struct.unpack(">I", pkt[off:off + 4])[0]
        spans.append((off, off + 17, size))
        off += 17 + size
    for trial in range(120):
        p = bytearray(pkt)
        ho, po, size = spans[rng.randrange(len(spans))]
        for _ in range(rng.randint(1, 3)):
            p[po + rng.randrange(size)] = rng.randrange(256)
        if trial % 2 == 0:
            p[ho + 13:ho + 17] = struct.pack(">I", zlib.crc32(bytes(p[po:po + size])) & 0xFFFFFFFF)
        p = bytes(p)
        da, db = reference.decode_status(p), oracle.decode_status(p)
        assert da.status == db.status
        assert da.slice_status == db.slice_status
        assert all(np.array_equal(x, y) for x, y in zip(da.planes, db.planes))


def _random_v8_config(rng):
    """A random V8 configuration: colour only (V8 carries no alpha and no CFA),
    segment granularity 8/16/32 blocks (reserved[3]) and tile heights whole
    plane / 16 / 32 / 64 block rows (reserved[4])."""
    w, h = rng.randint(1, 200), rng.randint(1, 120)
    pf = rng.choice([0, 0, 1, 2])
    bd = rng.choice([10, 10, 12, 16])
    ck = dict(qp=rng.choice([0, 2, 4, 8, 16, 30, 45, 63, 80]), pixel_format=pf, bit_depth=bd,
              profile=3 if pf == 0 else 5, qmatrix_id=rng.choice([0, 1, 2, 3]) if bd == 10 else 0)
    if bd == 16:
        ck["qp"] = rng.choice([30, 60, 80])
    if pf == 2:
        ck.update(color_range=1)
    kw = dict(bit_depth=bd, pixel_format=pf, limited=pf != 2)
    return w, h, kw, ck, rng.choice([0, 3, 4, 5]), rng.choice([0, 4, 5, 6])


def _v8(cfg, sb, tl):
    cfg.reserved[0] = 9
    cfg.reserved[3] = sb
    cfg.reserved[4] = tl
    return cfg


def _same_decode(a, b):
    return (a.status == b.status and a.slice_status == b.slice_status
            and a.info.concealed_slices == b.info.concealed_slices
            and all(np.array_equal(x, y) for x, y in zip(a.planes, b.planes)))


def test_oracle_v8_differential_vs_reference(oracle, reference):
    """V8 segmented rANS (reserved[0] = 9): packets, statistics and decoded
    planes equal the reference library's on random geometry, formats, QPs,
    segment sizes and tile heights."""
    rng = random.Random(8008)
    coded = 0
    for i in range(60):
        w, h, kw, ck, sb, tl = _random_v8_config(rng)
        planes = synth.make_frame_np(w, h, seed=100 + i, **kw)
        cfg = _v8(B.make_config(w, h, **ck), sb, tl)
        ra, pa, sa = reference.encode_status(cfg, planes)
        rb, pb, sbb = oracle.encode_status(cfg, planes)
        assert ra == rb, (w, h, ck, sb, tl)
        if ra != 0:
            continue
        coded += 1
        assert pa == pb, (w, h, ck, sb, tl)
        assert sa.as_dict() == sbb.as_dict()
        assert _same_decode(reference.decode_status(pa), oracle.decode_status(pa))
        ia, ib = reference.query(pa), oracle.query(pa)
        assert ia[0] == ib[0] and bytes(ia[1]) == bytes(ib[1])
    assert coded >= 40


def test_oracle_v8_concealment_vs_reference(oracle, reference):
    """Damaged V8 packets: bytes changed in a segment stream with the tile CRC
    re-sealed (the segment's own decode fails: that segment is concealed), with
    the CRC left stale (the whole tile is concealed), and in the directory or
    tables (structural rejects or tile-level failures): same status, per-tile
    status, concealed count and planes as the reference."""
    from v8_packets import layout, plane_blocks, reseal_tile
    rng = random.Random(88)
    w, h = 160, 96
    cfg = _v8(B.make_config(w, h, qp=4, qmatrix_id=4), 3, 4)
    pkt = reference.encode(cfg, synth.make_frame_np(w, h, seed=9))
    lay = layout(pkt, plane_blocks(w, h, 0))
    for trial in range(90):
        p = bytearray(pkt)
        pl = lay[rng.randrange(3)]
        kind = trial % 3
        if kind < 2:
            t = rng.randrange(len(pl["tiles"]))
            sf, sn = pl["tiles"][t]
            if sn == sf:
                continue
            so, ln = pl["segs"][rng.randrange(sf, sn)]
            p[pl["streams"] + so + rng.randrange(ln)] ^= 1 + rng.randrange(255)
            if kind == 0:
                reseal_tile(p, pl, t)
        else:
            p[rng.randrange(53, len(p))] ^= 1 + rng.randrange(255)
        p = bytes(p)
        assert _same_decode(reference.decode_status(p), oracle.decode_status(p)), trial
