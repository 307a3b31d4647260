"""Generate the committed golden fixtures from the reference library.

Run in a checkout that has the reference sources built into oracle/_ref
(`make -C oracle ref`):

    python tests/golden/make_golden.py

Each case stores its config, the input planes, the reference packet, the
reference decode of that packet, and - for damaged-packet cases - the damaged
packet with the reference's per-slice concealment status and pixels. The
fixtures are small (<= 96x64) so the CPU suite and the GPU parity tests can
compare against them without the reference being present.
"""
from __future__ import annotations

import json
import os
import random
import struct
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from topos_codec_b200 import binding as B, synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "libtopos_codec_ref.so")

# (name, width, height, synth kwargs, config kwargs)
CASES = [
    ("yuv422_10_qp8_qm4_deblock", 96, 64, {}, dict(qp=8, qmatrix_id=4, features=1)),
    ("yuv422_10_qp4_qm0_deblock_qpt2", 96, 64, {}, dict(qp=4, qmatrix_id=0, features=3)),
    ("yuv422_10_qp30_odd", 73, 39, {}, dict(qp=30, qmatrix_id=1, slice_rows=2)),
    ("yuv422_12_qp20", 64, 48, {"bit_depth": 12}, dict(qp=20, bit_depth=12, qmatrix_id=1)),
    ("yuv444_10_qp12", 48, 40, {"pixel_format": 1}, dict(qp=12, pixel_format=1)),
    ("gbr444_12_alpha16_qp2", 64, 48, {"bit_depth": 12, "pixel_format": 2, "limited": False, "alpha": True, "sigma": 12},
     dict(qp=2, bit_depth=12, pixel_format=2, profile=5, alpha_mode=1, alpha_bit_depth=16, color_range=1)),
    ("yuv444_12_alpha10_qp70", 56, 40, {"bit_depth": 12, "pixel_format": 1, "alpha": True},
     dict(qp=70, bit_depth=12, pixel_format=1, alpha_mode=2, alpha_bit_depth=10, slice_rows=3)),
    ("yuv422_16_qp24", 40, 24, {"bit_depth": 16, "limited": False}, dict(qp=24, bit_depth=16)),
    ("yuv422_10_tiny_1x1", 1, 1, {}, dict(qp=0)),
    ("yuv422_10_high_qp90", 96, 64, {}, dict(qp=90, qmatrix_id=1, qp_delta_chroma=3)),
]


def slice_spans(pkt: bytes):
    off, out = 53, []
    while off < len(pkt):
        size = struct.unpack(">I", pkt[off:off + 4])[0]
        out.append((off, off + 17, size))
        off += 17 + size
    return out


def damage(pkt: bytes, seed: int) -> bytes:
    """Corrupt payload bytes of ~1/3 of the slices; half of them keep a valid
    CRC so the entropy decoder itself must detect (or survive) the damage."""
    rng = random.Random(seed)
    p = bytearray(pkt)
    for k, (ho, po, size) in enumerate(slice_spans(pkt)):
        if size == 0 or rng.random() > 0.34:
            continue
        for _ in range(rng.randint(1, 3)):
            p[po + rng.randrange(size)] = rng.randrange(256)
        if k % 2 == 0:
            p[ho + 13:ho + 17] = struct.pack(">I", zlib.crc32(bytes(p[po:po + size])) & 0xFFFFFFFF)
    return bytes(p)


def main() -> None:
    ref = B.ToposCodec(REF)
    index = []
    for i, (name, w, h, skw, ckw) in enumerate(CASES):
        planes = synth.make_frame_np(w, h, seed=1000 + i, **skw)
        cfg = B.make_config(w, h, **ckw)
        pkt, stats = ref.encode_frame(cfg, planes)
        dec = ref.decode(pkt)
        bad = damage(pkt, 77 + i)
        dd = ref.decode_status(bad, fill=0)
        arrays = {f"in{p}": a for p, a in enumerate(planes)}
        arrays.update({f"dec{p}": a for p, a in enumerate(dec.planes)})
        arrays.update({f"bad{p}": a for p, a in enumerate(dd.planes)})
        arrays["packet"] = np.frombuffer(pkt, dtype=np.uint8)
        arrays["damaged"] = np.frombuffer(bad, dtype=np.uint8)
        arrays["bad_status"] = np.array(dd.slice_status, dtype=np.uint8)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        index.append({"name": name, "width": w, "height": h, "config": ckw, "stats": stats,
                      "damaged_rc": dd.status, "planes": len(planes)})
        print(name, len(pkt), "bytes; damaged rc", dd.status, "concealed", sum(dd.slice_status))
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1)


if __name__ == "__main__":
    main()
