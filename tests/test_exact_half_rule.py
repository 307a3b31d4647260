"""The exact-half delivery rule that the GPU decimation follows, checked on the
reference library alone (CPU, no GPU): the reference's half-size output must
equal its own full-size decode sampled by the rule.

Rule (reference color_store.h:538-559, transform_avx2.c:528-570): a colour
plane delivered at exactly half its size on both axes is stored per 8x8 block
as nx x ny target samples, of which only the first nx*ny entries of a 4-wide
row-major array are computed before entry iy*4 + ix is read. In a right-edge
block narrower than 8 pixels the entries at or past nx*ny keep older values:
the sample one block to the left in planes wider than a block; in planes one
block wide, the sample one block row up when the partial last block row
shares a slice band with it, else a zero residual (the mid-level sample)."""
import random

import numpy as np
import pytest

from test_oracle import _random_config
from topos_codec_b200 import binding as B, synth


def _rule(full, tw, th, mid, last_row_shares_band):
    vh, vw = full.shape
    out = np.empty((th, tw), np.int64)
    exact = tw * 2 == vw and th * 2 == vh
    for ty in range(th):
        for tx in range(tw):
            sy, sx = ty * vh // th, tx * vw // tw
            v = int(full[sy, sx])
            if exact:
                px0, py0 = (tx >> 2) * 8, (ty >> 2) * 8
                nx, ny = min(8, vw - px0) // 2, min(8, vh - py0) // 2
                k = (ty & 3) * 4 + (tx & 3)
                if nx < 4 and k >= nx * ny:
                    if vw > 8:
                        v = int(full[sy, sx - 8])
                    elif last_row_shares_band and ny < 4 and k < 4 * nx:
                        v = int(out[ty - 4, tx])
                    else:
                        v = mid
            out[ty, tx] = v
    return out


def _check(reference, w, h, ck, kw, shares):
    planes = synth.make_frame_np(w, h, seed=w * 131 + h, **kw)
    pkt = reference.encode(B.make_config(w, h, **ck), planes)
    full = B.decode_request(reference, pkt, B.make_request(0), fill=7)
    half = B.decode_request(reference, pkt, B.make_request(1, target=((w + 1) // 2, (h + 1) // 2)), fill=7)
    assert full.status == 0 and half.status == 0
    mid = 1 << (ck.get("bit_depth", 10) - 1)
    affected = 0
    for p in range(3):
        f, g = full.planes[p], half.planes[p]
        expect = _rule(f, g.shape[1], g.shape[0], mid, shares)
        plain = f[np.ix_(np.arange(g.shape[0]) * f.shape[0] // g.shape[0],
                         np.arange(g.shape[1]) * f.shape[1] // g.shape[1])]
        affected += int(not np.array_equal(expect, plain))
        assert np.array_equal(expect, g), (w, h, ck, p)
    return affected


def test_exact_half_rule_wide_planes(reference):
    rng = random.Random(5)
    affected = 0
    for _ in range(40):
        w, h, kw, ck = _random_config(rng)
        w, h = rng.randint(9, 160), rng.randint(9, 120)
        ck["features"] = ck.get("features", 0) & ~1  # no deblocking: samples are the stored ones
        affected += _check(reference, w, h, ck, kw, True)
    assert affected > 0  # the rule was exercised, not only plain sampling


@pytest.mark.parametrize("w,h,slice_rows,shares", [(12, 40, 1, False), (6, 44, 1, False), (4, 28, 1, False),
                                                   (6, 44, 2, True), (6, 60, 4, True)])
def test_exact_half_rule_one_block_wide(reference, w, h, slice_rows, shares):
    assert _check(reference, w, h, dict(qp=8, slice_rows=slice_rows), {}, shares) > 0
