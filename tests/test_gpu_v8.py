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
