"""Full-size frames of the benchmark workloads checked against the reference
library itself (oracle/_ref, built from the reference's own sources), not only
against the oracle restatement; and the reference's own C conformance driver
(golden_codec.c) linked against the GPU library, so a C program calls this
library through the C ABI exactly as it calls the reference.

Parity bar: packets byte-identical, decoded planes bit-identical, the same
statuses and per-slice concealment results."""
import os
import random
import struct
import subprocess

import numpy as np
import pytest

from conftest import REF_DIR, ROOT
from topos_codec_b200 import binding as B, synth

pytestmark = pytest.mark.gpu

GOLDEN_BIN = os.path.join(REF_DIR, "golden_codec_v7r2_intra.bin")


def _roundtrip_vs_reference(product, reference, cfg, planes):
    pr = reference.encode(cfg, planes)
    pg = product.encode(cfg, planes)
    assert pg == pr, "GPU packet differs from the reference library's"
    dr, dg = reference.decode(pr), product.decode(pr)
    assert dr.status == dg.status == 0
    for x, y in zip(dr.planes, dg.planes):
        assert np.array_equal(x, y)
    return pr


def test_1080p_qp8_qm4_deblock_vs_reference(product, reference):
    """The CPU-runnable workload: one 1920x1080 10-bit 4:2:2 frame, qp 8,
    quant matrix 4, DEBLOCK, default slices."""
    planes = synth.make_frame_np(1920, 1080, seed=0)
    cfg = B.make_config(1920, 1080, qp=8, qmatrix_id=4, features=1)
    _roundtrip_vs_reference(product, reference, cfg, planes)


def test_4k_hq_frames_vs_reference(product, reference):
    """Three frames of the 3840x2160 HQ benchmark batch (qp 4, flat matrix,
    DEBLOCK | QPT2), batched on the GPU, each against the reference's own
    single-frame encode and decode."""
    cfg = B.make_config(3840, 2160, qp=4, qmatrix_id=0, features=3)
    idx = [0, 29, 59]
    frames = [synth.make_frame_np(3840, 2160, seed=0, frame=i) for i in idx]
    rc, pk, rcs, _ = product.encode_batch([cfg] * len(frames), frames)
    assert rc == 0 and rcs == [0] * len(frames)
    for planes, pg in zip(frames, pk):
        pr = reference.encode(cfg, planes)
        assert pg == pr
    rc, dec = product.decode_batch(pk)
    assert rc == 0
    for pg, dg in zip(pk, dec):
        dr = reference.decode(pg)
        assert dr.status == 0
        for x, y in zip(dr.planes, dg.planes):
            assert np.array_equal(x, y)


def test_4k_hq_damaged_vs_reference(product, reference):
    """Reference packets of a 4K HQ frame with payload bytes changed in 1 % of
    the slices (at least two): same status, per-slice concealment and pixels."""
    cfg = B.make_config(3840, 2160, qp=4, qmatrix_id=0, features=3)
    pr = reference.encode(cfg, synth.make_frame_np(3840, 2160, seed=0, frame=3))
    spans, off = [], 53
    while off < len(pr):
        size = struct.unpack(">I", pr[off:off + 4])[0]
        spans.append((off + 17, size))
        off += 17 + size
    rng = random.Random(9)
    for trial in range(2):
        p = bytearray(pr)
        for po, size in rng.sample(spans, 2):
            p[po + rng.randrange(size)] ^= 1 + rng.randrange(255)
        p = bytes(p)
        dr, dg = reference.decode_status(p), product.decode_status(p)
        assert dr.status == dg.status == 1, trial
        assert dr.slice_status == dg.slice_status
        for x, y in zip(dr.planes, dg.planes):
            assert np.array_equal(x, y)


def test_reference_golden_driver_on_gpu_library(built, tmp_path):
    """The reference's C conformance driver (intra-r2 golden set: 10/12-bit,
    4:2:2/4:4:4/GBR, alpha modes 1/2) linked against the GPU library."""
    if not (os.path.exists(GOLDEN_BIN) and os.path.exists(os.path.join(REF_DIR, "obj", "golden_codec.o"))):
        pytest.skip("reference golden driver not built (oracle/_ref)")
    exe = str(tmp_path / "golden_on_gpu")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "golden-on",
                    f"LIB={B.PRODUCT_LIBRARY}", f"OUT={exe}"], check=True)
    r = subprocess.run([exe, "check", GOLDEN_BIN, "intra-r2"], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "16 records byte-exact" in r.stdout
