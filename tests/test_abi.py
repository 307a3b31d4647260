"""The C-ABI boundary, checked without a GPU: the library loads and exports
every symbol the public header declares, struct layouts match the reference
ABI, and the host-side rules (config validation, packet bound, structural
packet parse) agree with the oracle status for status."""
import ctypes
import os
import random
import re
import struct
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, reference_path
from topos_codec_b200 import binding as B, synth

HEADER = os.path.join(ROOT, "include", "topos_codec.h")
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include"))) if f.endswith(".h")]
REF_HEADER = reference_path("native", "include", "topos_codec.h")


def _declared_functions():
    text = "\n".join(open(h).read() for h in HEADERS)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:tc|tcg)_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(built):
    out = subprocess.run(["nm", "-D", "--defined-only", B.PRODUCT_LIBRARY], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    declared = _declared_functions()
    assert declared, "no declarations parsed"
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    # nothing internal leaks out of the library
    extra = [s for s in exported if not (s.startswith("tc_") or s.startswith("tcg_"))]
    assert not extra, extra


def test_library_loads_and_answers_queries(product):
    L = product._lib
    assert L.tc_abi_version() == 2
    caps = (ctypes.c_uint32 * 10)()
    assert L.tc_query_capabilities(caps) == 0
    assert caps[0] == 40 and caps[3] == 16384 and (caps[2] & 1) == 1
    L.tc_status_message.restype = ctypes.c_char_p
    assert L.tc_status_message(ctypes.c_int32(1)).startswith(b"concealment")
    assert L.tc_status_message(ctypes.c_int32(-99)) == b"unknown status"
    assert L.tc_query_support(3, 0, 10, 0) == 0
    assert L.tc_query_support(7, 0, 12, 0) == -5
    assert L.tc_query_support(4, 0, 10, 0) == -4
    assert L.tc_query_support(3, 0, 10, 3) == -7


LAYOUT_PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "topos_codec.h"
#define P(T, F) printf(#T "." #F " %zu\n", offsetof(T, F))
int main(void) {
  printf("cfg %zu in %zu st %zu out %zu bp %zu ver %zu caps %zu\n", sizeof(topos_frame_config),
         sizeof(topos_frame_input), sizeof(topos_frame_stats), sizeof(topos_frame_output),
         sizeof(topos_batch_packet), sizeof(topos_version_info), sizeof(topos_codec_capabilities));
  P(topos_frame_config, qp_base); P(topos_frame_config, sar_num); P(topos_frame_config, reserved);
  P(topos_frame_input, strides); P(topos_frame_stats, slice_count); P(topos_frame_stats, alpha_max_abs_error);
  P(topos_frame_output, concealed_slices); P(topos_frame_output, slice_status); P(topos_frame_output, reserved);
  return 0;
}
"""


def _layout(include_dir, tmp_path, tag):
    src = tmp_path / f"probe_{tag}.c"
    exe = tmp_path / f"probe_{tag}"
    src.write_text(LAYOUT_PROBE)
    subprocess.run(["gcc", "-std=c11", f"-I{include_dir}", str(src), "-o", str(exe)], check=True)
    return subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout


def test_struct_layouts(tmp_path):
    mine = _layout(os.path.dirname(HEADER), tmp_path, "mine")
    sizes = dict(zip(mine.split()[0:14:2], map(int, mine.split()[1:14:2])))
    assert sizes["cfg"] == ctypes.sizeof(B.FrameConfig)
    assert sizes["in"] == ctypes.sizeof(B.FrameInput)
    assert sizes["st"] == ctypes.sizeof(B.FrameStats)
    assert sizes["out"] == ctypes.sizeof(B.FrameOutput)
    if os.path.exists(REF_HEADER):
        assert mine == _layout(os.path.dirname(REF_HEADER), tmp_path, "ref")


def _rand_cfg(rng):
    c = B.make_config(rng.choice([0, 1, 7, 64, 1920, 16384, 16385]), rng.choice([0, 1, 9, 1080, 16384]),
                      qp=rng.choice([0, 8, 63, 64, 95, 96]), qmatrix_id=rng.choice([0, 1, 2, 3, 4, 5]),
                      pixel_format=rng.choice([0, 0, 1, 2, 3, 4]), bit_depth=rng.choice([0, 10, 12, 16, 8]),
                      profile=rng.choice([0, 3, 3, 5, 6, 7, 2]), slice_rows=rng.choice([0, 1, 2, 16, 255]),
                      alpha_mode=rng.choice([0, 0, 1, 2, 3]), alpha_bit_depth=rng.choice([0, 8, 10, 16]),
                      features=rng.choice([0, 1, 2, 3, 4]), color_matrix=rng.choice([0, 1, 5, 2]),
                      color_range=rng.choice([0, 1, 2]), chroma_siting=rng.choice([0, 1, 3]),
                      coding=rng.choice([8, 8, 8, 0, 1, 3, 9, 10, 12]))
    c.reserved[1] = rng.choice([0, 0, 0, 1, 2])
    c.reserved[3] = rng.choice([0, 0, 0, 1])
    c.struct_size = rng.choice([ctypes.sizeof(B.FrameConfig)] * 8 + [0, 12])
    return c


def test_config_validation_matches_oracle(product, oracle):
    rng = random.Random(11)
    seen = set()
    for _ in range(3000):
        c = _rand_cfg(rng)
        a, b = product.validate(c), oracle.validate(c)
        assert a == b, bytes(c)
        assert product.packet_bound(c) == oracle.packet_bound(c)
        seen.add(a)
    assert len(seen) >= 5


def test_structural_parse_matches_oracle(product, oracle):
    """Query-mode decode (header + slice map rules) on damaged headers."""
    rng = random.Random(5)
    names = [f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz")]
    for name in sorted(names):
        pkt = bytes(np.load(os.path.join(GOLDEN, name + ".npz"))["packet"])
        for trial in range(60):
            p = bytearray(pkt)
            mode = trial % 4
            if mode == 0:      # header field with a fixed-up CRC
                i = rng.randrange(4, 49)
                p[i] = rng.randrange(256)
                crc = __import__("zlib").crc32(bytes(p[:49])) & 0xFFFFFFFF
                p[49:53] = struct.pack(">I", crc)
            elif mode == 1:    # any header byte
                p[rng.randrange(53)] ^= 1 << rng.randrange(8)
            elif mode == 2:    # slice header bytes
                if len(p) > 70:
                    p[53 + rng.randrange(17)] = rng.randrange(256)
            else:              # truncation / extension
                p = p[: rng.randrange(len(p) + 1)] if rng.random() < 0.7 else p + b"\0" * rng.randint(1, 9)
            p = bytes(p)
            ra, ia = product.query(p)
            rb, ib = oracle.query(p)
            assert ra == rb, (name, trial)
            if ra == 0:
                assert bytes(ia) == bytes(ib)


REF_PY = reference_path("python")


def test_reference_python_binding_loads_this_library(built):
    """The reference's own Python binding binds every symbol it needs from this
    library (hot path for real, the rest as NOT_IMPLEMENTED exports) and its
    host-side answers match ours. Runs only where the reference is checked out."""
    import importlib
    import sys
    if not os.path.isdir(REF_PY):
        pytest.skip("reference Python package not present")
    sys.path.insert(0, REF_PY)
    try:
        tb = importlib.import_module("topos_codec.topos_binding")
    finally:
        sys.path.remove(REF_PY)
    codec = tb.ToposCodec(library=ctypes.CDLL(B.PRODUCT_LIBRARY))
    assert codec.abi_version == 2
    ours = B.ToposCodec(B.PRODUCT_LIBRARY)
    for w, h, kw in [(1920, 1080, dict(qp=8, qmatrix_id=4, features=1)), (3840, 2160, dict(qp=4, features=3)),
                     (4096, 2160, dict(qp=2, bit_depth=12, pixel_format=2, profile=5, alpha_mode=1,
                                       alpha_bit_depth=16, color_range=1))]:
        mine = B.make_config(w, h, **kw)
        theirs = tb._CFrameConfig.from_buffer_copy(bytes(mine))
        assert codec.config_validate(theirs) == ours.validate(mine) == 0
        assert codec.packet_bound(theirs) == ours.packet_bound(mine)
    lib = codec._lib
    lib.tc_frame_encode_sized.restype = ctypes.c_int32
    assert lib.tc_frame_encode_sized(None, None, 0, 0, 0, None, None, 0, None) == B.TC_ERR_INVALID_ARGUMENT
    lib.tc_decode_scale_dimensions.restype = ctypes.c_int32
    tw, th = ctypes.c_uint32(), ctypes.c_uint32()
    assert lib.tc_decode_scale_dimensions(3841, 2161, 2, ctypes.byref(tw), ctypes.byref(th)) == 0
    assert (tw.value, th.value) == (1281, 721)
    lib.tc_gop_context_observe.restype = ctypes.c_int32
    assert lib.tc_gop_context_observe(None, None, 0, None) == B.TC_ERR_NOT_IMPLEMENTED
    lib.tc_scalable_status_name.restype = ctypes.c_char_p
    assert lib.tc_scalable_status_name(1) == b"reference" and lib.tc_scalable_status_name(9) == b"unknown"


def _plan(L, sizes, decode=0):
    n = len(sizes)
    arr = (ctypes.c_uint64 * max(n, 1))(*sizes)
    starts = (ctypes.c_uint32 * 5)()
    k = int(L.tcg_pipeline_plan(ctypes.c_int32(decode), arr, ctypes.c_uint32(n), starts))
    return k, list(starts[: k + 1])


def test_pipeline_plan_splits_host_batches(product, monkeypatch):
    """Chunking of host-memory batches: no split below 256 MB of copies, one
    chunk per 64 MB up to four (encode) or three (decode), every chunk
    non-empty and contiguous, chunk bytes within one frame of an even share;
    TCG_PIPELINE forces the count (up to four)."""
    L = product._lib
    L.tcg_pipeline_plan.restype = ctypes.c_uint32
    monkeypatch.delenv("TCG_PIPELINE", raising=False)
    MB = 1 << 20
    assert _plan(L, [33 * MB] * 7) == (1, [0, 7])           # 231 MB: one piece
    assert _plan(L, [33 * MB] * 60)[0] == 4                  # 3840x2160 4:2:2 batch
    assert _plan(L, [63 * MB] * 60, decode=1)[0] == 3        # its packets and planes
    assert _plan(L, [300 * MB]) == (1, [0, 1])               # one frame never splits
    assert _plan(L, [160 * MB, 160 * MB]) == (2, [0, 1, 2])
    assert _plan(L, []) == (1, [0, 0])
    rng = random.Random(3)
    for trial in range(300):
        n = rng.randint(1, 70)
        sizes = [rng.choice([0, rng.randint(1, 80 * MB)]) for _ in range(n)]
        total = sum(sizes)
        decode = trial % 2
        k, st = _plan(L, sizes, decode)
        want = 1 if total < 256 * MB else min(3 if decode else 4, total // (64 * MB), n)
        assert k == max(1, want)
        assert st[0] == 0 and st[-1] == n and all(a < b for a, b in zip(st, st[1:]))
        if k > 1:
            big = max(sizes)
            for i in range(k - 1):  # every chunk but the last stops at its share
                assert sum(sizes[: st[i + 1]]) < total // k * (i + 1) + big or st[i + 1] - st[i] == 1
    monkeypatch.setenv("TCG_PIPELINE", "3")
    assert _plan(L, [1, 1, 1, 1, 1]) == (3, [0, 1, 2, 5])
    assert _plan(L, [1, 1]) == (2, [0, 1, 2])
    monkeypatch.setenv("TCG_PIPELINE", "9")
    assert _plan(L, [1] * 8, decode=1) == (4, [0, 2, 4, 6, 8])
    monkeypatch.setenv("TCG_PIPELINE", "0")
    assert _plan(L, [33 * MB] * 60) == (1, [0, 60])


def test_sized_encode_argument_checks_match_reference(product, reference):
    """tc_frame_encode_sized's checks before any encode, status for status with
    the reference library: NULL config, qp ranges (reversed, above 95),
    pixel format 3 and the temporal generations."""
    planes = [np.zeros((16, 16), np.uint16) for _ in range(3)]
    cases = []
    base = B.make_config(16, 16, qp=8, qmatrix_id=4, features=1)
    for lo, hi in [(30, 20), (0, 96), (96, 96)]:
        cases.append((base, lo, hi))
    for gen in (9, 10, 11):
        c = B.make_config(16, 16, qp=8)
        c.reserved[0] = gen
        cases.append((c, 0, 63))
    for cfg, lo, hi in cases:
        got = [x.encode_sized_status(cfg, planes, 1000, lo, hi, 4096)[0] for x in (product, reference)]
        assert got[0] == got[1] and got[0] < 0, (cfg.reserved[0], lo, hi, got)
    assert product._lib.tc_frame_encode_sized(None, None, 0, 0, 0, None, None, 0, None) == \
        reference._lib.tc_frame_encode_sized(None, None, 0, 0, 0, None, None, 0, None)


def _request_cases():
    """(request, label) pairs: every mode, scale and flag, and the invalid forms."""
    out = [(B.make_request(0), "full"), (B.make_request(0, flags=1), "full-drop-alpha")]
    for t in [(1, 1), (17, 9), (64, 48), (10 ** 5, 8), (8, 0)]:
        out.append((B.make_request(1, target=t), f"scaled {t}"))
    for sc in range(6):
        out.append((B.make_request(2, scale=sc), f"reduced {sc}"))
    out += [(B.make_request(3), "auto2k"), (B.make_request(3, target=(20, 10)), "auto2k target"),
            (B.make_request(2, scale=1, target=(4, 4)), "reduced with target"),
            (B.make_request(0, scale=1), "full with scale"), (B.make_request(4), "bad mode"),
            (B.make_request(0, quality=4), "bad quality"), (B.make_request(0, memory_type=2), "bad memory"),
            (B.make_request(0, flags=2), "bad flag"), (B.make_request(1, target=(8, 8), quality=3, memory_type=1), "ok")]
    bad = B.make_request(0)
    bad.reserved[2] = 1
    out.append((bad, "reserved"))
    bad = B.make_request(0)
    bad.struct_size = 8
    out.append((bad, "struct size"))
    return out


def test_decode_request_query_matches_reference(product, reference):
    """tc_frame_decode_request and tc_decoder_prepare_request in query mode
    (no output planes): status and frame information equal the reference
    library's for every mode, scale, flag and invalid request on the fixture
    packets (4:2:2, 4:4:4 + alpha, 1x1) and a V8 packet."""
    names = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    for lib in (product._lib, reference._lib):
        lib.tc_frame_decode_request.restype = ctypes.c_int32
        lib.tc_decoder_prepare_request.restype = ctypes.c_int32
        lib.tc_decoder_create.restype = ctypes.c_int32
    decs = []
    for lib in (product._lib, reference._lib):
        d = ctypes.c_void_p()
        assert lib.tc_decoder_create(None, ctypes.byref(d)) == 0
        decs.append(d)
    pkts = [(name, bytes(np.load(os.path.join(GOLDEN, name + ".npz"))["packet"])) for name in names]
    v8 = B.make_config(96, 64, qp=9, qmatrix_id=4)
    v8.reserved[0], v8.reserved[3], v8.reserved[4] = 9, 4, 5
    pkts.append(("v8", reference.encode(v8, synth.make_frame_np(96, 64, seed=5))))
    try:
        for name, pkt in pkts:
            buf = np.frombuffer(pkt, np.uint8)
            for req, label in _request_cases():
                got = []
                for lib, d in zip((product._lib, reference._lib), decs):
                    a, b = B.FrameOutput(), B.FrameOutput()
                    ra = int(lib.tc_frame_decode_request(ctypes.c_void_p(buf.ctypes.data), ctypes.c_size_t(len(pkt)),
                                                         ctypes.byref(req), None, None, ctypes.byref(a)))
                    rb = int(lib.tc_decoder_prepare_request(d, ctypes.c_void_p(buf.ctypes.data), ctypes.c_size_t(len(pkt)),
                                                            ctypes.byref(req), ctypes.byref(b)))
                    got.append((ra, bytes(a) if ra == 0 else None, rb, bytes(b) if rb == 0 else None))
                assert got[0] == got[1], (name, label, got[0][0], got[1][0], got[0][2], got[1][2])
    finally:
        product._lib.tc_decoder_destroy(decs[0])
        reference._lib.tc_decoder_destroy(decs[1])
