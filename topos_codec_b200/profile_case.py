"""One batched encode + decode of a small synthetic case, for kernel profiling.

    python -m topos_codec_b200.profile_case [--size 1920x1080] [--frames 1] [--qp 4] [--repeat 1] [--gbr]

Runs the same library path as bench.py (device-resident samples, packets and
planes) on a case small enough for a full-metric profiler capture, and prints
the per-kernel device times of the last repetition. --gbr codes 12-bit GBR
4:4:4 with a 16-bit alpha plane at qp 2 instead of 10-bit 4:2:2.
"""
from __future__ import annotations

import argparse
import ctypes
import json

import torch

from . import binding as B, synth


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", default="1920x1080")
    ap.add_argument("--frames", type=int, default=1)
    ap.add_argument("--qp", type=int, default=4)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--gbr", action="store_true")
    a = ap.parse_args()
    w, h = (int(v) for v in a.size.split("x"))
    n = a.frames
    gpu = B.ToposCodec(B.PRODUCT_LIBRARY)
    L = gpu._lib
    L.tcg_profile_read.argtypes = [ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_uint64)]
    if a.gbr:
        from .workloads import gbr_config
        cfg = gbr_config(w, h)
        kw = dict(bit_depth=12, pixel_format=2, limited=False, alpha=True, sigma=12)
    else:
        cfg = B.make_config(w, h, qp=a.qp, qmatrix_id=0 if w >= 3840 else 4, features=3 if w >= 3840 else 1)
        kw = {}
    frames = [[p.to(torch.uint16) for p in synth.make_frame(w, h, seed=0, frame=i, device="cuda", **kw)]
              for i in range(n)]
    cap = gpu.packet_bound(cfg)
    outs = [torch.empty(cap, dtype=torch.uint8, device="cuda") for _ in range(n)]
    dec = [[torch.empty(s, dtype=torch.uint16, device="cuda") for s in B.plane_shapes(cfg)] for _ in range(n)]
    cfgs = (B.FrameConfig * n)(*[cfg] * n)
    ins = (B.FrameInput * n)()
    for i, fr in enumerate(frames):
        ins[i].struct_size, ins[i].abi_version = ctypes.sizeof(B.FrameInput), 2
        for p, t in enumerate(fr):
            ins[i].planes[p], ins[i].strides[p] = t.data_ptr(), t.shape[1]
    optr = (ctypes.c_void_p * n)(*[t.data_ptr() for t in outs])
    caps = (ctypes.c_size_t * n)(*[cap] * n)
    st = (B.FrameStats * n)()
    rcs = (ctypes.c_int32 * n)()
    dptr = (ctypes.c_void_p * (4 * n))()
    for i in range(n):
        for p, t in enumerate(dec[i]):
            dptr[4 * i + p] = t.data_ptr()
    infos = (B.FrameOutput * n)()
    for r in range(a.repeat):
        if r == a.repeat - 1:
            L.tcg_profile_reset()
            L.tcg_profile_enable(1)
        rc = L.tcg_frame_encode_batch(cfgs, ins, n, optr, caps, st, rcs)
        assert rc == 0, gpu.last_error()
        pk = (B.BatchPacket * n)()
        for i in range(n):
            pk[i].data, pk[i].size = outs[i].data_ptr(), st[i].packet_size
        rc = L.tc_frame_decode_batch(pk, n, dptr, None, infos)
        assert rc == 0, gpu.last_error()
    L.tcg_profile_enable(0)
    res = {}
    for k in range(64):
        name, ms, cnt = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_uint64()
        if L.tcg_profile_read(k, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(cnt)) != 0:
            break
        if cnt.value:
            res[name.value.decode()] = round(ms.value, 3)
    print(json.dumps({"size": a.size, "frames": n, "packet_bytes": sum(s.packet_size for s in st), "kernels_ms": res}))


if __name__ == "__main__":
    main()
