"""Benchmark workloads beside the 4K HQ batch, measured through the C ABI.

* Mixed batch: 64 frames whose resolution (1280x720, 1920x1080, 3840x2160,
  7680x4320), tier (proxy, lt, 422, hq) and fixed QP (2..16) are drawn from a
  seeded generator; 10-bit 4:2:2 limited range. Tier mapping of the product
  layer: quantisation matrix 4 and DEBLOCK for every tier; at 3840 wide and
  up the 422 and HQ tiers take the flat matrix and the refined qp table.
* GBR 4:4:4 + alpha: 4096x2160 12-bit GBR full range, 16-bit alpha (hard
  ellipses with 4-pixel ramps), fixed QP 2, 32 frames; copies of packets with
  1 % of their slices byte-corrupted check the per-slice concealment status
  and pixels against the reference library.

* Size-targeted encode: 3840x2160 10-bit 4:2:2 HQ frames from host memory,
  one tc_frame_encode_sized call per frame with a byte target, beside the
  reference library on the host cores.
* Preview decode: the bench batch's packets decoded at half size
  (tc_frame_decode_batch_reduced), beside the reference library.

The first two are coded as one batched call and as one plain call per frame
on the same device-resident inputs; device time comes from the library's own
stream events (tcg_last_device_ms) and both forms must give identical bytes.
"""
from __future__ import annotations

import ctypes
import random
import struct
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, List, Sequence

import numpy as np

from . import binding as B, synth

MIXED_RES = [(1280, 720), (1920, 1080), (3840, 2160), (7680, 4320)]
MIXED_TIERS = ["proxy", "lt", "422", "hq"]


def mixed_config(w: int, h: int, tier: str, qp: int) -> B.FrameConfig:
    big = w >= 3840 and tier in ("422", "hq")
    return B.make_config(w, h, qp=qp, qmatrix_id=0 if big else 4, features=3 if big else 1)


def mixed_specs(n: int = 64, seed: int = 0):
    rng = random.Random(seed)
    return [(*rng.choice(MIXED_RES), rng.choice(MIXED_TIERS), rng.randint(2, 16)) for _ in range(n)]


def gbr_config(w: int = 4096, h: int = 2160) -> B.FrameConfig:
    return B.make_config(w, h, qp=2, bit_depth=12, pixel_format=2, profile=5, alpha_mode=1, alpha_bit_depth=16,
                         color_range=1)


def _lib(codec):
    L = codec._lib
    L.tcg_last_device_ms.restype = ctypes.c_double
    return L


def _inputs(frames) -> ctypes.Array:
    arr = (B.FrameInput * len(frames))()
    for i, planes in enumerate(frames):
        arr[i].struct_size = ctypes.sizeof(B.FrameInput)
        arr[i].abi_version = B.TOPOS_CODEC_ABI_VERSION
        for p, t in enumerate(planes):
            arr[i].planes[p] = t.data_ptr()
            arr[i].strides[p] = t.shape[1]
    return arr


def batched_vs_plain(codec, cfgs: Sequence[B.FrameConfig], frames, repeats: int = 2, v8: bool = False) -> Dict:
    """Encode and decode the frames (device-resident uint16 planes) batched and
    per frame. Returns device times, bit-exactness of the two forms and the
    batched packets (host bytes). v8: the frames are V8 packets, decoded in
    one batch by tcg_frame_decode_v8_batch."""
    import torch
    L = _lib(codec)
    n = len(cfgs)
    dev = frames[0][0].device
    carr = (B.FrameConfig * n)(*cfgs)
    ins = _inputs(frames)
    caps = [codec.packet_bound(c) for c in cfgs]
    outs = [torch.empty(c, dtype=torch.uint8, device=dev) for c in caps]
    optr = (ctypes.c_void_p * n)(*[t.data_ptr() for t in outs])
    ocap = (ctypes.c_size_t * n)(*caps)
    st = (B.FrameStats * n)()
    rcs = (ctypes.c_int32 * n)()
    dec = [[torch.empty(s, dtype=torch.uint16, device=dev) for s in B.plane_shapes(c)] for c in cfgs]
    dptr = (ctypes.c_void_p * (B.TC_FRAME_MAX_PLANES * n))()
    for i in range(n):
        for p, t in enumerate(dec[i]):
            dptr[B.TC_FRAME_MAX_PLANES * i + p] = t.data_ptr()
    infos = (B.FrameOutput * n)()

    def enc_batch() -> float:
        rc = int(L.tcg_frame_encode_batch(carr, ins, n, optr, ocap, st, rcs))
        if rc != 0:
            raise RuntimeError(f"batched encode failed [{rc}]: {codec.last_error()}")
        return L.tcg_last_device_ms()

    def dec_batch() -> float:
        arr = (B.BatchPacket * n)()
        for i in range(n):
            arr[i].data, arr[i].size = outs[i].data_ptr(), st[i].packet_size
        fn = L.tcg_frame_decode_v8_batch if v8 else L.tc_frame_decode_batch
        rc = int(fn(arr, n, dptr, None, infos))
        if rc not in (B.TC_OK, B.TC_WARN_CONCEALED):
            raise RuntimeError(f"batched decode failed [{rc}]: {codec.last_error()}")
        return L.tcg_last_device_ms()

    enc_batch()  # first batch of each size class also tunes the decode tiling
    dec_batch()
    enc_ms = min(enc_batch() for _ in range(repeats))
    dec_ms = min(dec_batch() for _ in range(repeats))
    pkts = [outs[i][: st[i].packet_size].cpu().numpy().tobytes() for i in range(n)]
    # plain per-frame path on the same inputs
    exact = True
    p_enc = p_dec = 0.0
    one = torch.empty(max(caps), dtype=torch.uint8, device=dev)
    s1 = B.FrameStats()
    for i in range(n):
        rc = int(L.tc_frame_encode(ctypes.byref(carr[i]), ctypes.byref(ins[i]), ctypes.c_void_p(one.data_ptr()),
                                   caps[i], ctypes.byref(s1)))
        p_enc += L.tcg_last_device_ms()
        exact = exact and rc == 0 and one[: s1.packet_size].cpu().numpy().tobytes() == pkts[i]
        got = [torch.empty_like(t) for t in dec[i]]
        ptrs = (ctypes.c_void_p * B.TC_FRAME_MAX_PLANES)(*[t.data_ptr() for t in got])
        info = B.FrameOutput()
        rc = int(L.tc_frame_decode(ctypes.c_void_p(outs[i].data_ptr()), st[i].packet_size, ptrs, None,
                                   ctypes.byref(info)))
        p_dec += L.tcg_last_device_ms()
        exact = exact and rc in (B.TC_OK, B.TC_WARN_CONCEALED) and all(
            torch.equal(a.view(torch.int16), b.view(torch.int16)) for a, b in zip(got, dec[i]))
    return {"frames": n, "batched_encode_ms": enc_ms, "batched_decode_ms": dec_ms, "plain_encode_ms": p_enc,
            "plain_decode_ms": p_dec, "batched_vs_plain": (p_enc + p_dec) / (enc_ms + dec_ms),
            "encode_fps": n / (enc_ms / 1e3), "decode_fps": n / (dec_ms / 1e3), "bit_exact": bool(exact),
            "packets": pkts}


def sized_vs_reference(product, reference, cfg: B.FrameConfig, frames, target: int, qp_min: int = 0,
                       qp_max: int = 63, ref_threads: int = 16) -> Dict:
    """tc_frame_encode_sized on host-memory frames, one call per frame in order
    (as an encoder would run it, after one untimed call on the first frame),
    through this library and the reference
    library (its slice pool at ref_threads): per-frame wall time, chosen qps,
    probe encodes and whether packets, qps and probe counts agree. The two
    libraries must start from the same cross-call hint history (for instance,
    neither has made a size-targeted call before), as the probe sequence
    depends on it."""
    import time
    out = np.empty(product.packet_bound(cfg), np.uint8)
    res = {}
    if reference is not None:
        reference._lib.tc_dev_set_thread_count(ctypes.c_int32(ref_threads))
    for name, codec in (("gpu", product), ("reference", reference)):
        if codec is None:
            continue
        L = codec._lib
        # one untimed call first (the same one in both libraries, so their
        # cross-call hint histories stay equal): buffer growth stays out of
        # the per-frame time
        rc, _, _, _, _ = codec.encode_sized_status(cfg, frames[0], target, qp_min, qp_max, out=out)
        if rc != 0:
            raise RuntimeError(f"{name} sized encode failed [{rc}]: {codec.last_error()}")
        i0 = L.tc_dev_sized_iters()
        t0 = time.perf_counter()
        got = []
        for f in frames:
            rc, pkt, st, qp, _ = codec.encode_sized_status(cfg, f, target, qp_min, qp_max, out=out)
            if rc != 0:
                raise RuntimeError(f"{name} sized encode failed [{rc}]: {codec.last_error()}")
            got.append((qp, pkt))
        el = time.perf_counter() - t0
        res[name] = {"ms_per_frame": 1e3 * el / len(frames), "qps": [q for q, _ in got],
                     "probes_per_frame": (L.tc_dev_sized_iters() - i0) / len(frames), "packets": got}
    r = {"frames": len(frames), "target_bytes": int(target), "qp_range": [qp_min, qp_max],
         "gpu_ms_per_frame": res["gpu"]["ms_per_frame"], "gpu_probes_per_frame": res["gpu"]["probes_per_frame"],
         "qps": res["gpu"]["qps"]}
    if "reference" in res:
        r["reference_ms_per_frame"] = res["reference"]["ms_per_frame"]
        r["reference_threads"] = ref_threads
        r["speedup_vs_reference"] = res["reference"]["ms_per_frame"] / res["gpu"]["ms_per_frame"]
        r["parity"] = res["gpu"]["packets"] == res["reference"]["packets"] and \
            res["gpu"]["probes_per_frame"] == res["reference"]["probes_per_frame"]
    b = sized_batch_vs_reference(product, reference, cfg, frames, target, qp_min, qp_max)
    if "reference_ms_per_frame" in r:
        # the reference's better rate: one call after another or all at once
        best = max(1e3 / r["reference_ms_per_frame"], b.get("reference_fps", 0.0))
        b["reference_best_fps"] = best
        b["speedup_vs_reference_best"] = b["gpu_fps"] / best
    r["batch"] = b
    return r


def sized_batch_vs_reference(product, reference, cfg: B.FrameConfig, frames, target: int, qp_min: int,
                             qp_max: int) -> Dict:
    """All frames at once (after one untimed batch): tcg_frame_encode_sized_batch against the reference's
    single calls run concurrently from one host thread per frame (its slice
    pool shared), both with an empty cross-call hint record (the reference with
    its hint and hint model off): frames/s and whether packets agree."""
    import time
    n = len(frames)
    L = product._lib
    L.tcg_frame_encode_sized_batch.restype = ctypes.c_int32
    cap = product.packet_bound(cfg)
    bufs = [np.empty(cap, np.uint8) for _ in range(n)]
    carr = (B.FrameConfig * n)(*[cfg] * n)
    iarr = (B.FrameInput * n)(*[product._input(f) for f in frames])
    tarr = (ctypes.c_uint32 * n)(*[target] * n)
    qps = (ctypes.c_uint8 * n)()
    optr = (ctypes.c_void_p * n)(*[b.ctypes.data for b in bufs])
    ocap = (ctypes.c_size_t * n)(*[cap] * n)
    st = (B.FrameStats * n)()
    rcs = (ctypes.c_int32 * n)()
    # one untimed batch first, so that the searches' buffer growth stays out of
    # the time (the batch's searches carry no hint history)
    for _ in range(2):
        t0 = time.perf_counter()
        rc = int(L.tcg_frame_encode_sized_batch(carr, iarr, ctypes.c_uint32(n), tarr, ctypes.c_uint8(qp_min),
                                                ctypes.c_uint8(qp_max), qps, optr, ocap, st, rcs))
        el = time.perf_counter() - t0
        if rc != 0:
            break
    if rc != 0:
        raise RuntimeError(f"sized batch failed [{rc}]: {product.last_error()}")
    got = [(qps[i], bufs[i][: st[i].packet_size].tobytes()) for i in range(n)]
    r = {"frames": n, "gpu_fps": n / el, "qps": [q for q, _ in got]}
    if reference is not None:
        R = reference._lib
        R.tc_dev_set_qp_hint(1)
        R.tc_dev_set_qp_hint_model(1)
        try:
            def one(f):
                out = np.empty(cap, np.uint8)
                rc, pkt, _, qp, _ = reference.encode_sized_status(cfg, f, target, qp_min, qp_max, out=out)
                return rc, qp, pkt
            t0 = time.perf_counter()
            with ThreadPoolExecutor(n) as ex:
                ref = list(ex.map(one, frames))
            el = time.perf_counter() - t0
        finally:
            R.tc_dev_set_qp_hint(0)
            R.tc_dev_set_qp_hint_model(0)
        r["reference_fps"] = n / el
        r["speedup_vs_reference"] = r["gpu_fps"] / r["reference_fps"]
        r["parity"] = all(rr[0] == 0 and (rr[1], rr[2]) == g for rr, g in zip(ref, got))
    return r


def preview_vs_reference(product, reference, pkts: List[bytes], scale: int = 1, repeats: int = 2,
                         ref_frames: int = 8) -> Dict:
    """Reduced-size (preview) decode of a batch: tc_frame_decode_batch_reduced
    on device-resident packets into device planes (device time from the
    library's stream events), against the reference library decoding a
    sample of the same packets frame-parallel on the host cores with
    tc_frame_decode_reduced; the sampled frames must agree sample for sample."""
    import os
    import time

    import torch
    n = len(pkts)
    L = product._lib
    L.tc_frame_decode_batch_reduced.restype = ctypes.c_int32
    dev = [torch.from_numpy(np.frombuffer(p, dtype=np.uint8).copy()).cuda() for p in pkts]
    arr = (B.BatchPacket * n)()
    for i, t in enumerate(dev):
        arr[i].data, arr[i].size = t.data_ptr(), len(pkts[i])
    infos = (B.FrameOutput * n)()
    rc = int(L.tc_frame_decode_batch_reduced(arr, n, scale, None, None, infos))
    if rc != 0:
        raise RuntimeError(f"preview query failed [{rc}]: {product.last_error()}")
    shapes = [B.ToposCodec.geometry(infos[i]) for i in range(n)]
    out = [[torch.empty(s, dtype=torch.uint16, device="cuda") for s in shapes[i]] for i in range(n)]
    ptrs = (ctypes.c_void_p * (4 * n))()
    for i in range(n):
        for p, t in enumerate(out[i]):
            ptrs[4 * i + p] = t.data_ptr()

    def run() -> float:
        r = int(L.tc_frame_decode_batch_reduced(arr, n, scale, ptrs, None, infos))
        if r not in (B.TC_OK, B.TC_WARN_CONCEALED):
            raise RuntimeError(f"preview decode failed [{r}]: {product.last_error()}")
        return L.tcg_last_device_ms()

    run()
    ms = min(run() for _ in range(repeats))
    res = {"frames": n, "scale": scale, "target": f"{infos[0].visible_width}x{infos[0].visible_height}",
           "gpu_ms": ms, "gpu_fps": n / (ms / 1e3)}
    if reference is not None:
        k = min(ref_frames, n)
        R = reference._lib
        R.tc_frame_decode_reduced.restype = ctypes.c_int32

        def one(i):
            planes = [np.empty(s, dtype=np.uint16) for s in shapes[i]]
            pp = (ctypes.c_void_p * 4)(*[a.ctypes.data for a in planes])
            buf = np.frombuffer(pkts[i], np.uint8)
            info = B.FrameOutput()
            r = int(R.tc_frame_decode_reduced(ctypes.c_void_p(buf.ctypes.data), ctypes.c_size_t(len(pkts[i])),
                                              ctypes.c_int32(scale), pp, None, ctypes.byref(info)))
            return r, planes
        threads = min(k, os.cpu_count() or 1)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            ref = list(ex.map(one, range(k)))
        el = time.perf_counter() - t0
        res["reference_fps"] = k / el
        res["reference_sample"] = f"{k} frames, {threads} threads"
        res["parity"] = all(r == 0 and all(np.array_equal(a, b.cpu().numpy()) for a, b in zip(planes, out[i]))
                            for i, (r, planes) in enumerate(ref))
    return res


def slice_spans(pkt: bytes):
    """(header offset, payload offset, payload size) of every slice of a packet."""
    off, out = 53, []
    while off + 17 <= len(pkt):
        size = struct.unpack(">I", pkt[off:off + 4])[0]
        out.append((off, off + 17, size))
        off += 17 + size
    return out


def corrupt_slices(pkts: List[bytes], fraction: float = 0.01, seed: int = 5) -> List[bytes]:
    """Copies of the packets with the given fraction of all slices (at least one)
    byte-corrupted at seeded payload positions; slice headers stay intact."""
    rng = random.Random(seed)
    spans = [(f, s) for f, p in enumerate(pkts) for s in slice_spans(p) if s[2] > 0]
    k = max(1, int(round(fraction * len(spans))))
    out = [bytearray(p) for p in pkts]
    for f, (_, po, size) in rng.sample(spans, k):
        i = po + rng.randrange(size)
        out[f][i] ^= 1 + rng.randrange(255)
    return [bytes(p) for p in out]


def concealment_parity(product, reference, pkts: List[bytes], threads: int = 8) -> Dict:
    """Decode damaged packets with both libraries: per-slice status, return code
    and pixels must agree."""
    with ThreadPoolExecutor(threads) as ex:
        ref = list(ex.map(reference.decode_status, pkts))
    ok = True
    concealed = 0
    for p, r in zip(pkts, ref):
        d = product.decode_status(p)
        concealed += sum(1 for s in r.slice_status if s != 0)
        ok = ok and d.status == r.status and d.slice_status == r.slice_status and all(
            np.array_equal(a, b) for a, b in zip(d.planes, r.planes))
    return {"frames": len(pkts), "concealed_slices": concealed, "parity": bool(ok)}
