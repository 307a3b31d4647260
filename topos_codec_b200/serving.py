"""Open-loop serving measurement over the library's request server.

Requests arrive as a Poisson process: half encodes, half decodes; frames of
1920x1080 (40 %), 3840x2160 (40 %) and 1280x720 (20 %), 10-bit 4:2:2, tiers
422 (qp 8, quant matrix 4) and HQ (qp 4; flat matrix and refined qp table at
3840 wide), chosen from a seeded generator. Sample planes and packets stay
resident in device memory; each request codes into its own output buffer.
The server measures each request's latency from submission to completion.
"""
from __future__ import annotations

import random
import threading
import time
from typing import Dict, List

from . import binding as B, synth

RESOLUTIONS = [((1920, 1080), 0.4), ((3840, 2160), 0.4), ((1280, 720), 0.2)]
TIERS = ["422", "hq"]


def tier_config(w: int, h: int, tier: str) -> B.FrameConfig:
    if tier == "hq":
        big = w >= 3840
        return B.make_config(w, h, qp=4, qmatrix_id=0 if big else 4, features=3 if big else 1)
    return B.make_config(w, h, qp=8, qmatrix_id=4, features=1)


class _Slot:
    """Device buffers for one request of one (resolution, tier, direction)."""

    def __init__(self, codec, torch, dev, w, h, tier, seed):
        self.cfg = tier_config(w, h, tier)
        self.w, self.h = w, h
        planes = synth.make_frame(w, h, seed=seed, frame=0, device=dev)
        self.planes = [p.to(torch.uint16).contiguous() for p in planes]
        self.cap = codec.packet_bound(self.cfg)
        self.out = torch.empty(self.cap, dtype=torch.uint8, device=dev)
        pkt = codec.encode(self.cfg, [p.cpu().numpy() for p in self.planes])
        self.pkt = torch.frombuffer(bytearray(pkt), dtype=torch.uint8).to(dev)
        self.dec = [torch.empty_like(p) for p in self.planes]


def run_trace(codec, rate_rps: float, duration_s: float, seed: int = 0, slots_per_kind: int = 8,
              max_batch_frames: int = 32) -> Dict:
    """Submit a Poisson request stream at rate_rps for duration_s; returns latency percentiles."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = random.Random(seed)
    kinds = [(wh, t) for wh, _ in RESOLUTIONS for t in TIERS]
    pools = {k: [_Slot(codec, torch, dev, k[0][0], k[0][1], k[1], seed + i) for i in range(slots_per_kind)]
             for k in kinds}
    free = {k: list(range(slots_per_kind)) for k in kinds}
    cv = threading.Condition()
    torch.cuda.synchronize()
    srv = B.Server(codec, max_batch_frames=max_batch_frames)
    lat: List[float] = []
    stats = {"encode": 0, "decode": 0, "errors": 0}
    pending: List = []
    done_evt = threading.Event()

    def waiter():
        while True:
            with cv:
                while not pending and not done_evt.is_set():
                    cv.wait()
                if not pending:
                    return
                key, idx, t = pending.pop(0)
            st, _, _, ms = srv.wait(t)
            with cv:
                lat.append(ms)
                if st not in (0, 1):
                    stats["errors"] += 1
                free[key].append(idx)
                cv.notify_all()

    th = threading.Thread(target=waiter)
    th.start()
    weights = [w for _, w in RESOLUTIONS]
    t0 = time.perf_counter()
    t_next = t0
    n = 0
    try:
        while True:
            t_next += rng.expovariate(rate_rps)
            if t_next - t0 > duration_s:
                break
            wh = rng.choices([r for r, _ in RESOLUTIONS], weights)[0]
            key = (wh, rng.choice(TIERS))
            enc = rng.random() < 0.5
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            with cv:
                while not free[key]:
                    cv.wait()
                idx = free[key].pop()
            s = pools[key][idx]
            if enc:
                t = srv.submit_encode(s.cfg, [(p.data_ptr(), p.shape[1]) for p in s.planes], s.out.data_ptr(), s.cap)
                stats["encode"] += 1
            else:
                t = srv.submit_decode(s.pkt.data_ptr(), s.pkt.numel(), [p.data_ptr() for p in s.dec])
                stats["decode"] += 1
            n += 1
            with cv:
                pending.append((key, idx, t))
                cv.notify_all()
    finally:
        done_evt.set()
        with cv:
            cv.notify_all()
        th.join()
        srv.close()
    wall = time.perf_counter() - t0
    lat.sort()

    def pct(p):
        return lat[min(len(lat) - 1, int(p * len(lat)))] if lat else None

    return {"offered_rps": rate_rps, "requests": n, "duration_s": round(wall, 2), "throughput_rps": n / wall,
            "p50_ms": pct(0.50), "p99_ms": pct(0.99), "p999_ms": pct(0.999), "max_ms": lat[-1] if lat else None,
            "encodes": stats["encode"], "decodes": stats["decode"], "errors": stats["errors"]}


def saturation_rps(codec, n: int = 48, seed: int = 1, max_batch_frames: int = 32) -> float:
    """Requests per second when n requests of the mix are all submitted at once
    (the best of two passes: the first also pays for one-time per-batch-size
    tuning)."""
    return max(_saturation_pass(codec, n, seed, max_batch_frames) for _ in range(2))


def _saturation_pass(codec, n: int, seed: int, max_batch_frames: int) -> float:
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = random.Random(seed)
    kinds = [(wh, t) for wh, _ in RESOLUTIONS for t in TIERS]
    per = max(1, n // len(kinds) + 1)
    pools = {k: [_Slot(codec, torch, dev, k[0][0], k[0][1], k[1], seed + i) for i in range(per)] for k in kinds}
    weights = [w for _, w in RESOLUTIONS]
    used = {k: 0 for k in kinds}
    torch.cuda.synchronize()
    srv = B.Server(codec, max_batch_frames=max_batch_frames)
    try:
        t0 = time.perf_counter()
        tickets = []
        for _ in range(n):
            wh = rng.choices([r for r, _ in RESOLUTIONS], weights)[0]
            key = (wh, rng.choice(TIERS))
            if used[key] >= per:
                key = min(used, key=used.get)
            s = pools[key][used[key]]
            used[key] += 1
            if rng.random() < 0.5:
                tickets.append(srv.submit_encode(s.cfg, [(p.data_ptr(), p.shape[1]) for p in s.planes],
                                                 s.out.data_ptr(), s.cap))
            else:
                tickets.append(srv.submit_decode(s.pkt.data_ptr(), s.pkt.numel(), [p.data_ptr() for p in s.dec]))
        for t in tickets:
            srv.wait(t)
        return n / (time.perf_counter() - t0)
    finally:
        srv.close()


def run_trace_plain(codec, rate_rps: float, duration_s: float, seed: int = 0) -> Dict:
    """The same Poisson request stream served by the plain per-frame calls, one
    request at a time in arrival order (the drop-in path without batching);
    latency runs from each request's arrival to its completion."""
    import ctypes
    import queue
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = random.Random(seed)
    kinds = [(wh, t) for wh, _ in RESOLUTIONS for t in TIERS]
    slots = {k: _Slot(codec, torch, dev, k[0][0], k[0][1], k[1], seed) for k in kinds}
    L = codec._lib
    torch.cuda.synchronize()
    q: "queue.Queue" = queue.Queue()
    lat: List[float] = []
    errors = [0]

    def worker():
        st = B.FrameStats()
        while True:
            item = q.get()
            if item is None:
                return
            key, enc, t_arr = item
            s = slots[key]
            if enc:
                fi = B.FrameInput()
                fi.struct_size, fi.abi_version = ctypes.sizeof(B.FrameInput), B.TOPOS_CODEC_ABI_VERSION
                for p, t in enumerate(s.planes):
                    fi.planes[p], fi.strides[p] = t.data_ptr(), t.shape[1]
                rc = int(L.tc_frame_encode(ctypes.byref(s.cfg), ctypes.byref(fi), ctypes.c_void_p(s.out.data_ptr()),
                                           s.cap, ctypes.byref(st)))
            else:
                ptrs = (ctypes.c_void_p * B.TC_FRAME_MAX_PLANES)(*[t.data_ptr() for t in s.dec])
                info = B.FrameOutput()
                rc = int(L.tc_frame_decode(ctypes.c_void_p(s.pkt.data_ptr()), s.pkt.numel(), ptrs, None,
                                           ctypes.byref(info)))
            if rc not in (0, 1):
                errors[0] += 1
            lat.append((time.perf_counter() - t_arr) * 1e3)

    th = threading.Thread(target=worker)
    th.start()
    weights = [w for _, w in RESOLUTIONS]
    t0 = time.perf_counter()
    t_next = t0
    n = 0
    while True:
        t_next += rng.expovariate(rate_rps)
        if t_next - t0 > duration_s:
            break
        wh = rng.choices([r for r, _ in RESOLUTIONS], weights)[0]
        key = (wh, rng.choice(TIERS))
        enc = rng.random() < 0.5
        delay = t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        q.put((key, enc, t_next))
        n += 1
    q.put(None)
    th.join()
    wall = time.perf_counter() - t0
    lat.sort()

    def pct(p):
        return lat[min(len(lat) - 1, int(p * len(lat)))] if lat else None

    return {"offered_rps": rate_rps, "requests": n, "duration_s": round(wall, 2), "throughput_rps": n / wall,
            "p50_ms": pct(0.50), "p99_ms": pct(0.99), "p999_ms": pct(0.999), "max_ms": lat[-1] if lat else None,
            "errors": errors[0]}


def plain_saturation_rps(codec, n: int = 48, seed: int = 1) -> float:
    """Requests per second of the plain per-frame calls on n requests of the mix back to back."""
    r = run_trace_plain(codec, rate_rps=1e6, duration_s=n / 1e6, seed=seed)
    return r["requests"] / max(r["duration_s"], 1e-9)

