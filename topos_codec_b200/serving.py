"""Open-loop serving measurement over the library's request server.

Requests arrive as a Poisson process: half encodes, half decodes; frames of
1920x1080 (40 %), 3840x2160 (40 %) and 1280x720 (20 %), 10-bit 4:2:2, tiers
422 (qp 8, quant matrix 4) and HQ (qp 4; flat matrix and refined qp table at
3840 wide), chosen from a seeded generator. generation="v8" codes the same
stream as V8 segmented-rANS packets (16-block segments, 32-row tiles; V8 has
no deblocking or refined qp table, so those features are off).

The load generator is open-loop: arrivals follow their schedule whatever the
server does. Input planes and packets are shared, read-only, per (resolution,
tier); every request gets its own output buffer from a pool that is provisioned
before the stream for a second of arrivals and grows when all are in
use, so a busy server never delays the next arrival. Past saturation an
arrival that finds 512 requests unfinished is shed and counted as dropped. Latency runs
from a request's scheduled arrival to the moment its completion is seen
(the generator's lag before submitting it plus the server's own
submission-to-completion time, which is also reported alone). Percentiles are given for the whole stream and per resolution and
direction.
"""
from __future__ import annotations

import random
import threading
import time
from typing import Dict, List

from . import binding as B, synth

RESOLUTIONS = [((1920, 1080), 0.4), ((3840, 2160), 0.4), ((1280, 720), 0.2)]
TIERS = ["422", "hq"]


def tier_config(w: int, h: int, tier: str, generation: str = "v7") -> B.FrameConfig:
    if generation == "v8":
        cfg = B.make_config(w, h, qp=4 if tier == "hq" else 8, qmatrix_id=0 if (tier == "hq" and w >= 3840) else 4)
        cfg.reserved[0] = 9
        return cfg
    if tier == "hq":
        big = w >= 3840
        return B.make_config(w, h, qp=4, qmatrix_id=0 if big else 4, features=3 if big else 1)
    return B.make_config(w, h, qp=8, qmatrix_id=4, features=1)


class _Kind:
    """Shared inputs of one (resolution, tier): sample planes and a packet in
    device memory; output buffers are handed out per request."""

    def __init__(self, codec, torch, dev, w, h, tier, seed, generation):
        self.cfg = tier_config(w, h, tier, generation)
        self.w, self.h = w, h
        self.torch, self.dev = torch, dev
        planes = synth.make_frame(w, h, seed=seed, frame=0, device=dev)
        self.planes = [p.to(torch.uint16).contiguous() for p in planes]
        pkt = codec.encode(self.cfg, [p.cpu().numpy() for p in self.planes])
        # every request of this kind codes the same planes, so its packet has
        # this size; the margin keeps the buffers far below the packet bound
        self.cap = min(codec.packet_bound(self.cfg), len(pkt) + (1 << 20))
        self.pkt = torch.frombuffer(bytearray(pkt), dtype=torch.uint8).to(dev)
        self.free_out: List = []
        self.free_dec: List = []

    def out(self):
        return self.free_out.pop() if self.free_out else self.torch.empty(self.cap, dtype=self.torch.uint8,
                                                                          device=self.dev)

    def dec(self):
        return self.free_dec.pop() if self.free_dec else [self.torch.empty_like(p) for p in self.planes]

    def provision(self, n_out: int, n_dec: int):
        """Allocate output buffers ahead of a stream, so that the device
        allocator's synchronising calls fall outside it."""
        while len(self.free_out) < n_out:
            self.free_out.append(self.torch.empty(self.cap, dtype=self.torch.uint8, device=self.dev))
        while len(self.free_dec) < n_dec:
            self.free_dec.append([self.torch.empty_like(p) for p in self.planes])


def _pct(xs, p):
    return xs[min(len(xs) - 1, int(p * len(xs)))] if xs else None


def _summary(lat: List[float]) -> Dict:
    lat = sorted(lat)
    return {"n": len(lat), "p50_ms": _pct(lat, 0.50), "p99_ms": _pct(lat, 0.99), "p999_ms": _pct(lat, 0.999),
            "max_ms": lat[-1] if lat else None}


def _kinds(codec, torch, dev, seed, generation):
    return {(wh, t): _Kind(codec, torch, dev, wh[0], wh[1], t, seed + i, generation)
            for i, (wh, t) in enumerate((wh, t) for wh, _ in RESOLUTIONS for t in TIERS)}


def run_trace(codec, rate_rps: float, duration_s: float, seed: int = 0, max_batch_frames: int = 32,
              generation: str = "v7", workers: int = 4, kinds=None, resolutions=None,
              max_outstanding: int = 512) -> Dict:
    """Submit a Poisson request stream at rate_rps for duration_s; returns the
    latency percentiles (whole stream, per resolution, per direction). An
    arrival that finds max_outstanding requests unfinished is shed (counted
    in "dropped", not submitted): past saturation the backlog would otherwise
    grow without bound."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = random.Random(seed)
    kinds = kinds or _kinds(codec, torch, dev, seed, generation)
    res_mix = resolutions or RESOLUTIONS
    # output buffers for a second of arrivals per (resolution, tier, direction)
    for (wh, share) in res_mix:
        for t in TIERS:
            if (wh, t) in kinds:
                n = int(rate_rps * share / len(TIERS) * 0.5 * 1.0) + 2
                kinds[(wh, t)].provision(n, n)
    torch.cuda.synchronize()
    srv = B.Server(codec, max_batch_frames=max_batch_frames, workers=workers)
    cv = threading.Condition()
    pending: List = []
    records: List = []   # (resolution, encode, client ms, server ms)
    errors = [0]
    closing = threading.Event()

    def waiter():
        while True:
            with cv:
                while not pending and not closing.is_set():
                    cv.wait()
                if not pending:
                    return
                kind, enc, buf, t_sched, t_sub, ticket = pending.pop(0)
            st, _, _, ms = srv.wait(ticket)
            with cv:
                # scheduled arrival to completion: the generator's lag before
                # submission plus the server's submission-to-completion time
                # (collectors take requests in submission order, so the time
                # one sees a completion could include the wait for older ones)
                records.append((kind[0], enc, (t_sub - t_sched) * 1e3 + ms, ms, (t_sub - t_sched) * 1e3,
                                t_sched - t0))
                if st not in (0, 1):
                    errors[0] += 1
                (kind_obj(kind).free_out if enc else kind_obj(kind).free_dec).append(buf)

    def kind_obj(k):
        return kinds[k]

    # several collectors, so one slow request does not hold back the buffers
    # of the faster ones submitted after it
    ths = [threading.Thread(target=waiter) for _ in range(8)]
    for th in ths:
        th.start()
    weights = [w for _, w in res_mix]
    t0 = time.perf_counter()
    t_next = t0
    n = 0
    dropped = 0
    try:
        while True:
            t_next += rng.expovariate(rate_rps)
            if t_next - t0 > duration_s:
                break
            wh = rng.choices([r for r, _ in res_mix], weights)[0]
            key = (wh, rng.choice(TIERS))
            enc = rng.random() < 0.5
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            k = kinds[key]
            with cv:
                if len(pending) >= max_outstanding:
                    dropped += 1
                    continue
                buf = k.out() if enc else k.dec()
            t_sub = time.perf_counter()
            if enc:
                ticket = srv.submit_encode(k.cfg, [(p.data_ptr(), p.shape[1]) for p in k.planes], buf.data_ptr(), k.cap)
            else:
                ticket = srv.submit_decode(k.pkt.data_ptr(), k.pkt.numel(), [p.data_ptr() for p in buf])
            n += 1
            with cv:
                pending.append((key, enc, buf, t_next, t_sub, ticket))
                cv.notify_all()
    finally:
        closing.set()
        with cv:
            cv.notify_all()
        for th in ths:
            th.join()
        srv.close()
    wall = time.perf_counter() - t0
    out = {"offered_rps": rate_rps, "requests": n, "duration_s": round(wall, 2), "throughput_rps": n / wall,
           "errors": errors[0], "dropped": dropped, "generation": generation}
    out.update(_summary([r[2] for r in records]))
    out["server_side"] = _summary([r[3] for r in records])
    out["submit_lag"] = _summary([r[4] for r in records])  # the generator's own delay
    # when the worst client latencies arrived (seconds into the stream)
    worst = sorted(records, key=lambda r: -r[2])[:8]
    out["worst"] = [{"at_s": round(r[5], 3), "ms": round(r[2], 1), "server_ms": round(r[3], 1),
                     "lag_ms": round(r[4], 1), "size": f"{r[0][0]}x{r[0][1]}", "encode": r[1]} for r in worst]
    out["by_resolution"] = {f"{w}x{h}": _summary([r[2] for r in records if r[0] == (w, h)]) for (w, h), _ in res_mix}
    out["by_direction"] = {"encode": _summary([r[2] for r in records if r[1]]),
                           "decode": _summary([r[2] for r in records if not r[1]])}
    return out


def saturation_rps(codec, n: int = 96, seed: int = 1, max_batch_frames: int = 32, generation: str = "v7",
                   workers: int = 4, kinds=None) -> float:
    """Requests per second when n requests of the mix are all submitted at once
    (the best of two passes: the first also pays for one-time per-batch-size
    tuning)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    kinds = kinds or _kinds(codec, torch, dev, seed, generation)
    return max(_saturation_pass(codec, n, seed, max_batch_frames, workers, kinds) for _ in range(2))


def peak_rps(codec, generation: str = "v7", kinds=None, seconds: float = 6.0, workers: int = 4) -> Dict:
    """The server's sustained peak: an open-loop stream offered at 1.5 times
    the burst rate (saturation_rps) for `seconds`, with arrivals past 256
    unfinished requests shed; the peak is the rate at which it completed
    requests (a burst drains queues built before it, so it overstates what a
    stream sustains)."""
    burst = saturation_rps(codec, generation=generation, kinds=kinds, workers=workers)
    r = run_trace(codec, rate_rps=1.5 * burst, duration_s=seconds, seed=3, generation=generation, kinds=kinds,
                  workers=workers, max_outstanding=256)
    return {"burst_rps": burst, "sustained_rps": min(burst, r["throughput_rps"]), "dropped": r["dropped"]}


def _saturation_pass(codec, n, seed, max_batch_frames, workers, kinds) -> float:
    import torch
    rng = random.Random(seed)
    weights = [w for _, w in RESOLUTIONS]
    torch.cuda.synchronize()
    srv = B.Server(codec, max_batch_frames=max_batch_frames, workers=workers)
    bufs = []
    try:
        t0 = time.perf_counter()
        tickets = []
        for _ in range(n):
            wh = rng.choices([r for r, _ in RESOLUTIONS], weights)[0]
            k = kinds[(wh, rng.choice(TIERS))]
            if rng.random() < 0.5:
                b = k.out()
                tickets.append(srv.submit_encode(k.cfg, [(p.data_ptr(), p.shape[1]) for p in k.planes],
                                                 b.data_ptr(), k.cap))
                bufs.append((k.free_out, b))
            else:
                b = k.dec()
                tickets.append(srv.submit_decode(k.pkt.data_ptr(), k.pkt.numel(), [p.data_ptr() for p in b]))
                bufs.append((k.free_dec, b))
        for t in tickets:
            srv.wait(t)
        return n / (time.perf_counter() - t0)
    finally:
        srv.close()
        for pool, b in bufs:
            pool.append(b)


def run_trace_plain(codec, rate_rps: float, duration_s: float, seed: int = 0, generation: str = "v7",
                    kinds=None) -> Dict:
    """The same Poisson request stream served by the plain per-frame calls, one
    request at a time in arrival order (the drop-in path without batching);
    latency runs from each request's scheduled arrival to its completion."""
    import ctypes
    import queue
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = random.Random(seed)
    kinds = kinds or _kinds(codec, torch, dev, seed, generation)
    outs = {k: (v.out(), v.dec()) for k, v in kinds.items()}
    L = codec._lib
    torch.cuda.synchronize()
    q: "queue.Queue" = queue.Queue()
    records: List = []
    errors = [0]

    def worker():
        st = B.FrameStats()
        while True:
            item = q.get()
            if item is None:
                return
            key, enc, t_arr = item
            k = kinds[key]
            out, dec = outs[key]
            if enc:
                fi = B.FrameInput()
                fi.struct_size, fi.abi_version = ctypes.sizeof(B.FrameInput), B.TOPOS_CODEC_ABI_VERSION
                for p, t in enumerate(k.planes):
                    fi.planes[p], fi.strides[p] = t.data_ptr(), t.shape[1]
                rc = int(L.tc_frame_encode(ctypes.byref(k.cfg), ctypes.byref(fi), ctypes.c_void_p(out.data_ptr()),
                                           k.cap, ctypes.byref(st)))
            else:
                ptrs = (ctypes.c_void_p * B.TC_FRAME_MAX_PLANES)(*[t.data_ptr() for t in dec])
                info = B.FrameOutput()
                rc = int(L.tc_frame_decode(ctypes.c_void_p(k.pkt.data_ptr()), k.pkt.numel(), ptrs, None,
                                           ctypes.byref(info)))
            if rc not in (0, 1):
                errors[0] += 1
            records.append((key[0], enc, (time.perf_counter() - t_arr) * 1e3))

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
    out = {"offered_rps": rate_rps, "requests": n, "duration_s": round(wall, 2), "throughput_rps": n / wall,
           "errors": errors[0], "generation": generation}
    out.update(_summary([r[2] for r in records]))
    out["by_resolution"] = {f"{w}x{h}": _summary([r[2] for r in records if r[0] == (w, h)]) for (w, h), _ in RESOLUTIONS}
    return out


def plain_saturation_rps(codec, n: int = 48, seed: int = 1, generation: str = "v7", kinds=None) -> float:
    """Requests per second of the plain per-frame calls on n requests of the mix back to back."""
    r = run_trace_plain(codec, rate_rps=1e6, duration_s=n / 1e6, seed=seed, generation=generation, kinds=kinds)
    return r["requests"] / max(r["duration_s"], 1e-9)


def single_frame_floor(codec, w: int = 1920, h: int = 1080, tier: str = "422", generation: str = "v7",
                       repeats: int = 5) -> Dict:
    """One frame encoded and decoded alone on an idle GPU through the plain
    calls (device-resident planes and packet): the latency floor of a request
    of that size, best of the repeats, wall clock of the call."""
    import ctypes
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    k = _Kind(codec, torch, dev, w, h, tier, 5, generation)
    out, dec = k.out(), k.dec()
    L = codec._lib
    fi = B.FrameInput()
    fi.struct_size, fi.abi_version = ctypes.sizeof(B.FrameInput), B.TOPOS_CODEC_ABI_VERSION
    for p, t in enumerate(k.planes):
        fi.planes[p], fi.strides[p] = t.data_ptr(), t.shape[1]
    ptrs = (ctypes.c_void_p * B.TC_FRAME_MAX_PLANES)(*[t.data_ptr() for t in dec])
    st, info = B.FrameStats(), B.FrameOutput()
    enc_ms, dec_ms = [], []
    torch.cuda.synchronize()
    for _ in range(repeats + 1):
        t0 = time.perf_counter()
        L.tc_frame_encode(ctypes.byref(k.cfg), ctypes.byref(fi), ctypes.c_void_p(out.data_ptr()), k.cap,
                          ctypes.byref(st))
        t1 = time.perf_counter()
        L.tc_frame_decode(ctypes.c_void_p(k.pkt.data_ptr()), k.pkt.numel(), ptrs, None, ctypes.byref(info))
        t2 = time.perf_counter()
        enc_ms.append((t1 - t0) * 1e3)
        dec_ms.append((t2 - t1) * 1e3)
    return {"size": f"{w}x{h}", "tier": tier, "generation": generation, "encode_ms": min(enc_ms[1:]),
            "decode_ms": min(dec_ms[1:])}
