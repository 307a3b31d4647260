"""Benchmark: 4K 10-bit 4:2:2 HQ intra encode + decode of a 60-frame batch.

Workload: 3840x2160 10-bit YUV 4:2:2 limited range, fixed QP 4, HQ tier mapping
(flat quantisation matrix, DEBLOCK + refined qp table), default slice layout
(16 block rows), 60 synthetic frames (seeded sinusoids + rectangles + Gaussian
noise, per-frame phase drift). One step = batched GPU encode of the 60 frames
followed by batched GPU decode of the 60 packets (the round trip). The metric
is round-trip frames/s; encode and decode rates are reported beside it, with
the plain per-frame GPU path on the same frames for comparison.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--serve-seconds S] [--no-serve] [--no-extra]
    python bench.py --case 3840x2160 --frames 2 [--repeat R] [--case-qp Q] [--case-gbr] [--case-v8]

Beside the headline the line reports (key `workloads`) a 64-frame mixed batch
(720p..8K, four tiers, qp 2..16) and a 32-frame 4096x2160 12-bit GBR 4:4:4 +
16-bit alpha batch, each batched against the plain per-frame path, the latter
also against the reference library on 8 frames and on damaged copies of its
packets; and (key `served`) open-loop request streams at 25/50/75/100 % of the
server's saturation beside the plain per-request path.

Under torchrun every rank codes its own 60-frame batch (weak scaling, no
collective on the data path); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, FRAMES = 3840, 2160, 60
CFG = dict(qp=4, qmatrix_id=0, features=3, profile=3)
METRIC = "4K 422 HQ enc/dec frames/s (batched vs plain GPU, bit-exact); served p50/p99 ms"
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtopos_codec_ref.so")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle_tc.so")


def plane_bytes(w=W, h=H):
    return w * h * 2 + 2 * ((w + 1) // 2) * h * 2


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples during the timed region (read-only queries)."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="tc_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        try:
            os.unlink(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ reference CPU path

def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def ref_simd_backend(lib):
    """The reference library's SIMD dispatch choice (dispatch.c:213)."""
    fn = lib._lib.tc_dev_simd_backend
    fn.restype = ctypes.c_char_p
    v = fn()
    return v.decode() if v else None


def cpu_mode_main(mode, seconds, nframes):
    """One as-is mode of the reference CPU path, run in its own process so its
    slice pool takes the thread count set for it (TOPOS_SLICE_THREADS is read
    once per process): prints one JSON line.
      slice  - tc_frame_encode then tc_frame_decode per frame, slice pool of
               min(cores, 16) threads (the reference's per-frame path)
      batch  - tc_frame_decode_batch over the frame set, same pool"""
    from topos_codec_b200 import binding as B, synth
    ref = B.ToposCodec(REF_LIB)
    cfg = B.make_config(W, H, **CFG)
    frames = [synth.make_frame_np(W, H, seed=0, frame=i) for i in range(nframes)]
    pkts = [ref.encode(cfg, f) for f in frames[:1]]  # warm-up (pool start, tables)
    ref.decode(pkts[0])
    out = {"mode": mode, "threads": int(os.environ.get("TOPOS_SLICE_THREADS", "0")), "frames": nframes,
           "simd_backend": ref_simd_backend(ref), "cpu_model": cpu_model()}
    if mode == "slice":
        t0 = time.perf_counter()
        n, pkts = 0, []
        while time.perf_counter() - t0 < seconds or n < 2:
            pkts.append(ref.encode(cfg, frames[n % nframes]))
            n += 1
        enc_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        m = 0
        while time.perf_counter() - t0 < seconds or m < 2:
            ref.decode(pkts[m % len(pkts)])
            m += 1
        dec_s = time.perf_counter() - t0
        out.update(encode_fps=n / enc_s, decode_fps=m / dec_s, encoded=n, decoded=m)
    else:
        pkts = [ref.encode(cfg, f) for f in frames]
        t0 = time.perf_counter()
        calls = 0
        while time.perf_counter() - t0 < seconds or calls < 1:
            rc, _ = ref.decode_batch(pkts)
            assert rc == 0
            calls += 1
        out.update(decode_fps=calls * len(pkts) / (time.perf_counter() - t0), batches=calls)
    print(json.dumps(out))


def cpu_modes(seconds=6.0, nframes=8):
    """The reference's as-is CPU modes, each in a subprocess of this script."""
    cores = os.cpu_count() or 1
    env = dict(os.environ, TOPOS_SLICE_THREADS=str(min(cores, 16)))
    res = {}
    for mode in ("slice", "batch"):
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-mode", mode, "--cpu-seconds", str(seconds),
                            "--frames", str(nframes)], capture_output=True, text=True, env=env)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        res[mode] = json.loads(lines[-1]) if r.returncode == 0 and lines else {"error": (r.stderr or r.stdout)[-300:]}
    return res


def reference_rate(frames_np, cfg, budget_s=10.0, threads=None):
    """Round-trip frames/s of the reference CPU library (built from its own
    sources into oracle/_ref) on the host cores: frame-parallel, one frame per
    worker thread, the reference's slice pool at one thread per call."""
    os.environ["TOPOS_SLICE_THREADS"] = "1"
    from topos_codec_b200 import binding as B
    ref = B.ToposCodec(REF_LIB)
    cores = threads or (os.cpu_count() or 1)
    n = len(frames_np)
    done, lock = [0], threading.Lock()
    t_end = [0.0]

    def work(i0):
        k = i0
        while True:
            with lock:
                if time.perf_counter() > t_end[0] and done[0] >= cores:
                    return
                done[0] += 1
            f = frames_np[k % n]
            pkt = ref.encode(cfg, f)
            ref.decode(pkt)
            k += cores

    t0 = time.perf_counter()
    t_end[0] = t0 + budget_s
    th = [threading.Thread(target=work, args=(i,)) for i in range(cores)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    el = time.perf_counter() - t0
    return done[0] / el, cores, done[0], el


# ------------------------------------------------------------------ profiling case

def kernel_case(args):
    """One batched encode + decode of a small case (device-resident samples,
    packets and planes; the same library path as the bench), repeated
    --repeat times; prints the per-kernel device times of the last repetition.
    Sized for a profiler capture: --case 3840x2160 --frames 2."""
    import torch
    from topos_codec_b200 import binding as B, synth
    w, h = (int(v) for v in args.case.split("x"))
    n = args.frames
    gpu = B.ToposCodec(B.PRODUCT_LIBRARY)
    L = gpu._lib
    L.tcg_profile_read.argtypes = [ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_uint64)]
    if args.case_gbr:
        from topos_codec_b200.workloads import gbr_config
        cfg = gbr_config(w, h)
        kw = dict(bit_depth=12, pixel_format=2, limited=False, alpha=True, sigma=12)
    elif args.case_v8:
        cfg = B.make_config(w, h, qp=args.case_qp, qmatrix_id=0 if w >= 3840 else 4)
        cfg.reserved[0] = 9  # V8 segmented rANS, 16-block segments, 32-row tiles
        kw = {}
    else:
        cfg = B.make_config(w, h, qp=args.case_qp, qmatrix_id=0 if w >= 3840 else 4, features=3 if w >= 3840 else 1)
        kw = {}
    frames = [[p.to(torch.uint16) for p in synth.make_frame(w, h, seed=0, frame=i, device="cuda", **kw)]
              for i in range(n)]
    cap = gpu.packet_bound(cfg)
    outs = [torch.empty(cap, dtype=torch.uint8, device="cuda") for _ in range(n)]
    dec = [[torch.empty(sh, dtype=torch.uint16, device="cuda") for sh in B.plane_shapes(cfg)] for _ in range(n)]
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
    for r in range(args.repeat):
        if r == args.repeat - 1:
            L.tcg_profile_reset()
            L.tcg_profile_enable(1)
        rc = L.tcg_frame_encode_batch(cfgs, ins, n, optr, caps, st, rcs)
        assert rc == 0, gpu.last_error()
        pk = (B.BatchPacket * n)()
        for i in range(n):
            pk[i].data, pk[i].size = outs[i].data_ptr(), st[i].packet_size
        dec_fn = L.tcg_frame_decode_v8_batch if args.case_v8 else L.tc_frame_decode_batch
        rc = dec_fn(pk, n, dptr, None, infos)
        assert rc == 0, gpu.last_error()
    L.tcg_profile_enable(0)
    res = {}
    for k in range(64):
        name, ms, cnt = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_uint64()
        if L.tcg_profile_read(k, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(cnt)) != 0:
            break
        if cnt.value:
            res[name.value.decode()] = round(ms.value, 3)
    # V8 kernels are counted in the slots of the V7-R2 kernels of the same stage
    print(json.dumps({"case": args.case, "generation": "v8" if args.case_v8 else "v7", "frames": n, "packet_bytes": sum(s.packet_size for s in st),
                      "kernels_ms": res}))


# ------------------------------------------------------------------ GPU path

def main():
    t_main = time.perf_counter()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="seconds per offered load (config: 60)")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the mixed-batch and GBR 4:4:4 + alpha workloads")
    ap.add_argument("--case", default=None, help="WxH: run one small batched round trip for a profiler capture "
                                                   "(with --frames, --repeat, --case-qp, --case-gbr) instead of the bench")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--case-qp", type=int, default=4)
    ap.add_argument("--case-gbr", action="store_true", help="12-bit GBR 4:4:4 + 16-bit alpha at qp 2")
    ap.add_argument("--case-v8", action="store_true", help="V8 segmented rANS packets instead of V7-R2")
    ap.add_argument("--cpu-mode", default=None, choices=["slice", "batch"], help=argparse.SUPPRESS)
    ap.add_argument("--cpu-seconds", type=float, default=6.0, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.cpu_mode:
        cpu_mode_main(args.cpu_mode, args.cpu_seconds, args.frames if args.frames != FRAMES else 8)
        return
    if args.case:
        kernel_case(args)
        return
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from topos_codec_b200 import binding as B, synth

    cfg = B.make_config(W, H, **CFG)
    config_desc = {"workload": f"3840x2160 10-bit 4:2:2 HQ qp4 x{args.frames} frames (round trip)",
                   "frames_per_rank": args.frames, "width": W, "height": H, "qp": 4, "qmatrix_id": 0,
                   "features": "DEBLOCK|QPT2", "slice_rows": 16, "l2": "inputs larger than L2 (>=2 GB per step)",
                   "parallelism": f"frame-sharded x{args.gpus}"}

    if args.impl == "reference":
        if rank != 0:
            return
        if not os.path.exists(REF_LIB):
            print(json.dumps({"impl": "reference", "unavailable": "reference library not built (oracle/_ref)"}))
            return
        frames = [synth.make_frame_np(W, H, seed=0, frame=i) for i in range(16)]
        for _ in range(args.warmup):
            reference_rate(frames[:1], cfg, budget_s=0.0, threads=1)
        rates = []
        for _ in range(args.steps):
            r, cores, n, el = reference_rate(frames, cfg, budget_s=10.0)
            rates.append(r)
        value = statistics.median(rates)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * args.frames / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16/int32",
            "data": "synthetic", "config": config_desc,
            "cpu_baseline": {"value": value, "unit": "frames/s", "cores": cores, "kind": "reference",
                             "sample": f"each step: frame-parallel encode+decode of 16 distinct frames on {cores} "
                                       "threads (slice pool 1 thread per call) for ~10 s",
                             "cpu_model": cpu_model()},
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    gpu = B.ToposCodec(B.PRODUCT_LIBRARY)
    L = gpu._lib
    L.tcg_last_device_ms.restype = ctypes.c_double
    L.tcg_kernel_launches.restype = ctypes.c_uint64
    L.tcg_profile_read.restype = ctypes.c_int32
    L.tcg_profile_read.argtypes = [ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_uint64)]
    L.tcg_device_init(local)

    nf = args.frames
    dev = torch.device("cuda", local)
    # inputs resident in HBM: uint16 planes
    frames_d = []
    from topos_codec_b200 import sharding
    for seed, i in sharding.rank_frames(rank, nf):
        ps = synth.make_frame(W, H, seed=seed, frame=i, device=dev)
        frames_d.append([p.to(torch.uint16) for p in ps])
    torch.cuda.synchronize()
    in_bytes = plane_bytes() * nf
    cap = plane_bytes() * 2 + (1 << 20)
    out_d = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in range(nf)]
    dec_d = [[torch.empty((H, w), dtype=torch.uint16, device=dev) for w in (W, W // 2, W // 2)] for _ in range(nf)]

    cfgs = (B.FrameConfig * nf)(*[cfg] * nf)

    def inputs_for(planes_list):
        arr = (B.FrameInput * nf)()
        for i, planes in enumerate(planes_list):
            arr[i].struct_size = ctypes.sizeof(B.FrameInput)
            arr[i].abi_version = 2
            for p, t in enumerate(planes):
                arr[i].planes[p] = t.data_ptr()
                arr[i].strides[p] = t.shape[1]
        return arr

    in_d = inputs_for(frames_d)
    outs_d = (ctypes.c_void_p * nf)(*[t.data_ptr() for t in out_d])
    caps = (ctypes.c_size_t * nf)(*[cap] * nf)
    stats = (B.FrameStats * nf)()
    rcs = (ctypes.c_int32 * nf)()
    dec_ptrs = (ctypes.c_void_p * (4 * nf))()
    for i in range(nf):
        for p in range(3):
            dec_ptrs[4 * i + p] = dec_d[i][p].data_ptr()
    infos = (B.FrameOutput * nf)()

    def encode_batch(inputs, outs):
        rc = L.tcg_frame_encode_batch(cfgs, inputs, nf, outs, caps, stats, rcs)
        if rc != 0:
            raise RuntimeError(f"encode batch failed [{rc}]: {gpu.last_error()}")
        return L.tcg_last_device_ms()

    def decode_batch(pkts, ptrs):
        arr = (B.BatchPacket * nf)()
        for i in range(nf):
            arr[i].data = pkts[i]
            arr[i].size = stats[i].packet_size
        rc = L.tc_frame_decode_batch(arr, nf, ptrs, None, infos)
        if rc != 0:
            raise RuntimeError(f"decode batch failed [{rc}]: {gpu.last_error()}")
        return L.tcg_last_device_ms()

    pkt_ptrs_d = [t.data_ptr() for t in out_d]

    def step():
        te = encode_batch(in_d, outs_d)
        td = decode_batch(pkt_ptrs_d, dec_ptrs)
        return te, td

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    pkt_bytes = sum(stats[i].packet_size for i in range(nf))

    # ---------------- timed region: device-resident batched round trip ----------------
    L.tcg_profile_reset()
    L.tcg_profile_enable(1)
    launches0 = L.tcg_kernel_launches()
    enc_ms, dec_ms = [], []
    with ClockSampler(local) as clk:
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            te, td = step()
            enc_ms.append(te)
            dec_ms.append(td)
        barrier()
        wall = time.perf_counter() - t0
    L.tcg_profile_enable(0)
    launches = L.tcg_kernel_launches() - launches0
    step_ms = (sum(enc_ms) + sum(dec_ms)) / args.steps
    step_ms, enc_avg, dec_avg = sharding.max_over_ranks([step_ms, sum(enc_ms) / args.steps, sum(dec_ms) / args.steps],
                                                         device=dev)
    value = nf * world / (step_ms / 1000.0)

    # per-kernel timings over the timed region
    kern = {}
    for k in range(64):
        name, ms, n = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_uint64()
        if L.tcg_profile_read(k, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(n)) != 0:
            break
        if n.value:
            kern[name.value.decode()] = {"ms": ms.value, "launches": n.value}

    # ---------------- bit-exactness: batched vs plain per-frame vs oracle ----------------
    batched_pkts = [out_d[i][: stats[i].packet_size].cpu().numpy().tobytes() for i in range(nf)]
    plain_enc_ms, plain_dec_ms, exact = 0.0, 0.0, True
    one_out = torch.empty(cap, dtype=torch.uint8, device=dev)
    st1 = B.FrameStats()
    for i in range(nf):
        rc = L.tc_frame_encode(ctypes.byref(cfg), ctypes.byref(in_d[i]), ctypes.c_void_p(one_out.data_ptr()), cap,
                               ctypes.byref(st1))
        plain_enc_ms += L.tcg_last_device_ms()
        if rc != 0 or one_out[: st1.packet_size].cpu().numpy().tobytes() != batched_pkts[i]:
            exact = False
        info = B.FrameOutput()
        plain_out = [torch.empty_like(dec_d[i][p]) for p in range(3)]
        ptrs1 = (ctypes.c_void_p * 4)(*[t.data_ptr() for t in plain_out], None)
        rc = L.tc_frame_decode(ctypes.c_void_p(out_d[i].data_ptr()), stats[i].packet_size, ptrs1, None, ctypes.byref(info))
        plain_dec_ms += L.tcg_last_device_ms()
        if rc != 0 or not all(torch.equal(a.view(torch.int16), b.view(torch.int16)) for a, b in zip(plain_out, dec_d[i])):
            exact = False
    oracle_ok = None
    if rank == 0 and os.path.exists(ORACLE_LIB):
        orc = B.ToposCodec(ORACLE_LIB)
        f0 = [p.cpu().numpy() for p in frames_d[0]]
        oracle_ok = orc.encode(cfg, f0) == batched_pkts[0]
        d0 = orc.decode(batched_pkts[0])
        oracle_ok = oracle_ok and all(np.array_equal(a, b.cpu().numpy()) for a, b in zip(d0.planes, dec_d[0]))
        exact = exact and oracle_ok

    # ---------------- e2e: host (pinned) buffers through the public API ----------------
    frames_h = [[p.cpu().pin_memory() for p in fr] for fr in frames_d]
    in_h = inputs_for(frames_h)
    out_h = [torch.empty(cap, dtype=torch.uint8).pin_memory() for _ in range(nf)]
    outs_h = (ctypes.c_void_p * nf)(*[t.data_ptr() for t in out_h])
    dec_h = [[torch.empty((H, w), dtype=torch.uint16).pin_memory() for w in (W, W // 2, W // 2)] for _ in range(nf)]
    dec_ptrs_h = (ctypes.c_void_p * (4 * nf))()
    for i in range(nf):
        for p in range(3):
            dec_ptrs_h[4 * i + p] = dec_h[i][p].data_ptr()
    pkt_ptrs_h = [t.data_ptr() for t in out_h]
    # the same warm-up as the device-resident steps: every context the chunked
    # host-memory calls rotate through holds its buffers before timing starts
    for _ in range(args.warmup):
        encode_batch(in_h, outs_h)
        decode_batch(pkt_ptrs_h, dec_ptrs_h)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        encode_batch(in_h, outs_h)
        decode_batch(pkt_ptrs_h, dec_ptrs_h)
    barrier()
    e2e_s = (time.perf_counter() - t0) / args.steps
    e2e_s = sharding.max_over_ranks([e2e_s], device=dev)[0]
    e2e_exact = all(out_h[i][: stats[i].packet_size].numpy().tobytes() == batched_pkts[i] for i in range(nf))
    e2e_exact = e2e_exact and all(torch.equal(dec_h[i][p].view(torch.int16), dec_d[i][p].cpu().view(torch.int16))
                                  for i in range(nf) for p in range(3))
    exact = exact and e2e_exact
    # host-memory batches are coded in pipelined chunks (copies of one chunk
    # overlap the kernels of another); report the split the library used
    L.tcg_pipeline_plan.restype = ctypes.c_uint32
    fb = (ctypes.c_uint64 * nf)(*[in_bytes // nf] * nf)
    e2e_chunks = int(L.tcg_pipeline_plan(0, fb, nf, (ctypes.c_uint32 * 5)()))
    fb = (ctypes.c_uint64 * nf)(*[(in_bytes + pkt_bytes) // nf] * nf)
    e2e_dchunks = int(L.tcg_pipeline_plan(1, fb, nf, (ctypes.c_uint32 * 5)()))

    # ---------------- roofline of the dominant kernel ----------------
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    top = max(kern.items(), key=lambda kv: kv[1]["ms"]) if kern else (None, None)
    roof = None
    if top[0] is not None:
        per_launch_ms = top[1]["ms"] / top[1]["launches"]
        # algorithmic bytes per launch: one launch codes the whole batch
        dec_side = top[0].startswith("k_d") or top[0].startswith("k_deblock")
        out_side = plane_bytes() * nf if dec_side else pkt_bytes
        algo = (pkt_bytes + plane_bytes() * nf) if dec_side else (in_bytes + pkt_bytes)
        achieved = algo / (per_launch_ms / 1000.0) / 1e9
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.txt")
        if os.path.exists(tp):
            for line in open(tp):
                if line.startswith(top[0] + " "):
                    try:
                        traffic = float(line.split()[1]) * nf
                    except ValueError:
                        pass
        roof = {"bound": "hbm", "kernel": top[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                "algorithmic_bytes_per_launch": algo, "launch_ms": per_launch_ms,
                "note": "serial rANS state chains bound this kernel by dependent-op latency, not HBM"}
        _ = out_side

    sections = {"main_s": round(time.perf_counter() - t_main, 1)}
    # ---------------- CPU baseline (rank 0, N=1 only) ----------------
    t_sec = time.perf_counter()
    cpu = None
    if rank == 0 and world == 1 and os.path.exists(REF_LIB):
        f_np = [[p.cpu().numpy() for p in frames_d[i]] for i in range(min(nf, 8))]
        r, cores, n, el = reference_rate(f_np, cfg, budget_s=12.0)
        modes = cpu_modes()
        cpu = {"value": r, "unit": "frames/s", "cores": cores, "kind": "reference",
               "sample": f"{n} frames encoded+decoded frame-parallel (one slice thread per call) in {el:.1f} s",
               "cpu_model": cpu_model(), "simd_backend": modes.get("slice", {}).get("simd_backend"),
               "modes": {"frame_parallel_round_trip_fps": r,
                         "per_frame_slice_parallel": modes.get("slice"),
                         "decode_batch": modes.get("batch")}}

    sections["cpu_baseline_s"] = round(time.perf_counter() - t_sec, 1)
    # ---------------- further workloads: mixed batch, GBR 4:4:4 + alpha ----------------
    t_sec = time.perf_counter()
    extra = {}
    if world == 1 and not args.no_extra:
        from concurrent.futures import ThreadPoolExecutor
        from topos_codec_b200 import workloads as WL
        specs = WL.mixed_specs(64, seed=0)
        mcfgs = [WL.mixed_config(w, h, t, q) for (w, h, t, q) in specs]
        mframes = [[p.to(torch.uint16).contiguous() for p in synth.make_frame(w, h, seed=11, frame=i, device=dev)]
                   for i, (w, h, _, _) in enumerate(specs)]
        r = WL.batched_vs_plain(gpu, mcfgs, mframes)
        r.pop("packets")
        r["workload"] = ("64 frames, resolution uniform over 1280x720/1920x1080/3840x2160/7680x4320, tier uniform "
                         "over proxy/lt/422/hq, qp uniform 2..16 (seed 0), 10-bit 4:2:2")
        r["resolutions"] = {f"{w}x{h}": sum(1 for s in specs if s[:2] == (w, h)) for (w, h) in WL.MIXED_RES}
        extra["mixed_batch"] = r
        del mframes
        gcfg = WL.gbr_config()
        gframes = [[p.to(torch.uint16).contiguous() for p in
                    synth.make_frame(4096, 2160, seed=21, frame=i, bit_depth=12, pixel_format=2, limited=False,
                                     alpha=True, sigma=12, device=dev)] for i in range(32)]
        r = WL.batched_vs_plain(gpu, [gcfg] * 32, gframes)
        gpk = r.pop("packets")
        r["workload"] = "32 frames 4096x2160 12-bit GBR 4:4:4 full range + 16-bit alpha, qp 2"
        if rank == 0 and os.path.exists(REF_LIB):
            ref = B.ToposCodec(REF_LIB)
            sub = [[p.cpu().numpy() for p in gframes[i]] for i in range(8)]
            with ThreadPoolExecutor(8) as ex:
                rpk = list(ex.map(lambda f: ref.encode(gcfg, f), sub))
            r["reference_packets_equal_8_frames"] = all(a == b for a, b in zip(rpk, gpk[:8]))
            r["damaged_decode_vs_reference"] = WL.concealment_parity(gpu, ref, WL.corrupt_slices(rpk, 0.01, seed=5))
            r["damaged_decode_vs_reference"]["corruption"] = "1 % of the slices of 8 reference packets, one payload byte each"
        extra["gbr4444_alpha"] = r
        del gframes
        # the bench batch coded as V8 (segmented rANS: 16-block segments, 32-row tiles; no deblocking or
        # refined qp table in V8): batched encode and batched decode beside the per-frame calls, and the
        # packets of two frames against the reference library's
        v8cfg = B.make_config(W, H, qp=4, qmatrix_id=0)
        v8cfg.reserved[0] = 9
        r = WL.batched_vs_plain(gpu, [v8cfg] * nf, frames_d, v8=True)
        v8pk = r.pop("packets")
        r["workload"] = f"the {nf} 3840x2160 10-bit 4:2:2 frames as V8 packets (qp 4, flat matrix), device-resident"
        r["encode_fps"] = nf / (r["batched_encode_ms"] / 1000.0)
        r["decode_fps"] = nf / (r["batched_decode_ms"] / 1000.0)
        if rank == 0 and os.path.exists(REF_LIB):
            ref = B.ToposCodec(REF_LIB)
            r["reference_packets_equal_2_frames"] = all(
                ref.encode(v8cfg, [p.cpu().numpy() for p in frames_d[i]]) == v8pk[i] for i in (0, nf - 1))
        extra["v8_batch"] = r
        del v8pk
        # size-targeted encode: 8 frames of the bench workload from host memory, target = the
        # first frame's packet at qp 24, qp searched over 0..63 (strict search, hints on)
        sframes = [[p.cpu().numpy() for p in frames_d[i]] for i in range(min(nf, 8))]
        c24 = B.make_config(W, H, **{**CFG, "qp": 24})
        target = len(gpu.encode(c24, sframes[0]))
        ref = B.ToposCodec(REF_LIB) if (rank == 0 and os.path.exists(REF_LIB)) else None
        r = WL.sized_vs_reference(gpu, ref, cfg, sframes, target, 0, 63, ref_threads=min(16, os.cpu_count() or 1))
        r["workload"] = ("3840x2160 10-bit 4:2:2 HQ from host memory, tc_frame_encode_sized per frame in order "
                         "after one untimed call, target = frame 0 at qp 24, qp 0..63")
        extra["sized_encode"] = r
        del sframes
        # preview decode: the batch's packets at half size (1920x1080, 24 zigzag coefficients kept)
        r = WL.preview_vs_reference(gpu, ref, batched_pkts, scale=1)
        r["workload"] = "the 60 3840x2160 HQ packets decoded at 1/2 size, device-resident"
        extra["preview_decode"] = r
        torch.cuda.empty_cache()
    sections["workloads_s"] = round(time.perf_counter() - t_sec, 1)

    # ---------------- serving: open-loop request streams at 25/50/75/100 % of saturation ----------------
    t_sec = time.perf_counter()
    served = None
    if world == 1 and not args.no_serve:
        # the earlier sections' idle call contexts hold their largest buffers;
        # the serving streams allocate their own through torch
        gpu._lib.tcg_release_idle_memory()
        torch.cuda.empty_cache()
        from topos_codec_b200 import serving
        floors = [serving.single_frame_floor(gpu, 1920, 1080, "422", g) for g in ("v7", "v8")]
        kinds = serving._kinds(gpu, torch, dev, 0, "v7")
        pk = serving.peak_rps(gpu, kinds=kinds)
        sat = pk["sustained_rps"]
        # a short discarded trace first: the decode-tiling tuner times the tilings
        # on the first batch of each batch-size class
        serving.run_trace(gpu, rate_rps=0.5 * sat, duration_s=3.0, seed=7, kinds=kinds)
        loads = {}
        for ld in (0.25, 0.5, 0.75, 1.0):
            loads[ld] = serving.run_trace(gpu, rate_rps=ld * sat, duration_s=args.serve_seconds, seed=int(ld * 100),
                                          kinds=kinds)
        served = dict(loads[0.5])
        psat = serving.plain_saturation_rps(gpu, kinds=kinds)
        plain_s = min(30.0, args.serve_seconds)
        plain = {"saturation_rps": psat,
                 "at_quarter_batched_saturation": serving.run_trace_plain(gpu, rate_rps=0.25 * sat,
                                                                          duration_s=plain_s, kinds=kinds),
                 "at_half_plain_saturation": serving.run_trace_plain(gpu, rate_rps=0.5 * psat, duration_s=plain_s,
                                                                     kinds=kinds)}
        del kinds
        torch.cuda.empty_cache()
        gpu._lib.tcg_release_idle_memory()
        # the same stream coded as V8 (segmented rANS): many short chains per frame
        k8 = serving._kinds(gpu, torch, dev, 0, "v8")
        pk8 = serving.peak_rps(gpu, generation="v8", kinds=k8)
        sat8 = pk8["sustained_rps"]
        serving.run_trace(gpu, rate_rps=0.5 * sat8, duration_s=3.0, seed=7, generation="v8", kinds=k8)
        v8_half = serving.run_trace(gpu, rate_rps=0.5 * sat8, duration_s=args.serve_seconds, seed=50,
                                    generation="v8", kinds=k8)
        del k8
        keys = ("offered_rps", "throughput_rps", "p50_ms", "p99_ms", "p999_ms", "errors", "dropped", "by_resolution",
                "server_side", "submit_lag")
        served.update({"load": 0.5, "saturation_rps": sat,
                       "mix": "50/50 encode/decode; 1080p 40 %, 2160p 40 %, 720p 20 %; 10-bit 4:2:2 tiers 422/HQ",
                       "latency": "client side, from each request's scheduled (open-loop Poisson) arrival to its "
                                  "completion; server_side: submission to completion",
                       "seconds_per_load": args.serve_seconds,
                       "loads": {str(k): {x: v[x] for x in keys} for k, v in loads.items()},
                       "plain_per_request": plain,
                       "single_frame_floor_1080p": floors,
                       "v8_at_half_saturation": dict({x: v8_half[x] for x in keys}, saturation_rps=sat8,
                                                     by_direction=v8_half["by_direction"])})

    sections["serving_s"] = round(time.perf_counter() - t_sec, 1)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16/int32", "data": "synthetic", "config": config_desc,
            "encode_fps": nf * world / (enc_avg / 1000.0), "decode_fps": nf * world / (dec_avg / 1000.0),
            "plain_encode_fps": nf / (plain_enc_ms / 1000.0), "plain_decode_fps": nf / (plain_dec_ms / 1000.0),
            "batched_vs_plain": (plain_enc_ms + plain_dec_ms) / step_ms,
            "bit_exact": exact, "oracle_frame0_exact": oracle_ok,
            "pixel_gbs": (in_bytes * 2) * world / (step_ms / 1000.0) / 1e9,
            "wall_s_timed": wall,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "kernels_ms": {k: round(v["ms"] / args.steps, 3) for k, v in kern.items()},
            "roofline": roof,
            "cpu_baseline": cpu,
            "served": served,
            "workloads": extra,
            "section_seconds": sections,
            "e2e": {"value": nf * world / e2e_s, "unit": "frames/s",
                    "h2d_bytes_per_step": int(in_bytes + pkt_bytes), "d2h_bytes_per_step": int(pkt_bytes + in_bytes),
                    "encode_chunks": e2e_chunks, "decode_chunks": e2e_dchunks},
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
