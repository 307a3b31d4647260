"""The continuous-batching server (tcg_server_*): encode and decode requests of
mixed sizes submitted together, while earlier ones are still on the GPU, give
exactly the results of the single-frame calls."""
import numpy as np
import pytest

from topos_codec_b200 import binding as B, synth

pytestmark = pytest.mark.gpu


def test_server_mixed_requests_match_single_calls(product):
    sizes = [(1920, 1080, 8), (640, 360, 6), (1280, 720, 12), (333, 77, 3), (3840, 2160, 4), (96, 64, 16)]
    cfgs, frames, want = [], [], []
    for i, (w, h, qp) in enumerate(sizes):
        cfg = B.make_config(w, h, qp=qp, qmatrix_id=0 if w >= 3840 else 4, features=3 if w >= 3840 else 1)
        fr = synth.make_frame_np(w, h, seed=300 + i)
        cfgs.append(cfg)
        frames.append(fr)
        want.append(product.encode(cfg, fr))
    want_dec = [product.decode(p) for p in want]
    srv = B.Server(product, max_batch_frames=4)
    try:
        for rnd in range(2):  # two rounds: a fresh server queue and one with warm contexts
            outs, tickets, dec_bufs, pkt_bufs = [], [], [], []
            for i, cfg in enumerate(cfgs):
                cap = product.packet_bound(cfg)
                out = np.zeros(cap, dtype=np.uint8)
                outs.append(out)
                tickets.append(("e", i, srv.submit_encode(cfg, frames[i], out.ctypes.data, cap)))
                # a decode of a different frame in the same mix
                j = (i + 1 + rnd) % len(sizes)
                pk = np.frombuffer(want[j], dtype=np.uint8).copy()
                planes = [np.zeros(p.shape, dtype=np.uint16) for p in want_dec[j].planes]
                pkt_bufs.append(pk)
                dec_bufs.append((j, planes))
                tickets.append(("d", len(dec_bufs) - 1,
                                srv.submit_decode(pk.ctypes.data, pk.size, [p.ctypes.data for p in planes])))
            for kind, i, t in tickets:
                st, stats, info, lat = srv.wait(t)
                assert lat > 0.0
                if kind == "e":
                    assert st == 0
                    assert outs[i][: stats.packet_size].tobytes() == want[i]
                else:
                    j, planes = dec_bufs[i]
                    assert st == 0 and info.visible_width == sizes[j][0]
                    for a, b in zip(planes, want_dec[j].planes):
                        assert np.array_equal(a, b)
    finally:
        srv.close()


def test_server_rejects_bad_packet(product):
    srv = B.Server(product)
    try:
        bad = np.frombuffer(b"TPIC" + bytes(60), dtype=np.uint8).copy()
        with pytest.raises(B.ToposCodecError):
            srv.submit_decode(bad.ctypes.data, bad.size, [0, 0, 0])
    finally:
        srv.close()


def test_server_v8_requests_match_single_calls(product):
    """V8 encode and decode requests beside V7-R2 ones give the single calls' results."""
    specs = [(1920, 1080, 9), (640, 360, 8), (1280, 720, 9), (320, 180, 8)]
    srv = B.Server(product, max_batch_frames=8)
    try:
        cfgs, frames, want = [], [], []
        for i, (w, h, em) in enumerate(specs):
            cfg = B.make_config(w, h, qp=6, qmatrix_id=4)
            cfg.reserved[0] = em
            fr = synth.make_frame_np(w, h, seed=700 + i)
            cfgs.append(cfg)
            frames.append(fr)
            want.append(product.encode(cfg, fr))
        want_dec = [product.decode(p) for p in want]
        tickets, outs, decs, pkts = [], [], [], []
        for i, cfg in enumerate(cfgs):
            cap = product.packet_bound(cfg)
            outs.append(np.zeros(cap, dtype=np.uint8))
            tickets.append(("e", i, srv.submit_encode(cfg, frames[i], outs[i].ctypes.data, cap)))
            pk = np.frombuffer(want[i], dtype=np.uint8).copy()
            pkts.append(pk)
            decs.append([np.zeros(p.shape, dtype=np.uint16) for p in want_dec[i].planes])
            tickets.append(("d", i, srv.submit_decode(pk.ctypes.data, pk.size, [p.ctypes.data for p in decs[i]])))
        for kind, i, t in tickets:
            st, stats, info, lat = srv.wait(t)
            assert st == 0
            if kind == "e":
                assert outs[i][: stats.packet_size].tobytes() == want[i]
            else:
                for a, b in zip(decs[i], want_dec[i].planes):
                    assert np.array_equal(a, b)
    finally:
        srv.close()


def test_server_takes_arrivals_while_batches_run(product):
    """Continuous batching: a small request submitted while a batch of large
    ones is on the GPU is taken by another worker and completes first, with
    the same bytes as its single call."""
    import time
    big_cfg = B.make_config(3840, 2160, qp=4, qmatrix_id=0, features=3)
    big = synth.make_frame_np(3840, 2160, seed=5)
    small_cfg = B.make_config(1280, 720, qp=8, qmatrix_id=4, features=1)
    small = synth.make_frame_np(1280, 720, seed=6)
    want = product.encode(small_cfg, small)
    srv = B.Server(product, max_batch_frames=8, workers=4)
    try:
        cap_b, cap_s = product.packet_bound(big_cfg), product.packet_bound(small_cfg)
        outs_b = [np.zeros(cap_b, dtype=np.uint8) for _ in range(2)]
        out_s = np.zeros(cap_s, dtype=np.uint8)
        tb = [srv.submit_encode(big_cfg, big, o.ctypes.data, cap_b) for o in outs_b]
        time.sleep(0.005)
        ts = srv.submit_encode(small_cfg, small, out_s.ctypes.data, cap_s)
        st, stats, _, lat_s = srv.wait(ts)
        assert st == 0 and out_s[: stats.packet_size].tobytes() == want
        lats_b = [srv.wait(t)[3] for t in tb]
        assert lat_s < min(lats_b)
    finally:
        srv.close()
