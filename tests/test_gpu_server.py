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
