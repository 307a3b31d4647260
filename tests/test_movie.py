"""MOV read path against the reference library built from its sources
(oracle/_ref): movies muxed by the reference (standard and faststart layouts,
alpha budget, several frame sizes) are read by both libraries; movie
information, every sample, timing, sync points, batched reads and the
statuses of truncated and damaged files agree. The GPU test decodes a movie
range through tcg_movie_decode_batch and checks it against the reference's
decode of the same samples."""
import ctypes

import numpy as np
import pytest

from topos_codec_b200 import binding as B, synth

READ = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t)
WRITE = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)
SEEKW = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t)


class IO(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32), ("ctx", ctypes.c_void_p),
                ("read", READ), ("write", WRITE), ("seek_write", SEEKW), ("length", ctypes.c_uint64),
                ("reserved", ctypes.c_uint32 * 4)]


class MovieConfig(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32),
                ("visible_width", ctypes.c_uint16), ("visible_height", ctypes.c_uint16),
                ("profile", ctypes.c_uint8), ("pixel_format", ctypes.c_uint8), ("bit_depth", ctypes.c_uint8),
                ("qmatrix_id", ctypes.c_uint8), ("qp_base", ctypes.c_uint8), ("qp_delta_luma", ctypes.c_int8),
                ("qp_delta_chroma", ctypes.c_int8), ("alpha_mode", ctypes.c_uint8),
                ("alpha_bit_depth", ctypes.c_uint8), ("alpha_premultiplied", ctypes.c_uint8),
                ("color_range", ctypes.c_uint8), ("color_primaries", ctypes.c_uint8),
                ("color_transfer", ctypes.c_uint8), ("color_matrix", ctypes.c_uint8),
                ("chroma_siting", ctypes.c_uint8), ("sar_num", ctypes.c_uint16), ("sar_den", ctypes.c_uint16),
                ("timescale", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 8)]


class MovieInfo(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32),
                ("visible_width", ctypes.c_uint16), ("visible_height", ctypes.c_uint16),
                ("profile", ctypes.c_uint8), ("pixel_format", ctypes.c_uint8), ("bit_depth", ctypes.c_uint8),
                ("qmatrix_id", ctypes.c_uint8), ("qp_base", ctypes.c_uint8), ("qp_delta_luma", ctypes.c_int8),
                ("qp_delta_chroma", ctypes.c_int8), ("alpha_mode", ctypes.c_uint8),
                ("alpha_bit_depth", ctypes.c_uint8), ("alpha_premultiplied", ctypes.c_uint8),
                ("color_range", ctypes.c_uint8), ("color_primaries", ctypes.c_uint8),
                ("color_transfer", ctypes.c_uint8), ("color_matrix", ctypes.c_uint8),
                ("chroma_siting", ctypes.c_uint8), ("sar_num", ctypes.c_uint16), ("sar_den", ctypes.c_uint16),
                ("timescale", ctypes.c_uint32), ("sample_count", ctypes.c_uint32), ("faststart", ctypes.c_uint32),
                ("index_bytes", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 8)]


class Source:
    """A byte string behind the topos_io read callback."""

    def __init__(self, data: bytes):
        self.buf = ctypes.create_string_buffer(bytes(data), max(len(data), 1))
        self.n = len(data)

        def rd(ctx, off, dst, n):
            if off + n > self.n:
                return -1
            ctypes.memmove(dst, ctypes.addressof(self.buf) + off, n)
            return 0
        self.cb = READ(rd)
        self.io = IO()
        self.io.struct_size, self.io.abi_version = ctypes.sizeof(IO), 2
        self.io.read = self.cb
        self.io.length = self.n


class Sink:
    def __init__(self):
        self.data = bytearray()

        def wr(ctx, src, n):
            self.data += ctypes.string_at(src, n)
            return 0

        def sw(ctx, off, src, n):
            self.data[off:off + n] = ctypes.string_at(src, n)
            return 0
        self.w, self.s = WRITE(wr), SEEKW(sw)
        self.io = IO()
        self.io.struct_size, self.io.abi_version = ctypes.sizeof(IO), 2
        self.io.write, self.io.seek_write = self.w, self.s


def _mux(reference, packets, fc: B.FrameConfig, timescale=24000, dur=1001):
    L = reference._lib
    mc = MovieConfig()
    mc.struct_size, mc.abi_version = ctypes.sizeof(MovieConfig), 2
    for f in ("visible_width", "visible_height", "profile", "pixel_format", "bit_depth", "qmatrix_id", "qp_base",
              "qp_delta_luma", "qp_delta_chroma", "alpha_mode", "alpha_bit_depth", "alpha_premultiplied"):
        setattr(mc, f, getattr(fc, f))
    rc, info = reference.query(packets[0])  # colour fields and aspect as the encoder wrote them
    assert rc == 0
    for f in ("color_range", "color_primaries", "color_transfer", "color_matrix", "chroma_siting", "sar_num",
              "sar_den"):
        setattr(mc, f, getattr(info, f))
    mc.timescale = timescale
    sink = Sink()
    m = ctypes.c_void_p()
    L.tc_mux_create.restype = ctypes.c_int32
    assert L.tc_mux_create(ctypes.byref(mc), ctypes.byref(sink.io), ctypes.byref(m)) == 0, reference.last_error()
    for i, p in enumerate(packets):
        buf = np.frombuffer(p, np.uint8)
        rc = L.tc_mux_add_packet(m, ctypes.c_void_p(buf.ctypes.data), ctypes.c_size_t(len(p)),
                                 ctypes.c_uint64(i * dur), ctypes.c_uint32(dur))
        assert rc == 0, reference.last_error()
    assert L.tc_mux_finish(m) == 0, reference.last_error()
    L.tc_mux_free(m)
    return bytes(sink.data)


def _faststart(reference, data: bytes) -> bytes:
    src, dst = Source(data), Sink()
    assert reference._lib.tc_movie_faststart(ctypes.byref(src.io), ctypes.byref(dst.io)) == 0, reference.last_error()
    return bytes(dst.data)


def _read_all(codec, data: bytes):
    """Everything the reader reports about a movie, or the open status."""
    L = codec._lib
    src = Source(data)
    mv = ctypes.c_void_p()
    rc = int(L.tc_movie_open(ctypes.byref(src.io), ctypes.byref(mv)))
    if rc != 0:
        return ("open", rc)
    try:
        info = MovieInfo()
        info.struct_size, info.abi_version = ctypes.sizeof(MovieInfo), 2
        out = [int(L.tc_movie_info(mv, ctypes.byref(info))), bytes(info)]
        n = info.sample_count
        for i in range(n):
            need = ctypes.c_size_t()
            r0 = int(L.tc_movie_packet(mv, i, None, ctypes.c_size_t(0), ctypes.byref(need)))
            buf = (ctypes.c_uint8 * max(need.value, 1))()
            r1 = int(L.tc_movie_packet(mv, i, buf, need, ctypes.byref(need)))
            pts, dur, sync, prev = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint8(), ctypes.c_uint32()
            r2 = int(L.tc_movie_packet_pts(mv, i, ctypes.byref(pts), ctypes.byref(dur)))
            r3 = int(L.tc_movie_packet_sync(mv, i, ctypes.byref(sync)))
            r4 = int(L.tc_movie_prev_sync(mv, i, ctypes.byref(prev)))
            out.append((r0, r1, need.value, bytes(buf) if r1 == 0 else None, r2, pts.value, dur.value, r3,
                        sync.value, r4, prev.value))
        for start, count in ((0, n), (1, max(0, n - 2)), (n - 1, 1), (n, 1), (0, n + 1)):
            need = ctypes.c_size_t()
            r0 = int(L.tc_movie_packet_batch(mv, start, count, None, ctypes.c_size_t(0), None, None, ctypes.byref(need)))
            arena = (ctypes.c_uint8 * max(need.value, 1))()
            offs = (ctypes.c_size_t * max(count, 1))()
            sizes = (ctypes.c_size_t * max(count, 1))()
            r1 = int(L.tc_movie_packet_batch(mv, start, count, arena, need, offs, sizes, ctypes.byref(need)))
            out.append(("batch", start, count, r0, r1, need.value, bytes(arena) if r1 == 0 else None,
                        list(offs) if r1 == 0 else None, list(sizes) if r1 == 0 else None))
        return tuple(out)
    finally:
        L.tc_movie_close(mv)


@pytest.fixture(scope="module")
def movies(reference):
    """(label, file bytes, frame config, packets) of movies the reference muxes."""
    out = []
    for label, w, h, kw, n in [("422 deblock", 320, 192, dict(qp=8, qmatrix_id=4, features=1), 5),
                               ("odd", 203, 77, dict(qp=12), 3)]:
        cfg = B.make_config(w, h, **kw)
        pk = [reference.encode(cfg, synth.make_frame_np(w, h, seed=300 + i)) for i in range(n)]
        data = _mux(reference, pk, cfg)
        out.append((label, data, cfg, pk))
        out.append((label + " faststart", _faststart(reference, data), cfg, pk))
    w, h = 96, 64
    cfg = B.make_config(w, h, qp=2, bit_depth=12, pixel_format=2, profile=5, alpha_mode=1, alpha_bit_depth=16,
                        color_range=1)
    pk = [reference.encode(cfg, synth.make_frame_np(w, h, seed=320 + i, bit_depth=12, pixel_format=2, limited=False,
                                                    alpha=True, sigma=12)) for i in range(3)]
    out.append(("444 alpha", _mux(reference, pk, cfg, timescale=30000, dur=1000), cfg, pk))
    return out


def test_movie_reads_match_reference(product, reference, movies):
    for label, data, _, pk in movies:
        a, b = _read_all(product, data), _read_all(reference, data)
        assert a == b, label
        assert a[0] == 0 and [x[3] for x in a[2:2 + len(pk)]] == pk, label


def test_movie_damage_statuses_match_reference(product, reference, movies):
    """Truncated files and single changed bytes (headers, tables, samples):
    the same open status, and when both open, the same reads."""
    import random
    rng = random.Random(4)
    for label, data, _, _ in movies[:3]:
        cuts = sorted({0, 7, 19, 20, 64, len(data) // 3, len(data) // 2, len(data) - 1} | {rng.randrange(len(data)) for _ in range(12)})
        for cut in cuts:
            a, b = _read_all(product, data[:cut]), _read_all(reference, data[:cut])
            assert a == b, (label, "cut", cut)
        moov = data.find(b"moov")
        for _ in range(60):
            d = bytearray(data)
            i = rng.randrange(moov - 4, len(d)) if moov > 0 and rng.random() < 0.7 else rng.randrange(len(d))
            d[i] ^= 1 << rng.randrange(8)
            a, b = _read_all(product, bytes(d)), _read_all(reference, bytes(d))
            assert a == b, (label, "byte", i)


@pytest.mark.gpu
def test_movie_decode_batch_vs_reference(product, reference, movies):
    for label, data, _, pk in movies:
        L = product._lib
        src = Source(data)
        mv = ctypes.c_void_p()
        assert L.tc_movie_open(ctypes.byref(src.io), ctypes.byref(mv)) == 0
        try:
            n = len(pk)
            infos = (B.FrameOutput * n)()
            L.tcg_movie_decode_batch.restype = ctypes.c_int32
            assert L.tcg_movie_decode_batch(mv, 0, n, None, None, infos) == 0
            planes = [[np.zeros(s, np.uint16) for s in B.ToposCodec.geometry(infos[i])] for i in range(n)]
            ptrs = (ctypes.c_void_p * (4 * n))()
            for i in range(n):
                for p, a in enumerate(planes[i]):
                    ptrs[4 * i + p] = a.ctypes.data
            assert L.tcg_movie_decode_batch(mv, 0, n, ptrs, None, infos) == 0, product.last_error()
            for i in range(n):
                want = reference.decode(pk[i])
                assert all(np.array_equal(x, y) for x, y in zip(want.planes, planes[i])), (label, i)
        finally:
            L.tc_movie_close(mv)
