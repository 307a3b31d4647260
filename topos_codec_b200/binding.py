"""ctypes binding for any library that exports the Topos Codec frame ABI.

Mirrors the reference Python binding's ``ToposCodec`` surface for the frame
path (python/topos_codec/topos_binding.py:2783-3360: ``encode``,
``encode_frame``, ``decode``, ``packet_bound``, ``last_error``) with the same
error behaviour: negative statuses raise ``ToposCodecError``; concealment is a
warning status returned beside the decoded frame. The same class drives the
GPU library (the product), and in tests the CPU oracle or the reference
library, so that parity tests read like the reference's own tests.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

TOPOS_CODEC_ABI_VERSION = 2
TC_FRAME_MAX_PLANES = 4
TC_MAX_SLICES = 512

TC_OK = 0
TC_WARN_CONCEALED = 1
TC_ERR_INVALID_ARGUMENT = -1
TC_ERR_OUT_OF_MEMORY = -2
TC_ERR_UNSUPPORTED_VERSION = -3
TC_ERR_LIMIT_EXCEEDED = -8
TC_ERR_MALFORMED = -9
TC_ERR_TRUNCATED = -10
TC_ERR_CHECKSUM_MISMATCH = -11
TC_ERR_BUFFER_TOO_SMALL = -15
TC_ERR_NOT_IMPLEMENTED = -16

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIBRARY = os.path.join(PACKAGE_DIR, "lib", "libtopos_codec.so")


class ToposCodecError(RuntimeError):
    def __init__(self, message: str, status: int = 0):
        super().__init__(message)
        self.status = status


class FrameConfig(ctypes.Structure):
    """topos_frame_config (reference native/include/topos_codec.h:177-224)."""
    _fields_ = [
        ("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32),
        ("visible_width", ctypes.c_uint16), ("visible_height", ctypes.c_uint16),
        ("profile", ctypes.c_uint8), ("pixel_format", ctypes.c_uint8),
        ("bit_depth", ctypes.c_uint8), ("qmatrix_id", ctypes.c_uint8),
        ("qp_base", ctypes.c_uint8), ("qp_delta_luma", ctypes.c_int8),
        ("qp_delta_chroma", ctypes.c_int8), ("slice_rows", ctypes.c_uint8),
        ("alpha_mode", ctypes.c_uint8), ("alpha_bit_depth", ctypes.c_uint8),
        ("alpha_premultiplied", ctypes.c_uint8), ("color_range", ctypes.c_uint8),
        ("color_primaries", ctypes.c_uint8), ("color_transfer", ctypes.c_uint8),
        ("color_matrix", ctypes.c_uint8), ("chroma_siting", ctypes.c_uint8),
        ("sar_num", ctypes.c_uint16), ("sar_den", ctypes.c_uint16),
        ("reserved", ctypes.c_uint32 * 8),
    ]


class FrameInput(ctypes.Structure):
    """topos_frame_input (reference native/include/topos_codec.h:231-237)."""
    _fields_ = [
        ("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32),
        ("planes", ctypes.c_void_p * TC_FRAME_MAX_PLANES),
        ("strides", ctypes.c_size_t * TC_FRAME_MAX_PLANES),
        ("reserved", ctypes.c_uint32 * 8),
    ]


class FrameStats(ctypes.Structure):
    """topos_frame_stats (reference native/include/topos_codec.h:240-254)."""
    _fields_ = [
        ("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32),
        ("packet_size", ctypes.c_uint32), ("color_payload_bytes", ctypes.c_uint32),
        ("alpha_payload_bytes", ctypes.c_uint32), ("color_header_bytes", ctypes.c_uint32),
        ("alpha_header_bytes", ctypes.c_uint32), ("slice_count", ctypes.c_uint16),
        ("qp_base", ctypes.c_uint8), ("reserved8", ctypes.c_uint8),
        ("alpha_max_abs_error", ctypes.c_uint16), ("reserved16", ctypes.c_uint16),
        ("reserved", ctypes.c_uint32 * 8),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_
                if name not in ("reserved", "struct_size", "abi_version")}


class FrameOutput(ctypes.Structure):
    """topos_frame_output (reference native/include/topos_codec.h:261-285)."""
    _fields_ = [
        ("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32),
        ("visible_width", ctypes.c_uint16), ("visible_height", ctypes.c_uint16),
        ("coded_width", ctypes.c_uint16), ("coded_height", ctypes.c_uint16),
        ("plane_count", ctypes.c_uint8), ("bit_depth", ctypes.c_uint8),
        ("profile", ctypes.c_uint8), ("pixel_format", ctypes.c_uint8),
        ("alpha_mode", ctypes.c_uint8), ("alpha_bit_depth", ctypes.c_uint8),
        ("color_range", ctypes.c_uint8), ("color_primaries", ctypes.c_uint8),
        ("color_transfer", ctypes.c_uint8), ("color_matrix", ctypes.c_uint8),
        ("chroma_siting", ctypes.c_uint8),
        ("concealed_slices", ctypes.c_uint16), ("slice_count", ctypes.c_uint16),
        ("sar_num", ctypes.c_uint16), ("sar_den", ctypes.c_uint16),
        ("slice_status", ctypes.c_uint8 * TC_MAX_SLICES),
        ("reserved", ctypes.c_uint32 * 8),
    ]


class BatchPacket(ctypes.Structure):
    """topos_batch_packet (reference native/include/topos_codec.h:387-390)."""
    _fields_ = [("data", ctypes.c_void_p), ("size", ctypes.c_size_t)]


def make_config(width: int, height: int, *, qp: int = 8, qmatrix_id: int = 0,
                pixel_format: int = 0, bit_depth: int = 10, profile: int = 3,
                slice_rows: int = 0, alpha_mode: int = 0, alpha_bit_depth: int = 0,
                features: int = 0, qp_delta_luma: int = 0, qp_delta_chroma: int = 0,
                color_range: int = 0, color_matrix: int = 0, color_primaries: int = 0,
                color_transfer: int = 0, chroma_siting: int = 0,
                coding: int = 8) -> FrameConfig:
    """A V7-R2 frame config (reserved[0] = 8; reserved[5] = DEBLOCK|QPT2 bits)."""
    c = FrameConfig()
    c.struct_size = ctypes.sizeof(FrameConfig)
    c.abi_version = TOPOS_CODEC_ABI_VERSION
    c.visible_width, c.visible_height = width, height
    c.profile, c.pixel_format, c.bit_depth = profile, pixel_format, bit_depth
    c.qmatrix_id, c.qp_base, c.slice_rows = qmatrix_id, qp, slice_rows
    c.qp_delta_luma, c.qp_delta_chroma = qp_delta_luma, qp_delta_chroma
    c.alpha_mode, c.alpha_bit_depth = alpha_mode, alpha_bit_depth
    c.color_range, c.color_matrix = color_range, color_matrix
    c.color_primaries, c.color_transfer, c.chroma_siting = color_primaries, color_transfer, chroma_siting
    c.reserved[0] = coding
    c.reserved[5] = features
    return c


def plane_shapes(cfg: FrameConfig) -> List[Tuple[int, int]]:
    """(height, width) of each visible input plane for a config."""
    w, h = cfg.visible_width, cfg.visible_height
    cw = (w + 1) // 2 if cfg.pixel_format == 0 else w
    n = 3 + (1 if cfg.alpha_mode else 0)
    return [(h, w), (h, cw), (h, cw), (h, w)][:n]


@dataclass
class DecodedFrame:
    planes: List[np.ndarray]
    info: FrameOutput
    status: int

    @property
    def slice_status(self) -> List[int]:
        return list(self.info.slice_status[: self.info.slice_count])


def _u16_ptr(a: np.ndarray) -> int:
    assert a.dtype == np.uint16
    return a.ctypes.data


class ToposCodec:
    """Typed wrapper around a library exporting the frame ABI."""

    def __init__(self, library: Optional[str] = None, *, mode: int = os.RTLD_LOCAL):
        path = library or PRODUCT_LIBRARY
        if not os.path.exists(path):
            raise ToposCodecError(f"library not found: {path} (build it first)")
        self.path = path
        self._lib = ctypes.CDLL(path, mode=mode)
        self._configure()

    def _configure(self) -> None:
        L = self._lib
        L.tc_frame_encode.restype = ctypes.c_int32
        L.tc_frame_encode.argtypes = [ctypes.POINTER(FrameConfig), ctypes.POINTER(FrameInput),
                                      ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(FrameStats)]
        L.tc_frame_decode.restype = ctypes.c_int32
        L.tc_frame_decode.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.POINTER(FrameOutput)]
        L.tc_frame_decode_batch.restype = ctypes.c_int32
        L.tc_frame_decode_batch.argtypes = [ctypes.POINTER(BatchPacket), ctypes.c_uint32,
                                            ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.POINTER(FrameOutput)]
        L.tc_frame_packet_bound.restype = ctypes.c_size_t
        L.tc_frame_packet_bound.argtypes = [ctypes.POINTER(FrameConfig)]
        L.tc_frame_config_validate.restype = ctypes.c_int32
        L.tc_frame_config_validate.argtypes = [ctypes.POINTER(FrameConfig)]
        L.tc_last_error.restype = ctypes.c_char_p
        L.tc_last_error.argtypes = []
        if hasattr(L, "tc_frame_encode_sized"):
            L.tc_frame_encode_sized.restype = ctypes.c_int32
            L.tc_frame_encode_sized.argtypes = [ctypes.POINTER(FrameConfig), ctypes.POINTER(FrameInput),
                                                ctypes.c_uint32, ctypes.c_uint8, ctypes.c_uint8,
                                                ctypes.POINTER(ctypes.c_uint8), ctypes.c_void_p, ctypes.c_size_t,
                                                ctypes.POINTER(FrameStats)]
        for name, res in (("tc_dev_sized_iters", ctypes.c_uint64), ("tc_dev_sized_calls", ctypes.c_uint64)):
            if hasattr(L, name):
                getattr(L, name).restype = res
                getattr(L, name).argtypes = []
        for name in ("tc_dev_set_sized_mode", "tc_dev_set_qp_hint", "tc_dev_set_qp_hint_model", "tc_dev_set_sized_m7"):
            if hasattr(L, name):
                getattr(L, name).restype = None
                getattr(L, name).argtypes = [ctypes.c_int32]
        self.has_encode_batch = hasattr(L, "tcg_frame_encode_batch")
        if self.has_encode_batch:
            L.tcg_frame_encode_batch.restype = ctypes.c_int32
            L.tcg_frame_encode_batch.argtypes = [ctypes.POINTER(FrameConfig), ctypes.POINTER(FrameInput),
                                                 ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.POINTER(FrameStats), ctypes.POINTER(ctypes.c_int32)]

    # ---- queries ----
    def last_error(self) -> str:
        return (self._lib.tc_last_error() or b"").decode("utf-8", "replace")

    def packet_bound(self, cfg: FrameConfig) -> int:
        return int(self._lib.tc_frame_packet_bound(ctypes.byref(cfg)))

    def validate(self, cfg: FrameConfig) -> int:
        return int(self._lib.tc_frame_config_validate(ctypes.byref(cfg)))

    # ---- encode ----
    @staticmethod
    def _input(planes: Sequence[np.ndarray]) -> FrameInput:
        fi = FrameInput()
        fi.struct_size = ctypes.sizeof(FrameInput)
        fi.abi_version = TOPOS_CODEC_ABI_VERSION
        for i, p in enumerate(planes):
            if p.dtype != np.uint16 or p.ndim != 2 or p.strides[1] != 2:
                raise ToposCodecError("planes must be 2-D uint16 arrays with unit column stride",
                                      TC_ERR_INVALID_ARGUMENT)
            fi.planes[i] = _u16_ptr(p)
            fi.strides[i] = p.strides[0] // 2
        return fi

    def encode_status(self, cfg: FrameConfig, planes: Sequence[np.ndarray],
                      out_cap: Optional[int] = None) -> Tuple[int, bytes, FrameStats]:
        fi = self._input(planes)
        cap = self.packet_bound(cfg) if out_cap is None else out_cap
        out = np.empty(max(cap, 1), dtype=np.uint8)
        st = FrameStats()
        rc = int(self._lib.tc_frame_encode(ctypes.byref(cfg), ctypes.byref(fi),
                                           out.ctypes.data if cap else None, cap, ctypes.byref(st)))
        pkt = out[: st.packet_size].tobytes() if rc == TC_OK else b""
        return rc, pkt, st

    def encode(self, cfg: FrameConfig, planes: Sequence[np.ndarray]) -> bytes:
        rc, pkt, _ = self.encode_status(cfg, planes)
        if rc != TC_OK:
            raise ToposCodecError(f"tc_frame_encode failed [{rc}]: {self.last_error()}", rc)
        return pkt

    def encode_sized_status(self, cfg: FrameConfig, planes: Sequence[np.ndarray], target_bytes: int,
                            qp_min: int = 0, qp_max: int = 95, out_cap: Optional[int] = None,
                            out: Optional[np.ndarray] = None):
        """tc_frame_encode_sized: (status, packet, stats, qp_used, output buffer). Without `out` the
        output buffer is a new one filled with 0xA5 (to see what a failing call leaves)."""
        fi = self._input(planes)
        cap = self.packet_bound(cfg) if out_cap is None else out_cap
        if out is None:
            out = np.full(max(cap, 1), 0xA5, dtype=np.uint8)
        cap = min(cap, out.size)
        st = FrameStats()
        qp_used = ctypes.c_uint8(0xEE)
        rc = int(self._lib.tc_frame_encode_sized(ctypes.byref(cfg), ctypes.byref(fi), target_bytes, qp_min, qp_max,
                                                 ctypes.byref(qp_used), out.ctypes.data, cap, ctypes.byref(st)))
        pkt = out[: st.packet_size].tobytes() if rc == TC_OK else b""
        return rc, pkt, st, qp_used.value, out

    def encode_sized(self, cfg: FrameConfig, planes: Sequence[np.ndarray], target_bytes: int, qp_min: int = 0,
                     qp_max: int = 95) -> Tuple[bytes, int]:
        rc, pkt, _, qp, _ = self.encode_sized_status(cfg, planes, target_bytes, qp_min, qp_max)
        if rc != TC_OK:
            raise ToposCodecError(f"tc_frame_encode_sized failed [{rc}]: {self.last_error()}", rc)
        return pkt, qp

    def encode_frame(self, cfg: FrameConfig, planes: Sequence[np.ndarray]) -> Tuple[bytes, dict]:
        rc, pkt, st = self.encode_status(cfg, planes)
        if rc != TC_OK:
            raise ToposCodecError(f"tc_frame_encode failed [{rc}]: {self.last_error()}", rc)
        return pkt, st.as_dict()

    def encode_batch(self, cfgs: Sequence[FrameConfig],
                     frames: Sequence[Sequence[np.ndarray]]) -> Tuple[int, List[bytes], List[int], List[dict]]:
        """tcg_frame_encode_batch (extension): all frames in one launch sequence."""
        if not self.has_encode_batch:
            raise ToposCodecError("library has no tcg_frame_encode_batch", TC_ERR_NOT_IMPLEMENTED)
        n = len(cfgs)
        carr = (FrameConfig * n)(*cfgs)
        iarr = (FrameInput * n)(*[self._input(f) for f in frames])
        caps = [self.packet_bound(c) for c in cfgs]
        bufs = [np.empty(max(c, 1), dtype=np.uint8) for c in caps]
        optr = (ctypes.c_void_p * n)(*[b.ctypes.data for b in bufs])
        ocap = (ctypes.c_size_t * n)(*caps)
        st = (FrameStats * n)()
        rcs = (ctypes.c_int32 * n)()
        rc = int(self._lib.tcg_frame_encode_batch(carr, iarr, n, optr, ocap, st, rcs))
        pkts = [bufs[i][: st[i].packet_size].tobytes() if rcs[i] == TC_OK else b"" for i in range(n)]
        return rc, pkts, list(rcs), [st[i].as_dict() for i in range(n)]

    # ---- decode ----
    def query(self, packet: bytes) -> Tuple[int, FrameOutput]:
        info = FrameOutput()
        buf = np.frombuffer(packet, dtype=np.uint8)
        rc = int(self._lib.tc_frame_decode(buf.ctypes.data if len(packet) else None, len(packet),
                                           None, None, ctypes.byref(info)))
        return rc, info

    @staticmethod
    def geometry(info: FrameOutput) -> List[Tuple[int, int]]:
        w, h = info.visible_width, info.visible_height
        cw = (w + 1) // 2 if info.pixel_format == 0 else w
        return [(h, w), (h, cw), (h, cw), (h, w)][: info.plane_count]

    def decode_status(self, packet: bytes, fill: int = 0) -> DecodedFrame:
        rc, info = self.query(packet)
        if rc != TC_OK:
            return DecodedFrame([], info, rc)
        planes = [np.full(s, fill, dtype=np.uint16) for s in self.geometry(info)]
        ptrs = (ctypes.c_void_p * TC_FRAME_MAX_PLANES)(*[p.ctypes.data for p in planes])
        buf = np.frombuffer(packet, dtype=np.uint8)
        info = FrameOutput()
        rc = int(self._lib.tc_frame_decode(buf.ctypes.data, len(packet), ptrs, None, ctypes.byref(info)))
        return DecodedFrame(planes, info, rc)

    def decode(self, packet: bytes) -> DecodedFrame:
        d = self.decode_status(packet)
        if d.status not in (TC_OK, TC_WARN_CONCEALED):
            raise ToposCodecError(f"tc_frame_decode failed [{d.status}]: {self.last_error()}", d.status)
        return d

    def decode_batch(self, packets: Sequence[bytes]) -> Tuple[int, List[DecodedFrame]]:
        n = len(packets)
        bufs = [np.frombuffer(p, dtype=np.uint8) for p in packets]
        arr = (BatchPacket * n)()
        for i, b in enumerate(bufs):
            arr[i].data = b.ctypes.data
            arr[i].size = len(packets[i])
        infos = (FrameOutput * n)()
        rc = int(self._lib.tc_frame_decode_batch(arr, n, None, None, infos))
        if rc != TC_OK:
            return rc, []
        planes = [[np.zeros(s, dtype=np.uint16) for s in self.geometry(infos[i])] for i in range(n)]
        ptrs = (ctypes.c_void_p * (n * TC_FRAME_MAX_PLANES))()
        for i in range(n):
            for p, a in enumerate(planes[i]):
                ptrs[i * TC_FRAME_MAX_PLANES + p] = a.ctypes.data
        infos = (FrameOutput * n)()
        rc = int(self._lib.tc_frame_decode_batch(arr, n, ptrs, None, infos))
        frames = []
        for i in range(n):
            one = FrameOutput()
            ctypes.memmove(ctypes.byref(one), ctypes.byref(infos[i]), ctypes.sizeof(FrameOutput))
            frames.append(DecodedFrame(planes[i], one, TC_OK))
        return rc, frames


class DecodeRequest(ctypes.Structure):
    """topos_decode_request (reference native/include/topos_codec.h:465-476)."""
    _fields_ = [("struct_size", ctypes.c_uint32), ("abi_version", ctypes.c_uint32), ("mode", ctypes.c_uint32),
                ("scale", ctypes.c_uint32), ("target_width", ctypes.c_uint32), ("target_height", ctypes.c_uint32),
                ("quality", ctypes.c_uint32), ("memory_type", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32 * 4)]


def make_request(mode: int = 0, scale: int = 0, target=(0, 0), flags: int = 0, quality: int = 0,
                 memory_type: int = 0) -> DecodeRequest:
    r = DecodeRequest()
    r.struct_size, r.abi_version = ctypes.sizeof(DecodeRequest), TOPOS_CODEC_ABI_VERSION
    r.mode, r.scale, r.quality, r.memory_type, r.flags = mode, scale, quality, memory_type, flags
    r.target_width, r.target_height = target
    return r


def decode_request(codec: "ToposCodec", packet: bytes, req: DecodeRequest, fill: int = 0) -> "DecodedFrame":
    """tc_frame_decode_request into host planes sized from its own query."""
    L = codec._lib
    L.tc_frame_decode_request.restype = ctypes.c_int32
    buf = np.frombuffer(packet, dtype=np.uint8)
    info = FrameOutput()
    rc = int(L.tc_frame_decode_request(ctypes.c_void_p(buf.ctypes.data if len(packet) else 0), ctypes.c_size_t(len(packet)),
                                       ctypes.byref(req), None, None, ctypes.byref(info)))
    if rc != TC_OK:
        return DecodedFrame([], info, rc)
    planes = [np.full(s, fill, dtype=np.uint16) for s in ToposCodec.geometry(info)]
    ptrs = (ctypes.c_void_p * TC_FRAME_MAX_PLANES)(*[p.ctypes.data for p in planes])
    info = FrameOutput()
    rc = int(L.tc_frame_decode_request(ctypes.c_void_p(buf.ctypes.data), ctypes.c_size_t(len(packet)), ctypes.byref(req),
                                       ptrs, None, ctypes.byref(info)))
    return DecodedFrame(planes, info, rc)


class Server:
    """Continuous-batching request server of the library (tcg_server_*).

    submit_encode/submit_decode take numpy arrays (host memory) or device
    pointers; the caller keeps the buffers alive until wait() returns.
    """

    def __init__(self, codec: "ToposCodec", max_bytes_in_flight: int = 0, max_batch_frames: int = 64,
                 workers: int = 4):
        L = codec._lib
        self._codec, self._lib = codec, L
        L.tcg_server_create_ex.restype = ctypes.c_int32
        L.tcg_server_create_ex.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_void_p)]
        L.tcg_server_destroy.restype = None
        L.tcg_server_destroy.argtypes = [ctypes.c_void_p]
        L.tcg_server_submit_encode.restype = ctypes.c_int32
        L.tcg_server_submit_encode.argtypes = [ctypes.c_void_p, ctypes.POINTER(FrameConfig), ctypes.POINTER(FrameInput),
                                               ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)]
        L.tcg_server_submit_decode.restype = ctypes.c_int32
        L.tcg_server_submit_decode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
        L.tcg_server_wait.restype = ctypes.c_int32
        L.tcg_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32),
                                      ctypes.POINTER(FrameStats), ctypes.POINTER(FrameOutput),
                                      ctypes.POINTER(ctypes.c_double)]
        h = ctypes.c_void_p()
        rc = int(L.tcg_server_create_ex(max_bytes_in_flight, max_batch_frames, workers, ctypes.byref(h)))
        if rc != TC_OK:
            raise ToposCodecError(f"tcg_server_create failed [{rc}]: {codec.last_error()}", rc)
        self._h = h
        self._keep = {}

    def close(self) -> None:
        if self._h:
            self._lib.tcg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def submit_encode(self, cfg: FrameConfig, planes, out_ptr: int, out_cap: int) -> int:
        """planes: numpy uint16 arrays, or (pointer, stride) pairs of device planes."""
        fi = FrameInput()
        fi.struct_size, fi.abi_version = ctypes.sizeof(FrameInput), TOPOS_CODEC_ABI_VERSION
        for i, p in enumerate(planes):
            if isinstance(p, np.ndarray):
                fi.planes[i], fi.strides[i] = p.ctypes.data, p.strides[0] // 2
            else:
                fi.planes[i], fi.strides[i] = p
        t = ctypes.c_uint64()
        rc = int(self._lib.tcg_server_submit_encode(self._h, ctypes.byref(cfg), ctypes.byref(fi), out_ptr, out_cap,
                                                    ctypes.byref(t)))
        if rc != TC_OK:
            raise ToposCodecError(f"submit_encode failed [{rc}]: {self._codec.last_error()}", rc)
        self._keep[t.value] = (planes, fi)
        return t.value

    def submit_decode(self, packet_ptr: int, size: int, plane_ptrs: Sequence[int]) -> int:
        ptrs = (ctypes.c_void_p * TC_FRAME_MAX_PLANES)(*list(plane_ptrs) + [None] * (TC_FRAME_MAX_PLANES - len(plane_ptrs)))
        t = ctypes.c_uint64()
        rc = int(self._lib.tcg_server_submit_decode(self._h, packet_ptr, size, ptrs, None, ctypes.byref(t)))
        if rc != TC_OK:
            raise ToposCodecError(f"submit_decode failed [{rc}]: {self._codec.last_error()}", rc)
        self._keep[t.value] = ptrs
        return t.value

    def wait(self, ticket: int):
        """(status, stats, info, latency_ms) of a finished request."""
        st, stats, info, lat = ctypes.c_int32(), FrameStats(), FrameOutput(), ctypes.c_double()
        rc = int(self._lib.tcg_server_wait(self._h, ticket, ctypes.byref(st), ctypes.byref(stats), ctypes.byref(info),
                                           ctypes.byref(lat)))
        self._keep.pop(ticket, None)
        if rc != TC_OK:
            raise ToposCodecError(f"wait failed [{rc}]: {self._codec.last_error()}", rc)
        return st.value, stats, info, lat.value
