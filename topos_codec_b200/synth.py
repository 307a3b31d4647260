"""Seeded synthetic frames with the shapes and value distributions of the
benchmark workloads (no public dataset is involved; these stand in for it).

Colour planes: a base level at the middle of the legal range, plus three random
low-frequency 2-D sinusoids (amplitude 150 LSB at 10-bit, scaled with bit
depth), twenty axis-aligned rectangles that replace the content with a uniform
random level, and Gaussian noise (sigma 6 LSB at 10-bit), clipped to the range
(limited: luma 64..940, chroma 64..960 at 10-bit; full: 0..2^bd-1). A per-frame
phase drift (0.05 rad per frame index) makes the frames of a batch differ.
Alpha: 0/65535 with eight hard-edged random ellipses and 4-pixel linear ramps.

The generator runs on torch (CPU or CUDA); it is deterministic for a given
(seed, frame index, device type).
"""
from __future__ import annotations

import math
from typing import List, Optional

import numpy as np
import torch


def _ranges(bit_depth: int, limited: bool):
    s = 1 << (bit_depth - 10)
    if limited:
        return (64 * s, 940 * s), (64 * s, 960 * s)
    full = (0, (1 << bit_depth) - 1)
    return full, full


def _plane(h: int, w: int, lo: int, hi: int, scale: float, sigma: float, phase: float,
           g: torch.Generator, device) -> torch.Tensor:
    r = lambda *s: torch.rand(*s, generator=g, device=device, dtype=torch.float64)
    y = torch.arange(h, device=device, dtype=torch.float64)[:, None]
    x = torch.arange(w, device=device, dtype=torch.float64)[None, :]
    img = torch.full((h, w), (lo + hi) / 2.0, device=device, dtype=torch.float64)
    for _ in range(3):
        fx, fy, ph = r(3).tolist()
        fx = (fx * 6.0 - 3.0) * 2 * math.pi / max(w, 1)
        fy = (fy * 6.0 - 3.0) * 2 * math.pi / max(h, 1)
        ph = ph * 2 * math.pi + phase
        img = img + 150.0 * scale * torch.sin(fx * x + fy * y + ph)
    for _ in range(20):
        x0, y0, ww, hh, lv = r(5).tolist()
        xa, ya = int(x0 * w), int(y0 * h)
        xb, yb = min(w, xa + 1 + int(ww * w / 3)), min(h, ya + 1 + int(hh * h / 3))
        img[ya:yb, xa:xb] = lo + lv * (hi - lo)
    img = img + sigma * scale * torch.randn(h, w, generator=g, device=device, dtype=torch.float64)
    return img.round().clamp(lo, hi).to(torch.int32)


def _alpha(h: int, w: int, g: torch.Generator, device) -> torch.Tensor:
    r = lambda *s: torch.rand(*s, generator=g, device=device, dtype=torch.float64)
    y = torch.arange(h, device=device, dtype=torch.float64)[:, None]
    x = torch.arange(w, device=device, dtype=torch.float64)[None, :]
    a = torch.zeros((h, w), device=device, dtype=torch.float64)
    for _ in range(8):
        cx, cy, rx, ry = r(4).tolist()
        cx, cy = cx * w, cy * h
        rx, ry = 4 + rx * w / 4, 4 + ry * h / 4
        # signed distance to the ellipse edge in pixels (approximate along the normal)
        d = (torch.sqrt(((x - cx) / rx) ** 2 + ((y - cy) / ry) ** 2) - 1.0) * min(rx, ry)
        a = torch.maximum(a, (1.0 - d / 4.0).clamp(0.0, 1.0))
    return (a * 65535.0).round().to(torch.int32)


def make_frame(width: int, height: int, *, seed: int = 0, frame: int = 0, bit_depth: int = 10,
               pixel_format: int = 0, limited: bool = True, alpha: bool = False,
               sigma: Optional[float] = None, device="cpu") -> List[torch.Tensor]:
    """Planes [Y,U,V(,A)] (or [G,B,R(,A)]) as uint16-valued int32 tensors."""
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed((seed * 1000003 + frame) & 0x7FFFFFFFFFFFFFFF)
    (llo, lhi), (clo, chi) = _ranges(bit_depth, limited)
    scale = float(1 << (bit_depth - 10))
    sig = 6.0 if sigma is None else sigma
    cw = (width + 1) // 2 if pixel_format == 0 else width
    phase = 0.05 * frame
    planes = [_plane(height, width, llo, lhi, scale, sig, phase, g, dev)]
    planes.append(_plane(height, cw, clo, chi, scale, sig, phase, g, dev))
    planes.append(_plane(height, cw, clo, chi, scale, sig, phase, g, dev))
    if alpha:
        planes.append(_alpha(height, width, g, dev))
    return planes


def to_numpy(planes: List[torch.Tensor]) -> List[np.ndarray]:
    return [np.ascontiguousarray(p.to("cpu").numpy().astype(np.uint16)) for p in planes]


def make_frame_np(width: int, height: int, **kw) -> List[np.ndarray]:
    return to_numpy(make_frame(width, height, **kw))
