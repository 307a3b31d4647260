"""V8 packet layout helpers for the tests (segment directory, tile tables,
streams, tile CRCs per colour plane; reference bitstream/packet.h:36-82).
Used to damage chosen segments or tiles and to re-seal a tile's CRC so that a
segment's own decode failure (not the tile CRC) is exercised."""
import struct
import zlib

HDR, EXT, DIR, TABLE = 53, 8, 12, 350


def layout(pkt, plane_blocks):
    """plane_blocks: [(cols, rows)] per colour plane. Returns a list per plane of
    dicts with dir/tables/streams/crc offsets, the segment (offset, length)
    list and the tiles' member segment ranges."""
    sb = 1 << pkt[HDR]
    tr = 0 if pkt[HDR + 1] == 0 else 1 << pkt[HDR + 1]
    off = HDR + EXT
    out = []
    for cols, rows in plane_blocks:
        blocks = cols * rows
        S = (blocks + sb - 1) // sb
        T = 1 if tr == 0 or rows == 0 else (rows + tr - 1) // tr
        d = off
        segs = [struct.unpack(">II", pkt[d + DIR * k:d + DIR * k + 8]) for k in range(S)]
        tab = d + DIR * S
        st = tab + TABLE * T
        crc = st + sum(ln for _, ln in segs)
        tiles = []
        for t in range(T):
            fb = 0 if tr == 0 else t * tr * cols
            fn = blocks if tr == 0 else (t + 1) * tr * cols
            sf, sn = min(fb // sb, S), min(fn // sb, S)
            tiles.append((sf, max(sn, sf)))
        out.append(dict(dir=d, tables=tab, streams=st, crc=crc, segs=segs, tiles=tiles, sb=sb))
        off = crc + 4 * T
    return out


def reseal_tile(p, pl, t):
    """Recompute tile t's CRC (table + member streams) in the bytearray p."""
    sf, sn = pl["tiles"][t]
    a = pl["streams"] + (pl["segs"][sf][0] if sn > sf else 0)
    n = sum(ln for _, ln in pl["segs"][sf:sn])
    c = zlib.crc32(bytes(p[pl["tables"] + TABLE * t:pl["tables"] + TABLE * (t + 1)]))
    c = zlib.crc32(bytes(p[a:a + n]), c)
    p[pl["crc"] + 4 * t:pl["crc"] + 4 * t + 4] = struct.pack(">I", c & 0xFFFFFFFF)


def plane_blocks(w, h, pixel_format):
    """(cols, rows) of the three colour planes of a w x h frame."""
    cw = ((w + 1) // 2 if pixel_format == 0 else w)
    pad = lambda v: (v + 7) // 8 * 8
    return [(pad(w) // 8, pad(h) // 8), (pad(cw) // 8, pad(h) // 8), (pad(cw) // 8, pad(h) // 8)]
