"""Readers for the image files of the export path (test infrastructure): 8-bit
RGB PNG (any filter, zlib stream), 24-bit TGA (raw or RLE, either vertical
origin) and scanline EXR without compression (HALF / FLOAT channels).  Each
returns the pixels in the row order of the buffer that was written: row 0 is
the buffer's first row."""
import struct
import zlib

import numpy as np


def read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", None
    while pos < len(data):
        n, typ = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        assert zlib.crc32(typ + body) & 0xFFFFFFFF == struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        if typ == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
            assert depth == 8 and ctype == 2 and interlace == 0
        elif typ == b"IDAT":
            idat += body
        elif typ == b"IEND":
            break
        pos += 12 + n
    raw = zlib.decompress(idat)
    stride = 3 * w
    out = np.zeros((h, stride), np.int32)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        f = raw[y * (stride + 1)]
        line = np.frombuffer(raw, np.uint8, stride, y * (stride + 1) + 1).astype(np.int32)
        cur = np.zeros(stride, np.int32)
        for x in range(stride):
            a = cur[x - 3] if x >= 3 else 0
            b = prev[x]
            c = prev[x - 3] if x >= 3 else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) // 2
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            cur[x] = (line[x] + p) & 0xFF
        out[y] = cur
        prev = cur
    return out.astype(np.uint8).reshape(h, w, 3)


def read_tga(path):
    data = open(path, "rb").read()
    idlen, cmtype, itype = data[0], data[1], data[2]
    w, h = struct.unpack("<HH", data[12:16])
    bpp, desc = data[16], data[17]
    assert cmtype == 0 and itype in (2, 10) and bpp == 24
    pos = 18 + idlen
    px = np.zeros((w * h, 3), np.uint8)
    i = 0
    if itype == 2:
        px[:] = np.frombuffer(data, np.uint8, w * h * 3, pos).reshape(-1, 3)
    else:
        while i < w * h:
            hdr = data[pos]
            pos += 1
            n = (hdr & 0x7F) + 1
            if hdr & 0x80:
                px[i:i + n] = np.frombuffer(data, np.uint8, 3, pos)
                pos += 3
            else:
                px[i:i + n] = np.frombuffer(data, np.uint8, 3 * n, pos).reshape(n, 3)
                pos += 3 * n
            i += n
    img = px.reshape(h, w, 3)[:, :, ::-1]  # BGR
    if not desc & 0x20:  # bottom-left origin: the first stored row is the last one
        img = img[::-1]
    return np.ascontiguousarray(img)


def read_exr(path):
    """(names, planes): channel names and their h x w float32 planes."""
    data = open(path, "rb").read()
    assert data[:4] == b"\x76\x2f\x31\x01"
    pos = 8
    attrs = {}
    while data[pos] != 0:
        e = data.index(b"\0", pos)
        name = data[pos:e].decode()
        t = data.index(b"\0", e + 1)
        typ = data[e + 1:t].decode()
        size = struct.unpack("<i", data[t + 1:t + 5])[0]
        attrs[name] = (typ, data[t + 5:t + 5 + size])
        pos = t + 5 + size
    pos += 1
    assert attrs["compression"][1][0] == 0, "compressed EXR"
    chl = attrs["channels"][1]
    chans, p = [], 0
    while chl[p] != 0:
        e = chl.index(b"\0", p)
        ptype = struct.unpack("<i", chl[e + 1:e + 5])[0]
        chans.append((chl[p:e].decode(), ptype))
        p = e + 17
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    offsets = struct.unpack("<%dQ" % h, data[pos:pos + 8 * h])
    planes = [np.zeros((h, w), np.float32) for _ in chans]
    for off in offsets:
        y, size = struct.unpack("<ii", data[off:off + 8])
        q = off + 8
        for k, (_, ptype) in enumerate(chans):
            if ptype == 1:
                planes[k][y - y0] = np.frombuffer(data, np.float16, w, q).astype(np.float32)
                q += 2 * w
            else:
                assert ptype == 2
                planes[k][y - y0] = np.frombuffer(data, np.float32, w, q)
                q += 4 * w
    return [c[0] for c in chans], planes


def half_bits(f):
    """float32 -> float16 bits as the EXR writers convert (ISPC reference rule):
    the mantissa truncated and rounded up in magnitude when the first dropped
    bit is set (so exact ties go up, not to even), float denormals to 0, NaN to
    a quiet NaN, overflow to infinity."""
    u = np.asarray(f, np.float32).view(np.uint32).astype(np.int64)
    sign, e, m = (u >> 31) & 1, (u >> 23) & 0xFF, u & 0x7FFFFF
    newexp = e - 127 + 15
    nan_inf = e == 255
    normal = (e != 0) & ~nan_inf
    out = np.where(nan_inf, (31 << 10) | np.where(m != 0, 0x200, 0), 0)
    out = np.where(normal & (newexp >= 31), 31 << 10, out)
    under = normal & (newexp <= 0)
    sh = 14 - newexp
    mant = m | 0x800000
    sub = np.where(sh <= 24, (mant >> np.clip(sh, 0, 63)) + ((mant >> np.clip(sh - 1, 0, 63)) & 1), 0)
    out = np.where(under, sub, out)
    norm = normal & (newexp > 0) & (newexp < 31)
    out = np.where(norm, ((newexp << 10) | (m >> 13)) + ((m >> 12) & 1), out)
    return (out | (sign << 15)).astype(np.uint16)
