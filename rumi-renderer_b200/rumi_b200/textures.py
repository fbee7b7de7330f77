"""Texture image files as the reference reads them.

* ``load_bmp`` restates ``LoadBmp`` (src/Kernel/bmp.cpp:3-57): the 54-byte header (with
  32-bit fields, as the reference's header struct reads on the platform it was written
  for), then the pixel rows from ``bitmap_data_offset`` in file order -- bottom row first,
  B,G,R[,A] -- contiguously when the width is a multiple of 4, else row by row skipping
  ``width % 4`` bytes after each row (the true padding for 24-bit rows; 32-bit rows with
  such widths are misread the same way the reference misreads them).
* ``load_hdr`` restates ``LoadHDR`` / ``ScanLine`` (src/Kernel/hdr.cpp:4-177): the
  ``#?RADIANCE`` signature, comment lines, ``FORMAT=32-bit_rle_rgbe``, ``EXPOSURE`` /
  ``GAMMA`` lines up to the blank line, ``-Y h +X w``, then new-style run-length scanlines
  only (2, 2, width >> 8, width & 255, four channel runs).  RGBE -> float is
  ``m * 2^(e - 136)`` (0 when e = 0).  Where the reference gives up on a scanline (old-style
  or flat scanlines, widths outside [8, 32767], and widths whose low byte is >= 128, which
  its signed ``char`` comparison rejects) it prints an error and leaves the rest of its
  buffer unwritten; here ValueError is raised instead.
* ``save_hdr`` writes files ``load_hdr`` (and the reference) reads: new-style RLE
  scanlines, runs where a byte repeats, literals elsewhere.
"""
from __future__ import annotations

import struct

import numpy as np


def load_bmp(path: str) -> np.ndarray:
    """(height, width, bytes_per_pixel) uint8 in LoadBmp's buffer order."""
    with open(path, "rb") as f:
        data = f.read()
    return load_bmp_bytes(data)


def load_bmp_bytes(data: bytes) -> np.ndarray:
    if len(data) < 54:
        raise ValueError("BMP header truncated")
    offset = struct.unpack_from("<I", data, 10)[0]
    width, height = struct.unpack_from("<ii", data, 18)
    bpp = struct.unpack_from("<H", data, 28)[0] // 8
    if width <= 0 or height <= 0 or bpp <= 0:
        raise ValueError("unsupported BMP dimensions")
    row = width * bpp
    out = np.zeros((height, row), np.uint8)
    if width % 4 == 0:
        n = min(len(data) - offset, row * height)
        flat = np.frombuffer(data, np.uint8, count=max(n, 0), offset=offset)
        out.reshape(-1)[:flat.size] = flat
    else:
        pos = offset
        for h in range(height):
            chunk = data[pos:pos + row]
            out[h, :len(chunk)] = np.frombuffer(chunk, np.uint8)
            pos += row + width % 4
    return out.reshape(height, width, bpp)


def _scanline(data: bytes, pos: int, width: int):
    """ScanLine: one new-style RLE scanline -> (4, width) bytes and the next position."""
    if width < 8 or width > 0x7FFF:
        raise ValueError("HDR scanline width outside [8, 32767]")
    if pos + 4 > len(data):
        raise ValueError("HDR scanline truncated")
    r0, r1, r2, r3 = data[pos:pos + 4]
    pos += 4
    if r0 != 2 or r1 != 2 or (r2 & 0x80):
        raise ValueError("HDR scanline is not new-style run-length encoded")
    # the reference reads these bytes as signed char: a low byte >= 128 never matches
    if r3 >= 128 or ((r2 << 8) | r3) != width:
        raise ValueError("HDR scanline width does not match (or its low byte is >= 128)")
    line = np.zeros(4 * width, np.uint8)
    k = 0
    for ch in range(4):
        end = (ch + 1) * width
        while k < end:
            if pos + 2 > len(data):
                raise ValueError("HDR scanline truncated")
            c, v = data[pos], data[pos + 1]
            pos += 2
            if c > 128:
                c -= 128
                if c > end - k:
                    raise ValueError("HDR run overflows the scanline")
                line[k:k + c] = v
                k += c
            else:
                if c == 0 or c > end - k:
                    raise ValueError("HDR literal overflows the scanline")
                line[k] = v
                k += 1
                c -= 1
                if c > 0:
                    if pos + c > len(data):
                        raise ValueError("HDR scanline truncated")
                    line[k:k + c] = np.frombuffer(data, np.uint8, count=c, offset=pos)
                    pos += c
                    k += c
    return line.reshape(4, width), pos


def load_hdr(path: str) -> np.ndarray:
    """(height, width, 3) float32, first scanline first, R,G,B."""
    with open(path, "rb") as f:
        data = f.read()
    return load_hdr_bytes(data)


def load_hdr_bytes(data: bytes) -> np.ndarray:
    pos = 0

    def getline():
        nonlocal pos
        nl = data.find(b"\n", pos, pos + 255)
        end = nl + 1 if nl >= 0 else min(pos + 255, len(data))
        s = data[pos:end]
        pos = end
        return s

    if getline() != b"#?RADIANCE\n":
        raise ValueError("not a Radiance HDR file")
    line = getline()
    while line[:1] == b"#":
        line = getline()
    if line != b"FORMAT=32-bit_rle_rgbe\n":
        raise ValueError("HDR format is not 32-bit_rle_rgbe")
    while True:
        line = getline()
        if line[:8] == b"EXPOSURE" or line[:5] == b"GAMMA":
            continue
        if line[:1] == b"\n":
            break
        if not line:
            raise ValueError("HDR header truncated")
    res = getline().split()
    if len(res) != 4 or res[0] != b"-Y" or res[2] != b"+X":
        raise ValueError("HDR resolution line must be -Y h +X w")
    height, width = int(res[1]), int(res[3])
    out = np.zeros((height, width, 3), np.float32)
    for h in range(height):
        sl, pos = _scanline(data, pos, width)
        e = sl[3].astype(np.int32)
        f = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0)
        for c in range(3):
            out[h, :, c] = (sl[c].astype(np.float64) * f).astype(np.float32)
    return out


def _rle_channel(b: np.ndarray) -> bytes:
    out = bytearray()
    i, n = 0, len(b)
    while i < n:
        j = i
        while j < n and j - i < 127 and b[j] == b[i]:
            j += 1
        if j - i >= 3:
            out += bytes([128 + (j - i), int(b[i])])
            i = j
            continue
        j = i + 1
        while j < n and j - i < 128 and not (j + 2 < n and b[j] == b[j + 1] == b[j + 2]):
            j += 1
        out += bytes([j - i]) + bytes(b[i:j].tolist())
        i = j
    return bytes(out)


def rgbe_from_float(rgb: np.ndarray) -> np.ndarray:
    """Float RGB -> RGBE bytes (shared exponent of the largest channel)."""
    rgb = np.asarray(rgb, np.float64)
    m = rgb.max(-1)
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    nz = m > 1e-32
    mant, ex = np.frexp(m[nz])
    scale = mant * 256.0 / m[nz]
    out[nz, :3] = np.clip(rgb[nz] * scale[:, None], 0, 255).astype(np.uint8)
    out[nz, 3] = (ex + 128).astype(np.uint8)
    return out


def save_hdr(path: str, rgbe: np.ndarray, comment: bytes = b"# written by rumi_b200", extra: bytes = b"") -> None:
    """Writes (height, width, 4) RGBE bytes as a new-style RLE Radiance file; `comment`
    lines go before the FORMAT line, `extra` lines (EXPOSURE=..., ...) after it."""
    rgbe = np.asarray(rgbe, np.uint8)
    h, w = rgbe.shape[:2]
    out = bytearray(b"#?RADIANCE\n" + comment + b"\nFORMAT=32-bit_rle_rgbe\n" + extra + b"\n")
    out += b"-Y %d +X %d\n" % (h, w)
    for y in range(h):
        out += bytes([2, 2, w >> 8, w & 0xFF])
        for c in range(4):
            out += _rle_channel(rgbe[y, :, c])
    with open(path, "wb") as f:
        f.write(bytes(out))
