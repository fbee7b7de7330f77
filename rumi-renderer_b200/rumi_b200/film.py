"""Film output: tonemapping (Film::Save), the fireflies post-filter (FirefliesFiltering)
and BMP files.

The two image operations run on the GPU through the C-ABI (rumi_film_tonemap,
rumi_film_fireflies).  ``save_bmp`` writes what the reference's SaveBmp
(src/Kernel/bmp.cpp:59-97) means to write -- the film's rows in order, B,G,R(,A) -- with a
correct 54-byte header (32-bit fields; the reference's ``unsigned long`` fields are 64-bit
on LP64 Linux and corrupt it) and rows padded to 4 bytes as the format requires.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from . import _capi


def tonemap(film, n_samples: int, gamma: float = 2.2, bytes_per_pixel: int = 3) -> np.ndarray:
    """(H, W, 3) B,G,R pixel sums -> (H, W, bytes_per_pixel) uint8 as Film::Save converts them."""
    f = np.ascontiguousarray(film, np.float32)
    H, W = f.shape[0], f.shape[1]
    out = np.zeros((H, W, bytes_per_pixel), np.uint8)
    L = _capi.load()
    _capi.check(L.rumi_film_tonemap(f.ctypes.data_as(C.c_void_p), W, H, int(n_samples), float(gamma),
                                    bytes_per_pixel, out.ctypes.data_as(C.c_void_p), 0, None), "rumi_film_tonemap")
    return out


def fireflies(img) -> np.ndarray:
    """FirefliesFiltering on an (H, W, 3 or 4) uint8 image in the film's row order."""
    a = np.ascontiguousarray(img, np.uint8)
    H, W, bpp = a.shape
    out = np.empty_like(a)
    L = _capi.load()
    _capi.check(L.rumi_film_fireflies(a.ctypes.data_as(C.c_void_p), W, H, bpp, out.ctypes.data_as(C.c_void_p), 0,
                                      None), "rumi_film_fireflies")
    return out


def save_bmp(path: str, img) -> None:
    """Writes an (H, W, 3 or 4) uint8 image as a BMP, rows in the order given."""
    a = np.ascontiguousarray(img, np.uint8)
    H, W, bpp = a.shape
    row = W * bpp
    pad = (-row) % 4
    data = b"".join(a[h].tobytes() + b"\0" * pad for h in range(H))
    header = b"BM" + struct.pack("<IHHI", 54 + len(data), 0, 0, 54)
    header += struct.pack("<IiiHHIIiiII", 40, W, H, 1, 8 * bpp, 0, len(data), 0, 0, 0, 0)
    with open(path, "wb") as f:
        f.write(header + data)


def load_bmp(path: str) -> np.ndarray:
    """Reads a BMP written by save_bmp: (H, W, bytes_per_pixel) uint8, rows in file order."""
    with open(path, "rb") as f:
        b = f.read()
    if b[:2] != b"BM":
        raise ValueError("not a BMP file")
    off = struct.unpack_from("<I", b, 10)[0]
    W, H = struct.unpack_from("<ii", b, 18)
    bpp = struct.unpack_from("<H", b, 28)[0] // 8
    row = W * bpp
    stride = row + (-row) % 4
    return np.stack([np.frombuffer(b, np.uint8, row, off + h * stride).reshape(W, bpp) for h in range(abs(H))])
