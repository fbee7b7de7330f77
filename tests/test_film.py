"""Film output: tonemapping and the fireflies filter on the GPU against the reference's
own Film::Save / FirefliesFiltering (run through oracle/_ref on the same pixel sums), and
the BMP writer (host)."""
import ctypes as C
import os

import numpy as np
import pytest

import refimpl
from rumi_b200 import film as F


def test_bmp_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    for H, W, bpp in ((5, 7, 3), (4, 8, 3), (3, 5, 4)):
        img = rng.integers(0, 256, (H, W, bpp), dtype=np.uint8)
        p = str(tmp_path / f"a{W}.bmp")
        F.save_bmp(p, img)
        size = os.path.getsize(p)
        assert size == 54 + H * (W * bpp + (-(W * bpp)) % 4)
        np.testing.assert_array_equal(F.load_bmp(p), img)


def _reference(tmp_path, film, spp, gamma, bpp):
    L = refimpl.lib()
    L.ref_film_save_filter.restype = C.c_int
    L.ref_film_save_filter.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p,
                                       C.c_void_p, C.c_void_p]
    H, W = film.shape[:2]
    t = np.zeros((H, W, bpp), np.uint8)
    f = np.zeros((H, W, bpp), np.uint8)
    assert L.ref_film_save_filter(str(tmp_path).encode(), W, H, bpp, spp, gamma,
                                  np.ascontiguousarray(film, np.float32).ctypes.data_as(C.c_void_p),
                                  t.ctypes.data_as(C.c_void_p), f.ctypes.data_as(C.c_void_p)) == 0
    return t, f


def _film(seed, H, W, spp):
    """Pixel sums with a spread of values, some far above 1 (saturating) -- only away from
    the border, where the reference's fireflies filter stays inside its buffer."""
    rng = np.random.default_rng(seed)
    film = (rng.random((H, W, 3)) ** 3 * 0.9 * spp).astype(np.float32)
    for _ in range(12):
        h, w = rng.integers(2, H - 2), rng.integers(2, W - 2)
        film[h, w] = 50.0 * spp
        if rng.random() < 0.4:  # a white neighbour: not a firefly
            film[h + 1, w] = 50.0 * spp
    film[rng.random((H, W)) < 0.03] *= 0.0
    return film


@pytest.mark.gpu
@pytest.mark.skipif(not refimpl.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("spp,gamma,bpp", [(16, 2.2, 3), (25, 1.0, 3), (64, 2.2, 4)])
def test_tonemap_and_fireflies_match_the_reference(tmp_path, spp, gamma, bpp):
    H, W = 40, 48
    film = _film(spp, H, W, spp)
    ref_t, ref_f = _reference(tmp_path, film, spp, gamma, bpp)
    t = F.tonemap(film, spp, gamma, bpp)
    # the GPU's powf and the host's may differ in the last bit: a byte may then truncate one
    # step lower or higher
    diff = np.abs(t.astype(int) - ref_t.astype(int))
    assert diff.max() <= 1 and (diff > 0).mean() < 0.002, ((diff > 0).mean(), diff.max())
    # the filter on the reference's own bytes: exact in B,G,R (the reference leaves a fourth
    # byte of its output buffer unwritten; here it keeps the input's)
    got = F.fireflies(ref_t)
    np.testing.assert_array_equal(got[..., :3], ref_f[..., :3])
    assert (ref_f[..., :3] != ref_t[..., :3]).any()  # some fireflies were removed
