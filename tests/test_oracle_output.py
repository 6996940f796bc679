"""Output development in the CPU oracle: apply_optics (output.rs:159-190,
pinned to its tests output.rs:193-233), the AgX / ACES tone curves and the
sRGB quantisation of tone_map (output.rs:7-113) against an independent float64
restatement, and the PNG writer."""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.output import png_name, read_png, write_png
from rustracer_b200.renderer import develop_params


def test_optics_identity_when_off():
    img = np.zeros((4, 4, 3), np.float32)
    img[..., 0] = np.arange(16).reshape(4, 4)
    np.testing.assert_allclose(O.apply_optics(img, 0.0, 0.0), img, atol=1e-7)


def test_vignette_darkens_corners_not_center():
    out = O.apply_optics(np.ones((4, 4, 3), np.float32), 0.4, 0.0)
    assert 0.9 < out[1, 1, 0] < 1.0
    assert abs(out[0, 0, 0] - 0.6) < 1e-6


def test_barrel_distortion_pulls_corners_inward():
    w = h = 9
    img = np.zeros((h, w, 3), np.float32)
    img[..., 0] = np.arange(w)[None, :]
    out = O.apply_optics(img, 0.0, 0.2)
    assert out[0, 0, 0] > img[0, 0, 0]
    assert abs(out[4, 4, 0] - img[4, 4, 0]) < 1e-6


def _srgb(x):
    x = np.fmax(x, 0.0)                  # f32::max: a NaN (pow of a negative curve value) becomes 0
    return np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(x, 1 / 2.4) - 0.055)


def _quant(x):
    return (np.clip(_srgb(x), 0.0, 0.999) * 256.0).astype(np.uint8)


def _aces(c):
    A = np.array([[0.59719, 0.35458, 0.04823], [0.07600, 0.90834, 0.01566], [0.02840, 0.13383, 0.83777]])
    B = np.array([[1.60475, -0.53108, -0.07367], [-0.10208, 1.10813, -0.00605], [-0.00327, -0.07276, 1.07602]])
    x = np.maximum(c @ A.T, 0.0)
    return ((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14)) @ B.T


def _agx(c):
    A = np.array([[0.842479062253094, 0.0784335999999992, 0.0792237451477643],
                  [0.0423282422610123, 0.878468636469772, 0.0791661274605434],
                  [0.0423756549057051, 0.0784336, 0.879142973793104]])
    B = np.array([[1.19687900512017, -0.0980208811401368, -0.0990297440797205],
                  [-0.0528968517574562, 1.15190312990417, -0.0989611768448433],
                  [-0.0529716355144234, -0.0980434501171241, 1.15107567775604]])
    x = np.clip((np.log2(np.maximum(c @ A.T, 1e-10)) + 12.47393) / 16.5, 0.0, 1.0)
    x2, x4 = x * x, x ** 4
    k = 15.5 * x4 * x2 - 40.14 * x4 * x + 31.96 * x4 - 6.868 * x2 * x + 0.4298 * x2 + 0.1191 * x - 0.00232
    luma = k @ np.array([0.2126, 0.7152, 0.0722])
    with np.errstate(invalid="ignore"):
        k = luma[..., None] + 1.4 * (np.power(k, 1.35) - luma[..., None])
    return k @ B.T


@pytest.mark.parametrize("tm,fn", [("agx", _agx), ("aces", _aces)])
def test_tone_curves_match_a_float64_restatement(tm, fn):
    rng = np.random.default_rng(1)
    img = np.exp(rng.normal(-1.0, 2.0, (37, 53, 3))).astype(np.float32)
    img[0, :5] = 0.0                                       # black stays black
    got = O.develop(develop_params(53, 37, 1.5, tm), linear=img)
    want = _quant(fn(img.astype(np.float64) * 1.5))
    diff = np.abs(got.astype(int) - want.astype(int))
    assert diff.max() <= 1 and (diff == 0).mean() > 0.99
    assert (got[0, :5] == want[0, :5]).all()


def test_accumulators_are_divided_by_their_counts():
    rng = np.random.default_rng(2)
    mean = rng.random((8, 9, 3)).astype(np.float32)
    cnt = rng.integers(0, 5, (8, 9)).astype(np.uint32)
    s = mean * np.maximum(cnt, 1)[..., None]
    p = develop_params(9, 8, 1.0, "aces")
    assert np.array_equal(O.develop(p, sum_=s, count=cnt),
                          O.develop(p, linear=s / np.maximum(cnt, 1)[..., None].astype(np.float32)))


def test_png_round_trip_and_name(tmp_path):
    a = (np.random.default_rng(0).random((6, 11, 3)) * 255).astype(np.uint8)
    p = write_png(str(tmp_path / "x.png"), a)
    assert np.array_equal(read_png(p), a)
    assert png_name("Benchmark Scene", 64) == "render_benchmark_scene_0064spp.png"
