"""The Physical (Preetham) sky of the CPU oracle: internal consistency of the
sun disc, the cone sampling and its pdf, and the ground blend
(renderer.rs:231-362; the reference has no unit tests for the sky)."""
import math

import numpy as np

from oracle import oracle as O
from tests.helpers import physical_sky_scene

COS_SUN_MAX = np.float32(0.9999892)


def _sun(el, az):
    el, az = math.radians(el), math.radians(az)
    d = np.array([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)])
    return d / np.linalg.norm(d)


def test_sun_disc_and_pdf():
    s = O.OracleScene(physical_sky_scene(elevation=35.0, azimuth=30.0))
    sun = _sun(35.0, 30.0)
    rgb, pdf = s.bg_eval_n(np.stack([sun, np.array([0.0, 1.0, 0.0]), np.array([0.3, -0.5, 0.2])]))
    disc = rgb[0]
    assert disc[0] > 0 and abs(disc[1] / disc[0] - 0.95) < 1e-5 and abs(disc[2] / disc[0] - 0.85) < 1e-5
    assert disc[0] > 50 * rgb[1].max()                       # the disc outshines the zenith sky
    assert pdf[0] == np.float32(1.0) / (np.float32(2.0 * math.pi) * (np.float32(1.0) - COS_SUN_MAX)) or \
        abs(pdf[0] * 2 * math.pi * (1 - 0.9999892) - 1.0) < 1e-3
    assert pdf[1] == 0.0 and pdf[2] == 0.0
    assert (rgb[2] > 0).all()                                 # below the horizon: blend towards the ground tone


def test_sun_cone_samples_lie_in_the_disc():
    s = O.OracleScene(physical_sky_scene(elevation=35.0, azimuth=30.0))
    rng = np.random.default_rng(3)
    d = s.sun_sample(rng.random((20000, 2)))
    sun = _sun(35.0, 30.0)
    cos = d @ sun / np.linalg.norm(d, axis=1)
    assert (cos > 0.9999892 - 2e-6).all()
    # uniform in solid angle: cos θ uniform on [COS_SUN_MAX, 1]
    u = (1.0 - cos) / (1.0 - 0.9999892)
    assert abs(u.mean() - 0.5) < 0.02


def test_sky_brightness_follows_the_sun():
    lo = O.OracleScene(physical_sky_scene(elevation=5.0))
    hi = O.OracleScene(physical_sky_scene(elevation=60.0))
    up = np.array([[0.0, 1.0, 0.0]])
    assert hi.bg_eval_n(up)[0].sum() > lo.bg_eval_n(up)[0].sum()
