"""Output development on the GPU against the CPU oracle: apply_optics +
tone_map (output.rs:84-190) byte for byte up to one level (the device log2f /
powf differ from the CPU's in the last bits), from linear images and from the
device accumulators, and the PNG written by save_png."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.output import read_png, save_png
from rustracer_b200.renderer import GpuScene, develop_params, pass_params
from rustracer_b200.scene import make_camera
from tests.helpers import physical_sky_scene

pytestmark = pytest.mark.gpu


def _close(a, b):
    d = np.abs(a.astype(int) - b.astype(int))
    assert d.max() <= 1, d.max()
    assert (d == 0).mean() > 0.995, (d == 0).mean()


@pytest.mark.parametrize("tm", ["agx", "aces"])
@pytest.mark.parametrize("vig,dist", [(0.0, 0.0), (0.3, 0.05), (1.0, 1.0)])
def test_gpu_develop_linear_matches_oracle(tm, vig, dist):
    rng = np.random.default_rng(5)
    img = np.exp(rng.normal(-1.0, 2.0, (61, 97, 3))).astype(np.float32)
    g = GpuScene(physical_sky_scene())
    got = g.develop(97, 61, linear=img, exposure=1.3, tonemapper=tm, vignette=vig, distortion=dist)
    want = O.develop(develop_params(97, 61, 1.3, tm, vig, dist), linear=img)
    _close(got, want)


def test_gpu_develop_accumulators_and_png(tmp_path):
    sb = physical_sky_scene()
    g = GpuScene(sb)
    cam = make_camera((0.0, 1.2, 3.5), (0.0, 0.4, 0.0), vfov=40.0, aspect=1.5)
    s, _, c = g.render_accumulate(cam, pass_params(96, 64, 0, 16, 4, 8, 1, 1.0, 3))
    got = g.develop(96, 64, exposure=0.8, vignette=0.25, distortion=0.02)
    want = O.develop(develop_params(96, 64, 0.8, "agx", 0.25, 0.02), sum_=s, count=c)
    _close(got, want)
    path = save_png(g, 96, 64, "Sky Test", 16, exposure=0.8, vignette=0.25, distortion=0.02,
                    path=str(tmp_path / "out.png"))
    assert np.array_equal(read_png(path), got)


def test_gpu_develop_device_tensors():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(6)
    img = np.exp(rng.normal(-1.0, 1.5, (33, 45, 3))).astype(np.float32)
    g = GpuScene(physical_sky_scene())
    host = g.develop(45, 33, linear=img, tonemapper="aces")
    dev = g.develop(45, 33, linear=torch.from_numpy(img).cuda(), tonemapper="aces")
    assert dev.is_cuda and np.array_equal(dev.cpu().numpy(), host)


def test_gpu_develop_rejects_bad_parameters():
    g = GpuScene(physical_sky_scene())
    with pytest.raises(Exception):
        g.develop(8, 8, linear=np.zeros((8, 8, 3), np.float32), vignette=1.5)
    with pytest.raises(Exception):
        g.develop(8, 8)                       # no accumulators of this size yet
