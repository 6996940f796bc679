"""rt_render_pass_noalloc: the sample-pass entry point for hosts that may not
allocate device memory while they run (real-time loops that must not stall on
cudaMalloc, processes whose device memory belongs to a framework's caching
allocator, plugin hosts that pass only their own buffers).  Its output must
match rt_render_pass on the same inputs, on consecutive calls that share the
library's fixed scratch array.  Collected last so that a failure here comes
after every other test has run."""
import numpy as np
import pytest

from rustracer_b200 import configs
from rustracer_b200.renderer import GpuScene, RtError, pass_params

pytestmark = pytest.mark.gpu


def test_noalloc_matches_render_pass_on_consecutive_calls():
    import torch
    sb, st = configs.box_scene(width=96, height=80)
    g = GpuScene(sb)
    for call, (first, seed) in enumerate([(0, 3), (4, 11)]):
        p = pass_params(96, 80, first, 4, 2, 8, 4, 1.0, seed)
        ref = torch.zeros((4, 80, 96, 3), device="cuda")
        out = torch.full((4, 80, 96, 3), float("nan"), device="cuda")
        g.render_pass(st["camera"], p, out=ref)
        g.render_pass_noalloc(st["camera"], p, out)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.isfinite(a).all(), f"call {call}: non-finite output"
        np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-7, err_msg=f"call {call}")
        assert b.sum() > 0


@pytest.mark.parametrize("w,h,n", [(128, 128, 4), (256, 256, 1)])
def test_noalloc_refills_its_path_pool(w, h, n):
    """Frames of more samples than the fixed array's 32,768 path slots: the
    retire kernel hands each freed slot the next sample, through the shared
    array, until all w·h·n samples are drawn (two calls in a row)."""
    import torch
    assert w * h * n > 32768
    sb, st = configs.box_scene(width=w, height=h)
    g = GpuScene(sb)
    for call, (first, seed) in enumerate([(0, 21), (n, 22)]):
        p = pass_params(w, h, first, n, 2, 8, 4, 1.0, seed)
        ref = torch.zeros((n, h, w, 3), device="cuda")
        out = torch.full((n, h, w, 3), float("nan"), device="cuda")
        g.render_pass(st["camera"], p, out=ref)
        g.render_pass_noalloc(st["camera"], p, out)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.isfinite(a).all(), f"call {call}: non-finite output"
        np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-7, err_msg=f"call {call}")
        assert b.sum() > 0


def test_noalloc_rejects_frames_beyond_its_scratch():
    import torch
    sb, st = configs.box_scene(width=512, height=512)
    g = GpuScene(sb)
    out = torch.zeros((1, 512, 512, 3), device="cuda")
    with pytest.raises(RtError) as e:
        g.render_pass_noalloc(st["camera"], pass_params(512, 512, 0, 1, 1, 8, 4, 1.0, 1), out)
    assert e.value.code == 2 and "65536" in str(e.value)
