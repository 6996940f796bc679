"""The path-guiding network on the GPU against its CPU restatement
(oracle/guide.py): network outputs, mixture densities and draws, the
gradient of the loss over every parameter, one Adam step; then, on the
slit-light room, that guided rendering stays unbiased, with the relMSE of the
trained guide against cosine bounces at equal samples reported."""
import numpy as np
import pytest

from oracle import guide as OG
from rustracer_b200 import configs
from rustracer_b200.guiding import relmse, render_guided
from rustracer_b200.renderer import GpuScene, guide_params, pass_params
from tests.test_gpu_render import assert_tiles_agree

pytestmark = pytest.mark.gpu

RES = OG.resolutions(16, 1.447)           # 16 → ≈4096 cells: every level hashed or dense exercised
LO, INV = np.zeros(3, np.float32), np.ones(3, np.float32)


def _scene():
    sb, _ = configs.box_scene(width=32, height=32)
    gs = GpuScene(sb)
    gs.guide_init(guide_params(lr=1e-2, domain=((0, 0, 0), (1, 1, 1)), batch=1024, min_resolution=16,
                               level_scale=1.447, alpha_max=OG.AMAX, log_kappa_max=OG.LKMAX))
    return gs


def _params(seed=11):
    p = OG.init_params(seed)
    rng = np.random.default_rng(seed + 1)
    p[OG.N_MLP:] = rng.uniform(-0.5, 0.5, p.size - OG.N_MLP).astype(np.float32)   # features that matter
    return p


def _queries(n, seed=2):
    """Positions (a few outside the box: clamped), unit normals and unit
    outgoing directions ω_o (the one-blob input)."""
    rng = np.random.default_rng(seed)
    P = rng.uniform(-0.05, 1.05, (n, 3)).astype(np.float32)
    N = rng.normal(size=(n, 3))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    WO = rng.normal(size=(n, 3))
    WO /= np.linalg.norm(WO, axis=1, keepdims=True)
    return P, N.astype(np.float32), WO.astype(np.float32)


def test_guide_network_outputs_match_oracle():
    gs = _scene()
    p = _params()
    gs.guide_set_params(p)
    assert np.array_equal(gs.guide_get_params(), p)
    P, N, WO = _queries(4096)
    gpu = gs.guide_eval(np.concatenate([P, N, WO], 1))
    X = OG.encode(p, RES, LO, INV, P, WO)
    cpu, _ = OG.forward(p, X)
    cpu = cpu[:, :41]
    scale = cpu.std()
    err = np.abs(gpu - cpu)
    assert np.isfinite(gpu).all()
    assert np.quantile(err, 0.99) < 1e-3 * scale, np.quantile(err, 0.99) / scale
    assert err.max() < 5e-2 * scale, err.max() / scale


def test_guide_density_and_draws():
    gs = _scene()
    gs.guide_set_params(_params(21))
    n = 1 << 18
    P, N, WO = _queries(n, 4)
    q = np.concatenate([P, N, WO], 1)
    raw = gs.guide_eval(q)
    rng = np.random.default_rng(9)
    D = rng.normal(size=(n, 3))
    D /= np.linalg.norm(D, axis=1, keepdims=True)
    pdf = gs.guide_pdf(q, D)
    ref = OG.guide_pdf(raw, N, D)
    assert np.allclose(pdf, ref, rtol=2e-3, atol=1e-6)
    u = rng.random((n, 4)).astype(np.float32)
    out = gs.guide_sample(q, u)
    d = out[:, :3]
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)
    assert np.allclose(out[:, 3], gs.guide_pdf(q, d), rtol=1e-6)
    assert np.allclose(out[:, 3], OG.guide_pdf(raw, N, d), rtol=2e-3, atol=1e-6)
    # E[cos⁺/p] over draws from p is ∫ cos⁺ = π for every row's mixture
    est = np.maximum((d * N).sum(1), 0) / out[:, 3]
    assert abs(est.mean() / np.pi - 1) < 1e-2, est.mean() / np.pi


def _samples(n, seed=6):
    rng = np.random.default_rng(seed)
    P, N, WO = _queries(n, seed)
    D = rng.normal(size=(n, 3))
    D /= np.linalg.norm(D, axis=1, keepdims=True)
    D = np.where(((D * N).sum(1) < 0)[:, None] & (rng.random((n, 1)) < 0.8), -D, D)
    w = rng.exponential(1.0, n)
    w[rng.random(n) < 0.1] = 0.0
    return np.concatenate([P, N, WO, D, w[:, None]], 1).astype(np.float32)


def _rel(a, b):
    return np.linalg.norm(a.astype(np.float64) - b) / max(np.linalg.norm(b.astype(np.float64)), 1e-30)


def test_guide_gradient_matches_oracle():
    gs = _scene()
    p = _params(31)
    gs.guide_set_params(p)
    s = _samples(1500)
    loss, g = gs.guide_loss_grad(s)
    lref, gref = OG.loss_and_grad(p, RES, LO, INV, s)
    assert abs(loss / lref - 1) < 1e-3
    for name, sl in (("W0", slice(0, 4096)), ("W1", slice(4096, 8192)), ("W2", slice(8192, 12288)),
                     ("W3", slice(12288, OG.N_MLP)), ("table", slice(OG.N_MLP, None))):
        r = _rel(g[sl], gref[sl])
        assert r < 2e-2, (name, r)
    assert np.array_equal(g[12288 + 41 * 64:OG.N_MLP], np.zeros(7 * 64, np.float32))   # padded outputs


def test_guide_adam_step_matches_oracle():
    gs = _scene()
    p = _params(41)
    gs.guide_set_params(p)
    s = _samples(1024, 8)
    _, g = gs.guide_loss_grad(s)
    gs.guide_train(s, steps=1)
    p1 = gs.guide_get_params()
    ref, _, _ = OG.adam(p, np.zeros_like(p), np.zeros_like(p), g, 1)
    big = np.abs(g) > 1e-4 * np.abs(g).max()
    assert big.sum() > 1000
    assert np.allclose(p1[big], ref[big], rtol=0, atol=1e-6 + 1e-3 * 1e-2)
    assert np.abs(p1 - ref).max() <= 2.0e-2 + 1e-6            # sign of a near-zero gradient at worst
    assert np.array_equal(p1[g == 0], p[g == 0])


def _vmf_draw(mu, k, n, rng):
    u1, u2 = rng.random(n), rng.random(n)
    c = 1 + np.log(u1 + (1 - u1) * np.exp(-2 * k)) / k
    t = np.cross(mu, [1.0, 0.0, 0.0] if abs(mu[0]) < 0.9 else [0.0, 1.0, 0.0])
    t /= np.linalg.norm(t)
    b = np.cross(mu, t)
    s = np.sqrt(np.maximum(1 - c * c, 0))
    return (c[:, None] * mu + s[:, None] * (np.cos(2 * np.pi * u2)[:, None] * t + np.sin(2 * np.pi * u2)[:, None] * b))


def test_guide_training_learns_a_known_distribution():
    """Records from two points, each with its own vMF lobe (κ 40) and unit
    weights: Adam steps raise the mean log-density of fresh draws at each
    point from the untrained level towards the lobe's own (≈ 0.75 with
    α ≤ 0.9), and each point's density prefers its own lobe's draws."""
    gs = _scene()
    rng = np.random.default_rng(17)
    mus = np.array([[0.3, -0.2, 0.93], [-0.5, 0.4, 0.77]])
    mus /= np.linalg.norm(mus, axis=1, keepdims=True)
    pts = np.array([[0.2, 0.3, 0.4], [0.7, 0.6, 0.5]])
    n = 4096
    rows, q, fresh = [], [], []
    for mu, pt in zip(mus, pts):
        P = np.tile(pt, (n, 1))
        N = np.tile([0.0, 0.0, 1.0], (n, 1))
        WO = np.tile([0.0, 0.6, 0.8], (n, 1))
        rows.append(np.concatenate([P, N, WO, _vmf_draw(mu, 40.0, n, rng), np.ones((n, 1))], 1))
        q.append(np.concatenate([P[:2048], N[:2048], WO[:2048]], 1))
        fresh.append(_vmf_draw(mu, 40.0, 2048, rng))
    s = np.concatenate(rows).astype(np.float32)
    before = [np.log(gs.guide_pdf(q[i], fresh[i])).mean() for i in range(2)]
    gs.guide_train(s, steps=200)
    after = [np.log(gs.guide_pdf(q[i], fresh[i])).mean() for i in range(2)]
    cross = [np.log(gs.guide_pdf(q[i], fresh[1 - i])).mean() for i in range(2)]
    print(f"mean log p of the targets' draws: {before} -> {after} (other point's lobe: {cross})")
    for i in range(2):
        assert after[i] > before[i] + 1.5
        assert after[i] > 0.3
        assert after[i] > cross[i] + 1.0


def test_guided_render_is_unbiased_and_measures_its_gain():
    w = h = 64
    sb, st = configs.guided_box_scene(width=w, height=h, max_depth=24)
    gs = GpuScene(sb)
    cam, hero = st["camera"], st["hero"]
    base = pass_params(w, h, 0, 1, 8, 24, hero, 1.0, 5)
    _, _, stats = render_guided(gs, cam, base, 48, train_spp=48, train_per_call=4,
                                guide=guide_params(batch=16384, steps_per_pass=16, seed=3))
    assert stats["steps"] == 12 * 16 and stats["samples"] > 2_000     # records that gathered light
    gs.guide_mode(1)
    spp = 256
    gi = gs.render_pass(cam, pass_params(w, h, 1000, spp, 16, 24, hero, 1.0, 7))
    gs.guide_mode(0)
    pi = gs.render_pass(cam, pass_params(w, h, 1000, spp, 16, 24, hero, 1.0, 8))
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, pi)                                   # guided bounces leave the mean alone
    ref = gs.render_pass(cam, pass_params(w, h, 0, 4096, 64, 24, hero, 1.0, 9)).mean(0)
    e_g, e_p = relmse(gi.mean(0), ref), relmse(pi.mean(0), ref)
    print(f"relMSE at {spp} spp: guided {e_g:.4g}, plain {e_p:.4g} (ratio {e_g / e_p:.3f})")
    # on this room the trained guide is about even with cosine bounces at equal
    # samples (5-15 % better at 320×180 and 1280×720); training is not
    # deterministic (records are appended by atomics) and a 64×64 relMSE is a
    # noisy estimate (0.74-1.12 of plain seen), so only a clear loss fails
    assert e_g < 1.35 * e_p


@pytest.mark.parametrize("background", ["physical", "envmap"])
def test_guided_sun_and_env_nee_stay_unbiased(background):
    """The guide density also enters the sun-NEE weights of a Physical sky and
    the env-map NEE weights: after a short training, guided tiles agree with
    cosine bounces within 3 SE."""
    from rustracer_b200.scene import Material, SceneBuilder, make_camera
    sb = SceneBuilder()
    floor = sb.add_material(Material.lambertian((0.6, 0.6, 0.6)))
    red = sb.add_material(Material.lambertian((0.7, 0.25, 0.2)))
    sb.add_quad((-3.0, 0.0, -3.0), (0.0, 0.0, 6.0), (6.0, 0.0, 0.0), floor)
    sb.add_quad((-1.5, 0.0, -1.0), (3.0, 0.0, 0.0), (0.0, 1.5, 0.0), red)        # a wall casting shadows
    sb.add_sphere((0.3, 0.4, 0.2), 0.4, floor)
    if background == "physical":
        sb.set_physical(40.0, 35.0, 3.0)
    else:
        env, _ = configs.sky_env(256, 128, sun_peak=50.0, seed=4)
        sb.set_env(env)
    w = h = 48
    cam = make_camera((0.0, 1.2, 3.0), (0.0, 0.4, 0.0), vfov=45.0, aspect=1.0)
    gs = GpuScene(sb)
    base = pass_params(w, h, 0, 1, 4, 8, 4, 1.0, 5)
    render_guided(gs, cam, base, 16, train_spp=16, guide=guide_params(batch=16384, steps_per_pass=16, seed=2))
    gs.guide_mode(1)
    gi = gs.render_pass(cam, pass_params(w, h, 100, 128, 11, 8, 4, 1.0, 7))
    gs.guide_mode(0)
    pi = gs.render_pass(cam, pass_params(w, h, 100, 128, 11, 8, 4, 1.0, 8))
    assert np.isfinite(gi).all() and gi.mean() > 0
    assert_tiles_agree(gi, pi)


def test_guided_gem_room_with_photons_stays_unbiased():
    """Guided bounces beside the caustic photon map's injection, PBR lobes,
    analytic gems and the dusk sky's sun NEE (the reference's benchmark room
    at a reduced size): guided tiles agree with cosine bounces within 3 SE."""
    from rustracer_b200 import photons
    sb, st = configs.gem_room_scene(width=96, height=64)
    gs = GpuScene(sb)
    assert gs.photon_build(photons.caustic_params(sb, st["photons"], st["radius"], seed=1)) > 1000
    cam = st["camera"]
    render_guided(gs, cam, pass_params(96, 64, 0, 1, 4, 16, 1, 1.0, 5), 16, train_spp=16,
                  guide=guide_params(batch=16384, seed=2))
    gs.guide_mode(1)
    gi = gs.render_pass(cam, pass_params(96, 64, 100, 96, 8, 16, 1, 1.0, 7))
    gs.guide_mode(0)
    pi = gs.render_pass(cam, pass_params(96, 64, 100, 96, 8, 16, 1, 1.0, 8))
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, pi)


def test_guide_entry_points_take_device_buffers():
    """rt_guide_eval / _pdf / _sample with RT_MEM_DEVICE pointers (CUDA
    tensors) give what the host-memory calls give."""
    import ctypes as C
    import torch
    from rustracer_b200 import abi
    from rustracer_b200.renderer import lib
    gs = _scene()
    gs.guide_set_params(_params(51))
    P, N, WO = _queries(3000, 12)
    q = np.concatenate([P, N, WO], 1).astype(np.float32)
    rng = np.random.default_rng(3)
    D = rng.normal(size=(3000, 3)).astype(np.float32)
    D /= np.linalg.norm(D, axis=1, keepdims=True)
    u = rng.random((3000, 4)).astype(np.float32)
    qd, dd, ud = (torch.from_numpy(x).cuda() for x in (q, D, u))
    raw_d = torch.zeros((3000, 41), device="cuda")
    pdf_d = torch.zeros(3000, device="cuda")
    smp_d = torch.zeros((3000, 4), device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())
    assert lib().rt_guide_eval(gs.h, ptr(qd), 3000, ptr(raw_d), abi.RT_MEM_DEVICE) == 0
    assert lib().rt_guide_pdf(gs.h, ptr(qd), ptr(dd), 3000, ptr(pdf_d), abi.RT_MEM_DEVICE) == 0
    assert lib().rt_guide_sample(gs.h, ptr(qd), ptr(ud), 3000, ptr(smp_d), abi.RT_MEM_DEVICE) == 0
    torch.cuda.synchronize()
    assert np.array_equal(raw_d.cpu().numpy(), gs.guide_eval(q))
    assert np.array_equal(pdf_d.cpu().numpy(), gs.guide_pdf(q, D))
    assert np.array_equal(smp_d.cpu().numpy(), gs.guide_sample(q, u))
