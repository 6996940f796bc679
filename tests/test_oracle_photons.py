"""CPU oracle of the caustic photon map (src/photon.rs) against the reference's
photon tests, plus the k-NN rule; no GPU needed."""
import numpy as np

from oracle import oracle as O
from rustracer_b200 import photons
from rustracer_b200.scene import Material, SceneBuilder


def glass_over_floor(floor_half=0.6):
    """photon.rs:345-364 with the infinite plane replaced by a finite floor quad
    (infinite planes are not in the GPU path; the reference excludes them from
    the photon bounds, a finite floor around the sphere plays the same role)."""
    sb = SceneBuilder()
    white = sb.add_material(Material.lambertian((0.7, 0.7, 0.7)))
    glass = sb.add_material(Material.dielectric(1.5))
    h = floor_half
    sb.add_quad((-h, 0.0, -h), (0, 0, 2 * h), (2 * h, 0, 0), white)
    sb.add_sphere((0.0, 1.0, 0.0), 0.5, glass)
    return sb


def test_photon_disk_hugs_geometry_and_stores_caustics():
    s = O.OracleScene(glass_over_floor())
    p = photons.photon_params([photons.disk_emitter((0, 1, 0), (10, 10, 10), 20000)], 0.5, seed=1)
    n = s.photon_build(p)
    assert n > 2000, n                                        # photon.rs:362-363
    pos, power, nor, idx = s.photon_export()
    assert np.isfinite(pos).all() and np.isfinite(power).all()
    assert (np.diff(idx) > 0).all()                           # emission order
    assert np.allclose(pos[:, 1], 0.0, atol=1e-4)             # all on the floor
    assert (nor[:, 1] > 0.99).all()
    # caustic under the sphere: positive, finite irradiance
    irr = s.photon_gather(np.array([[0, 0, 0, 0, 1, 0]], np.float32))[0]
    assert np.isfinite(irr).all() and irr[0] > 0


def test_photon_gather_matches_brute_force():
    rng = np.random.default_rng(3)
    n = 4000
    pos = rng.uniform(-1, 1, size=(n, 3)).astype(np.float32)
    pos[:, 1] = 0
    power = rng.uniform(0, 1, size=(n, 3)).astype(np.float32)
    nor = np.tile(np.array([0, 1, 0], np.float32), (n, 1))
    nor[::7] = (0, -1, 0)                                     # some on the opposite side
    s = O.OracleScene(glass_over_floor())
    s.photon_set(pos, power, nor, np.arange(n), radius=0.2)
    q = np.zeros((50, 6), np.float32)
    q[:, 0] = rng.uniform(-0.8, 0.8, 50)
    q[:, 2] = rng.uniform(-0.8, 0.8, 50)
    q[:, 4] = 1.0
    got = s.photon_gather(q)
    r2 = np.float32(0.04)
    for i in range(50):
        d2 = ((pos - q[i, :3]) ** 2).sum(1)
        m = (d2 < r2) & (nor[:, 1] > 0)
        want = (power[m] * (1 - d2[m] / r2)[:, None]).sum(0) * 2 / (np.pi ** 2 * r2)
        np.testing.assert_allclose(got[i], want, rtol=1e-4, atol=1e-6)


def test_knn_rule_sorted_with_index_ties():
    rng = np.random.default_rng(4)
    n = 3000
    pos = np.round(rng.uniform(-1, 1, size=(n, 3)) * 8) / 8            # many exact distance ties
    pos = pos.astype(np.float32)
    s = O.OracleScene(glass_over_floor())
    s.photon_set(pos, np.ones((n, 3), np.float32), np.tile([0, 1, 0], (n, 1)), np.arange(n), radius=0.3)
    q = rng.uniform(-1, 1, size=(40, 3)).astype(np.float32)
    idx, d2 = s.knn(q, 16, 0.5)
    for i in range(40):
        dd = ((pos - q[i]) ** 2).sum(1).astype(np.float32)
        order = np.lexsort((np.arange(n), dd))
        order = order[dd[order] <= np.float32(0.25)][:16]
        assert list(idx[i][: len(order)]) == list(order)
        assert (idx[i][len(order):] == -1).all()


def test_projection_map_keeps_the_expected_caustic_power():
    """Light-quad photons sent toward the stone's bounding sphere (power ×
    2·cosθ·(1 − cos θ_max)) store ~20× more photons than the full hemisphere,
    with the same expected total stored power (within 4 standard errors)."""
    from rustracer_b200 import configs
    sb, st = configs.gem_scene(width=32, height=18, env_w=64, env_h=32)
    s = O.OracleScene(sb)
    tot = {}
    for proj, n in ((False, 2_000_000), (True, 200_000)):
        cnt = s.photon_build(st["photon_params"](11, n, projection=proj))
        _, pw, _, _ = s.photon_export()
        lum = pw @ np.array([0.2126, 0.7152, 0.0722])
        # the map's total power is a sum over n photons (stored or not), so its
        # standard error is sqrt(n · Var) with the unstored photons at 0
        per = np.zeros(n)
        per[:cnt] = lum * n
        tot[proj] = (lum.sum(), per.std() / np.sqrt(n), cnt)
    (a, sa, na), (b, sb_, nb) = tot[False], tot[True]
    assert (nb / 200_000) > 10 * (na / 2_000_000), (na, nb)   # far more stored per emitted photon
    assert abs(a - b) < 4.0 * np.hypot(sa, sb_), (a, b, sa, sb_)


def test_photon_shards_partition_the_emission_order():
    """first_photon / shard_photons: the shards' stored photons are exactly
    the unsharded build's, split by emission index."""
    from rustracer_b200 import configs
    sb, st = configs.gem_scene(width=32, height=18, env_w=64, env_h=32)
    s = O.OracleScene(sb)
    p = st["photon_params"](2, 50000)
    s.photon_build(p)
    ref = s.photon_export()
    parts = []
    for r in range(3):
        s.photon_build(photons.shard_params(p, 3, r))
        parts.append(s.photon_export())
    for k in range(4):
        assert np.array_equal(np.concatenate([q[k] for q in parts]), ref[k])
