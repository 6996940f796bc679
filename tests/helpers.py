"""Scene fixtures shared by the CPU-oracle tests and the GPU parity tests."""
import numpy as np

from rustracer_b200.scene import Material, SceneBuilder

INF = np.float32(np.inf)


def ray(o, d, tmin=0.001, tmax=np.inf):
    return np.array(list(o) + list(d) + [tmin, tmax], dtype=np.float32)


def rays(*rs):
    return np.stack(rs).astype(np.float32)


def unit_quad_scene():
    """quad.rs:115-122: q=(0,0,0), u=(1,0,0), v=(0,1,0)."""
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_quad((0, 0, 0), (1, 0, 0), (0, 1, 0), m)
    return sb


def xy_triangle_scene(normals=None):
    """triangle.rs:231-238: v0=(0,0,0), v1=(2,0,0), v2=(0,2,0)."""
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_mesh(np.array([[0, 0, 0], [2, 0, 0], [0, 2, 0]], np.float64), np.array([[0, 1, 2]]), m, normals)
    return sb


def spheres_scene(centers, r=1.0):
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    for c in centers:
        sb.add_sphere(c, r, m)
    return sb


def random_rays(n, seed, center=(0, 0, 0), radius=3.0, spread=0.5, tmin=0.001):
    """Rays from a sphere of `radius` around `center` aimed at jittered points near it."""
    rng = np.random.default_rng(seed)
    o = rng.normal(size=(n, 3))
    o = o / np.linalg.norm(o, axis=1, keepdims=True) * radius + np.asarray(center)
    tgt = rng.normal(size=(n, 3)) * spread + np.asarray(center)
    d = tgt - o
    r = np.concatenate([o, d, np.full((n, 1), tmin), np.full((n, 1), np.inf)], 1)
    return r.astype(np.float32)


def camera_rays(cam, w, h, seed=0):
    """Primary rays through pixel centres jittered by a seeded uniform offset."""
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(w), np.arange(h))
    u = (ii.ravel() + rng.random(w * h)) / max(w - 1, 1)
    v = (jj.ravel() + rng.random(w * h)) / max(h - 1, 1)
    o = np.array(cam.origin, np.float32)
    ll, hz, vt = (np.array(x, np.float32) for x in (cam.lower_left, cam.horizontal, cam.vertical))
    d = ll[None] + u[:, None].astype(np.float32) * hz[None] + v[:, None].astype(np.float32) * vt[None] - o[None]
    r = np.concatenate([np.broadcast_to(o, d.shape), d, np.full((len(d), 1), 0.001), np.full((len(d), 1), np.inf)], 1)
    return r.astype(np.float32)


def tile_means(img, tile=16):
    """Per-tile mean over (H, W, 3) → (H/tile, W/tile, 3)."""
    h, w, _ = img.shape
    return img[: h // tile * tile, : w // tile * tile].reshape(h // tile, tile, w // tile, tile, 3).mean(axis=(1, 3))


def medium_sphere_scene(density=1.0, blocker=False, kind="constant"):
    """volume.rs:281-325: a medium in the unit sphere at the origin, optionally
    with an opaque sphere (-2, 0, 0) r 0.5 in front of it."""
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_medium(kind, "sphere", density, (1, 1, 1), center=(0, 0, 0), radius=1.0)
    if blocker:
        sb.add_sphere((-2.0, 0.0, 0.0), 0.5, m)
    return sb


def physical_sky_scene(elevation=35.0, azimuth=30.0, turbidity=3.0, roughness=0.3):
    """An open scene under the Physical sky: a diffuse floor, a rough conductor
    sphere and a diffuse sphere (sun NEE at diffuse and conductor vertices)."""
    from rustracer_b200.configs import gold_like_nk
    sb = SceneBuilder()
    sb.set_physical(azimuth, elevation, turbidity)
    floor = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    n, k = gold_like_nk()
    metal = sb.add_material(Material.spectral_metal_nk(380.0, 50.0, n, k, roughness=roughness))
    white = sb.add_material(Material.lambertian((0.8, 0.8, 0.8)))
    sb.add_quad((-5.0, 0.0, -5.0), (0.0, 0.0, 10.0), (10.0, 0.0, 0.0), floor)
    sb.add_sphere((-0.6, 0.5, 0.0), 0.5, metal)
    sb.add_sphere((0.6, 0.4, 0.2), 0.4, white)
    return sb
