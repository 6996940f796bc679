"""Seeded synthetic workloads (the reference ships no data set for them).

Each generator returns (SceneBuilder, render settings dict).  Sizes and value
distributions follow the workload definitions:

  box        256×256 open-front 1×1×1 Lambertian room, diffuse + dispersive glass
             sphere, 0.25² 6500 K blackbody ceiling light ×15; 16 spp, depth 8,
             4 hero wavelengths over 380–780 nm.
  icosphere  icosphere with 8 subdivisions (1,310,720 triangles), radial Perlin
             displacement (amplitude 0.08, 4 octaves, frequency 3), GGX conductor
             roughness 0.2 with a gold-like n,k on 8 wavelengths; diffuse floor
             (albedo 0.5); 2048×1024 float32 sky (gradient 0.2→1.0 plus a 0.5°
             sun lobe of peak 5e4); 1920×1080, 64 spp, depth 12.

The Perlin noise is the lattice-gradient noise of src/perlin.rs:21-92 (random
unit gradients, three 256-entry permutations, Hermite-smoothed trilinear
interpolation), seeded from numpy instead of thread_rng.
"""
import functools
import math

import numpy as np

from .scene import Material, SceneBuilder, make_camera, scene_from_toml_dict

F32 = np.float32


# ── Perlin (perlin.rs:21-92), vectorised ────────────────────────────────────
class Perlin:
    def __init__(self, seed):
        rng = np.random.default_rng(seed)
        v = rng.uniform(-1.0, 1.0, size=(256, 3))
        self.ranvec = v / np.linalg.norm(v, axis=1, keepdims=True)
        self.perm = [rng.permutation(256) for _ in range(3)]

    def noise(self, p):
        p = np.asarray(p, dtype=np.float64)
        fl = np.floor(p)
        f = p - fl
        s = f * f * (3.0 - 2.0 * f)
        ijk = fl.astype(np.int64)
        acc = np.zeros(len(p))
        for di in (0, 1):
            for dj in (0, 1):
                for dk in (0, 1):
                    idx = (self.perm[0][(ijk[:, 0] + di) & 255] ^ self.perm[1][(ijk[:, 1] + dj) & 255]
                           ^ self.perm[2][(ijk[:, 2] + dk) & 255])
                    g = self.ranvec[idx]
                    wv = s - np.array([di, dj, dk], dtype=np.float64)
                    wgt = ((di * s[:, 0] + (1 - di) * (1 - s[:, 0])) * (dj * s[:, 1] + (1 - dj) * (1 - s[:, 1]))
                           * (dk * s[:, 2] + (1 - dk) * (1 - s[:, 2])))
                    acc += wgt * (g * wv).sum(1)
        return acc

    def fbm(self, p, octaves):
        acc = np.zeros(len(p))
        w = 1.0
        q = np.asarray(p, dtype=np.float64)
        for _ in range(octaves):
            acc += w * self.noise(q)
            w *= 0.5
            q = q * 2.0
        return acc


# ── icosphere ────────────────────────────────────────────────────────────────
def icosphere(levels):
    """Unit icosphere: 20·4^levels faces, shared vertices (midpoint cache)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    V = np.array(verts, dtype=np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    Fc = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                   [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                   [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(levels):
        nv = len(V)
        e = np.concatenate([Fc[:, [0, 1]], Fc[:, [1, 2]], Fc[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (nv + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // (nv + 1), uniq % (nv + 1)
        mid = V[a] + V[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        V = np.concatenate([V, mid])
        nf = len(Fc)
        m01, m12, m20 = nv + inv[:nf], nv + inv[nf:2 * nf], nv + inv[2 * nf:]
        Fc = np.concatenate([
            np.stack([Fc[:, 0], m01, m20], 1),
            np.stack([Fc[:, 1], m12, m01], 1),
            np.stack([Fc[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1)])
    return V, Fc


def vertex_normals(V, Fc):
    fn = np.cross(V[Fc[:, 1]] - V[Fc[:, 0]], V[Fc[:, 2]] - V[Fc[:, 0]])
    N = np.zeros_like(V)
    for k in range(3):
        np.add.at(N, Fc[:, k], fn)
    return N / np.linalg.norm(N, axis=1, keepdims=True)


# ── synthetic environment map ────────────────────────────────────────────────
def sky_env(width=2048, height=1024, sun_dir=None, sun_peak=5e4, sun_fwhm_deg=0.5, seed=7):
    """Equirect float32 sky: luminance 0.2 at and below the horizon rising to
    1.0 at the zenith, plus a Gaussian sun lobe (FWHM 0.5°, peak 5e4).  Texel
    directions follow the reference's mapping (renderer.rs:145-151)."""
    if sun_dir is None:
        rng = np.random.default_rng(seed)
        az = rng.uniform(0, 2 * math.pi)
        el = math.radians(rng.uniform(25.0, 55.0))
        sun_dir = (math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az))
    s = np.asarray(sun_dir, dtype=np.float64)
    s /= np.linalg.norm(s)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = math.pi * v[:, None]
    phi = 2.0 * math.pi * (u[None, :] - 0.5)
    dx = np.sin(theta) * np.sin(phi)
    dy = np.cos(theta) * np.ones_like(phi)
    dz = np.sin(theta) * np.cos(phi)
    grad = 0.2 + 0.8 * np.clip(dy, 0.0, 1.0)
    cosg = np.clip(dx * s[0] + dy * s[1] + dz * s[2], -1.0, 1.0)
    ang = np.degrees(np.arccos(cosg))
    sigma = sun_fwhm_deg / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    sun = sun_peak * np.exp(-0.5 * (ang / sigma) ** 2)
    sky = np.stack([grad * 0.85 + sun, grad * 0.92 + sun * 0.96, grad * 1.0 + sun * 0.88], axis=-1)
    return sky.astype(F32), tuple(s)


def gold_like_nk(n_samples=8, start=380.0, step=50.0):
    """n,k of gold (src/spectrum.rs:218-219) resampled on a uniform grid."""
    from . import abi  # noqa: F401
    gold_n = [1.69, 1.65, 1.54, 1.33, 0.97, 0.54, 0.30, 0.23, 0.20, 0.19, 0.18, 0.16, 0.16]
    gold_k = [1.91, 1.94, 1.95, 1.92, 1.80, 1.93, 2.41, 3.00, 3.56, 4.07, 4.56, 4.99, 5.41]
    lam = start + step * np.arange(n_samples)
    src = 380.0 + 25.0 * np.arange(13)
    return (np.interp(lam, src, gold_n).tolist(), np.interp(lam, src, gold_k).tolist())


# ── workloads ────────────────────────────────────────────────────────────────
def box_scene(width=256, height=256, spp=16, max_depth=8, hero=4, seed=1):
    sb = SceneBuilder()
    sb.name = "box"
    sb.spectral_range = 1 if hero > 1 else 0
    white = sb.add_material(Material.lambertian((0.73, 0.73, 0.73)))
    red = sb.add_material(Material.lambertian((0.65, 0.05, 0.05)))
    green = sb.add_material(Material.lambertian((0.12, 0.45, 0.15)))
    sb.add_quad((0, 0, 0), (1, 0, 0), (0, 0, 1), white)      # floor
    sb.add_quad((0, 1, 0), (1, 0, 0), (0, 0, 1), white)      # ceiling
    sb.add_quad((0, 0, 1), (1, 0, 0), (0, 1, 0), white)      # back wall
    sb.add_quad((1, 0, 0), (0, 0, 1), (0, 1, 0), red)        # left wall (image left)
    sb.add_quad((0, 0, 0), (0, 0, 1), (0, 1, 0), green)      # right wall
    light = sb.add_material(Material.blackbody(6500.0, 15.0))
    sb.add_light_quad((0.375, 1.0 - 1e-3, 0.375), (0.25, 0, 0), (0, 0, 0.25), light)
    diffuse = sb.add_material(Material.lambertian((0.73, 0.73, 0.73)))
    glass = sb.add_material(Material.spectral_dielectric_cauchy(1.5, 0.0042))
    sb.add_sphere((0.3, 0.18, 0.6), 0.18, diffuse)
    sb.add_sphere((0.7, 0.18, 0.35), 0.18, glass)
    sb.set_solid((0.0, 0.0, 0.0))
    cam = make_camera((0.5, 0.5, -1.4), (0.5, 0.5, 0.5), vfov=40.0, aspect=width / height)
    settings = dict(width=width, height=height, spp=spp, max_depth=max_depth, hero=hero, seed=seed, camera=cam,
                    name="box 256x256 16spp depth8 hero4")
    return sb, settings


def icosphere_scene(width=1920, height=1080, spp=64, max_depth=12, hero=4, seed=2, levels=8,
                    env_w=2048, env_h=1024):
    sb = SceneBuilder()
    sb.name = "icosphere"
    sb.spectral_range = 1 if hero > 1 else 0
    V, Fc = icosphere(levels)
    per = Perlin(seed)
    disp = per.fbm(V * 3.0, 4)
    V = V * (1.0 + 0.08 * disp)[:, None]
    N = vertex_normals(V, Fc)
    n, k = gold_like_nk()
    metal = sb.add_material(Material.spectral_metal_nk(380.0, 50.0, n, k, roughness=0.2))
    sb.add_mesh(V, Fc, metal, N)
    floor = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_quad((-10.0, -1.1, -10.0), (0.0, 0.0, 20.0), (20.0, 0.0, 0.0), floor)
    env, sun = sky_env(env_w, env_h, seed=seed)
    sb.set_env(env)
    cam = make_camera((0.0, 0.45, 3.6), (0.0, -0.15, 0.0), vfov=40.0, aspect=width / height)
    settings = dict(width=width, height=height, spp=spp, max_depth=max_depth, hero=hero, seed=seed, camera=cam,
                    name=f"icosphere{levels} {len(Fc)} tris {width}x{height} {spp}spp depth{max_depth} hero{hero}",
                    n_tris=len(Fc), sun_dir=sun)
    return sb, settings


def perlin_density_grid(res=128, seed=7, freq=4.0, octaves=4, empty=0.1):
    """A res³ grid (z, y, x) of fractal Perlin noise at the voxel centres of the
    unit cube, mapped to [0, 1]: the lowest `empty` fraction of the voxels is 0
    (clear gaps), the 99.5th percentile and above is 1.  (Cached: a copy.)"""
    return _density_grid(res, seed, freq, octaves, empty).copy()


@functools.lru_cache(maxsize=4)
def _density_grid(res, seed, freq, octaves, empty):
    per = Perlin(seed)
    c = (np.arange(res) + 0.5) / res
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    P = np.stack([x.ravel(), y.ravel(), z.ravel()], 1) * freq
    n = per.fbm(P, octaves).reshape(res, res, res)
    lo, hi = np.quantile(n, [empty, 0.995])
    return np.clip((n - lo) / (hi - lo), 0.0, 1.0).astype(F32)


def grid_box_scene(width=128, height=128, spp=16, max_depth=24, hero=4, seed=5, res=32, sigma_max=4.0):
    """The box room with a voxel-grid medium in its lower half: a res³
    fractal-noise grid scaled to σ_t ∈ [0, sigma_max], albedo 0.9, HG g = 0.3."""
    sb, st = box_scene(width, height, spp, max_depth, hero, seed)
    sb.name = "grid box"
    sb.spheres.clear()
    sb.add_medium("grid", "box", sigma_max, (0.9, 0.9, 0.9), g=0.3, p_min=(0.0, 0.0, 0.0), p_max=(1.0, 0.5, 1.0),
                  grid=perlin_density_grid(res, seed=seed))
    st["name"] = f"grid box {res}^3 {width}x{height} {spp}spp depth{max_depth} hero{hero}"
    return sb, st


def media_box_scene(width=256, height=256, spp=16, max_depth=24, hero=4, seed=5, density=4.0):
    """The box room with participating media (volume.rs): a Perlin-noise medium
    filling the lower half (density scale `density`, albedo 0.9, g = 0.3) and a
    constant-density sphere (σ = 2, albedo 0.8, g = −0.2) above it."""
    sb, st = box_scene(width, height, spp, max_depth, hero, seed)
    sb.name = "media box"
    sb.spheres.clear()                                   # keep the room and the light
    sb.add_medium("noise", "box", density, (0.9, 0.9, 0.9), g=0.3, noise_scale=4.0, threshold=0.05,
                  p_min=(0.0, 0.0, 0.0), p_max=(1.0, 0.5, 1.0), seed=seed)
    sb.add_medium("constant", "sphere", 2.0, (0.8, 0.8, 0.8), g=-0.2, center=(0.5, 0.7, 0.55), radius=0.15)
    st["name"] = f"media box {width}x{height} {spp}spp depth{max_depth} hero{hero}"
    return sb, st


def brilliant_planes(radius=0.5, table_pct=57.0, crown_angle=34.5, pavilion_angle=40.75, girdle_pct=3.0,
                     star_angle=22.0, upper_girdle_angle=42.0, lower_girdle_angle=41.5, girdle_facets=32):
    """Half-spaces of a 57-facet round brilliant: the table, 8 star, 8 bezel
    and 16 upper-girdle facets of the crown, 16 lower-girdle facets and 8
    pavilion mains, plus a girdle of `girdle_facets` vertical planes.  Bezels
    and pavilion mains sit at azimuths k·45° and leave the girdle edge there at
    the crown and pavilion angles; the table height is where a bezel reaches
    the table radius (table_pct % of the girdle diameter); stars lie on the
    table's octagon edges between the bezels; the girdle halves leave the
    girdle at k·45° + 22.5° ± 11.25°, steeper than the mains.  Returns a list
    of (unit outward normal, point on the plane, facet kind)."""
    r = radius
    ca, pa = math.radians(crown_angle), math.radians(pavilion_angle)
    t_r = table_pct / 100.0 * r
    gh = girdle_pct / 100.0 * 2.0 * r
    y_gt, y_gb = 0.5 * gh, -0.5 * gh
    y_tab = y_gt + (r - t_r) * math.tan(ca)

    def tilted(phi, alpha, rho, y, up):
        n = (math.sin(alpha) * math.cos(phi), math.cos(alpha) if up else -math.cos(alpha), math.sin(alpha) * math.sin(phi))
        return n, (rho * math.cos(phi), y, rho * math.sin(phi))

    P = [((0.0, 1.0, 0.0), (0.0, y_tab, 0.0), "table")]
    half = math.pi / 8.0
    for k in range(8):
        th = k * math.pi / 4.0
        P.append(tilted(th, ca, r, y_gt, True) + ("bezel",))
        P.append(tilted(th, pa, r, y_gb, False) + ("pavilion",))
        P.append(tilted(th + half, math.radians(star_angle), t_r * math.cos(half), y_tab, True) + ("star",))
        for sgn in (-1.0, 1.0):
            phi = th + half + sgn * half / 2.0
            P.append(tilted(phi, math.radians(upper_girdle_angle), r, y_gt, True) + ("upper_girdle",))
            P.append(tilted(phi, math.radians(lower_girdle_angle), r, y_gb, False) + ("lower_girdle",))
    for j in range(girdle_facets):
        a = (j + 0.5) * 2.0 * math.pi / girdle_facets
        P.append(((math.cos(a), 0.0, math.sin(a)), (math.cos(a) * r, 0.0, math.sin(a) * r), "girdle"))
    return P


def round_brilliant(radius=0.5, table_pct=57.0, crown_angle=34.5, pavilion_angle=40.75, girdle_pct=3.0,
                    split=3, center=(0.0, 0.0, 0.0), **facet_angles):
    """The 57-facet round brilliant of brilliant_planes as a closed triangle
    mesh: the half-spaces are intersected (scipy's half-space intersection),
    the solid's hull triangulated with outward winding, and every triangle
    split into split² (the solid is unchanged): 254 hull triangles, 2,286 at
    the default split.  Returns (vertices (n,3), faces (m,3))."""
    from scipy.spatial import ConvexHull, HalfspaceIntersection
    P = brilliant_planes(radius, table_pct, crown_angle, pavilion_angle, girdle_pct, **facet_angles)
    hs = []
    for nv, g, _ in P:
        nv = np.asarray(nv, np.float64)
        nv = nv / np.linalg.norm(nv)
        hs.append(list(nv) + [-float(nv @ np.asarray(g, np.float64))])      # n·x − d ≤ 0
    hi = HalfspaceIntersection(np.array(hs), np.zeros(3))
    V = hi.intersections
    hull = ConvexHull(V)
    V = hull.points
    F = hull.simplices.copy()
    ctr = V.mean(axis=0)
    for i, (a, b, c) in enumerate(F):
        nrm = np.cross(V[b] - V[a], V[c] - V[a])
        if nrm @ (V[a] - ctr) < 0:
            F[i] = (a, c, b)
    used = np.unique(F)
    remap = -np.ones(len(V), np.int64)
    remap[used] = np.arange(len(used))
    V, F = V[used], remap[F]
    if split > 1:
        V, F = _split_n(V, F, split)
    return V + np.asarray(center, np.float64), F


def brilliant_facets(V, F, radius=0.5, **kw):
    """Facet kind of every triangle of a round_brilliant mesh (centred at the
    origin), by the plane it lies on."""
    P = brilliant_planes(radius, **kw)
    kinds = []
    for a, b, c in F:
        m = (V[a] + V[b] + V[c]) / 3.0
        nrm = np.cross(V[b] - V[a], V[c] - V[a])
        nrm = nrm / np.linalg.norm(nrm)
        best = min(P, key=lambda p: np.abs(np.asarray(p[0]) / np.linalg.norm(p[0]) - nrm).sum()
                   + abs(np.dot(np.asarray(p[0]) / np.linalg.norm(p[0]), m - np.asarray(p[1]))))
        kinds.append(best[2])
    return kinds


def _split_n(V, F, k):
    """Split each triangle into k² by a k-step barycentric grid (shared edge
    points are merged, so the mesh stays closed)."""
    V = [tuple(v) for v in V]
    index = {}

    def point(a, b, c, i, j):
        # barycentric grid point (i, j, k − i − j) over corners a, b, c, keyed by
        # its exact rational position on the shared edge or face
        w = {a: k - i - j, b: i, c: j}
        key = tuple(sorted((p, q) for p, q in w.items() if q))
        if key not in index:
            pos = sum(np.asarray(V[p]) * q for p, q in w.items()) / k
            index[key] = len(V)
            V.append(tuple(pos))
        return index[key]

    out = []
    for a, b, c in F:
        g = {}
        for i in range(k + 1):
            for j in range(k + 1 - i):
                if i == 0 and j == 0:
                    g[(i, j)] = a
                elif i == k:
                    g[(i, j)] = b
                elif j == k:
                    g[(i, j)] = c
                else:
                    g[(i, j)] = point(a, b, c, i, j)
        for i in range(k):
            for j in range(k - i):
                out.append((g[(i, j)], g[(i + 1, j)], g[(i, j + 1)]))
                if i + j < k - 1:
                    out.append((g[(i + 1, j)], g[(i + 1, j + 1)], g[(i, j + 1)]))
    return np.array(V, np.float64), np.array(out, np.int64)


def _split4(V, F):
    V = list(map(tuple, V))
    mid = {}
    def m(a, b):
        key = (min(a, b), max(a, b))
        if key not in mid:
            mid[key] = len(V)
            V.append(tuple((np.asarray(V[a]) + np.asarray(V[b])) * 0.5))
        return mid[key]
    out = []
    for a, b, c in F:
        ab, bc, ca = m(a, b), m(b, c), m(c, a)
        out += [(a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)]
    return np.array(V, np.float64), np.array(out, np.int64)


def env_caustic_dir(env, seed=0xC0FFEE, n=8):
    """The env-map caustic source of rebuild_caustics (scene.rs:53-66): the unit sum
    of (0, 1, 0) and n directions drawn ∝ luminance·sinθ (a seeded stream standing
    in for the reference's SmallRng), and the map's radiance there × π."""
    h, w, _ = env.shape
    lum = 0.2126 * env[..., 0] + 0.7152 * env[..., 1] + 0.0722 * env[..., 2]
    wgt = (lum * np.sin(math.pi * (np.arange(h) + 0.5) / h)[:, None]).ravel().astype(np.float64)
    rng = np.random.default_rng(seed)
    idx = rng.choice(wgt.size, size=n, p=wgt / wgt.sum())
    d = np.array([0.0, 1.0, 0.0])
    for k in idx:
        j, i = divmod(int(k), w)
        theta = math.pi * (j + rng.random()) / h
        phi = 2.0 * math.pi * ((i + rng.random()) / w - 0.5)
        d = d + np.array([math.sin(theta) * math.sin(phi), math.cos(theta), math.sin(theta) * math.cos(phi)])
    d = d / np.linalg.norm(d)
    v = math.acos(max(-1.0, min(1.0, d[1]))) / math.pi
    u = (0.5 + math.atan2(d[0], d[2]) / (2 * math.pi)) % 1.0
    col = env[min(int(v * h), h - 1), min(int(u * w), w - 1)] * math.pi
    return tuple(d), tuple(float(c) for c in col)


def gem_scene(width=1280, height=720, spp=256, max_depth=32, hero=4, seed=3, env_w=1024, env_h=512,
              photons=2_000_000, knn_k=64, radius_max=0.01):
    """The gem workload: a 57-facet round brilliant (girdle Ø1, table 57 %,
    crown 34.5°, pavilion 40.75°, girdle 3 %; 2,286 triangles) in the diamond
    preset's Cauchy dispersion (B 2.351, C 0.0230: n_D 2.417, n_F − n_C 0.044;
    scene_file.rs:686) on an albedo-0.8 plane, two 0.3² blackbody lights at
    5500 K, the sky env at 0.1, and a caustic photon map of 2M photons emitted
    from the two lights toward the stone's bounding sphere (a projection map;
    k-NN 64 within r ≤ 0.01).  The reference's rebuild_caustics would emit
    from the env map's disk here (scene.rs:52-73), which sends nearly every
    photon past the stone; the lights are the workload's caustic source.  st["photon_params"](seed) gives the build's
    RtPhotonParams; st["env_dir"] / st["env_color"] keep the env-disk source."""
    sb = SceneBuilder()
    sb.name = "gem"
    sb.spectral_range = 1 if hero > 1 else 0
    V, Fc = round_brilliant(center=(0.0, 0.45, 0.0))
    diamond = sb.add_material(Material.spectral_dielectric_cauchy(2.351, 0.0230))
    sb.add_mesh(V, Fc, diamond)
    plane = sb.add_material(Material.lambertian((0.8, 0.8, 0.8)))
    sb.add_quad((-2.0, 0.0, -2.0), (0.0, 0.0, 4.0), (4.0, 0.0, 0.0), plane)
    light = sb.add_material(Material.blackbody(5500.0, 25.0))
    sb.add_light_quad((-1.35, 2.2, -0.65), (0.3, 0, 0), (0, 0, 0.3), light)
    sb.add_light_quad((0.95, 1.9, 0.45), (0.3, 0, 0), (0, 0, 0.3), light)
    env, _ = sky_env(env_w, env_h, seed=seed)
    env = (env * 0.1).astype(F32)
    sb.set_env(env)
    cam = make_camera((0.0, 1.55, 2.2), (0.0, 0.35, 0.0), vfov=32.0, aspect=width / height)
    d, col = env_caustic_dir(env)
    from . import photons as _ph

    gem_sphere = _ph.bounding_sphere(V)

    def photon_params(seed=1, n=photons, projection=True):
        return _ph.light_params(sb, n, radius_max, knn_k=knn_k, seed=seed,
                                target=gem_sphere if projection else None)
    st = dict(width=width, height=height, spp=spp, max_depth=max_depth, hero=hero, seed=seed, camera=cam,
              name=f"gem {len(Fc)} tris {width}x{height} {spp}spp depth{max_depth} hero{hero}",
              n_tris=len(Fc), photons=photons, knn_k=knn_k, radius_max=radius_max, env_dir=d, env_color=col,
              photon_params=photon_params)
    return sb, st


def latlong_ball(center, radius, nu=35, nv=21):
    """A closed latitude-longitude ball mesh: 2·nu·(nv − 2) quad triangles plus
    two pole fans = 1,400 faces for the defaults."""
    V = [[center[0], center[1] + radius, center[2]]]
    for j in range(1, nv):
        th = math.pi * j / nv
        for i in range(nu):
            ph = 2.0 * math.pi * i / nu
            V.append([center[0] + radius * math.sin(th) * math.cos(ph), center[1] + radius * math.cos(th),
                      center[2] + radius * math.sin(th) * math.sin(ph)])
    V.append([center[0], center[1] - radius, center[2]])
    F = []
    ring = lambda j, i: 1 + (j - 1) * nu + (i % nu)
    for i in range(nu):
        F.append([0, ring(1, i + 1), ring(1, i)])
    for j in range(1, nv - 1):
        for i in range(nu):
            a, b, c, d = ring(j, i), ring(j, i + 1), ring(j + 1, i), ring(j + 1, i + 1)
            F += [[a, b, c], [b, d, c]]
    bottom = len(V) - 1
    for i in range(nu):
        F.append([bottom, ring(nv - 1, i), ring(nv - 1, i + 1)])
    return np.array(V), np.array(F)


def gem_room_scene(width=1200, height=800, spp=128, max_depth=50, photons=500_000, gather_radius=0.5):
    """The reference's benchmark room (scenes/bench.toml): a 10 × 5 × 11 room
    with a checker floor, red and blue side walls, a back wall with a window,
    a ceiling with an opening around a 6500 K blackbody panel, a dusk
    Physical sky (sun elevation 10.2°, turbidity 4.5), a round brilliant
    diamond and a princess-cut sapphire as [[gems]], a brushed-gold PBR ball
    and a caustic photon map (500k photons, radius 0.5).  The reference's
    1,400-face OBJ ball is replaced by a generated 1,400-face ball of the
    same centre and radius."""
    white = {"type": "lambertian", "color": [0.80, 0.80, 0.80]}
    quad = lambda c, u, v, m: {"shape": {"type": "quad", "corner": c, "u": u, "v": v}, "material": m}
    doc = {
        "name": "Benchmark",
        "camera": {"look_from": [0.0, 3.4, -9.0], "look_at": [0.0, 2.247, 1.1993], "vfov": 36.0, "aperture": 0.0,
                   "focus_dist": 10.0},
        "background": {"type": "physical", "sun_azimuth": 0.0, "sun_elevation": 10.2, "turbidity": 4.5},
        "objects": [
            quad([-5.0, 0.0, -2.0], [10.0, 0.0, 0.0], [0.0, 0.0, 11.0],
                 {"type": "checker", "even": [0.12, 0.12, 0.12], "odd": [0.88, 0.88, 0.88], "scale": 0.8}),
            quad([-5.0, 0.0, -2.0], [0.0, 0.0, 11.0], [0.0, 5.0, 0.0], {"type": "lambertian", "color": [0.65, 0.10, 0.05]}),
            quad([5.0, 0.0, -2.0], [0.0, 0.0, 11.0], [0.0, 5.0, 0.0], {"type": "lambertian", "color": [0.05, 0.15, 0.65]}),
            quad([-5.0, 0.0, 9.0], [10.0, 0.0, 0.0], [0.0, 1.2, 0.0], white),
            quad([-5.0, 4.2, 9.0], [10.0, 0.0, 0.0], [0.0, 0.8, 0.0], white),
            quad([-5.0, 1.2, 9.0], [3.0, 0.0, 0.0], [0.0, 3.0, 0.0], white),
            quad([2.0, 1.2, 9.0], [3.0, 0.0, 0.0], [0.0, 3.0, 0.0], white),
            quad([-5.0, 5.0, -2.0], [10.0, 0.0, 0.0], [0.0, 0.0, 1.5], white),
            quad([-5.0, 5.0, 2.5], [10.0, 0.0, 0.0], [0.0, 0.0, 6.5], white),
            quad([-5.0, 5.0, -0.5], [3.5, 0.0, 0.0], [0.0, 0.0, 3.0], white),
            quad([1.5, 5.0, -0.5], [3.5, 0.0, 0.0], [0.0, 0.0, 3.0], white),
        ],
        "lights": [{"corner": [-1.5, 5.0, -0.5], "u": [3.0, 0.0, 0.0], "v": [0.0, 0.0, 3.0], "color": [8.0, 8.0, 8.0],
                    "temp_k": 6500.0, "intensity": 8.0}],
        "gems": [
            {"report": "round brilliant diamond", "measurements_mm": [9.00, 9.00, 5.60], "table_pct": 57.0,
             "crown_pct": 14.5, "pavilion_pct": 43.0, "color_grade": "D", "cut": "brilliant", "material": "diamond",
             "center": [0.0, 1.30, 2.5], "scale_mm": 0.3},
            {"report": "princess sapphire", "measurements_mm": [6.00, 5.90, 4.20], "table_pct": 65.0,
             "crown_pct": 12.0, "pavilion_pct": 50.0, "color_grade": "D", "cut": "princess", "material": "sapphire",
             "rotate_y": 25.0, "center": [-3.0, 0.90, 1.0], "scale_mm": 0.3},
        ],
    }
    sb = scene_from_toml_dict(doc)
    gold = sb.add_material(Material.pbr((1.0, 0.78, 0.34), roughness=0.25, metallic=1.0))
    V, F = latlong_ball((3.0, 1.2, 1.0), 1.2)
    sb.add_mesh(V, F, gold)
    sb.name = "Benchmark"
    aspect = width / height
    # CameraState::autofocus (camera.rs:139-143) does not matter with aperture 0
    cam = make_camera(doc["camera"]["look_from"], doc["camera"]["look_at"], vfov=36.0, aspect=aspect)
    return sb, dict(name="gem room", camera=cam, width=width, height=height, spp=spp, max_depth=max_depth, hero=1,
                    photons=photons, radius=gather_radius)


def guided_box_scene(width=1280, height=720, spp=64, max_depth=24, hero=4, seed=9, density=4.0, gem=True,
                     medium=True, grid_res=128, emission=600.0):
    """The hard-transport workload of the learned proposal: the box room whose
    ceiling has only a 0.05 × 0.1 slit (x ∈ [0.475, 0.525], z ∈ [0.45, 0.55]),
    with a 0.1² blackbody light (6500 K × `emission`) in a closed light box
    0.5 above it, a 57-facet round brilliant (radius 0.12, diamond
    dispersion) and a 128³ fractal-Perlin density grid in the lower half
    (σ_t ∈ [0, density], albedo 0.9, g = 0.3; delta tracking against
    per-brick majorants, ratio-tracked shadows).  grid_res = 0 puts the
    reference's procedural noise medium (volume.rs) there instead.  The light
    reaches the room only as the beam through the slit (a patch about 0.3
    across on the floor, and the medium along it); every other surface is lit
    from that patch, which cosine bounces find rarely and light sampling
    cannot reach."""
    sb = SceneBuilder()
    sb.name = "guided box"
    sb.spectral_range = 1 if hero > 1 else 0
    white = sb.add_material(Material.lambertian((0.73, 0.73, 0.73)))
    red = sb.add_material(Material.lambertian((0.65, 0.05, 0.05)))
    green = sb.add_material(Material.lambertian((0.12, 0.45, 0.15)))
    sb.add_quad((0, 0, 0), (1, 0, 0), (0, 0, 1), white)      # floor
    sb.add_quad((0, 0, 1), (1, 0, 0), (0, 1, 0), white)      # back wall
    sb.add_quad((1, 0, 0), (0, 0, 1), (0, 1, 0), red)        # left wall (image left)
    sb.add_quad((0, 0, 0), (0, 0, 1), (0, 1, 0), green)      # right wall
    # the ceiling at y = 1 around the slit
    sb.add_quad((0.0, 1.0, 0.0), (0.475, 0.0, 0.0), (0.0, 0.0, 1.0), white)
    sb.add_quad((0.525, 1.0, 0.0), (0.475, 0.0, 0.0), (0.0, 0.0, 1.0), white)
    sb.add_quad((0.475, 1.0, 0.0), (0.05, 0.0, 0.0), (0.0, 0.0, 0.45), white)
    sb.add_quad((0.475, 1.0, 0.55), (0.05, 0.0, 0.0), (0.0, 0.0, 0.45), white)
    # the light box above the slit: four walls and a lid, the light just below the lid
    lo, hi, top = 0.35, 0.65, 1.5
    sb.add_quad((lo, 1.0, lo), (hi - lo, 0.0, 0.0), (0.0, top - 1.0, 0.0), white)
    sb.add_quad((lo, 1.0, hi), (hi - lo, 0.0, 0.0), (0.0, top - 1.0, 0.0), white)
    sb.add_quad((lo, 1.0, lo), (0.0, 0.0, hi - lo), (0.0, top - 1.0, 0.0), white)
    sb.add_quad((hi, 1.0, lo), (0.0, 0.0, hi - lo), (0.0, top - 1.0, 0.0), white)
    sb.add_quad((lo, top, lo), (hi - lo, 0.0, 0.0), (0.0, 0.0, hi - lo), white)
    light = sb.add_material(Material.blackbody(6500.0, emission))
    sb.add_light_quad((0.45, top - 1e-3, 0.45), (0.1, 0, 0), (0, 0, 0.1), light)
    diffuse = sb.add_material(Material.lambertian((0.73, 0.73, 0.73)))
    sb.add_sphere((0.3, 0.18, 0.6), 0.18, diffuse)
    if gem:
        V, Fc = round_brilliant(radius=0.12, center=(0.68, 0.62, 0.45))
        diamond = sb.add_material(Material.spectral_dielectric_cauchy(2.351, 0.0230))
        sb.add_mesh(V, Fc, diamond)
    if medium and grid_res:
        sb.add_medium("grid", "box", density, (0.9, 0.9, 0.9), g=0.3, p_min=(0.0, 0.0, 0.0), p_max=(1.0, 0.5, 1.0),
                      grid=perlin_density_grid(grid_res, seed=seed))
    elif medium:
        sb.add_medium("noise", "box", density, (0.9, 0.9, 0.9), g=0.3, noise_scale=4.0, threshold=0.05,
                      p_min=(0.0, 0.0, 0.0), p_max=(1.0, 0.5, 1.0), seed=seed)
    sb.set_solid((0.0, 0.0, 0.0))
    cam = make_camera((0.5, 0.5, -1.4), (0.5, 0.5, 0.5), vfov=40.0, aspect=width / height)
    st = dict(width=width, height=height, spp=spp, max_depth=max_depth, hero=hero, seed=seed, camera=cam)
    st["name"] = (f"guided box (ceiling slit under a light box, gem, {grid_res}^3 grid medium) {width}x{height} "
                  f"{spp}spp depth{max_depth} hero{hero}")
    return sb, st


CONFIGS = {"box": box_scene, "icosphere": icosphere_scene, "media_box": media_box_scene, "grid_box": grid_box_scene,
           "gem": gem_scene,
           "gem_room": gem_room_scene, "guided_box": guided_box_scene}
