"""Host-side scene model: the flat structure-of-arrays description handed to
librtb200.so through rt_scene_create (include/rt_api.h).

It mirrors what the reference's loader builds (src/scene_file.rs:899-1132):
objects with materials and scale → rotate → translate transforms, NEE light
quads inserted into the world AND the light list (scene_file.rs:1056-1067),
backgrounds, and the spectral_dielectric (ior, dispersion) → Cauchy (B, C)
conversion (scene_file.rs:1161-1174).  Transforms (src/transform.rs) are applied
here to the primitives — the GPU path traces world-space primitives only — and
meshes join the world BVH directly instead of nesting a per-mesh BVH
(src/mesh.rs:91).

Canonical primitive ids (used for hit records and for tie-breaking) are:
triangles first, then quads, then spheres, each in insertion order.
"""
import ctypes as C
import math
import os

import numpy as np

from . import abi

F32 = np.float32


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


class Material:
    """Constructors for RtMaterial records (material.rs / texture.rs)."""

    @staticmethod
    def _new(t):
        m = abi.RtMaterial()
        m.type = t
        m.checker_scale = 1.0
        m.intensity = 1.0
        return m

    @staticmethod
    def lambertian(color):                                   # material.rs:85-102
        m = Material._new(abi.RT_MAT_LAMBERTIAN)
        m.albedo = _f3(color)
        return m

    @staticmethod
    def checker(even, odd, scale=1.0):                       # texture.rs:32-37
        m = Material._new(abi.RT_MAT_CHECKER)
        m.albedo = _f3(even)
        m.odd = _f3(odd)
        m.checker_scale = float(scale)
        return m

    @staticmethod
    def dielectric(ior):                                     # material.rs:323-332
        m = Material._new(abi.RT_MAT_DIELECTRIC)
        m.cauchy_b = float(ior)
        return m

    @staticmethod
    def spectral_dielectric_cauchy(b, c, absorption=(0.0, 0.0, 0.0)):   # material.rs:357-403
        m = Material._new(abi.RT_MAT_SPECTRAL_DIELECTRIC)
        m.cauchy_b = float(b)
        m.cauchy_c = float(c)
        m.absorption = _f3(absorption)
        return m

    @staticmethod
    def spectral_dielectric(ior, dispersion=0.0, absorption=(0.0, 0.0, 0.0)):
        """TOML form: (ior at the d-line, nF-nC-style spread) → Cauchy B, C
        exactly as scene_file.rs:1161-1174 computes them in f32."""
        c = F32(dispersion) / F32(3.250)
        b = F32(ior) - c / (F32(0.58756) * F32(0.58756))
        return Material.spectral_dielectric_cauchy(float(b), float(c), absorption)

    @staticmethod
    def spectral_metal(variant="gold", roughness=0.0):       # material.rs:427-554
        m = Material._new(abi.RT_MAT_SPECTRAL_METAL)
        m.metal = {"gold": abi.RT_METAL_GOLD, "copper": abi.RT_METAL_COPPER,
                   "silver": abi.RT_METAL_SILVER}.get(str(variant).lower(), abi.RT_METAL_GOLD)
        m.roughness = float(roughness)
        return m

    @staticmethod
    def spectral_metal_nk(start_nm, step_nm, n, k, roughness=0.0):
        """Conductor with a custom n,k table on a uniform wavelength grid."""
        if len(n) != len(k) or not (2 <= len(n) <= abi.RT_MAX_NK):
            raise ValueError("custom n,k table needs 2..16 samples")
        m = Material._new(abi.RT_MAT_SPECTRAL_METAL)
        m.metal = abi.RT_METAL_CUSTOM
        m.roughness = float(roughness)
        m.nk_count = len(n)
        m.nk_start = float(start_nm)
        m.nk_step = float(step_nm)
        for i, (a, b) in enumerate(zip(n, k)):
            m.nk_n[i] = float(a)
            m.nk_k[i] = float(b)
        return m

    @staticmethod
    def diffuse_light(color):                                # material.rs:14-25
        m = Material._new(abi.RT_MAT_DIFFUSE_LIGHT)
        m.albedo = _f3(color)
        return m

    @staticmethod
    def blackbody(temp_k, intensity=1.0):                    # material.rs:40-83
        m = Material._new(abi.RT_MAT_BLACKBODY_LIGHT)
        m.temp_k = float(temp_k)
        m.intensity = float(intensity)
        return m

    @staticmethod
    def pbr(albedo=(0.8, 0.8, 0.8), roughness=0.5, metallic=0.0, anisotropy=0.0, anisotropy_angle=0.0,
            clearcoat=0.0, clearcoat_roughness=0.03, film_thickness=0.0, film_ior=1.5, sheen=0.0, sheen_tint=0.5,
            emission=(0.0, 0.0, 0.0), emission_strength=0.0):
        """PbrMaterial with scalar parameters (material.rs:680-1050); the
        defaults are PbrMaterial::default and the TOML `pbr` defaults."""
        m = Material._new(abi.RT_MAT_PBR)
        m.albedo = _f3(albedo)
        m.roughness = float(roughness)
        m.metallic = float(metallic)
        m.anisotropy = float(anisotropy)
        m.anisotropy_angle = float(anisotropy_angle)
        m.clearcoat = float(clearcoat)
        m.clearcoat_roughness = float(clearcoat_roughness)
        m.film_thickness = float(film_thickness)
        m.film_ior = float(film_ior)
        m.sheen = float(sheen)
        m.sheen_tint = float(sheen_tint)
        m.emission = _f3(emission)
        m.emission_strength = float(emission_strength)
        return m


def _euler_fwd(angles_deg):
    """Rotate::euler (transform.rs:204-213): fwd = Ry · Rx · Rz, degrees."""
    rx, ry, rz = [math.radians(a) for a in angles_deg]
    sx, cx = math.sin(rx), math.cos(rx)
    sy, cy = math.sin(ry), math.cos(ry)
    sz, cz = math.sin(rz), math.cos(rz)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]], dtype=np.float64)
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]], dtype=np.float64)
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]], dtype=np.float64)
    return Ry @ (Rx @ Rz)


class Transform:
    """scale → rotate (Euler about the local origin) → translate (scene_file.rs:1036-1042)."""

    def __init__(self, scale=None, rotate=None, rotate_y=None, spin=None, translate=None):
        self.scale = 1.0 if scale is None else float(scale)
        ang = list(rotate) if rotate is not None else [0.0, 0.0, 0.0]
        if rotate_y is not None:
            ang[1] += float(rotate_y)
        if spin is not None:
            ang[1] += float(spin)
        self.R = _euler_fwd(ang) if any(a != 0.0 for a in ang) else np.eye(3)
        self.t = np.zeros(3) if translate is None else np.asarray(translate, dtype=np.float64)

    @property
    def identity(self):
        return self.scale == 1.0 and np.array_equal(self.R, np.eye(3)) and not self.t.any()

    def point(self, p):
        return (np.asarray(p, dtype=np.float64) * self.scale) @ self.R.T + self.t

    def vector(self, v):
        return (np.asarray(v, dtype=np.float64) * self.scale) @ self.R.T

    def normal(self, n):
        return np.asarray(n, dtype=np.float64) @ self.R.T


class SceneBuilder:
    """Collects primitives, materials, lights and the background, then emits an
    RtSceneDesc whose pointers stay valid while this object lives."""

    def __init__(self):
        self.materials = []
        self.tri_v = []          # list of (n,9) float32
        self.tri_n = []          # list of (n,9) float32 or None
        self.tri_mat = []
        self.tri_uv = []         # list of (n,6) float32 or None (the reference's default UVs)
        self.tri_tan = []        # list of (n,9) float32 or None ((1, 0, 0) tangents)
        self.textures = []       # RtTexture records (materials refer to them 1-based)
        self._tex_keep = []
        self.quads = []          # (Q, u, v, mat)
        self.spheres = []        # (c, r, mat)
        self._lights = []        # ("quad"|"sphere", local index)
        self.bg = {"type": abi.RT_BG_SOLID, "color": (0.0, 0.0, 0.0)}
        self.env = None          # (h, w, 3) float32
        self.spectral_range = 0
        self.name = "scene"
        self.camera = None       # dict(look_from, look_at, vfov, aperture, focus_dist)
        self.caustics = None
        self.media = []          # abi.RtMedium
        self.convex = []         # dicts: object-space planes (k,4) float32, mat, polish, box, placement
        self.shapes = []         # RtShape records

    # materials ---------------------------------------------------------
    def add_material(self, m):
        self.materials.append(m)
        return len(self.materials) - 1

    # primitives --------------------------------------------------------
    def add_sphere(self, center, radius, mat, xf=None):
        c = np.asarray(center, dtype=np.float64)
        r = float(radius)
        if xf is not None and not xf.identity:
            c = xf.point(c)
            r = r * xf.scale
        self.spheres.append((c.astype(F32), F32(r), mat))
        return len(self.spheres) - 1

    # participating media (volume.rs:78-263, scene_file.rs:297-336) ------
    def add_medium(self, kind, boundary, density, color, g=0.0, noise_scale=1.0, threshold=0.0, center=None,
                   radius=None, p_min=None, p_max=None, seed=0, grid=None):
        """A constant ("constant"), Perlin-noise ("noise") or voxel-grid
        ("grid") medium inside a sphere (center, radius) or an axis-aligned box
        (p_min, p_max).  The noise medium's Perlin tables are drawn from `seed`
        (the reference draws them from the thread RNG, perlin.rs:22-33).  A grid
        medium (box only; no reference counterpart) takes `grid` as a (nz, ny,
        nx) array: σ_t = density × the trilinear interpolation of its values."""
        m = abi.RtMedium()
        m.type = {"constant": abi.RT_MEDIUM_CONSTANT, "noise": abi.RT_MEDIUM_NOISE, "grid": abi.RT_MEDIUM_GRID}[kind]
        if kind == "grid":
            if boundary != "box" or grid is None:
                raise ValueError("a grid medium needs a box boundary and a grid")
            gr = np.ascontiguousarray(np.asarray(grid, dtype=F32))
            if gr.ndim != 3:
                raise ValueError("grid must be a (nz, ny, nx) array")
            self._tex_keep.append(gr)
            m.grid = gr.ctypes.data
            m.grid_res[:] = [gr.shape[2], gr.shape[1], gr.shape[0]]
        m.boundary = {"sphere": abi.RT_BOUND_SPHERE, "box": abi.RT_BOUND_BOX}[boundary]
        if boundary == "sphere":
            m.center = _f3(center)
            m.radius = float(radius)
        else:
            m.p_min = _f3(p_min)
            m.p_max = _f3(p_max)
        m.density = float(density)
        m.color = _f3(color)
        m.g = float(g)
        m.noise_scale = float(noise_scale)
        m.threshold = float(threshold)
        vec, perm = perlin_tables(seed)
        m.perlin_vec[:] = [float(x) for x in vec.reshape(-1)]
        m.perlin_perm[:] = [int(x) for x in perm.reshape(-1)]
        self.media.append(m)
        return len(self.media) - 1

    # analytic convex solids (diamond.rs:198-253) ----------------------
    def add_convex(self, planes, mat, box_lo, box_hi, polish=0.0, scale=1.0, rot=None, pivot=(0.0, 0.0, 0.0),
                   translate=(0.0, 0.0, 0.0)):
        """A convex polyhedron given by object-space outward half-spaces
        (n.xyz, d), interior n·x ≤ d, and an object-space box that contains it,
        placed at x_world = rot·(scale·x − pivot) + pivot + translate."""
        pl = np.ascontiguousarray(np.asarray(planes, dtype=F32).reshape(-1, 4))
        R = np.eye(3) if rot is None else np.asarray(rot, dtype=np.float64).reshape(3, 3)
        self.convex.append(dict(planes=pl, mat=mat, polish=float(polish), lo=tuple(map(float, box_lo)),
                                hi=tuple(map(float, box_hi)), scale=float(scale), rot=R,
                                pivot=tuple(map(float, pivot)), translate=tuple(map(float, translate))))
        return len(self.convex) - 1

    def add_diamond(self, center, radius, mat, table_pct=53.0, crown_angle=34.5, pavilion_angle=40.75, polish=0.0,
                    oval_ratio=1.0, girdle_facets=16, girdle_finish="uniform", girdle_pct=2.0, scale=1.0,
                    rotate=None, pivot=None, translate=(0.0, 0.0, 0.0)):
        """Diamond::new (diamond.rs:93-195): the round/oval brilliant's
        half-spaces, placed as the scene file does (scene_file.rs:924-930,
        1036-1042): a uniform scale about the origin, an Euler rotation in
        degrees about `pivot` (the gem's own center when None), then a
        translation."""
        planes, lo, hi = diamond_planes(center, radius, table_pct, crown_angle, pavilion_angle, oval_ratio,
                                        girdle_facets, girdle_finish, girdle_pct)
        pol = min(max(polish, 0.0), 0.25) if math.isfinite(polish) else 0.0       # diamond.rs:193
        ang = [0.0, 0.0, 0.0] if rotate is None else [float(a) for a in rotate]
        R = _euler_fwd(ang) if any(a != 0.0 for a in ang) else np.eye(3)
        return self.add_convex(planes, mat, lo, hi, polish=pol, scale=scale, rot=R,
                               pivot=center if pivot is None else pivot, translate=translate)

    def add_step_cut(self, center, half_a, half_b, mat, polish=0.0, scale=1.0, rotate=None, pivot=None,
                     translate=(0.0, 0.0, 0.0), **params):
        """StepCut::new (step_cut.rs:232-392): a step-family cut with semi-length
        `half_a` along x and semi-width `half_b` along z, placed like
        `add_diamond`; `params` are step_cut_planes' proportions."""
        planes, lo, hi = step_cut_planes(center, half_a, half_b, **params)
        pol = min(max(polish, 0.0), 0.25) if math.isfinite(polish) else 0.0       # step_cut.rs:390
        ang = [0.0, 0.0, 0.0] if rotate is None else [float(a) for a in rotate]
        R = _euler_fwd(ang) if any(a != 0.0 for a in ang) else np.eye(3)
        return self.add_convex(planes, mat, lo, hi, polish=pol, scale=scale, rot=R,
                               pivot=center if pivot is None else pivot, translate=translate)

    def add_texture_image(self, rgb8):
        """An 8-bit RGB image texture (H, W, 3), row 0 = top; returns its 1-based id."""
        img = np.ascontiguousarray(np.asarray(rgb8, np.uint8)[..., :3])
        t = abi.RtTexture()
        t.type, t.height, t.width = abi.RT_TEX_IMAGE, img.shape[0], img.shape[1]
        t.rgb8 = img.ctypes.data_as(C.POINTER(C.c_uint8))
        self._tex_keep.append(img)
        self.textures.append(t)
        return len(self.textures)

    def add_texture_mottle(self, lo, hi, scale=3.0, seed=0x5EED):
        """Texture::Mottle (texture.rs:52-55) with seeded Perlin tables; returns its 1-based id."""
        t = abi.RtTexture()
        t.type, t.scale = abi.RT_TEX_MOTTLE, float(scale)
        t.lo, t.hi = _f3(lo), _f3(hi)
        vec, perm = perlin_tables(seed)
        t.perlin_vec = (C.c_float * 768)(*vec.reshape(-1).tolist())
        t.perlin_perm = (C.c_int32 * 768)(*perm.reshape(-1).tolist())
        self.textures.append(t)
        return len(self.textures)

    def add_shape(self, kind, mat, center, radius=0.0, height=0.0, normal=(0.0, 1.0, 0.0), wave_amplitude=0.0,
                  wave_scale=1.0, xf=None):
        """Cylinder / Cone / Disk / InfinitePlane (cylinder.rs, cone.rs, disk.rs,
        plane.rs) in object space, placed by the objects' SRT transform."""
        kinds = {"cylinder": abi.RT_SHAPE_CYLINDER, "cone": abi.RT_SHAPE_CONE, "disk": abi.RT_SHAPE_DISK,
                 "infinite_plane": abi.RT_SHAPE_PLANE}
        r = abi.RtShape()
        r.type, r.mat = kinds[kind], mat
        r.center, r.normal = _f3(center), _f3(normal)
        r.radius, r.height = float(radius), float(height)
        r.wave_amplitude, r.wave_scale = float(wave_amplitude), float(wave_scale)
        xf = xf or Transform()
        r.scale = xf.scale
        r.rot = (C.c_float * 9)(*[float(v) for v in np.asarray(xf.R, np.float64).reshape(-1)])
        r.translate = _f3(xf.t)
        self.shapes.append(r)
        return len(self.shapes) - 1

    def add_quad(self, corner, u, v, mat, xf=None):
        q, uu, vv = (np.asarray(a, dtype=np.float64) for a in (corner, u, v))
        if xf is not None and not xf.identity:
            q, uu, vv = xf.point(q), xf.vector(uu), xf.vector(vv)
        self.quads.append((q.astype(F32), uu.astype(F32), vv.astype(F32), mat))
        return len(self.quads) - 1

    def add_box(self, p0, p1, mat, xf=None):
        """make_box (quad.rs:201-215): six quads."""
        p0, p1 = np.asarray(p0, dtype=F32), np.asarray(p1, dtype=F32)
        mn, mx = np.minimum(p0, p1), np.maximum(p0, p1)
        dx = np.array([mx[0] - mn[0], 0, 0], dtype=F32)
        dy = np.array([0, mx[1] - mn[1], 0], dtype=F32)
        dz = np.array([0, 0, mx[2] - mn[2]], dtype=F32)
        self.add_quad([mn[0], mn[1], mx[2]], dx, dy, mat, xf)
        self.add_quad([mx[0], mn[1], mx[2]], -dz, dy, mat, xf)
        self.add_quad([mx[0], mn[1], mn[2]], -dx, dy, mat, xf)
        self.add_quad([mn[0], mn[1], mn[2]], dz, dy, mat, xf)
        self.add_quad([mn[0], mx[1], mx[2]], dx, -dz, mat, xf)
        self.add_quad([mn[0], mn[1], mn[2]], dx, dz, mat, xf)

    def add_mesh(self, verts, faces, mat, vnormals=None, xf=None, uvs=None):
        """Indexed triangle mesh; vertex normals are normalised at load with a
        face-normal fallback (mesh.rs:68-73); zero-area faces are skipped.
        `uvs` (per vertex) also give per-vertex tangents from the UV-space
        derivatives (mesh.rs:33-54)."""
        V = np.asarray(verts, dtype=np.float64)
        Fi = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
        tan = None
        if uvs is not None:
            tan = mesh_tangents(V.astype(F32), Fi, np.asarray(uvs, F32))
        if xf is not None and not xf.identity:
            V = xf.point(V)
        Vf = V.astype(F32)
        v0, v1, v2 = Vf[Fi[:, 0]], Vf[Fi[:, 1]], Vf[Fi[:, 2]]
        fn_raw = np.cross((v1 - v0).astype(F32), (v2 - v0).astype(F32))
        l2 = (fn_raw.astype(np.float64) ** 2).sum(1)
        keep = l2 >= 1e-16
        Fi, v0, v1, v2, fn_raw, l2 = Fi[keep], v0[keep], v1[keep], v2[keep], fn_raw[keep], l2[keep]
        tv = np.concatenate([v0, v1, v2], axis=1).astype(F32)
        tn = None
        if vnormals is not None:
            N = np.asarray(vnormals, dtype=np.float64)
            if xf is not None and not xf.identity:
                N = xf.normal(N)
            face_n = fn_raw / np.sqrt(l2)[:, None]
            cols = []
            for k in range(3):
                nk = N[Fi[:, k]]
                ln = (nk ** 2).sum(1)
                ok = ln > 1e-12
                nk = np.where(ok[:, None], nk / np.sqrt(np.where(ok, ln, 1.0))[:, None], face_n)
                cols.append(nk)
            tn = np.concatenate(cols, axis=1).astype(F32)
        self.tri_v.append(np.ascontiguousarray(tv))
        self.tri_n.append(tn)
        self.tri_mat.append(np.full(len(tv), mat, dtype=np.int32))
        if uvs is not None:
            UV = np.asarray(uvs, F32)
            self.tri_uv.append(np.concatenate([UV[Fi[:, k]] for k in range(3)], axis=1).astype(F32))
            T = tan if xf is None or xf.identity else xf.vector(tan.astype(np.float64)).astype(F32)
            self.tri_tan.append(np.concatenate([T[Fi[:, k]] for k in range(3)], axis=1).astype(F32))
        else:
            self.tri_uv.append(None)
            self.tri_tan.append(None)
        return len(tv)

    def add_light_quad(self, corner, u, v, mat):
        """[[lights]] entry: the quad joins the world and the NEE list."""
        qi = self.add_quad(corner, u, v, mat)
        self._lights.append(("quad", qi))
        return qi

    def add_light_sphere(self, center, radius, mat):
        si = self.add_sphere(center, radius, mat)
        self._lights.append(("sphere", si))
        return si

    # background --------------------------------------------------------
    def set_physical(self, sun_azimuth=0.0, sun_elevation=30.0, turbidity=3.0):
        """Background::Physical from the TOML angles (scene_file.rs:917-927): the sun
        direction (cos el · sin az, sin el, cos el · cos az), normalised."""
        el, az = math.radians(sun_elevation), math.radians(sun_azimuth)
        d = np.array([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)], np.float32)
        d = d / np.float32(np.linalg.norm(d))
        self.bg = {"type": abi.RT_BG_PHYSICAL, "sun_dir": tuple(float(x) for x in d), "turbidity": float(turbidity)}

    def set_solid(self, color):
        self.bg = {"type": abi.RT_BG_SOLID, "color": tuple(color)}

    def set_gradient(self, top, bottom):
        self.bg = {"type": abi.RT_BG_GRADIENT, "top": tuple(top), "bottom": tuple(bottom)}

    def set_env(self, rgb, rotate_y=0.0, visible=None):
        """rgb: (H, W, 3) float32 equirect, row 0 = +Y.  visible: None or a dict
        {'type': 'solid', 'color': ...} / {'type': 'gradient', 'top':..., 'bottom':...}."""
        self.env = np.ascontiguousarray(np.asarray(rgb, dtype=F32))
        self.bg = {"type": abi.RT_BG_ENVMAP, "rot": float(rotate_y), "visible": visible}

    # emission ----------------------------------------------------------
    @property
    def n_tris(self):
        return int(sum(len(t) for t in self.tri_v))

    def light_prim_ids(self):
        nt, nq = self.n_tris, len(self.quads)
        out = []
        for kind, i in self._lights:
            out.append(nt + i if kind == "quad" else nt + nq + i)
        return np.asarray(out, dtype=np.int32)

    def desc(self):
        """Build the RtSceneDesc; the arrays are cached on self to keep them alive."""
        nt = self.n_tris
        if nt:
            self._tv = np.ascontiguousarray(np.concatenate(self.tri_v).astype(F32))
            if all(n is not None for n in self.tri_n):
                self._tn = np.ascontiguousarray(np.concatenate(self.tri_n).astype(F32))
            elif any(n is not None for n in self.tri_n):
                parts = []
                for v, n in zip(self.tri_v, self.tri_n):
                    if n is None:
                        e1 = v[:, 3:6] - v[:, 0:3]
                        e2 = v[:, 6:9] - v[:, 0:3]
                        fn = np.cross(e1, e2)
                        fn = fn / np.linalg.norm(fn, axis=1, keepdims=True)
                        n = np.concatenate([fn, fn, fn], axis=1)
                    parts.append(n.astype(F32))
                self._tn = np.ascontiguousarray(np.concatenate(parts))
            else:
                self._tn = None
            self._tm = np.ascontiguousarray(np.concatenate(self.tri_mat).astype(np.int32))
            if any(u is not None for u in self.tri_uv):
                # mesh.rs:75-81: without texcoords the corners get (0,0) (1,0) (0.5,1), tangents (1,0,0)
                duv = np.array([0, 0, 1, 0, 0.5, 1], F32)
                dtan = np.array([1, 0, 0] * 3, F32)
                self._tuv = np.ascontiguousarray(np.concatenate(
                    [u if u is not None else np.tile(duv, (len(v), 1)) for u, v in zip(self.tri_uv, self.tri_v)]))
                self._ttan = np.ascontiguousarray(np.concatenate(
                    [t if t is not None else np.tile(dtan, (len(v), 1)) for t, v in zip(self.tri_tan, self.tri_v)]))
            else:
                self._tuv = self._ttan = None
        else:
            self._tuv = self._ttan = None
            self._tv = np.zeros((0, 9), F32)
            self._tn = None
            self._tm = np.zeros(0, np.int32)
        if self.quads:
            self._qv = np.ascontiguousarray(np.array([np.concatenate([q, u, v]) for q, u, v, _ in self.quads], dtype=F32))
            self._qm = np.array([m for *_, m in self.quads], dtype=np.int32)
        else:
            self._qv = np.zeros((0, 9), F32)
            self._qm = np.zeros(0, np.int32)
        if self.spheres:
            self._sv = np.ascontiguousarray(np.array([[c[0], c[1], c[2], r] for c, r, _ in self.spheres], dtype=F32))
            self._sm = np.array([m for *_, m in self.spheres], dtype=np.int32)
        else:
            self._sv = np.zeros((0, 4), F32)
            self._sm = np.zeros(0, np.int32)
        self._mats = (abi.RtMaterial * max(1, len(self.materials)))(*self.materials)
        self._lp = self.light_prim_ids()
        d = abi.RtSceneDesc()
        d.bvh_builder = getattr(self, "bvh_builder", abi.RT_BVH_DEVICE)
        d.n_tris = nt
        d.tri_v = abi.fptr(self._tv)
        d.tri_n = abi.fptr(self._tn)
        d.tri_mat = abi.iptr(self._tm)
        d.n_quads = len(self.quads)
        d.quad_quv = abi.fptr(self._qv)
        d.quad_mat = abi.iptr(self._qm)
        d.n_spheres = len(self.spheres)
        d.sphere = abi.fptr(self._sv)
        d.sphere_mat = abi.iptr(self._sm)
        d.n_mats = len(self.materials)
        d.mats = C.cast(self._mats, C.POINTER(abi.RtMaterial))
        d.n_lights = len(self._lp)
        d.light_prims = abi.iptr(self._lp)
        bg = abi.RtBackground()
        bg.type = self.bg["type"]
        bg.visible_type = -1
        if bg.type == abi.RT_BG_SOLID:
            bg.color = _f3(self.bg["color"])
        elif bg.type == abi.RT_BG_PHYSICAL:
            bg.sun_dir = _f3(self.bg["sun_dir"])
            bg.turbidity = self.bg["turbidity"]
        elif bg.type == abi.RT_BG_GRADIENT:
            bg.top = _f3(self.bg["top"])
            bg.bottom = _f3(self.bg["bottom"])
        else:
            h, w, _ = self.env.shape
            bg.env_w, bg.env_h = w, h
            bg.env_rgb = abi.fptr(self.env)
            bg.env_rot_y_deg = self.bg["rot"]
            vis = self.bg.get("visible")
            if vis:
                if vis["type"] == "solid":
                    bg.visible_type = abi.RT_BG_SOLID
                    bg.visible_color = _f3(vis["color"])
                else:
                    bg.visible_type = abi.RT_BG_GRADIENT
                    bg.visible_top = _f3(vis["top"])
                    bg.visible_bottom = _f3(vis["bottom"])
        d.bg = bg
        d.spectral_range = int(self.spectral_range)
        if self.convex:
            offs, recs = 0, []
            for c in self.convex:
                r = abi.RtConvex()
                r.plane_offset, r.n_planes, r.mat, r.polish = offs, len(c["planes"]), c["mat"], c["polish"]
                r.box_lo, r.box_hi = _f3(c["lo"]), _f3(c["hi"])
                r.scale = c["scale"]
                r.rot = (C.c_float * 9)(*[float(v) for v in c["rot"].reshape(-1)])
                r.pivot, r.translate = _f3(c["pivot"]), _f3(c["translate"])
                recs.append(r)
                offs += len(c["planes"])
            self._cvx = (abi.RtConvex * len(recs))(*recs)
            self._cvp = np.ascontiguousarray(np.concatenate([c["planes"] for c in self.convex]).astype(F32))
            d.n_convex = len(recs)
            d.convex = C.cast(self._cvx, C.POINTER(abi.RtConvex))
            d.convex_planes = abi.fptr(self._cvp)
        if self._tuv is not None:
            d.tri_uv = abi.fptr(self._tuv)
            d.tri_tangent = abi.fptr(self._ttan)
        if self.textures:
            self._texs = (abi.RtTexture * len(self.textures))(*self.textures)
            d.n_textures = len(self.textures)
            d.textures = C.cast(self._texs, C.POINTER(abi.RtTexture))
        if self.shapes:
            self._shapes = (abi.RtShape * len(self.shapes))(*self.shapes)
            d.n_shapes = len(self.shapes)
            d.shapes = C.cast(self._shapes, C.POINTER(abi.RtShape))
        self._media = (abi.RtMedium * max(1, len(self.media)))(*self.media)
        d.n_media = len(self.media)
        d.media = C.cast(self._media, C.POINTER(abi.RtMedium)) if self.media else None
        self._desc = d
        return d


# ── camera (camera.rs:24-45) ────────────────────────────────────────────────
def make_camera(look_from, look_at, vup=(0.0, 1.0, 0.0), vfov=40.0, aspect=1.0,
                aperture=0.0, focus_dist=None, aperture_blades=0):
    """Camera::new in f32 arithmetic; returns an RtCamera."""
    f = lambda x: np.asarray(x, dtype=F32)
    lf, la, up = f(look_from), f(look_at), f(vup)
    if focus_dist is None:
        focus_dist = max(float(np.linalg.norm((lf - la).astype(np.float64))), 0.01)
    fd = F32(focus_dist)
    h = F32(math.tan(float(F32(vfov) * F32(math.pi / 180.0)) / 2.0))
    vh = F32(2.0) * h
    vw = F32(aspect) * vh

    def unit(a):
        return (a / F32(np.sqrt(F32((a * a).sum())))).astype(F32)

    w = unit((lf - la).astype(F32))
    u = unit(np.cross(up, w).astype(F32))
    v = np.cross(w, u).astype(F32)
    horizontal = (fd * vw * u).astype(F32)
    vertical = (fd * vh * v).astype(F32)
    lower_left = (lf - horizontal / F32(2) - vertical / F32(2) - fd * w).astype(F32)
    cam = abi.RtCamera()
    cam.origin = _f3(lf)
    cam.lower_left = _f3(lower_left)
    cam.horizontal = _f3(horizontal)
    cam.vertical = _f3(vertical)
    cam.u = _f3(u)
    cam.v = _f3(v)
    cam.lens_radius = float(F32(aperture) / F32(2))
    cam.aperture_blades = int(aperture_blades)         # ≥ 3: polygonal aperture (camera.rs:48-50)
    return cam


# ── OBJ + HDR readers ────────────────────────────────────────────────────────
def mesh_tangents(V, F, UV):
    """Per-vertex tangents from UV-space derivatives, summed over the faces and
    normalised with a (1, 0, 0) fallback (mesh.rs:33-54), in f32."""
    f = np.float32
    acc = np.zeros((len(V), 3), f)
    for i0, i1, i2 in F:
        e1, e2 = (V[i1] - V[i0]).astype(f), (V[i2] - V[i0]).astype(f)
        du1, dv1 = UV[i1, 0] - UV[i0, 0], UV[i1, 1] - UV[i0, 1]
        du2, dv2 = UV[i2, 0] - UV[i0, 0], UV[i2, 1] - UV[i0, 1]
        den = f(du1 * dv2 - dv1 * du2)
        if abs(den) < f(1e-8):
            continue
        t = (e1 * dv2 - e2 * dv1) * (f(1.0) / den)
        acc[i0] += t
        acc[i1] += t
        acc[i2] += t
    l2 = (acc * acc).sum(1)
    ok = l2 > f(1e-8)
    out = np.tile(np.array([1, 0, 0], f), (len(V), 1))
    out[ok] = acc[ok] / np.sqrt(l2[ok])[:, None]
    return out


def load_obj(path, with_uv=False):
    """Minimal Wavefront OBJ reader: positions, optional normals, polygon faces
    fan-triangulated with a single index per corner (the effect of tobj's
    GPU_LOAD_OPTIONS in mesh.rs:14).  Returns (verts, faces, vnormals|None)."""
    vs, vn, vt, faces, fnorm, ftex = [], [], [], [], [], []
    with open(path) as fh:
        for line in fh:
            if line.startswith("v "):
                vs.append([float(x) for x in line.split()[1:4]])
            elif line.startswith("vn "):
                vn.append([float(x) for x in line.split()[1:4]])
            elif line.startswith("vt "):
                vt.append([float(x) for x in line.split()[1:3]])
            elif line.startswith("f "):
                idx, nidx, tidx = [], [], []
                for tok in line.split()[1:]:
                    parts = tok.split("/")
                    i = int(parts[0])
                    idx.append(i - 1 if i > 0 else len(vs) + i)
                    if len(parts) >= 2 and parts[1]:
                        j = int(parts[1])
                        tidx.append(j - 1 if j > 0 else len(vt) + j)
                    if len(parts) >= 3 and parts[2]:
                        j = int(parts[2])
                        nidx.append(j - 1 if j > 0 else len(vn) + j)
                for k in range(1, len(idx) - 1):
                    faces.append([idx[0], idx[k], idx[k + 1]])
                    if len(nidx) == len(idx):
                        fnorm.append([nidx[0], nidx[k], nidx[k + 1]])
                    if len(tidx) == len(idx):
                        ftex.append([tidx[0], tidx[k], tidx[k + 1]])
    V = np.asarray(vs, dtype=np.float64)
    Fa = np.asarray(faces, dtype=np.int64)
    has_n = bool(vn) and len(fnorm) == len(faces)
    has_t = with_uv and bool(vt) and len(ftex) == len(faces)
    if has_n or has_t:
        # single-index vertices: one per distinct (position, uv, normal) triple
        # of the corners, as tobj's GPU_LOAD_OPTIONS builds them (mesh.rs:14)
        Fn = np.asarray(fnorm, np.int64) if has_n else np.zeros_like(Fa)
        Ft = np.asarray(ftex, np.int64) if has_t else np.zeros_like(Fa)
        key = np.stack([Fa.reshape(-1), Ft.reshape(-1), Fn.reshape(-1)], 1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        V2 = V[uniq[:, 0]]
        N2 = np.asarray(vn, np.float64)[uniq[:, 2]] if has_n else None
        out = (V2, inv.reshape(-1, 3), N2)
        if with_uv:
            return out + ((np.asarray(vt, np.float64)[uniq[:, 1]] if has_t else None),)
        return out
    return (V, Fa, None, None) if with_uv else (V, Fa, None)


def load_hdr(path):
    """Radiance RGBE (.hdr) reader with new-style RLE; returns (H, W, 3) float32."""
    with open(path, "rb") as fh:
        data = fh.read()
    pos = 0
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end]
        pos = end + 1
        if line.strip() == b"":
            break
    end = data.index(b"\n", pos)
    dims = data[pos:end].split()
    pos = end + 1
    H, W = int(dims[1]), int(dims[3])
    # the scanline decoder is native (rt_rgbe_decode in librtb200.so)
    from .renderer import lib
    out = np.zeros((H, W, 3), F32)
    body = np.frombuffer(data, np.uint8)[pos:]
    rc = lib().rt_rgbe_decode(body.ctypes.data_as(C.POINTER(C.c_uint8)), C.c_size_t(len(body)), W, H,
                              out.ctypes.data_as(C.POINTER(C.c_float)))
    if rc != 0:
        raise ValueError(f"{path}: corrupt RGBE scanlines")
    return out


# ── TOML loader (scene_file.rs:621-1216, the subset the GPU path supports) ───
def load_texture(path):
    """An image file as (H, W, 3) uint8 RGB (texture.rs:21-23): PNG, or a
    Radiance .hdr clamped to [0, 1] and quantised."""
    if path.lower().endswith(".hdr"):
        return (np.clip(load_hdr(path), 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)
    from .output import read_png
    return read_png(path)


def _material_from_toml(m, base, sb):
    t = m["type"]
    if t == "lambertian":
        return Material.lambertian(m["color"])
    if t == "checker":
        return Material.checker(m["even"], m["odd"], m.get("scale", 1.0))
    if t == "dielectric":
        return Material.dielectric(m["ior"])
    if t == "spectral_dielectric":
        return Material.spectral_dielectric(m["ior"], m.get("dispersion", 0.0), m.get("absorption", (0, 0, 0)))
    if t == "spectral_metal":
        if "n" in m and "k" in m:
            return Material.spectral_metal_nk(m.get("lambda_start", 380.0), m.get("lambda_step", 25.0),
                                              m["n"], m["k"], m.get("roughness", 0.0))
        return Material.spectral_metal(m.get("variant", "gold"), m.get("roughness", 0.0))
    if t == "diffuse_light":
        return Material.diffuse_light(m["color"])
    if t == "image":                                                 # scene_file.rs:1152-1153
        mat = Material.lambertian((0.0, 0.0, 0.0))
        mat.albedo_tex = sb.add_texture_image(load_texture(_resolve(base, m["path"])))
        return mat
    if t == "noise":                                                 # scene_file.rs:1149-1150: Texture::Mottle
        mat = Material.lambertian((0.0, 0.0, 0.0))
        mat.albedo_tex = sb.add_texture_mottle(m["lo"], m["hi"], m.get("scale", 3.0))
        return mat
    if t == "metal":                                                 # scene_file.rs:1155-1156
        return Material.pbr(m["color"], roughness=m.get("fuzz", 0.0), metallic=1.0)
    if t == "textured_pbr":                                          # scene_file.rs:1189-1199
        mat = Material.pbr(roughness=m.get("roughness", 0.5), metallic=m.get("metallic", 0.0))
        mat.albedo_tex = sb.add_texture_image(load_texture(_resolve(base, m["albedo_path"])))
        for key, field in (("roughness_path", "roughness_tex"), ("metallic_path", "metallic_tex"),
                           ("ao_path", "ao_tex"), ("normal_path", "normal_tex")):
            if m.get(key):
                setattr(mat, field, sb.add_texture_image(load_texture(_resolve(base, m[key]))))
        return mat
    if t == "pbr":                                                   # scene_file.rs:380-406, 1179-1187
        return Material.pbr(m["albedo"], m.get("roughness", 0.5), m.get("metallic", 0.0), m.get("anisotropy", 0.0),
                            m.get("anisotropy_angle", 0.0), m.get("clearcoat", 0.0),
                            m.get("clearcoat_roughness", 0.03), m.get("film_thickness", 0.0),
                            m.get("film_ior", 1.5), m.get("sheen", 0.0), m.get("sheen_tint", 0.5),
                            m.get("emission", (0.0, 0.0, 0.0)), m.get("emission_strength", 0.0))
    raise ValueError(f"material type '{t}' is not supported by the GPU path")


def load_toml(path):
    """Parse a scene TOML (the reference's schema, scene_file.rs:31-601) into a
    SceneBuilder.  Raises ValueError for fields the GPU path does not support."""
    import tomllib
    with open(path, "rb") as fh:
        doc = tomllib.load(fh)
    return scene_from_toml_dict(doc, os.path.dirname(os.path.abspath(path)))


def _resolve(base, p):
    cand = os.path.join(base, p)
    return cand if os.path.exists(cand) else p


def diamond_planes(center, radius, table_pct=53.0, crown_angle=34.5, pavilion_angle=40.75, oval_ratio=1.0,
                   girdle_facets=16, girdle_finish="uniform", girdle_pct=2.0):
    """The half-spaces and bounding box of Diamond::new (diamond.rs:93-195), in
    f32: the table, a crown and a pavilion facet through every girdle edge
    (every other one with a knife-edge girdle), and the band's vertical planes
    (the girdle n-gon when faceted, a 64-gon shell otherwise)."""
    f = np.float32
    cx, cy, cz = (f(c) for c in center)
    r, q = f(radius), f(max(oval_ratio, 0.05))
    table_r = f(table_pct / 100.0) * r
    crown_h = (r - table_r) * f(math.tan(math.radians(crown_angle)))
    pav_h = r * f(math.tan(math.radians(pavilion_angle)))
    girdle_h = f(min(max(girdle_pct / 100.0 * 2.0 * float(r), 0.0), 0.3 * float(r)))
    n = (max(int(girdle_facets), 4) // 2) * 2
    m = n // 2
    band_m = n if girdle_finish == "faceted" else 64
    planes = []

    def unit(v):
        v = np.asarray(v, f)
        return (v / f(math.sqrt(float(v @ v)))).astype(f)

    def push(nv, g):
        # the oval is the round stone stretched by q along x ABOUT ITS CENTER;
        # the reference stretches about the origin (q·g.x), which moves an
        # off-axis oval away from its own bounding box — the one deliberate
        # difference; round stones (q = 1) and ovals at x = 0 are unchanged
        nw = unit([f(nv[0]) / q, f(nv[1]), f(nv[2])])
        gx = f(g[0]) if q == f(1.0) else cx + q * (f(g[0]) - cx)
        gw = np.array([gx, f(g[1]), f(g[2])], f)
        planes.append([nw[0], nw[1], nw[2], f(nw @ gw)])

    push((0.0, 1.0, 0.0), (cx, cy + f(0.5) * girdle_h + crown_h, cz))
    wavy = girdle_h > 0 and girdle_finish == "faceted"
    band_h = lambda k: f(0.0) if (wavy and k % 2 == 1) else girdle_h
    crown_n = n if girdle_h > 0 else m
    for k in range(crown_n):
        th = f(k) * f(2.0 * math.pi) / f(crown_n)
        sn, c = f(math.sin(th)), f(math.cos(th))
        push(unit([c * crown_h, r - table_r, sn * crown_h]), (cx + c * r, cy + f(0.5) * band_h(k), cz + sn * r))
    pav_n = n if girdle_h > 0 else m
    for k in range(pav_n):
        ph = f(k) * f(2.0 * math.pi) / f(n) if girdle_h > 0 else f(k) * f(2.0 * math.pi) / f(m) + f(math.pi) / f(m)
        sn, c = f(math.sin(ph)), f(math.cos(ph))
        push(unit([c * pav_h, -r, sn * pav_h]), (cx + c * r, cy - f(0.5) * band_h(k), cz + sn * r))
    if girdle_h > 0:
        for j in range(band_m):
            a = f(j) * f(2.0 * math.pi) / f(band_m)
            sn, c = f(math.sin(a)), f(math.cos(a))
            push((c, 0.0, sn), (cx + c * r, cy, cz + sn * r))
    P = np.array(planes, f)
    if girdle_h > 0:
        circ_r = r / f(math.cos(math.pi / band_m))
        lo = (cx - circ_r * q, cy - (f(0.5) * girdle_h + pav_h), cz - circ_r)
        hi = (cx + circ_r * q, cy + (f(0.5) * girdle_h + crown_h), cz + circ_r)
    else:
        from scipy.spatial import HalfspaceIntersection
        hs = np.concatenate([P[:, :3].astype(np.float64), -P[:, 3:4].astype(np.float64)], 1)
        V = HalfspaceIntersection(hs, np.array([cx, cy, cz], np.float64)).intersections
        lo, hi = tuple(V.min(0) - 1e-4), tuple(V.max(0) + 1e-4)
    return P, lo, hi


def _f32_rad(deg):
    return np.float32(deg) * np.float32(np.float32(math.pi) / np.float32(180.0))


def step_outline_vertices(outline, a, b):
    """StepOutline::vertices (step_cut.rs:38-108): the girdle outline in XZ
    relative to the centre, sorted by angle about the vertex centroid.
    `outline` is ("rect", corner_pct) | ("rounded_rect", corner_pct, segs) |
    ("triangle",) | ("hexagon",) | ("pointed_oval", segs, pear) |
    ("polygon", [[x, z], ...])."""
    f = np.float32
    a, b = f(a), f(b)
    kind = outline[0]
    if kind == "rect":
        c = min(f(outline[1]) / f(100.0) * min(a, b), f(0.45) * min(a, b))
        if c <= f(1e-6):
            v = [(a, b), (a, -b), (-a, -b), (-a, b)]
        else:
            v = [(a - c, b), (a, b - c), (a, -(b - c)), (a - c, -b), (-(a - c), -b), (-a, -(b - c)), (-a, b - c),
                 (-(a - c), b)]
    elif kind == "rounded_rect":
        r = min(f(outline[1]) / f(100.0) * min(a, b), f(0.45) * min(a, b))
        segs = max(int(outline[2]), 1)
        v = []
        for sx in (f(1.0), f(-1.0)):
            for sz in (f(1.0), f(-1.0)):
                ccx, ccz = sx * (a - r), sz * (b - r)
                for j in range(segs + 1):
                    ang = f(j) / f(segs) * f(math.pi / 2)
                    v.append((ccx + sx * r * f(math.cos(ang)), ccz + sz * r * f(math.sin(ang))))
    elif kind == "triangle":
        v = []
        for k in range(3):
            th = f(math.pi / 2) + f(k) * f(2.0) * f(math.pi) / f(3.0)
            v.append((a * f(math.cos(th)), b * f(math.sin(th))))
    elif kind == "hexagon":
        v = []
        for k in range(6):
            th = f(k) * f(math.pi) / f(3.0)
            v.append((a * f(math.cos(th)), b * f(math.sin(th))))
    elif kind == "pointed_oval":
        segs, pear = int(outline[1]), bool(outline[2])
        n = max(segs, 4) * 2
        v = []
        for i in range(n):
            th = f(2.0) * f(math.pi) * f(i) / f(n)
            c, sn = f(math.cos(th)), f(math.sin(th))
            pw = (f(0.6) if c >= 0 else f(1.0)) if pear else f(0.65)
            sg = f(1.0) if c > 0 or (c == 0 and math.copysign(1.0, c) > 0) else f(-1.0)
            v.append((a * sg * f(abs(float(c)) ** float(pw)), b * sn))
    elif kind == "polygon":
        v = [(f(x), f(z)) for x, z in outline[1]]
    else:
        raise ValueError(f"unknown step outline '{kind}'")
    n = f(len(v))
    cx = f(0.0)
    for p in v:
        cx = cx + p[0]
    cz = f(0.0)
    for p in v:
        cz = cz + p[1]
    cx, cz = cx / n, cz / n
    return sorted(v, key=lambda p: f(math.atan2(float(p[1] - cz), float(p[0] - cx))))


def _validate_outline(v, scale):
    """validate_outline (step_cut.rs:183-225): dedupe adjacent vertices, then
    at least 3 distinct vertices, no zero edge, non-zero area, convex."""
    f = np.float32
    eps = f(1e-6) * f(scale)
    hyp = lambda p, q: f(math.hypot(float(p[0] - q[0]), float(p[1] - q[1])))
    out = []
    for p in v:
        if out and hyp(p, out[-1]) < eps:
            continue
        out.append(p)
    if len(out) > 1 and hyp(out[0], out[-1]) < eps:
        out.pop()
    n = len(out)
    if n < 3:
        raise ValueError("outline needs at least 3 distinct vertices")
    for i in range(n):
        if hyp(out[i], out[(i + 1) % n]) < eps:
            raise ValueError("outline has a zero-length edge")
    area2 = f(0.0)
    for i in range(n):
        p, q = out[i], out[(i + 1) % n]
        area2 = area2 + (p[0] * q[1] - q[0] * p[1])
    if abs(area2) < eps * eps:
        raise ValueError("outline has zero area")
    for i in range(n):
        p, q, r = out[i], out[(i + 1) % n], out[(i + 2) % n]
        cross = (q[0] - p[0]) * (r[1] - q[1]) - (q[1] - p[1]) * (r[0] - q[0])
        if cross * area2 < 0:
            raise ValueError("polygon outline must be convex")
    return out


def step_cut_planes(center, half_a, half_b, table_pct=65.0, crown_angle=35.0, pavilion_angle=42.0,
                    outline=("rect", 12.0), crown_steps=3, pavilion_steps=3, culet_pct=8.0, step_spread=0.25,
                    chevrons=0, girdle_pct=0.0):
    """The half-spaces and bounding box of StepCut::new (step_cut.rs:232-392),
    in f32: per outline edge an optional vertical girdle face, crown and
    pavilion rows whose runs are normalised so the table and culet insets are
    exact, chevron planes at the outline vertices, and the table/culet caps.
    Defaults are StepCutParams::default (step_cut.rs:147-163)."""
    f = np.float32
    if not (half_a > 0 and half_b > 0 and math.isfinite(half_a) and math.isfinite(half_b)):
        raise ValueError("StepCut: half extents must be positive and finite")
    cx, cy, cz = (f(c) for c in center)
    a, b = f(half_a), f(half_b)
    k = min(max(f(table_pct) / f(100.0), f(0.05)), f(0.95))
    kc = min(max(f(culet_pct) / f(100.0), f(0.0)), f(0.5))
    s_in, sp = b * (f(1.0) - k), b * (f(1.0) - kc)
    tan_c, tan_p = f(math.tan(float(_f32_rad(crown_angle)))), f(math.tan(float(_f32_rad(pavilion_angle))))
    crown_h, pav_h = s_in * tan_c, sp * tan_p
    gp = f(girdle_pct)
    girdle_h = min(max(gp / f(100.0) * f(2.0) * b, f(0.0)), f(0.3) * b)
    if not (math.isfinite(girdle_pct) and 0.0 <= girdle_pct < 100.0):
        raise ValueError(f"StepCut: girdle_pct must be in [0, 100), got {girdle_pct}")
    if not (crown_h > 0 and pav_h > 0):
        raise ValueError(f"StepCut: crown/pavilion angles must be in (0, 90) degrees, got {crown_angle} / {pavilion_angle}")
    verts = _validate_outline(step_outline_vertices(outline, a, b), max(a, b))
    nv = len(verts)
    gcx, gcz = f(0.0), f(0.0)
    for p in verts:
        gcx = gcx + p[0]
    for p in verts:
        gcz = gcz + p[1]
    gcx, gcz = gcx / f(nv), gcz / f(nv)

    def norm2(x, z):
        l = f(math.sqrt(float(x * x + z * z)))
        return (x / l, z / l) if l > f(1e-12) else (f(0.0), f(0.0))

    def unit(x, y, z):
        l = f(math.sqrt(float(x * x + y * y + z * z)))
        return (x / l, y / l, z / l)

    dot = lambda u, w: u[0] * w[0] + u[1] * w[1] + u[2] * w[2]
    edges = []
    for i in range(nv):
        p, q = verts[i], verts[(i + 1) % nv]
        m = norm2(q[1] - p[1], -(q[0] - p[0]))
        if m[0] * (p[0] - gcx) + m[1] * (p[1] - gcz) < 0:
            m = (-m[0], -m[1])
        edges.append((m, m[0] * p[0] + m[1] * p[1]))
    cs, ps = max(int(crown_steps), 1), max(int(pavilion_steps), 1)
    spread = min(max(f(step_spread), f(0.0)), f(0.9))
    factor = lambda i, rows: f(1.0) if rows <= 1 else f(1.0) + spread * (f(1.0) - f(2.0) * f(i) / f(rows - 1))
    dv, dvp = crown_h / f(cs), pav_h / f(ps)
    sum_c = f(0.0)
    for i in range(cs):
        sum_c = sum_c + dv / (tan_c * factor(i, cs))
    sum_p = f(0.0)
    for i in range(ps):
        sum_p = sum_p + dvp / (tan_p * factor(i, ps))
    norm_c, norm_p = s_in / sum_c, sp / sum_p
    planes = []
    for m, h in edges:
        if girdle_h > 0:
            planes.append((m[0], f(0.0), m[1], m[0] * cx + m[1] * cz + h))
        dist, y = h, f(0.5) * girdle_h
        for i in range(cs):
            dh = dv / (tan_c * factor(i, cs)) * norm_c
            n = unit(m[0] * dv, dh, m[1] * dv)
            planes.append(n + (dot(n, (cx + m[0] * dist, cy + y, cz + m[1] * dist)),))
            dist, y = dist - dh, y + dv
        dist, y = h, f(-0.5) * girdle_h
        for i in range(ps):
            dh = dvp / (tan_p * factor(i, ps)) * norm_p
            n = unit(m[0] * dvp, -dh, m[1] * dvp)
            planes.append(n + (dot(n, (cx + m[0] * dist, cy + y, cz + m[1] * dist)),))
            dist, y = dist - dh, y - dvp
    ctr = (cx, cy, cz)
    for i in range(nv):
        v, vp, vn = verts[i], verts[(i + nv - 1) % nv], verts[(i + 1) % nv]
        u1, u2 = norm2(vp[0] - v[0], vp[1] - v[1]), norm2(vn[0] - v[0], vn[1] - v[1])
        bis = (u1[0] + u2[0], u1[1] + u2[1])
        if bis[0] * bis[0] + bis[1] * bis[1] < f(1e-12):
            continue
        t = (-bis[1], bis[0])
        c3 = (cx + v[0], cy, cz + v[1])
        tc = (cx + v[0] * k, cy + f(0.5) * girdle_h + crown_h, cz + v[1] * k)
        cc = (cx + v[0] * kc, cy - f(0.5) * girdle_h - pav_h, cz + v[1] * kc)
        for j in range(int(chevrons)):
            fr = f(j + 1) / f(chevrons)
            for tgt in (tc, cc):
                pp = tuple(c3[a_] + (tgt[a_] - c3[a_]) * fr for a_ in range(3))
                w = (pp[0] - c3[0], pp[1] - c3[1], pp[2] - c3[2])
                # d3 × w with d3 = (t.x, 0, t.z)
                n = unit(f(0.0) * w[2] - t[1] * w[1], t[1] * w[0] - t[0] * w[2], t[0] * w[1] - f(0.0) * w[0])
                if dot(n, ctr) > dot(n, c3):
                    n = (-n[0], -n[1], -n[2])
                planes.append(n + (dot(n, c3),))
    planes.append((f(0.0), f(1.0), f(0.0), cy + f(0.5) * girdle_h + crown_h))
    planes.append((f(0.0), f(-1.0), f(0.0), -(cy - f(0.5) * girdle_h - pav_h)))
    xs, zs = [p[0] for p in verts], [p[1] for p in verts]
    top, bottom = f(0.5) * girdle_h + s_in * tan_c, f(0.5) * girdle_h + sp * tan_p
    lo = (float(cx + min(xs)), float(cy - bottom), float(cz + min(zs)))
    hi = (float(cx + max(xs)), float(cy + top), float(cz + max(zs)))
    return np.array(planes, f), lo, hi


# step-family presets for [[gems]] cut = "..." (scene_file.rs:738-766):
# outline, culet_pct, crown steps, pavilion steps, step spread, default chevrons
STEP_CUT_PRESETS = {
    "step": (("rect", 12.0), 8.0, 3, 3, 0.25, 0),
    "princess": (("rect", 0.0), 0.0, 4, 4, 0.15, 3),
    "asscher": (("rect", 22.0), 8.0, 3, 3, 0.20, 0),
    "radiant": (("rect", 12.0), 0.0, 4, 4, 0.15, 2),
    "baguette": (("rect", 4.0), 8.0, 2, 2, 0.10, 0),
    "cushion": (("rounded_rect", 30.0, 4), 8.0, 3, 3, 0.15, 0),
    "trillion": (("triangle",), 0.0, 4, 4, 0.15, 2),
    "marquise": (("pointed_oval", 24, False), 0.0, 4, 4, 0.15, 2),
    "pear": (("pointed_oval", 24, True), 0.0, 4, 4, 0.15, 2),
}


def step_outline_from_toml(name, corner_pct, corner_segs, oval_segs, pear, points):
    """step_outline_name (scene_file.rs:700-715)."""
    if name == "rect":
        return ("rect", corner_pct)
    if name == "rounded_rect":
        return ("rounded_rect", corner_pct, corner_segs)
    if name in ("triangle", "hexagon"):
        return (name,)
    if name == "marquise":
        return ("pointed_oval", oval_segs, False)
    if name == "pear":
        return ("pointed_oval", oval_segs, pear)
    if name == "polygon":
        if points is None:
            raise ValueError('outline = "polygon" requires `points`')
        return ("polygon", points)
    raise ValueError(f"unknown step_cut outline '{name}' (expected rect, rounded_rect, triangle, hexagon, "
                     "marquise, pear, polygon)")


def validate_diamond_params(radius, table_pct, crown_angle, pavilion_angle, girdle_pct, what):
    """validate_diamond_params (scene_file.rs:772-791): NaN/inf and
    out-of-range cut parameters are errors."""
    ok = lambda v: isinstance(v, (int, float)) and math.isfinite(v)
    if not (ok(radius) and radius > 0.0):
        raise ValueError(f"{what}: radius must be positive and finite, got {radius}")
    if not (ok(table_pct) and 0.0 < table_pct < 100.0):
        raise ValueError(f"{what}: table_pct must be in (0, 100), got {table_pct}")
    if not (ok(crown_angle) and 0.0 < crown_angle < 90.0):
        raise ValueError(f"{what}: crown angle must be in (0, 90) deg, got {crown_angle}")
    if not (ok(pavilion_angle) and 0.0 < pavilion_angle < 90.0):
        raise ValueError(f"{what}: pavilion angle must be in (0, 90) deg, got {pavilion_angle}")
    if not (ok(girdle_pct) and 0.0 <= girdle_pct < 100.0):
        raise ValueError(f"{what}: girdle_pct must be in [0, 100), got {girdle_pct}")


def parse_girdle_finish(s, what):
    """parse_girdle_finish (scene_file.rs:651-658)."""
    v = None if s is None else str(s).lower()
    if v in (None, ""):
        return "uniform"
    if v == "faceted":
        return "faceted"
    if v in ("polished", "bruted"):
        return "polished"
    raise ValueError(f"{what}: girdle_finish must be faceted|polished|bruted, got '{v}'")


# gem material presets (scene_file.rs:681-697): Cauchy B, C (µm²) and the body
# absorption per scene unit at scale_mm = 0.001
GEM_PRESETS = {
    "diamond": (2.351, 0.0230, (0.0, 0.0, 0.0)),
    "sapphire": (1.741, 0.0094, (650.0, 320.0, 25.0)),
    "ruby": (1.741, 0.0094, (25.0, 550.0, 450.0)),
    "emerald": (1.556, 0.0073, (480.0, 25.0, 380.0)),
}


def gem_preset(name):
    if name not in GEM_PRESETS:
        raise ValueError(f"unknown gem material '{name}' (expected diamond, sapphire, ruby or emerald)")
    return GEM_PRESETS[name]


def gem_absorption(g, preset_abs):
    """gem_absorption (scene_file.rs:721-736): preset body colour plus the D..Z
    grade tint, both rescaled by 0.001/scale_mm, plus an explicit absorption
    (per scene unit, not rescaled); f32 like the reference."""
    f = np.float32
    grade = str(g.get("color_grade", "D")).strip().upper()[:1]
    sigma = {"D": 0.0, "E": 0.0, "F": 0.0, "G": 50.0, "H": 80.0, "I": 120.0, "J": 170.0, "K": 230.0,
             "L": 300.0, "M": 300.0}.get(grade, 400.0)
    tint = np.array([1.0, 0.75, 0.35], f) * f(sigma)
    unit_fix = f(0.001) / f(g.get("scale_mm", 0.001))
    extra = np.asarray(g.get("absorption", (0.0, 0.0, 0.0)), f)
    return (np.asarray(preset_abs, f) + tint) * unit_fix + extra


def gem_geometry(g):
    """The size and cut of a [[gems]] entry (build_gem, scene_file.rs:793-850):
    radius, oval ratio, crown/pavilion angles, girdle facets/finish/pct."""
    f = np.float32
    scale_mm = g.get("scale_mm", 0.001)
    if g.get("measurements_mm") is not None:
        m = [f(v) for v in g["measurements_mm"]]
        if m[0] <= 0 or m[1] <= 0:
            raise ValueError("measurements_mm must be positive")
        L, W = (m[0], m[1]) if m[0] >= m[1] else (m[1], m[0])
        w_mm, ratio = W, (L / W if (L - W) / W > f(0.02) else f(1.0))
    elif g.get("carat") is not None:
        ct = f(g["carat"])
        if ct <= 0:
            raise ValueError("carat must be positive")
        w_mm, ratio = f(np.cbrt(ct / f(0.00355))), f(1.0)           # ct ≈ 0.00355 · d_mm³
    else:
        raise ValueError("provide either carat or measurements_mm")
    if not scale_mm > 0:
        raise ValueError("scale_mm must be positive")
    radius = f(0.5) * w_mm * f(scale_mm)
    table_pct = g.get("table_pct", 53.0)
    if not 0.0 < table_pct < 100.0:
        raise ValueError(f"table_pct must be in (0, 100), got {table_pct}")
    girdle_pct = g.get("girdle_pct", 2.0)
    table_r = f(table_pct / 100.0) * radius
    crown_angle = g.get("crown_angle", 34.5)
    if g.get("crown_pct") is not None:           # IGI: % of the minor axis → facet angle
        crown_angle = math.degrees(math.atan(float(f(g["crown_pct"]) / f(100.0) * w_mm * f(scale_mm) / (radius - table_r))))
    pavilion_angle = g.get("pavilion_angle", 40.75)
    if g.get("pavilion_pct") is not None:
        pavilion_angle = math.degrees(math.atan(float(f(g["pavilion_pct"]) / f(100.0) * w_mm * f(scale_mm) / radius)))
    validate_diamond_params(float(radius), table_pct, crown_angle, pavilion_angle, girdle_pct, f"gem '{g.get('report', '')}'")
    finish = parse_girdle_finish(g.get("girdle_finish"), f"gem '{g.get('report', '')}'")
    facets = g.get("girdle_facets") or (64 if ratio > 1.05 else 16)
    return dict(radius=float(radius), oval_ratio=float(ratio), table_pct=table_pct, crown_angle=crown_angle,
                pavilion_angle=pavilion_angle, girdle_facets=int(facets), girdle_finish=finish, girdle_pct=girdle_pct)


def add_gem(sb, g):
    """A [[gems]] entry from a grading report (build_gem, scene_file.rs:793-931):
    a round/oval brilliant or a step-family preset cut in a preset or
    overridden spectral dielectric, placed by scale → rotate about its center
    → translate."""
    cut = g.get("cut", "brilliant")
    geo = gem_geometry(g)
    name = g.get("material", "diamond")
    if name == "checker":                       # debug materials (scene_file.rs:862-868)
        mat = Material.checker((0.9, 0.9, 0.9), (0.05, 0.05, 0.05), 12.0)
    elif name == "opaque":
        mat = Material.lambertian((0.8, 0.8, 0.8))
    else:
        b, c, pabs = gem_preset(name)
        b = g["cauchy_b"] if g.get("cauchy_b") is not None else b
        c = g["cauchy_c"] if g.get("cauchy_c") is not None else c
        mat = Material.spectral_dielectric_cauchy(b, c, tuple(float(v) for v in gem_absorption(g, pabs)))
    ang = [0.0, 0.0, 0.0] if g.get("rotate") is None else [float(a) for a in g["rotate"]]
    ang[1] += float(g.get("rotate_y") or 0.0) + float(g.get("spin") or 0.0)
    place = dict(polish=g.get("polish", 0.02), scale=g.get("scale") or 1.0, rotate=ang,
                 translate=g.get("translate") or (0.0, 0.0, 0.0))
    if cut == "brilliant":
        return sb.add_diamond(g["center"], geo["radius"], sb.add_material(mat), geo["table_pct"], geo["crown_angle"],
                              geo["pavilion_angle"], oval_ratio=geo["oval_ratio"], girdle_facets=geo["girdle_facets"],
                              girdle_finish=geo["girdle_finish"], girdle_pct=geo["girdle_pct"], **place)
    if cut not in STEP_CUT_PRESETS:                 # step_cut_preset (scene_file.rs:741-766)
        raise ValueError(f"unknown gem cut '{cut}' (expected brilliant, step, princess, asscher, radiant, baguette, "
                         "cushion, trillion, marquise or pear)")
    outline, culet, cs, ps, spread, chev = STEP_CUT_PRESETS[cut]
    try:
        return sb.add_step_cut(g["center"], geo["radius"] * geo["oval_ratio"], geo["radius"], sb.add_material(mat),
                               table_pct=geo["table_pct"], crown_angle=geo["crown_angle"],
                               pavilion_angle=geo["pavilion_angle"], outline=outline, crown_steps=cs,
                               pavilion_steps=ps, culet_pct=culet, step_spread=spread,
                               chevrons=g["chevrons"] if g.get("chevrons") is not None else chev,
                               girdle_pct=geo["girdle_pct"], **place)
    except ValueError as e:
        raise ValueError(f"gem '{g.get('report', '')}': {e}") from None


def perlin_tables(seed):
    """Perlin::new (perlin.rs:22-33) from a seeded generator: 256 random unit
    vectors (components uniform in [-1, 1), normalised) and three Fisher–Yates
    permutations of 0..255."""
    rng = np.random.default_rng(seed)
    vec = rng.uniform(-1.0, 1.0, size=(256, 3)).astype(F32)
    vec = (vec / np.linalg.norm(vec, axis=1, keepdims=True)).astype(F32)
    perm = np.zeros((3, 256), np.int32)
    for a in range(3):
        p = np.arange(256)
        for i in range(255, 0, -1):
            j = int(rng.integers(0, i + 1))
            p[i], p[j] = p[j], p[i]
        perm[a] = p
    return vec, perm


_VOLUMES = {"constant_volume_sphere": ("constant", "sphere"), "constant_volume_box": ("constant", "box"),
            "noise_volume_sphere": ("noise", "sphere"), "noise_volume_box": ("noise", "box")}


def scene_from_toml_dict(doc, base="."):
    sb = SceneBuilder()
    sb.name = doc.get("name", "Custom Scene")
    cam = doc["camera"]
    lf, la = cam["look_from"], cam["look_at"]
    sb.camera = dict(look_from=lf, look_at=la, vfov=cam.get("vfov", 40.0), aperture=cam.get("aperture", 0.0),
                     focus_dist=cam.get("focus_dist"), aperture_blades=cam.get("aperture_blades", 0))
    bg = doc.get("background", {"type": "solid", "color": [0, 0, 0]})
    if bg["type"] == "solid":
        sb.set_solid(bg["color"])
    elif bg["type"] == "physical":
        sb.set_physical(bg.get("sun_azimuth", 0.0), bg.get("sun_elevation", 30.0), bg.get("turbidity", 3.0))
    elif bg["type"] == "env_map":
        img = load_hdr(_resolve(base, bg["path"]))
        sb.set_env(img, bg.get("rotate_y", 0.0) or 0.0, bg.get("visible"))
    else:
        raise ValueError(f"background type '{bg['type']}' is not supported by the GPU path")
    for i, obj in enumerate(doc.get("objects", [])):
        sh = obj["shape"]
        if sh["type"] in _VOLUMES:                                  # scene_file.rs:962-983
            kind, bound = _VOLUMES[sh["type"]]
            xf = Transform(obj.get("scale"), obj.get("rotate"), obj.get("rotate_y"), obj.get("spin"), obj.get("translate"))
            if not xf.identity:
                raise ValueError(f"objects[{i}]: transformed volumes are not supported by the GPU path")
            sb.add_medium(kind, bound, sh["density"], sh["color"], g=sh.get("g", 0.0),
                          noise_scale=sh.get("noise_scale", 1.0), threshold=sh.get("threshold", 0.0),
                          center=sh.get("center"), radius=sh.get("radius"), p_min=sh.get("p_min"),
                          p_max=sh.get("p_max"), seed=i)
            continue
        if "material" not in obj:
            raise ValueError(f"objects[{i}]: material is required for this shape type")
        mat = sb.add_material(_material_from_toml(obj["material"], base, sb))
        xf = Transform(obj.get("scale"), obj.get("rotate"), obj.get("rotate_y"), obj.get("spin"), obj.get("translate"))
        st = sh["type"]
        mt = obj["material"]
        # light_area > 0 for an emissive material (quad.rs:98-100, PbrMaterial::is_emissive)
        emissive = (mt["type"] == "diffuse_light" and any(c > 0 for c in mt["color"])) or \
            (mt["type"] == "pbr" and mt.get("emission_strength", 0.0) > 0 and
             float(np.dot(mt.get("emission", (0, 0, 0)), (0.2126, 0.7152, 0.0722))) > 0)
        if st == "sphere":
            si = sb.add_sphere(sh["center"], sh["radius"], mat, xf)
            if emissive:
                sb._lights.append(("sphere", si))
        elif st == "quad":
            qi = sb.add_quad(sh["corner"], sh["u"], sh["v"], mat, xf)
            if emissive:
                sb._lights.append(("quad", qi))
        elif st == "box":
            sb.add_box(sh["p_min"], sh["p_max"], mat, xf)
        elif st == "mesh":
            V, Fa, N, UV = load_obj(_resolve(base, sh["path"]), with_uv=True)
            sb.add_mesh(V, Fa, mat, N, xf, uvs=UV)
        elif st in ("cylinder", "cone"):                            # scene_file.rs:997-1000
            sb.add_shape(st, mat, sh["center"], radius=sh["radius"], height=sh["height"], xf=xf)
        elif st == "disk":                                          # scene_file.rs:1001-1002
            if float(np.dot(sh["normal"], sh["normal"])) <= 1e-12:
                raise ValueError(f"objects[{i}]: disk normal must be non-zero")
            sb.add_shape("disk", mat, sh["center"], radius=sh["radius"], normal=sh["normal"], xf=xf)
        elif st == "infinite_plane":                                # scene_file.rs:1023-1024
            if float(np.dot(sh["normal"], sh["normal"])) <= 1e-12:
                raise ValueError(f"objects[{i}]: plane normal must be non-zero")
            sb.add_shape("infinite_plane", mat, sh["point"], normal=sh["normal"],
                         wave_amplitude=sh.get("wave_amplitude", 0.0), wave_scale=sh.get("wave_scale", 1.0), xf=xf)
        elif st == "step_cut":                                      # scene_file.rs:1013-1021
            ol = step_outline_from_toml(sh.get("outline") or "rect", sh.get("corner_pct", 12.0),
                                        sh.get("corner_segs", 4), sh.get("oval_segs", 24), sh.get("pear", False),
                                        sh.get("points"))
            ang = [0.0, 0.0, 0.0] if obj.get("rotate") is None else [float(a) for a in obj["rotate"]]
            ang[1] += float(obj.get("rotate_y") or 0.0) + float(obj.get("spin") or 0.0)
            try:
                sb.add_step_cut(sh["center"], np.float32(0.5) * np.float32(sh["length"]),
                                np.float32(0.5) * np.float32(sh["width"]), mat, polish=sh.get("polish", 0.02),
                                scale=obj.get("scale") or 1.0, rotate=ang, pivot=(0.0, 0.0, 0.0),
                                translate=obj.get("translate") or (0.0, 0.0, 0.0),
                                table_pct=sh.get("table_pct", 53.0), crown_angle=sh.get("crown_angle", 34.5),
                                pavilion_angle=sh.get("pavilion_angle", 40.75), outline=ol,
                                crown_steps=sh.get("crown_steps", 3), pavilion_steps=sh.get("pavilion_steps", 3),
                                culet_pct=sh.get("culet_pct", 8.0), step_spread=sh.get("step_spread", 0.25),
                                chevrons=sh.get("chevrons", 0), girdle_pct=sh.get("girdle_pct", 2.0))
            except ValueError as e:
                raise ValueError(f"objects[{i}].shape: {e}") from None
        elif st == "diamond":                                       # scene_file.rs:1003-1011
            validate_diamond_params(sh["radius"], sh.get("table_pct", 53.0), sh.get("crown_angle", 34.5),
                                    sh.get("pavilion_angle", 40.75), sh.get("girdle_pct", 2.0), f"objects[{i}]")
            ang = [0.0, 0.0, 0.0] if obj.get("rotate") is None else [float(a) for a in obj["rotate"]]
            ang[1] += float(obj.get("rotate_y") or 0.0) + float(obj.get("spin") or 0.0)
            sb.add_diamond(sh["center"], sh["radius"], mat, sh.get("table_pct", 53.0), sh.get("crown_angle", 34.5),
                           sh.get("pavilion_angle", 40.75), polish=sh.get("polish", 0.02),
                           oval_ratio=sh.get("oval_ratio", 1.0), girdle_facets=sh.get("girdle_facets", 16),
                           girdle_finish=parse_girdle_finish(sh.get("girdle_finish"), f"objects[{i}]"),
                           girdle_pct=sh.get("girdle_pct", 2.0), scale=obj.get("scale") or 1.0, rotate=ang,
                           pivot=(0.0, 0.0, 0.0), translate=obj.get("translate") or (0.0, 0.0, 0.0))
        else:
            raise ValueError(f"objects[{i}]: shape '{st}' is not supported by the GPU path")
    for lc in doc.get("lights", []):
        if "temp_k" in lc:
            m = Material.blackbody(lc["temp_k"], lc.get("intensity", 1.0))
        else:
            m = Material.diffuse_light(lc["color"])
        sb.add_light_quad(lc["corner"], lc["u"], lc["v"], sb.add_material(m))
    for i, g in enumerate(doc.get("gems", [])):                     # scene_file.rs:1048-1052
        try:
            add_gem(sb, g)
        except ValueError as e:
            raise ValueError(f"gems[{i}]: {e}") from None
    sb.caustics = doc.get("caustics")
    return sb
