"""ctypes wrapper of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY:
imported by tests/, __graft_entry__.smoke() and bench.py's CPU legs, never by
the rustracer_b200 package.
"""
import ctypes as C
import os

import numpy as np

from rustracer_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            from . import build as _b  # noqa
        if not os.path.exists(path):
            import importlib.util
            spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(HERE, "build.py"))
            m = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(m)
            m.build()
        L = C.CDLL(path)
        vp, f, i32, i64, u32 = C.c_void_p, C.c_float, C.c_int32, C.c_int64, C.c_uint32
        fp = C.POINTER(C.c_float)
        L.orc_last_error.restype = C.c_char_p
        L.orc_scene_create.argtypes = [C.POINTER(abi.RtSceneDesc), C.POINTER(vp)]
        L.orc_scene_destroy.argtypes = [vp]
        L.orc_develop.argtypes = [fp, fp, C.POINTER(C.c_uint32), C.POINTER(abi.RtDevelopParams), C.POINTER(C.c_uint8)]
        L.orc_apply_optics.argtypes = [fp, C.c_uint32, C.c_uint32, C.c_float, C.c_float, fp]
        L.orc_tex_sample.argtypes = [vp, i32, i32, fp, i64, fp]
        L.orc_hit_uv.argtypes = [vp, fp, i64, fp]
        L.orc_pbr_scatter.argtypes = [C.POINTER(abi.RtMaterial), fp, i64, C.POINTER(i32), fp, fp, fp, fp, fp]
        L.orc_bvh_export.argtypes = [vp, fp, C.POINTER(i64), C.POINTER(i32), C.POINTER(i64)]
        L.orc_trace_closest.argtypes = [vp, fp, i64, C.POINTER(abi.RtHit), i32, i32]
        L.orc_trace_any.argtypes = [vp, fp, i64, C.POINTER(C.c_uint8), i32]
        L.orc_trace_stats.argtypes = [vp, fp, i64, C.POINTER(i64), i32]
        L.orc_trace_transmittance.argtypes = [vp, fp, i64, fp, i32]
        L.orc_hg_sample.argtypes = [fp, i64, fp]
        L.orc_bg_eval_n.argtypes = [vp, fp, i64, fp, fp]
        L.orc_sun_sample.argtypes = [vp, fp, i64, fp]
        L.orc_render_pass.argtypes = [vp, C.POINTER(abi.RtCamera), C.POINTER(abi.RtPassParams), fp,
                                      C.POINTER(C.c_uint8), i32, u32, u32, C.POINTER(i64)]
        L.orc_accumulate.argtypes = [fp, fp, C.POINTER(u32), fp, C.POINTER(C.c_uint8), i64, f, u32, f]
        L.orc_mark_converged.argtypes = [C.POINTER(C.c_uint8), C.POINTER(u32), fp, fp, i64, f]
        L.orc_mark_converged.restype = i64
        for name, nargs in [("orc_fresnel_dielectric", 2), ("orc_fresnel_conductor", 3), ("orc_cauchy_ior", 3),
                            ("orc_planck_raw", 2), ("orc_ggx_ndf", 2), ("orc_smith_g1", 2),
                            ("orc_smith_lambda", 2), ("orc_e_ss", 2), ("orc_energy_comp", 2)]:
            fn = getattr(L, name)
            fn.argtypes = [f] * nargs
            fn.restype = f
        L.orc_elut_export.argtypes = [fp]
        L.orc_spectral_to_rgb.argtypes = [f, i32, fp]
        L.orc_spectral_fire_rgb.argtypes = [f, i32, fp]
        L.orc_metal_ior.argtypes = [i32, f, fp, fp]
        L.orc_vndf_sample.argtypes = [fp, f, f, f, f, fp]
        L.orc_env_sample.argtypes = [vp, fp, fp]
        L.orc_env_pdf.argtypes = [vp, fp]
        L.orc_env_pdf.restype = f
        L.orc_env_sample_dir.argtypes = [vp, fp, fp, fp]
        L.orc_bg_eval.argtypes = [vp, fp, fp]
        L.orc_env_eval.argtypes = [vp, fp, fp]
        L.orc_lights_pdf_value.argtypes = [vp, fp, fp]
        L.orc_lights_pdf_value.restype = f
        L.orc_rng.argtypes = [C.c_uint64, u32, u32, u32, C.POINTER(u32), fp]
        ip = C.POINTER(C.c_int32)
        L.orc_photon_build.argtypes = [vp, C.POINTER(abi.RtPhotonParams), C.POINTER(i64), i32]
        L.orc_photon_set.argtypes = [vp, fp, fp, fp, ip, i64, f, u32]
        L.orc_photon_export.argtypes = [vp, fp, fp, fp, ip, C.POINTER(i64)]
        L.orc_photon_gather.argtypes = [vp, fp, i64, fp, i32]
        L.orc_knn.argtypes = [vp, fp, i64, i32, f, ip, fp, i32]
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def vec3_call(name, *args, range_mode=0):
    out = np.zeros(3, np.float32)
    getattr(lib(), name)(*args, range_mode, _fp(out))
    return out


def spectral_to_rgb(lam, range_mode=0):
    return vec3_call("orc_spectral_to_rgb", C.c_float(lam), range_mode=range_mode)


def spectral_fire_rgb(lam, range_mode=0):
    return vec3_call("orc_spectral_fire_rgb", C.c_float(lam), range_mode=range_mode)


def metal_ior(metal, lam):
    n, k = C.c_float(), C.c_float()
    lib().orc_metal_ior(metal, lam, C.byref(n), C.byref(k))
    return n.value, k.value


def scalar(name, *args):
    return getattr(lib(), "orc_" + name)(*[C.c_float(a) for a in args])


def elut():
    out = np.zeros((64, 64), np.float32)
    lib().orc_elut_export(_fp(out))
    return out


def pbr_scatter(mat, wo, n, xi, spec_wi=None):
    """PbrMaterial::scatter (material.rs:790-920) for rows of (wo, n, 4 random
    numbers): lobe (0 none, 1 specular, 2 diffuse), attenuation, direction, and
    specular_brdf_cos / specular_sampling_pdf at spec_wi (else the sampled
    direction)."""
    wo = np.asarray(wo, np.float32).reshape(-1, 3)
    k = len(wo)
    a = np.zeros((k, 10), np.float32)
    a[:, :3] = wo
    a[:, 3:6] = np.broadcast_to(np.asarray(n, np.float32), (k, 3))
    a[:, 6:10] = np.asarray(xi, np.float32).reshape(k, 4)
    lobe = np.zeros(k, np.int32)
    att, d, bc = (np.zeros((k, 3), np.float32) for _ in range(3))
    pdf = np.zeros(k, np.float32)
    swi = None if spec_wi is None else np.ascontiguousarray(np.asarray(spec_wi, np.float32).reshape(k, 3))
    lib().orc_pbr_scatter(C.byref(mat), _fp(a), k, lobe.ctypes.data_as(C.POINTER(C.c_int32)), _fp(att), _fp(d),
                          None if swi is None else _fp(swi), _fp(bc), _fp(pdf))
    return lobe, att, d, bc, pdf


def develop(params, linear=None, sum_=None, count=None):
    """apply_optics + tone_map (output.rs:84-190): a linear (H, W, 3) image of
    per-sample means, or accumulators sum (H, W, 3) / max(count, 1)."""
    h, w = params.height, params.width
    out = np.zeros((h, w, 3), np.uint8)
    lp = None if linear is None else _fp(np.ascontiguousarray(linear, np.float32))
    sp = None if sum_ is None else _fp(np.ascontiguousarray(sum_, np.float32))
    cp = None if count is None else np.ascontiguousarray(count, np.uint32).ctypes.data_as(C.POINTER(C.c_uint32))
    lib().orc_develop(lp, sp, cp, C.byref(params), out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return out


def apply_optics(img, vignette, distortion):
    """apply_optics (output.rs:159-190) on a linear (H, W, 3) image."""
    img = np.ascontiguousarray(img, np.float32)
    h, w = img.shape[:2]
    out = np.zeros_like(img)
    lib().orc_apply_optics(_fp(img), w, h, float(vignette), float(distortion), _fp(out))
    return out


def hg_sample(w, g, xi1, xi2):
    """hg_sample (volume.rs:39-62) for arrays of incident directions and numbers."""
    w = np.asarray(w, np.float32).reshape(-1, 3)
    n = len(w)
    a = np.zeros((n, 6), np.float32)
    a[:, :3] = w
    a[:, 3] = g
    a[:, 4] = xi1
    a[:, 5] = xi2
    out = np.zeros((n, 3), np.float32)
    lib().orc_hg_sample(_fp(a), n, _fp(out))
    return out


def rng(seed, pixel, sample, dim):
    u, f = C.c_uint32(), C.c_float()
    lib().orc_rng(seed, pixel, sample, dim, C.byref(u), C.byref(f))
    return u.value, f.value


class OracleScene:
    """Oracle scene built from a SceneBuilder (same RtSceneDesc as the GPU path)."""

    def __init__(self, builder):
        self._builder = builder
        self._desc = builder.desc()
        self.h = C.c_void_p()
        rc = lib().orc_scene_create(C.byref(self._desc), C.byref(self.h))
        if rc != 0:
            raise ValueError(lib().orc_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            lib().orc_scene_destroy(self.h)
            self.h = C.c_void_p()

    def bvh(self):
        nn, nl = C.c_int64(), C.c_int64()
        lib().orc_bvh_export(self.h, None, C.byref(nn), None, C.byref(nl))
        nodes = np.zeros((nn.value, 56), np.float32)
        leaves = np.zeros(nl.value, np.int32)
        lib().orc_bvh_export(self.h, _fp(nodes), C.byref(nn), leaves.ctypes.data_as(C.POINTER(C.c_int32)),
                             C.byref(nl))
        return nodes, leaves

    def trace_closest(self, rays, brute=False, threads=os.cpu_count()):
        rays = _f(rays).reshape(-1, 8)
        hits = (abi.RtHit * len(rays))()
        lib().orc_trace_closest(self.h, _fp(rays), len(rays), hits, 1 if brute else 0, threads)
        a = np.frombuffer(hits, dtype=np.dtype([("prim", np.int32), ("t", np.float32), ("b1", np.float32),
                                                ("b2", np.float32)]))
        return a.copy()

    def tex_sample(self, tex_id, uv, p=None, mode=-1):
        """Texture::value (mode −1) or the PBR samplers (0 sRGB, 1 raw, 2 red)
        at rows of (u, v) and points p."""
        uv = np.asarray(uv, np.float32).reshape(-1, 2)
        a = np.zeros((len(uv), 5), np.float32)
        a[:, :2] = uv
        if p is not None:
            a[:, 2:] = np.asarray(p, np.float32).reshape(-1, 3)
        out = np.zeros((len(uv), 3), np.float32)
        rc = lib().orc_tex_sample(self.h, int(tex_id), int(mode), _fp(a), len(a), _fp(out))
        if rc:
            raise ValueError("bad texture id")
        return out

    def hit_uv(self, rays):
        """(u, v, tangent xyz) of each ray's closest hit record."""
        rays = _f(rays).reshape(-1, 8)
        out = np.zeros((len(rays), 5), np.float32)
        lib().orc_hit_uv(self.h, _fp(rays), len(rays), _fp(out))
        return out

    def trace_any(self, rays, threads=os.cpu_count()):
        rays = _f(rays).reshape(-1, 8)
        occ = np.zeros(len(rays), np.uint8)
        lib().orc_trace_any(self.h, _fp(rays), len(rays), occ.ctypes.data_as(C.POINTER(C.c_uint8)), threads)
        return occ

    def trace_transmittance(self, rays, threads=os.cpu_count()):
        """world.transmittance (bvh.rs:532-575) per ray: 0 if occluded, else Π media."""
        rays = _f(rays).reshape(-1, 8)
        out = np.zeros(len(rays), np.float32)
        lib().orc_trace_transmittance(self.h, _fp(rays), len(rays), _fp(out), threads)
        return out

    def bg_eval_n(self, dirs):
        """Background::eval (renderer.rs:196-208) and the sun pdf per direction."""
        dirs = _f(dirs).reshape(-1, 3)
        rgb = np.zeros((len(dirs), 3), np.float32)
        pdf = np.zeros(len(dirs), np.float32)
        lib().orc_bg_eval_n(self.h, _fp(dirs), len(dirs), _fp(rgb), _fp(pdf))
        return rgb, pdf

    def sun_sample(self, r):
        r = _f(r).reshape(-1, 2)
        out = np.zeros((len(r), 3), np.float32)
        lib().orc_sun_sample(self.h, _fp(r), len(r), _fp(out))
        return out

    def trace_stats(self, rays, threads=os.cpu_count()):
        rays = _f(rays).reshape(-1, 8)
        out = np.zeros((len(rays), 4), np.int64)
        lib().orc_trace_stats(self.h, _fp(rays), len(rays), out.ctypes.data_as(C.POINTER(C.c_int64)), threads)
        return out

    def render_pass(self, cam, params, threads=os.cpu_count(), rows=None, converged=None):
        n = max(1, params.n_samples)
        out = np.zeros((n, params.height, params.width, 3), np.float32)
        cnt = np.zeros(2, np.int64)
        rb, re = (0, 0) if rows is None else rows
        conv = None if converged is None else np.ascontiguousarray(converged, dtype=np.uint8)
        lib().orc_render_pass(self.h, C.byref(cam), C.byref(params), _fp(out),
                              None if conv is None else conv.ctypes.data_as(C.POINTER(C.c_uint8)),
                              threads, rb, re, cnt.ctypes.data_as(C.POINTER(C.c_int64)))
        self.last_counters = cnt
        return out

    # ── caustic photon map ─────────────────────────────────────────────────
    def photon_build(self, params, threads=os.cpu_count()):
        n = C.c_int64()
        rc = lib().orc_photon_build(self.h, C.byref(params), C.byref(n), threads)
        if rc != 0:
            raise ValueError(f"photon build failed ({rc})")
        return n.value

    def photon_set(self, pos, power, nor, index=None, radius=0.1, knn_k=0):
        pos, power, nor = _f(pos).reshape(-1, 3), _f(power).reshape(-1, 3), _f(nor).reshape(-1, 3)
        idx = None if index is None else np.ascontiguousarray(index, dtype=np.int32)
        lib().orc_photon_set(self.h, _fp(pos), _fp(power), _fp(nor),
                             None if idx is None else idx.ctypes.data_as(C.POINTER(C.c_int32)), len(pos), radius, knn_k)

    def photon_export(self):
        n = C.c_int64()
        lib().orc_photon_export(self.h, None, None, None, None, C.byref(n))
        pos, power, nor = (np.zeros((n.value, 3), np.float32) for _ in range(3))
        idx = np.zeros(n.value, np.int32)
        lib().orc_photon_export(self.h, _fp(pos), _fp(power), _fp(nor), idx.ctypes.data_as(C.POINTER(C.c_int32)),
                                C.byref(n))
        return pos, power, nor, idx

    def photon_gather(self, queries, threads=os.cpu_count()):
        q = _f(queries).reshape(-1, 6)
        out = np.zeros((len(q), 3), np.float32)
        lib().orc_photon_gather(self.h, _fp(q), len(q), _fp(out), threads)
        return out

    def knn(self, queries, k, rmax, threads=os.cpu_count()):
        q = _f(queries).reshape(-1, 3)
        idx = np.zeros((len(q), k), np.int32)
        d2 = np.zeros((len(q), k), np.float32)
        lib().orc_knn(self.h, _fp(q), len(q), k, rmax, idx.ctypes.data_as(C.POINTER(C.c_int32)), _fp(d2), threads)
        return idx, d2

    def env_sample(self, d):
        out = np.zeros(3, np.float32)
        lib().orc_env_sample(self.h, _fp(_f(d)), _fp(out))
        return out

    def env_pdf(self, d):
        return lib().orc_env_pdf(self.h, _fp(_f(d)))

    def env_sample_dir(self, xi):
        d = np.zeros(3, np.float32)
        pdf = C.c_float()
        lib().orc_env_sample_dir(self.h, _fp(_f(xi)), _fp(d), C.byref(pdf))
        return d, pdf.value

    def bg_eval(self, d):
        out = np.zeros(3, np.float32)
        lib().orc_bg_eval(self.h, _fp(_f(d)), _fp(out))
        return out

    def env_eval(self, d):
        out = np.zeros(3, np.float32)
        lib().orc_env_eval(self.h, _fp(_f(d)), _fp(out))
        return out

    def lights_pdf_value(self, o, d):
        return lib().orc_lights_pdf_value(self.h, _fp(_f(o)), _fp(_f(d)))


class Accumulator:
    """accumulate_sample / mark_converged state (main.rs:603-677) on the CPU."""

    def __init__(self, npix):
        self.acc = np.zeros((npix, 3), np.float32)
        self.m2 = np.zeros((npix, 3), np.float32)
        self.n = np.zeros(npix, np.uint32)
        self.conv = np.zeros(npix, np.uint8)

    def add(self, scratch, clamp=0.0, min_samples=4, floor=5.0):
        s = _f(scratch).reshape(-1, 3)
        lib().orc_accumulate(_fp(self.acc), _fp(s), self.n.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(self.m2),
                             self.conv.ctypes.data_as(C.POINTER(C.c_uint8)), len(s), clamp, min_samples, floor)

    def mark_converged(self, thresh=0.05):
        return lib().orc_mark_converged(self.conv.ctypes.data_as(C.POINTER(C.c_uint8)),
                                        self.n.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(self.m2),
                                        _fp(self.acc), len(self.n), thresh)
