"""Host-side mirror of the reference's render entry points over librtb200.so.

    render_tiles(scratch, converged, sample_idx, strata, width, height, camera,
                 world, background, lights, bg_scale, photon_map, frame_time)
    (src/renderer.rs:655-669)

becomes GpuScene(builder).render_tiles(...): the world/background/lights are the
scene handle, created once (scene_file::build + BvhTree::from_list); every call
renders sample passes on the GPU.  There is no CPU fallback: without the CUDA
library or a GPU every call raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librtb200.so")
_lib = None


class RtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rt error {code}: {msg}")
        self.code = code


def lib():
    """Load librtb200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m rustracer_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, u32, f = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_float
        L.rt_version.restype = i32
        L.rt_device_count.argtypes = [C.POINTER(i32)]
        L.rt_scene_create.argtypes = [C.POINTER(abi.RtSceneDesc), i32, C.POINTER(vp)]
        L.rt_scene_destroy.argtypes = [vp]
        L.rt_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
        L.rt_scene_bvh_stats.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i32), C.POINTER(C.c_double)]
        L.rt_scene_bvh_export.argtypes = [vp, C.POINTER(f), C.POINTER(i64), C.POINTER(i32), C.POINTER(i64)]
        L.rt_trace_closest.argtypes = [vp, vp, i64, vp, i32]
        L.rt_trace_any.argtypes = [vp, vp, i64, vp, i32]
        L.rt_trace_transmittance.argtypes = [vp, vp, i64, vp, i32]
        L.rt_render_pass.argtypes = [vp, C.POINTER(abi.RtCamera), C.POINTER(abi.RtPassParams), vp, vp, i32]
        L.rt_render_accumulate.argtypes = [vp, C.POINTER(abi.RtCamera), C.POINTER(abi.RtPassParams), f, u32, f, i32,
                                           vp, vp, vp, i32]
        L.rt_develop.argtypes = [vp, vp, C.POINTER(abi.RtDevelopParams), vp, i32]
        L.rt_scene_build_time.argtypes = [vp, C.POINTER(C.c_double)]
        L.rt_rgbe_decode.argtypes = [C.POINTER(C.c_uint8), C.c_size_t, i32, i32, C.POINTER(C.c_float)]
        L.rt_last_render_stats.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)]
        L.rt_render_pass_noalloc.argtypes = [vp, C.POINTER(abi.RtCamera), C.POINTER(abi.RtPassParams), vp]
        L.rt_render_batch.argtypes = [vp, C.POINTER(abi.RtBatchJob), i32, C.POINTER(abi.RtPassParams), u32, vp, vp,
                                      vp, vp, i32]
        L.rt_photon_build.argtypes = [vp, C.POINTER(abi.RtPhotonParams), C.POINTER(i64)]
        L.rt_photon_set.argtypes = [vp, vp, vp, vp, vp, i64, f, u32]
        L.rt_photon_clear.argtypes = [vp]
        L.rt_photon_build_times.argtypes = [vp, C.POINTER(C.c_float)]
        L.rt_photon_export.argtypes = [vp, vp, vp, vp, vp, C.POINTER(i64)]
        L.rt_photon_gather.argtypes = [vp, vp, i64, vp, i32]
        L.rt_knn.argtypes = [vp, vp, i64, i32, f, vp, vp, i32]
        L.rt_set_profiling.argtypes = [vp, i32]
        L.rt_kernel_times.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(i64)]
        L.rt_capture_rays.argtypes = [vp, C.POINTER(abi.RtCamera), C.POINTER(abi.RtPassParams), u32, vp, i64,
                                      C.POINTER(i64)]
        L.rt_set_tuning.argtypes = [vp, C.POINTER(abi.RtTuning)]
        L.rt_render_accumulate_async.argtypes = [vp, C.POINTER(abi.RtCamera), C.POINTER(abi.RtPassParams), f, u32, f,
                                                 i32, vp, vp, vp, vp]
        L.rt_sync.argtypes = [vp]
        L.rt_get_tuning.argtypes = [vp, C.POINTER(abi.RtTuning)]
        L.rt_set_caller_stream.argtypes = [vp, vp]
        L.rt_guide_init.argtypes = [vp, C.POINTER(abi.RtGuideParams)]
        L.rt_guide_mode.argtypes = [vp, i32]
        L.rt_guide_params.argtypes = [vp, vp, i32]
        L.rt_guide_eval.argtypes = [vp, vp, i64, vp, i32]
        L.rt_guide_pdf.argtypes = [vp, vp, vp, i64, vp, i32]
        L.rt_guide_sample.argtypes = [vp, vp, vp, i64, vp, i32]
        L.rt_guide_loss_grad.argtypes = [vp, vp, i64, C.POINTER(f), vp]
        L.rt_guide_train.argtypes = [vp, vp, i64, i32, C.POINTER(f)]
        L.rt_guide_stats.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), C.POINTER(C.c_double)]
        _lib = L
    return _lib


def device_count():
    n = C.c_int32(0)
    lib().rt_device_count(C.byref(n))
    return n.value


def _ptr(a):
    """(pointer, mem flag) for a numpy array or a CUDA torch tensor."""
    if isinstance(a, np.ndarray):
        return C.c_void_p(a.ctypes.data), abi.RT_MEM_HOST
    try:
        import torch
        if isinstance(a, torch.Tensor):
            if a.is_cuda:
                return C.c_void_p(a.data_ptr()), abi.RT_MEM_DEVICE
            return C.c_void_p(a.data_ptr()), abi.RT_MEM_HOST
    except ImportError:
        pass
    raise TypeError("expected a numpy array or a torch tensor")


def _torch_stream(*arrays):
    """cudaStream_t of torch's current stream on the device of the first CUDA
    tensor among `arrays` (None when none is a CUDA tensor)."""
    for a in arrays:
        if a is not None and not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False):
            import torch
            return torch.cuda.current_stream(a.device).cuda_stream
    return None


def develop_params(width, height, exposure=1.0, tonemapper="agx", vignette=0.0, distortion=0.0):
    """RtDevelopParams; tonemapper "agx" (the reference's default) or "aces"."""
    tm = {"agx": abi.RT_TONEMAP_AGX, "aces": abi.RT_TONEMAP_ACES}
    if tonemapper not in tm:
        raise ValueError(f"unknown tonemapper '{tonemapper}' (agx or aces)")
    p = abi.RtDevelopParams()
    p.width, p.height, p.exposure, p.tonemapper = int(width), int(height), float(exposure), tm[tonemapper]
    p.vignette, p.distortion = float(vignette), float(distortion)
    return p


def pass_params(width, height, sample_idx=0, n_samples=1, strata=None, max_depth=50, hero=1, bg_scale=1.0,
                seed=0, spp_total=None, frame_time=None):
    """RtPassParams; strata defaults to ⌊√spp⌋ of the whole render (main.rs:64)."""
    p = abi.RtPassParams()
    p.width, p.height = int(width), int(height)
    p.sample_idx, p.n_samples = int(sample_idx), int(n_samples)
    if strata is None:
        strata = int(np.sqrt(np.float32(spp_total if spp_total else n_samples)))
    p.strata = int(strata)
    p.max_depth = int(max_depth)
    p.hero_count = int(hero)
    p.bg_scale = float(bg_scale)
    p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    if frame_time is not None:
        p.use_frame_time = 1
        p.t0, p.t1 = float(frame_time[0]), float(frame_time[1])
    return p


def guide_params(lr=1e-3, batch=65536, steps_per_pass=8, record_capacity=1 << 24, min_resolution=4,
                 level_scale=1.32, seed=1, domain=None, beta1=0.9, beta2=0.99, epsilon=1e-8, alpha_max=0.5,
                 log_kappa_max=5.0):
    """RtGuideParams with the learned proposal's defaults: 16 levels from 4 to
    ≈257 cells across the scene (finer levels memorise single records: a
    record's direction is one noisy draw, and at ~4096 cells each record gets
    a cell of its own), Adam lr 1e-3 (1e-2 and 3e-3 sharpened the lobes on
    noisy records), α ≤ 0.5 and κ ≤ e^5 (a defensive share for the cosine
    lobe and no needle lobes); domain None: the scene bounds."""
    p = abi.RtGuideParams()
    if domain is not None:
        lo, hi = domain
        p.domain_min[:] = [float(x) for x in lo]
        p.domain_max[:] = [float(x) for x in hi]
    p.learning_rate, p.beta1, p.beta2, p.epsilon = lr, beta1, beta2, epsilon
    p.batch, p.steps_per_pass, p.record_capacity = batch, steps_per_pass, record_capacity
    p.min_resolution, p.level_scale, p.seed = min_resolution, level_scale, seed
    p.alpha_max, p.log_kappa_max = alpha_max, log_kappa_max
    return p


class GpuScene:
    """A scene resident on one GPU (RtScene handle)."""

    def __init__(self, builder, device=0):
        self._builder = builder
        self._desc = builder.desc()
        self.h = C.c_void_p()
        rc = lib().rt_scene_create(C.byref(self._desc), int(device), C.byref(self.h))
        if rc != 0:
            msg = self.last_error()
            if self.h.value:
                lib().rt_scene_destroy(self.h)
                self.h = C.c_void_p()
            raise RtError(rc, msg)

    def last_error(self):
        buf = C.create_string_buffer(512)
        lib().rt_last_error(self.h, buf, 512)
        return buf.value.decode()

    def _check(self, rc):
        if rc != 0:
            raise RtError(rc, self.last_error())

    def _order(self, *arrays):
        """Make the library's calls wait for torch's current stream when CUDA
        tensors are passed (their producers may still be queued there)."""
        st = _torch_stream(*arrays)
        if st is not None:
            self._check(lib().rt_set_caller_stream(self.h, C.c_void_p(st)))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().rt_scene_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ── BVH ──────────────────────────────────────────────────────────────
    def bvh_stats(self):
        nn, nl, md, sah = C.c_int64(), C.c_int64(), C.c_int32(), C.c_double()
        lib().rt_scene_bvh_stats(self.h, C.byref(nn), C.byref(nl), C.byref(md), C.byref(sah))
        return dict(nodes=nn.value, leaves=nl.value, max_depth=md.value, sah_cost=sah.value)

    def build_time_ms(self):
        """Wall time of the BVH build at scene creation (rt_scene_build_time)."""
        ms = C.c_double()
        lib().rt_scene_build_time(self.h, C.byref(ms))
        return ms.value

    def bvh(self):
        nn, nl = C.c_int64(), C.c_int64()
        lib().rt_scene_bvh_export(self.h, None, C.byref(nn), None, C.byref(nl))
        nodes = np.zeros((nn.value, 56), np.float32)
        leaves = np.zeros(nl.value, np.int32)
        lib().rt_scene_bvh_export(self.h, nodes.ctypes.data_as(C.POINTER(C.c_float)), C.byref(nn),
                                  leaves.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(nl))
        return nodes, leaves

    # ── ray-level entry points ───────────────────────────────────────────
    def trace_closest(self, rays, out=None):
        """rays: (n, 8) float32 (origin, direction, t_min, t_max) numpy or CUDA tensor.
        Returns a structured array (prim, t, b1, b2) or fills `out` (n, 4) int32 tensor."""
        n = int(rays.shape[0])
        if isinstance(rays, np.ndarray):
            rays = np.ascontiguousarray(rays, dtype=np.float32)
            hits = np.zeros(n, dtype=np.dtype([("prim", np.int32), ("t", np.float32), ("b1", np.float32),
                                               ("b2", np.float32)]))
            self._check(lib().rt_trace_closest(self.h, C.c_void_p(rays.ctypes.data), n,
                                               C.c_void_p(hits.ctypes.data), abi.RT_MEM_HOST))
            return hits
        rp, mem = _ptr(rays)
        op, _ = _ptr(out)
        self._order(rays, out)
        self._check(lib().rt_trace_closest(self.h, rp, n, op, mem))
        return out

    def trace_any(self, rays):
        rays = np.ascontiguousarray(rays, dtype=np.float32)
        occ = np.zeros(len(rays), np.uint8)
        self._check(lib().rt_trace_any(self.h, C.c_void_p(rays.ctypes.data), len(rays), C.c_void_p(occ.ctypes.data),
                                       abi.RT_MEM_HOST))
        return occ

    def trace_transmittance(self, rays):
        """world.transmittance (bvh.rs:532-575) per ray: 0 behind an opaque
        primitive, else the product of the media's transmittances."""
        rays = np.ascontiguousarray(rays, dtype=np.float32)
        tr = np.zeros(len(rays), np.float32)
        self._check(lib().rt_trace_transmittance(self.h, C.c_void_p(rays.ctypes.data), len(rays),
                                                 C.c_void_p(tr.ctypes.data), abi.RT_MEM_HOST))
        return tr

    # ── sample passes ────────────────────────────────────────────────────
    def render_pass(self, cam, params, out=None, converged=None):
        """params.n_samples passes; returns (n_samples, height, width, 3) float32."""
        n = max(1, params.n_samples)
        if out is None:
            out = np.zeros((n, params.height, params.width, 3), np.float32)
        op, mem = _ptr(out)
        cp = None
        if converged is not None:
            cp, _ = _ptr(converged)
        self._order(out, converged)
        self._check(lib().rt_render_pass(self.h, C.byref(cam), C.byref(params), op, cp, mem))
        return out

    def render_pass_noalloc(self, cam, params, out):
        """rt_render_pass without device allocation: `out` is a CUDA tensor of
        (n_samples, height, width, 3) float32; width·height ≤ 65536.  For hosts
        that must not allocate device memory while running (see rt_api.h)."""
        op, mem = _ptr(out)
        if mem != abi.RT_MEM_DEVICE:
            raise TypeError("render_pass_noalloc writes device memory: pass a CUDA tensor")
        self._order(out)
        self._check(lib().rt_render_pass_noalloc(self.h, C.byref(cam), C.byref(params), op))
        return out

    def render_tiles(self, scratch, converged, sample_idx, strata, width, height, camera, bg_scale=1.0,
                     max_depth=50, hero=1, seed=0):
        """The reference's render_tiles signature (renderer.rs:655-669): one pass into scratch (H, W, 3)."""
        p = pass_params(width, height, sample_idx, 1, strata, max_depth, hero, bg_scale, seed)
        out = scratch.reshape(1, height, width, 3)
        self.render_pass(camera, p, out=out, converged=converged)
        return scratch

    def render_accumulate(self, cam, params, firefly_clamp=0.0, firefly_min_samples=4, firefly_floor=5.0,
                          reset=True, outputs=None):
        """Render params.n_samples passes and accumulate on the device (main.rs:603-643).
        Returns (sum (H,W,3), m2 (H,W,3), count (H,W)) as numpy, or fills `outputs` tensors."""
        H, W = params.height, params.width
        if outputs is None:
            s = np.zeros((H, W, 3), np.float32)
            m = np.zeros((H, W, 3), np.float32)
            c = np.zeros((H, W), np.uint32)
        else:
            s, m, c = outputs
        sp, mem = _ptr(s)
        mp, _ = _ptr(m)
        cp, _ = _ptr(c)
        self._order(s, m, c)
        self._check(lib().rt_render_accumulate(self.h, C.byref(cam), C.byref(params), float(firefly_clamp),
                                               int(firefly_min_samples), float(firefly_floor), 1 if reset else 0,
                                               sp, mp, cp, mem))
        return s, m, c

    def render_accumulate_async(self, cam, params, outputs, firefly_clamp=0.0, firefly_min_samples=4,
                                firefly_floor=5.0, reset=True, stream=None):
        """rt_render_accumulate_async: queue the render on the scene's stream
        after torch's current stream (or `stream`, a torch.cuda.Stream), which
        then waits for it; returns at once.  outputs: CUDA tensors (sum, m2,
        count) that must stay alive until the work is done.  sync() reports
        the device status and the statistics."""
        import torch
        s, m, c = outputs
        st = stream if stream is not None else torch.cuda.current_stream(s.device)
        self._check(lib().rt_render_accumulate_async(self.h, C.byref(cam), C.byref(params), float(firefly_clamp),
                                                     int(firefly_min_samples), float(firefly_floor),
                                                     1 if reset else 0, C.c_void_p(s.data_ptr()),
                                                     C.c_void_p(m.data_ptr()), C.c_void_p(c.data_ptr()),
                                                     C.c_void_p(st.cuda_stream)))

    def sync(self):
        """rt_sync: wait for the handle's queued work; raises on a device error of
        the last asynchronous call."""
        self._check(lib().rt_sync(self.h))

    def render_batch(self, jobs, shared, window=0, outputs=None):
        """A packed batch of requests on this scene (rt_render_batch).  jobs:
        dicts with cam, width, height, spp and optionally strata (⌊√spp⌋),
        sample_idx (0) and seed (0); shared: RtPassParams for max_depth,
        hero_count and bg_scale.  Returns a list of (sum (h,w,3), m2 (h,w,3),
        count (h,w)) per request — views of the packed outputs, numpy or the
        CUDA tensors given as outputs=(sum, m2, count), flat — and done_ms, the
        device time at which each request's last pass ended."""
        arr = (abi.RtBatchJob * len(jobs))()
        sizes = []
        for k, j in enumerate(jobs):
            b = arr[k]
            b.cam = j["cam"]
            b.width, b.height, b.spp = int(j["width"]), int(j["height"]), int(j["spp"])
            b.strata = int(j.get("strata", int(np.sqrt(np.float32(b.spp)))))
            b.sample_idx = int(j.get("sample_idx", 0))
            b.seed = int(j.get("seed", 0)) & 0xFFFFFFFFFFFFFFFF
            sizes.append((b.height, b.width))
        tot = sum(h * w for h, w in sizes)
        if outputs is None:
            outputs = (np.zeros(tot * 3, np.float32), np.zeros(tot * 3, np.float32), np.zeros(tot, np.uint32))
        s, m, c = outputs
        sp, mem = _ptr(s)
        mp, _ = _ptr(m)
        cp, _ = _ptr(c)
        done = np.zeros(len(jobs), np.float32)
        self._order(s, m, c)
        self._check(lib().rt_render_batch(self.h, arr, len(jobs), C.byref(shared), int(window), sp, mp, cp,
                                          C.c_void_p(done.ctypes.data), mem))
        out, o = [], 0
        for h, w in sizes:
            out.append((s[o * 3:(o + h * w) * 3].reshape(h, w, 3), m[o * 3:(o + h * w) * 3].reshape(h, w, 3),
                        c[o:o + h * w].reshape(h, w)))
            o += h * w
        return out, done

    def develop(self, width, height, linear=None, exposure=1.0, tonemapper="agx", vignette=0.0, distortion=0.0,
                out=None):
        """apply_optics + tone_map (output.rs:84-190) on the device: the scene's
        accumulators (linear=None) or a linear (H, W, 3) image → uint8 (H, W, 3)."""
        p = develop_params(width, height, exposure, tonemapper, vignette, distortion)
        if linear is not None and isinstance(linear, np.ndarray):
            linear = np.ascontiguousarray(linear, np.float32)
        if out is None:
            if linear is not None and not isinstance(linear, np.ndarray):
                import torch
                out = torch.empty((height, width, 3), dtype=torch.uint8, device=linear.device)
            else:
                out = np.zeros((height, width, 3), np.uint8)
        op, mem = _ptr(out)
        lp = None
        if linear is not None:
            lp, lmem = _ptr(linear)
            if lmem != mem:
                raise ValueError("linear and out must both be host arrays or both device tensors")
        self._order(linear, out)
        self._check(lib().rt_develop(self.h, lp, C.byref(p), op, mem))
        return out

    def last_stats(self):
        ms, e, s, l = C.c_double(), C.c_int64(), C.c_int64(), C.c_int64()
        lib().rt_last_render_stats(self.h, C.byref(ms), C.byref(e), C.byref(s), C.byref(l))
        return dict(ms=ms.value, ext_rays=e.value, shadow_rays=s.value, launches=l.value)

    # ── caustic photon map (photon.rs, scene.rs:35-74) ────────────────────
    def photon_build(self, params):
        """rebuild_caustics on the GPU; returns the number of stored photons."""
        n = C.c_int64()
        self._check(lib().rt_photon_build(self.h, C.byref(params), C.byref(n)))
        return n.value

    def photon_set(self, pos, power, nor, index=None, radius=0.1, knn_k=0):
        pos, power, nor = (np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1, 3)) for a in (pos, power, nor))
        idx = None if index is None else np.ascontiguousarray(index, dtype=np.int32)
        self._check(lib().rt_photon_set(self.h, C.c_void_p(pos.ctypes.data), C.c_void_p(power.ctypes.data),
                                        C.c_void_p(nor.ctypes.data),
                                        None if idx is None else C.c_void_p(idx.ctypes.data), len(pos), float(radius),
                                        int(knn_k)))

    def photon_stage_ms(self):
        """Device ms of the last photon build's stages: (trace, compaction, tree)."""
        ms = (C.c_float * 3)()
        self._check(lib().rt_photon_build_times(self.h, ms))
        return tuple(ms)

    def photon_clear(self):
        self._check(lib().rt_photon_clear(self.h))

    def photon_export(self):
        n = C.c_int64()
        self._check(lib().rt_photon_export(self.h, None, None, None, None, C.byref(n)))
        pos, power, nor = (np.zeros((n.value, 3), np.float32) for _ in range(3))
        idx = np.zeros(n.value, np.int32)
        self._check(lib().rt_photon_export(self.h, C.c_void_p(pos.ctypes.data), C.c_void_p(power.ctypes.data),
                                           C.c_void_p(nor.ctypes.data), C.c_void_p(idx.ctypes.data), C.byref(n)))
        return pos, power, nor, idx

    def photon_gather(self, queries):
        q = np.ascontiguousarray(np.asarray(queries, np.float32).reshape(-1, 6))
        out = np.zeros((len(q), 3), np.float32)
        self._check(lib().rt_photon_gather(self.h, C.c_void_p(q.ctypes.data), len(q), C.c_void_p(out.ctypes.data),
                                           abi.RT_MEM_HOST))
        return out

    def knn(self, queries, k, rmax):
        q = np.ascontiguousarray(np.asarray(queries, np.float32).reshape(-1, 3))
        idx = np.zeros((len(q), k), np.int32)
        d2 = np.zeros((len(q), k), np.float32)
        self._check(lib().rt_knn(self.h, C.c_void_p(q.ctypes.data), len(q), int(k), float(rmax),
                                 C.c_void_p(idx.ctypes.data), C.c_void_p(d2.ctypes.data), abi.RT_MEM_HOST))
        return idx, d2

    # ── diagnostics ──────────────────────────────────────────────────────
    # ── launch tuning (rt_set_tuning) ─────────────────────────────────────
    def set_tuning(self, max_paths=0, trace_blocks_per_sm=0, shade_blocks_per_sm=0, max_iterations=0,
                   stack_limit=0, stack_ring=0, node_format=0, graph=0):
        t = abi.RtTuning(int(max_paths), int(trace_blocks_per_sm), int(shade_blocks_per_sm), int(max_iterations),
                         int(stack_limit), int(stack_ring), int(node_format), int(graph))
        self._check(lib().rt_set_tuning(self.h, C.byref(t)))

    def get_tuning(self):
        t = abi.RtTuning()
        self._check(lib().rt_get_tuning(self.h, C.byref(t)))
        return dict(max_paths=t.max_paths, trace_blocks_per_sm=t.trace_blocks_per_sm,
                    shade_blocks_per_sm=t.shade_blocks_per_sm, max_iterations=t.max_iterations,
                    stack_limit=t.stack_limit, stack_ring=t.stack_ring, node_format=t.node_format, graph=t.graph)

    # ── path guiding (rt_guide_*) ─────────────────────────────────────────
    def guide_init(self, params=None):
        """Create the guide network with fresh parameters (mode off)."""
        self._gp = params if params is not None else guide_params()
        self._check(lib().rt_guide_init(self.h, C.byref(self._gp)))

    def guide_mode(self, mode):
        """0: plain cosine bounces, 1: guided (frozen), 2: guided + training after each render call."""
        self._check(lib().rt_guide_mode(self.h, int(mode)))

    def guide_get_params(self):
        out = np.zeros(abi.RT_GUIDE_PARAMS, np.float32)
        self._check(lib().rt_guide_params(self.h, C.c_void_p(out.ctypes.data), 0))
        return out

    def guide_set_params(self, params):
        params = np.ascontiguousarray(params, np.float32)
        assert params.size == abi.RT_GUIDE_PARAMS
        self._check(lib().rt_guide_params(self.h, C.c_void_p(params.ctypes.data), 1))

    def guide_eval(self, q):
        """Network outputs (n × 41) at q (n × 9: position, unit normal, unit ω_o)."""
        q = np.ascontiguousarray(np.asarray(q, np.float32).reshape(-1, 9))
        out = np.zeros((len(q), 41), np.float32)
        self._check(lib().rt_guide_eval(self.h, C.c_void_p(q.ctypes.data), len(q), C.c_void_p(out.ctypes.data),
                                        abi.RT_MEM_HOST))
        return out

    def guide_pdf(self, q, dirs):
        q = np.ascontiguousarray(np.asarray(q, np.float32).reshape(-1, 9))
        d = np.ascontiguousarray(np.asarray(dirs, np.float32).reshape(-1, 3))
        out = np.zeros(len(q), np.float32)
        self._check(lib().rt_guide_pdf(self.h, C.c_void_p(q.ctypes.data), C.c_void_p(d.ctypes.data), len(q),
                                       C.c_void_p(out.ctypes.data), abi.RT_MEM_HOST))
        return out

    def guide_sample(self, q, u):
        q = np.ascontiguousarray(np.asarray(q, np.float32).reshape(-1, 9))
        u = np.ascontiguousarray(np.asarray(u, np.float32).reshape(-1, 4))
        out = np.zeros((len(q), 4), np.float32)
        self._check(lib().rt_guide_sample(self.h, C.c_void_p(q.ctypes.data), C.c_void_p(u.ctypes.data), len(q),
                                          C.c_void_p(out.ctypes.data), abi.RT_MEM_HOST))
        return out

    def guide_loss_grad(self, samples):
        """(loss, gradient) of samples n × 13 (position, normal, ω_o, direction, weight)."""
        s = np.ascontiguousarray(np.asarray(samples, np.float32).reshape(-1, 13))
        g = np.zeros(abi.RT_GUIDE_PARAMS, np.float32)
        loss = C.c_float()
        self._check(lib().rt_guide_loss_grad(self.h, C.c_void_p(s.ctypes.data), len(s), C.byref(loss),
                                             C.c_void_p(g.ctypes.data)))
        return loss.value, g

    def guide_train(self, samples, steps=1):
        s = np.ascontiguousarray(np.asarray(samples, np.float32).reshape(-1, 13))
        loss = C.c_float()
        self._check(lib().rt_guide_train(self.h, C.c_void_p(s.ctypes.data), len(s), int(steps), C.byref(loss)))
        return loss.value

    def guide_stats(self):
        r, n, st, ms = C.c_int64(), C.c_int64(), C.c_int64(), C.c_double()
        self._check(lib().rt_guide_stats(self.h, C.byref(r), C.byref(n), C.byref(st), C.byref(ms)))
        return dict(records=r.value, samples=n.value, steps=st.value, train_ms=ms.value)

    def set_profiling(self, enable=True):
        self._check(lib().rt_set_profiling(self.h, 1 if enable else 0))

    def kernel_times(self):
        """{stage: (ms, launches)} of the last render call (profiling on)."""
        ms = (C.c_double * 4)()
        n = (C.c_int64 * 4)()
        self._check(lib().rt_kernel_times(self.h, ms, n))
        names = ("generate", "extend", "shade", "shadow")
        return {k: (ms[i], n[i]) for i, k in enumerate(names)}

    def capture_rays(self, cam, params, depth, max_rays):
        out = np.zeros((max_rays, 8), np.float32)
        n = C.c_int64()
        self._check(lib().rt_capture_rays(self.h, C.byref(cam), C.byref(params), int(depth),
                                          C.c_void_p(out.ctypes.data), int(max_rays), C.byref(n)))
        return out[: n.value]
