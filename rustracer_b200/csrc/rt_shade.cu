// rt_shade.cu — wavefront stages around the traversal kernels:
//   generate  : camera rays for every (pixel, sample) of the chunk
//               (render_tiles body, src/renderer.rs:692-726; Camera::get_ray, src/camera.rs:47-59)
//   shade     : one bounce of ray_color (src/renderer.rs:379-580) for every
//               path in the queue — emission with its MIS weight, material
//               scattering, next-event estimation (the shadow ray is queued and
//               its contribution parked in the path), Russian roulette — and
//               warp-aggregated compaction of the surviving paths
//   finalize  : fold the last parked contributions, write the pass output
//   accumulate: accumulate_sample (src/main.rs:603-643) over the passes in order
#include "rt_internal.h"
#include "rt_media.cuh"
#include "rt_sky.cuh"
#include "rt_ggx.cuh"
#include "rt_texture.cuh"

using namespace rtd;

namespace {

// ── spectrum (src/spectrum.rs) ──────────────────────────────────────────────
RT_D void cmf_lerp(const DevScene& S, float lambda, float xyz[3]) {
    float t = clampf_((lambda - 380.0f) / 5.0f, 0.0f, (float)(S.n_spec - 1));
    int i = min((int)t, S.n_spec - 2);
    float frac = t - (float)i;
    float4 a = __ldg(S.cmf + i), b = __ldg(S.cmf + i + 1);
    xyz[0] = a.x + frac * (b.x - a.x);
    xyz[1] = a.y + frac * (b.y - a.y);
    xyz[2] = a.z + frac * (b.z - a.z);
}
RT_D void xyz_srgb(float x, float y, float z, float o[3]) {
    o[0] = fmaxf(3.2406f * x - 1.5372f * y - 0.4986f * z, 0.0f);
    o[1] = fmaxf(-0.9689f * x + 1.8758f * y + 0.0415f * z, 0.0f);
    o[2] = fmaxf(0.0557f * x - 0.2040f * y + 1.0570f * z, 0.0f);
}
RT_D float3 spectral_to_rgb(const DevScene& S, float lambda) {
    float xyz[3], c[3];
    cmf_lerp(S, lambda, xyz);
    xyz_srgb(xyz[0], xyz[1], xyz[2], c);
    return mk(c[0] * S.norms[0], c[1] * S.norms[1], c[2] * S.norms[2]);
}
RT_D float3 spectral_fire_rgb(const DevScene& S, float lambda) {
    float xyz[3], c[3];
    cmf_lerp(S, lambda, xyz);
    float w = fmaxf(powf(xyz[1], 0.5f), 0.08f);
    xyz_srgb(xyz[0], xyz[1], xyz[2], c);
    c[0] *= w; c[1] *= w; c[2] *= w;
    float lum = 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
    for (int k = 0; k < 3; k++) c[k] = c[k] * 0.5f + lum * 0.5f;
    return mk(c[0] * S.fire_norms[0], c[1] * S.fire_norms[1], c[2] * S.fire_norms[2]);
}
RT_D float planck_raw(float l, float tk) {
    float x = 14388000.0f / (l * tk);
    float l2 = l * l, l4 = l2 * l2;
    return 1.0f / (l * l4 * fmaxf(expf(x) - 1.0f, 1e-30f));
}
RT_D void metal_ior(const DevMaterial& m, float lambda, float* n, float* k) {
    float t = clampf_((lambda - m.nk_start) / m.nk_step, 0.0f, (float)(m.nk_count - 1));
    int i = min((int)t, m.nk_count - 2);
    float f = t - (float)i;
    *n = m.nk_n[i] + f * (m.nk_n[i + 1] - m.nk_n[i]);
    *k = m.nk_k[i] + f * (m.nk_k[i + 1] - m.nk_k[i]);
}
RT_D float fresnel_conductor(float ci, float n, float k) {
    float cos2 = ci * ci, sin2 = fmaxf(1.0f - cos2, 0.0f);
    float n2 = n * n, k2 = k * k;
    float t0 = n2 - k2 - sin2;
    float ab = sqrtf(t0 * t0 + 4.0f * n2 * k2);
    float t1 = ab + cos2;
    float a = sqrtf(fmaxf(0.5f * (ab + t0), 0.0f));
    float t2 = 2.0f * ci * a;
    float rs = (t1 - t2) / fmaxf(t1 + t2, 1e-12f);
    float t3 = cos2 * ab + sin2 * sin2;
    float t4 = t2 * sin2;
    float rp = rs * (t3 - t4) / fmaxf(t3 + t4, 1e-12f);
    return clampf_(0.5f * (rp + rs), 0.0f, 1.0f);
}
RT_D float fresnel_dielectric(float ci, float eta) {
    float sin2_i = fmaxf(1.0f - ci * ci, 0.0f);
    float sin2_t = eta * eta * sin2_i;
    if (sin2_t >= 1.0f) return 1.0f;
    float ct = sqrtf(1.0f - sin2_t);
    float rs = (eta * ci - ct) / (eta * ci + ct);
    float rp = (eta * ct - ci) / (eta * ct + ci);
    return (rs * rs + rp * rp) * 0.5f;
}
// ── environment (renderer.rs:84-179) ────────────────────────────────────────
RT_D float3 env_unrot(const DevScene& S, float3 d) {
    return mk(d.x * S.env_cos_r - d.z * S.env_sin_r, d.y, d.x * S.env_sin_r + d.z * S.env_cos_r);
}
RT_D float3 env_rot(const DevScene& S, float3 d) {
    return mk(d.x * S.env_cos_r + d.z * S.env_sin_r, d.y, -d.x * S.env_sin_r + d.z * S.env_cos_r);
}
// rem_euclid(1.0): a − ⌊a⌋ is exact, so this equals the fmod form
RT_D float rem1(float a) { return a - floorf(a); }
RT_D void env_uv(const DevScene& S, float3 dir, float* u, float* v) {
    float3 d = env_unrot(S, unit3(dir));
    *u = rem1(0.5f + atan2f(d.x, d.z) / (2.0f * PI_F));
    *v = acosf(clampf_(d.y, -1.0f, 1.0f)) / PI_F;
}
RT_D float3 env_lookup_uv(const DevScene& S, float u, float v) {
    float x = u * (float)S.env_w - 0.5f, y = v * (float)S.env_h - 0.5f;
    float fx0 = floorf(x), fy0 = floorf(y);
    int x0 = (int)fx0, y0 = (int)fy0;
    float fx = x - fx0, fy = y - fy0;
    int xa = x0 % S.env_w; if (xa < 0) xa += S.env_w;
    int xb = (x0 + 1) % S.env_w; if (xb < 0) xb += S.env_w;
    int ya = min(max(y0, 0), S.env_h - 1), yb = min(max(y0 + 1, 0), S.env_h - 1);
    float4 c00 = __ldg(S.env + (size_t)ya * S.env_w + xa), c10 = __ldg(S.env + (size_t)ya * S.env_w + xb);
    float4 c01 = __ldg(S.env + (size_t)yb * S.env_w + xa), c11 = __ldg(S.env + (size_t)yb * S.env_w + xb);
    float3 a = mk(c00.x, c00.y, c00.z) * (1.0f - fx) + mk(c10.x, c10.y, c10.z) * fx;
    float3 b = mk(c01.x, c01.y, c01.z) * (1.0f - fx) + mk(c11.x, c11.y, c11.z) * fx;
    return a * (1.0f - fy) + b * fy;
}
RT_D float env_pdf_at(const DevScene& S, uint32_t k) {
    return __ldg(S.env + k).w * (float)((uint32_t)S.env_w * (uint32_t)S.env_h) * S.env_inv_total
           / (2.0f * PI_F * PI_F);
}
RT_D float3 env_lookup(const DevScene& S, float3 dir) {
    float u, v;
    env_uv(S, dir, &u, &v);
    return env_lookup_uv(S, u, v);
}
RT_D float env_pdf_uv(const DevScene& S, float u, float v) {
    int i = min((int)(u * (float)S.env_w), S.env_w - 1);
    int j = min((int)(v * (float)S.env_h), S.env_h - 1);
    i = max(i, 0); j = max(j, 0);
    return env_pdf_at(S, (uint32_t)j * S.env_w + i);
}
RT_D float env_dir_pdf(const DevScene& S, float3 dir) {
    if (!S.has_env) return 0.0f;
    float u, v;
    env_uv(S, dir, &u, &v);
    return env_pdf_uv(S, u, v);
}
// Alias-table draw with the same discrete texel distribution (lum·sinθ / Σ)
// as the reference's two-level CDF inversion, then the same sub-texel jitter.
RT_D float3 env_sample_dir(const DevScene& S, float x1, float x2, float x3, float x4, float* pdf) {
    uint32_t N = (uint32_t)S.env_w * (uint32_t)S.env_h;
    uint32_t k = min((uint32_t)(x1 * (float)N), N - 1);
    float2 pa = __ldg(S.env_alias + k);
    if (!(x2 < pa.x)) k = __float_as_uint(pa.y);
    uint32_t i = k % (uint32_t)S.env_w, j = k / (uint32_t)S.env_w;
    float u = ((float)i + x3) / (float)S.env_w;
    float v = ((float)j + x4) / (float)S.env_h;
    float sp, cp, st, ct;
    sincosf(2.0f * PI_F * (u - 0.5f), &sp, &cp);
    sincosf(PI_F * v, &st, &ct);
    *pdf = env_pdf_at(S, k);
    return env_rot(S, mk(st * sp, ct, st * cp));
}
RT_D float3 bg_type_eval(int type, const float* color, const float* top, const float* bottom, float3 dir) {
    if (type == RT_BG_SOLID) return mk(color[0], color[1], color[2]);
    float t = (clampf_(dir.y, -1.0f, 1.0f) + 1.0f) * 0.5f;
    return mk(bottom[0], bottom[1], bottom[2]) * (1.0f - t) + mk(top[0], top[1], top[2]) * t;
}
RT_D float3 bg_eval(const DevScene& S, float3 dir) {
    if (S.bg_type == RT_BG_ENVMAP) {
        if (S.vis_type >= 0) return bg_type_eval(S.vis_type, S.vis_color, S.vis_top, S.vis_bottom, dir);
        return env_lookup(S, dir);
    }
    return bg_type_eval(S.bg_type, S.bg_color, S.bg_top, S.bg_bottom, dir);
}

// ── light list (hittable.rs:156-225, quad.rs:82-96, sphere.rs:87-109) ───────
struct LRec { float t; float3 p, normal; int mat; };
RT_D bool light_hit(const DevLight& L, float3 o, float3 d, float tmin, float tmax, LRec* rec) {
    float t, a, b;
    float3 outward;
    if (L.type == RT_PRIM_QUAD) {
        if (!quad_test(L.g, o, d, tmin, tmax, &t, &a, &b)) return false;
        outward = mk(L.g[0].x, L.g[0].y, L.g[0].z);
    } else {
        if (!sphere_test(L.g[0], o, d, tmin, tmax, &t)) return false;
        outward = (ray_at(o, d, t) - mk(L.g[0].x, L.g[0].y, L.g[0].z)) / L.g[0].w;
    }
    rec->t = t;
    rec->p = ray_at(o, d, t);
    rec->normal = dot3(d, outward) < 0.0f ? outward : -outward;
    rec->mat = L.mat;
    return true;
}
RT_D bool lights_hit(const DevScene& S, float3 o, float3 d, LRec* out) {
    float closest = INFINITY;
    bool any = false;
    for (int i = 0; i < S.n_lights; i++) {
        LRec r;
        if (light_hit(S.lights[i], o, d, 0.001f, closest, &r)) { closest = r.t; *out = r; any = true; }
    }
    return any;
}
RT_D float light_pdf_value(const DevLight& L, float3 o, float3 d) {
    if (L.type == RT_PRIM_SPHERE) {
        float3 tc = mk(L.g[0].x, L.g[0].y, L.g[0].z) - o;
        float d2 = len2(tc), r2 = L.g[0].w * L.g[0].w;
        if (d2 <= r2) return 0.0f;
        float ctm = sqrtf(1.0f - r2 / d2);
        return 1.0f / (2.0f * PI_F * (1.0f - ctm));
    }
    LRec r;
    if (!light_hit(L, o, d, 0.001f, INFINITY, &r)) return 0.0f;
    float dist2 = len2(r.p - o);
    float ct = fabsf(dot3(unit3(d), r.normal));
    if (ct < 1e-8f) return 0.0f;
    return dist2 / (ct * L.g[4].z);
}
RT_D float lights_pdf_value(const DevScene& S, float3 o, float3 d) {
    if (S.n_lights == 0) return 0.0f;
    float w = 1.0f / (float)S.n_lights, sum = 0.0f;
    for (int i = 0; i < S.n_lights; i++) sum += w * light_pdf_value(S.lights[i], o, d);
    return sum;
}
RT_D float3 light_generate(const DevLight& L, float3 o, float r1, float r2) {
    if (L.type == RT_PRIM_QUAD) {
        float3 Q = mk(L.g[1].x, L.g[1].y, L.g[1].z), u = mk(L.g[1].w, L.g[2].x, L.g[2].y);
        float3 v = mk(L.g[2].z, L.g[2].w, L.g[3].x);
        return unit3((Q + r1 * u + r2 * v) - o);
    }
    float3 tc = mk(L.g[0].x, L.g[0].y, L.g[0].z) - o;
    float d2 = len2(tc), rr = L.g[0].w * L.g[0].w;
    if (d2 <= rr) return unit3(tc);
    float ctm = sqrtf(1.0f - rr / d2);
    float sphi, cphi;
    sincosf(2.0f * PI_F * r1, &sphi, &cphi);
    float ct = 1.0f - r2 * (1.0f - ctm);
    float st = sqrtf(fmaxf(1.0f - ct * ct, 0.0f));
    return onb_local_w(unit3(tc), mk(cphi * st, sphi * st, ct));
}

// ── hero-wavelength bookkeeping (see the header of the CPU checker) ─────────
enum { TINT_NONE = 0, TINT_CMF = 1, TINT_FIRE = 2 };
RT_D float3 tint_rgb(const DevScene& S, int tint, float lam) {
    return tint == TINT_CMF ? spectral_to_rgb(S, lam) : spectral_fire_rgb(S, lam);
}
RT_D float lam_k(const DevScene& S, float lam0, int k, int H) {
    // the offset lies in [0, 2·range): one conditional subtraction (exact by
    // Sterbenz's lemma) equals fmod
    float x = lam0 - S.lam_lo + (float)k * (S.lam_range / (float)H);
    return S.lam_lo + (x >= S.lam_range ? x - S.lam_range : x);
}
RT_D float3 spec_factor(const DevScene& S, int tint, float4 w, float lam0, int H) {
    float ws[4] = {w.x, w.y, w.z, w.w};
    if (tint == TINT_NONE) {
        float m = 0.0f;
        for (int i = 0; i < H; i++) m += ws[i];
        float v = m / (float)H;
        return mk(v, v, v);
    }
    float3 acc = mk(0.f, 0.f, 0.f);
    for (int i = 0; i < H; i++) if (ws[i] != 0.0f) acc = acc + tint_rgb(S, tint, lam_k(S, lam0, i, H)) * ws[i];
    return acc / (float)H;
}
RT_D float3 emission(const DevScene& S, const DevMaterial& m, int tint, float4 w, float lam0, int H) {
    if (m.type == RT_MAT_DIFFUSE_LIGHT) return mk(m.albedo[0], m.albedo[1], m.albedo[2]) * spec_factor(S, tint, w, lam0, H);
    if (m.type == RT_MAT_PBR) return mk(m.emission[0], m.emission[1], m.emission[2]) * spec_factor(S, tint, w, lam0, H);
    if (m.type == RT_MAT_BLACKBODY_LIGHT) {
        if (tint == TINT_NONE) return mk(m.bb_avg[0], m.bb_avg[1], m.bb_avg[2]) * spec_factor(S, tint, w, lam0, H);
        float ws[4] = {w.x, w.y, w.z, w.w};
        float3 acc = mk(0.f, 0.f, 0.f);
        for (int i = 0; i < H; i++) {
            if (ws[i] == 0.0f) continue;
            float l = lam_k(S, lam0, i, H);
            float sc = planck_raw(l, m.temp_k) * m.bb_norm * m.intensity;
            acc = acc + tint_rgb(S, tint, l) * (ws[i] * sc);
        }
        return acc / (float)H;
    }
    return mk(0.f, 0.f, 0.f);
}

RT_D uint32_t warp_append(uint32_t* counter, bool pred) {
    uint32_t m = __ballot_sync(__activemask(), pred);
    uint32_t lane = threadIdx.x & 31u;
    int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (m && (int)lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(__activemask(), base, leader < 0 ? 0 : leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

// Block-wide reservation in NC append-only queues: each thread asks for
// cnt[c] entries of queue c and gets its first position in off[c].  One global
// atomic per queue per call (warp scans, then a scan over the warps in shared
// memory), instead of one per warp.  Every thread of the block must call it.
template <int NC, int NW>
struct BlockQ {
    uint32_t wsum[NC][NW];
    uint32_t base[NC];
};
template <int NC, int NW>
RT_D void block_reserve(BlockQ<NC, NW>& sh, uint32_t* const (&ctr)[NC], const uint32_t (&cnt)[NC],
                        uint32_t (&off)[NC]) {
    uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) {
        uint32_t v = cnt[c];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, d);
            if (lane >= (uint32_t)d) v += t;
        }
        incl[c] = v;
        if (lane == 31) sh.wsum[c][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NC) {
        int c = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) { uint32_t t = sh.wsum[c][w]; sh.wsum[c][w] = run; run += t; }
        uint32_t* q = ctr[0];
#pragma unroll
        for (int k = 1; k < NC; k++) if (c == k) q = ctr[k];
        sh.base[c] = run ? atomicAdd(q, run) : 0u;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < NC; c++) off[c] = sh.base[c] + sh.wsum[c][warp] + incl[c] - cnt[c];
    __syncthreads();
}

}  // namespace

// ── generate ────────────────────────────────────────────────────────────────
// Camera ray of sample g of the group into path slot `pid` (Camera::get_ray,
// camera.rs:93-127, with the stratified jitter of renderer.rs:262-283).
#ifndef RT_TILE_SWIZZLE
#define RT_TILE_SWIZZLE 1
#endif
// Generation order of the pixels: 8×4 tiles, tiles row by row, so a warp's 32
// camera rays cover a compact tile (coherent traversal) rather than a 32-pixel
// strip.  A bijection of 0 .. W·H−1 for any W, H (edge tiles are smaller).
RT_D uint32_t tile_order_pixel(uint32_t j, uint32_t W, uint32_t H) {
#if RT_TILE_SWIZZLE
    uint32_t band = j / (W * 4u);
    uint32_t hb = min(4u, H - band * 4u);
    uint32_t idx = j - band * W * 4u;
    uint32_t chunk = idx / (8u * hb);
    uint32_t wc = min(8u, W - chunk * 8u);
    uint32_t rem = idx - chunk * 8u * hb;
    uint32_t row = rem / wc, col = rem - row * wc;
    return (band * 4u + row) * W + chunk * 8u + col;
#else
    (void)W; (void)H;
    return j;
#endif
}

// The request of a packed batch that cursor value g belongs to (the last
// whose first ≤ g)
RT_D uint32_t batch_job(const RenderLaunch& R, uint64_t g) {
    uint32_t lo = 0, hi = R.n_jobs - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (R.jobs[mid].first <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

RT_D void init_path(const DevScene& S, const PathState& P, const RenderLaunch& R, uint32_t pid, uint64_t g) {
    uint32_t job = 0, width = R.width, height = R.height, nact = R.nactive, strata = R.strata;
    uint32_t sample0 = R.sample_idx;
    uint64_t seed = R.seed;
    const RtCamera* cp = &R.cam;
    if (R.n_jobs) {
        job = batch_job(R, g);
        const JobDev& J = R.jobs[job];
        g -= J.first;
        width = J.width; height = J.height; nact = J.npix; strata = J.strata;
        sample0 = J.sample_idx; seed = J.seed; cp = &J.cam;
    }
    uint32_t k = (uint32_t)(g / nact), j = (uint32_t)(g - (uint64_t)k * nact);
    uint32_t i = R.active ? __ldg(R.active + j) : tile_order_pixel(j, width, height);
    uint32_t row = i / width, col = i - row * width;
    uint32_t sample = sample0 + k;
    P.L[pid] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pend0[pid] = make_float4(0.f, 0.f, 0.f, 0.f);
    P.pend1[pid] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (R.photons) P.pendC[pid] = make_float4(0.f, 0.f, 0.f, 0.f);
    Rng rng = make_rng(seed, i, sample);
    float wd = (float)max(width - 1u, 1u), hd = (float)max(height - 1u, 1u);
    uint32_t s2 = strata * strata, ray_y = height - 1u - row;
    float uj, vj;
    if (s2 > 0) {
        uint32_t off = (i * 0x9E3779B9u) % s2;
        uint32_t si = (sample + off) % s2;
        uj = ((float)(si % strata) + rnd(rng, D_JIT_U)) / (float)strata;
        vj = ((float)(si / strata) + rnd(rng, D_JIT_V)) / (float)strata;
    } else {
        uj = rnd(rng, D_JIT_U); vj = rnd(rng, D_JIT_V);
    }
    float u = ((float)col + uj) / wd, v = ((float)ray_y + vj) / hd;
    const RtCamera& c = *cp;
    float3 cu = mk(c.u[0], c.u[1], c.u[2]), cv = mk(c.v[0], c.v[1], c.v[2]);
    float3 org = mk(c.origin[0], c.origin[1], c.origin[2]);
    float3 rd;
    if (c.aperture_blades >= 3) {
        // sample_polygon (camera.rs:66-79): a fan wedge of the N-gon, then a folded
        // uniform triangle sample
        float nb = (float)c.aperture_blades, rot = PI_F / nb;
        float k = (float)(rnd_u32(rng, D_LENS_K) % (uint32_t)c.aperture_blades);
        float s1, c1, s2, c2;
        sincosf(2.0f * PI_F * k / nb + rot, &s1, &c1);
        sincosf(2.0f * PI_F * (k + 1.0f) / nb + rot, &s2, &c2);
        float r1 = rnd(rng, D_LENS_R), r2 = rnd(rng, D_LENS_P);
        if (r1 + r2 > 1.0f) { r1 = 1.0f - r1; r2 = 1.0f - r2; }
        rd = c.lens_radius * (mk(c1, s1, 0.0f) * r1 + mk(c2, s2, 0.0f) * r2);
    } else {
        float lr = sqrtf(rnd(rng, D_LENS_R));
        float ls, lc;
        sincosf(2.0f * PI_F * rnd(rng, D_LENS_P), &ls, &lc);
        rd = c.lens_radius * mk(lr * lc, lr * ls, 0.0f);
    }
    float3 off = cu * rd.x + cv * rd.y;
    float3 ll = mk(c.lower_left[0], c.lower_left[1], c.lower_left[2]);
    float3 hz = mk(c.horizontal[0], c.horizontal[1], c.horizontal[2]);
    float3 vt = mk(c.vertical[0], c.vertical[1], c.vertical[2]);
    float3 o = org + off;
    float3 d = ll + u * hz + v * vt - org - off;
    int H = (int)R.hero;
    float lam0 = S.lam_lo + S.lam_range * rnd(rng, D_LAMBDA);
    if (lam0 >= S.lam_lo + S.lam_range) lam0 = nextafterf(S.lam_lo + S.lam_range, 0.0f);
    P.ray_o[pid] = make_float4(o.x, o.y, o.z, 0.f);
    P.ray_d[pid] = make_float4(d.x, d.y, d.z, 0.f);
    P.thr[pid] = make_float4(1.f, 1.f, 1.f, 1.f);
    P.wts[pid] = make_float4(1.f, H > 1 ? 1.f : 0.f, H > 2 ? 1.f : 0.f, H > 3 ? 1.f : 0.f);
    P.meta[pid] = make_uint4(i, k, PF_PREV_SPEC | (H > 1 ? PF_SEC_ALIVE : 0u) | (job << PF_JOB_SHIFT),
                             __float_as_uint(lam0));
    if (R.guide.mode == 2) P.rec[pid] = rtg::REC_NONE;
}

__global__ void k_generate(DevScene S, PathState A, const RenderLaunch* __restrict__ Rp, uint32_t* count0) {
    const RenderLaunch& R = *Rp;
    const uint32_t pool = R.pool;
    if (blockIdx.x == 0 && threadIdx.x == 0) { *R.gen_next = pool; *count0 = pool; }
    for (uint32_t pid = blockIdx.x * blockDim.x + threadIdx.x; pid < pool; pid += gridDim.x * blockDim.x)
        init_path(S, A, R, pid, pid);
}

// ── retire + refill ─────────────────────────────────────────────────────────
// An ended path folds its last parked contributions (caustic, area-light NEE,
// env NEE — the order of renderer.rs:461-540) and writes its sample; for each
// ended path the next ungenerated sample, if any, is appended to the next set.
#define RETIRE_BLOCK 256
__global__ void __launch_bounds__(RETIRE_BLOCK) k_retire(DevScene S, PathState B, PathState Rt,
                                                         const RenderLaunch* __restrict__ Rp, uint32_t* ctr,
                                                         uint32_t* hdr, uint32_t* clear_block, uint32_t* cout) {
    const RenderLaunch& R = *Rp;
    __shared__ BlockQ<1, RETIRE_BLOCK / 32> shq;
    __shared__ unsigned long long gbase;
    uint32_t n = ctr[CTR_RETIRE_COUNT];
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) {
            atomicAdd((unsigned long long*)(hdr + HDR_EXT), (unsigned long long)ctr[CTR_COUNT]);
            atomicAdd((unsigned long long*)(hdr + HDR_SHADOW), (unsigned long long)ctr[CTR_SHADOW_COUNT]);
        }
        if (threadIdx.x < RT_CTR_STRIDE) clear_block[threadIdx.x] = 0u;
    }
    uint32_t* qctr[1] = {cout};
    for (uint32_t t0 = blockIdx.x * RETIRE_BLOCK; t0 < n; t0 += gridDim.x * RETIRE_BLOCK) {
        uint32_t j = t0 + threadIdx.x;
        bool act = j < n;
        if (act) {
            float4 L = Rt.L[j], a = Rt.pend0[j], b = Rt.pend1[j];
            if (R.photons) { float4 c = Rt.pendC[j]; L.x += c.x; L.y += c.y; L.z += c.z; }
            L.x += a.x; L.y += a.y; L.z += a.z;
            L.x += b.x; L.y += b.y; L.z += b.z;
            uint4 meta = Rt.meta[j];
            float* out;
            if (R.n_jobs) {
                const JobDev& J = R.jobs[meta.z >> PF_JOB_SHIFT];
                out = J.scratch + ((size_t)meta.y * J.npix + meta.x) * 3;
            } else {
                out = R.scratch + ((size_t)meta.y * R.npix + meta.x) * 3;
            }
            out[0] = L.x; out[1] = L.y; out[2] = L.z;
            if (R.guide.mode == 2) {
                // weights of the path's guide records: radiance gathered after
                // each vertex over the throughput there
                float sl = L.x + L.y + L.z;
                uint32_t r = Rt.rec[j];
                for (int k = 0; k < RT_MAX_DEPTH && r != rtg::REC_NONE; k++) {
                    float base = R.guide.rec_b[r].w, ts = R.guide.rec_a[r].w;
                    if (base >= 0.0f && ts > 0.0f) R.guide.rec_w[r] = fmaxf(sl - base, 0.0f) / ts;
                    r = __float_as_uint(R.guide.rec_c[r].w);
                }
            }
        }
        // one claim of new samples per block: the tile's ended paths are
        // t0 .. t0 + min(n − t0, RETIRE_BLOCK) − 1, in thread order
        uint32_t tile_n = min(n - t0, (uint32_t)RETIRE_BLOCK);
        if (threadIdx.x == 0) gbase = atomicAdd(R.gen_next, (unsigned long long)tile_n);
        __syncthreads();
        uint64_t g = gbase + threadIdx.x;
        bool fresh = act && g < R.total;
        uint32_t cnt[1] = {fresh}, off[1];
        block_reserve(shq, qctr, cnt, off);
        if (fresh) init_path(S, B, R, off[0], g);
    }
}

// ── converged pixels ─────────────────────────────────────────────────────────
__global__ void k_active_list(const uint8_t* __restrict__ conv, uint32_t W, uint32_t H, uint32_t* list,
                              uint32_t* count) {
    uint32_t npix = W * H;
    for (uint32_t b0 = blockIdx.x * blockDim.x; b0 < npix; b0 += gridDim.x * blockDim.x) {
        uint32_t j = b0 + threadIdx.x;
        uint32_t i = j < npix ? tile_order_pixel(j, W, H) : 0u;
        bool a = j < npix && !conv[i];
        uint32_t slot = warp_append(count, a);
        if (a) list[slot] = i;
    }
}

__global__ void k_zero_converged(const uint8_t* __restrict__ conv, uint32_t npix, uint32_t nsamp, float* scratch) {
    uint64_t total = (uint64_t)npix * nsamp;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t i = (uint32_t)(e % npix);
        if (conv[i]) { float* o = scratch + e * 3; o[0] = 0.f; o[1] = 0.f; o[2] = 0.f; }
    }
}

// ── classify: bin the paths of this bounce by material class ────────────────
// Warp-aggregated appends (ballot + popc + one atomic per class per warp) into
// one queue per class, so each shading kernel below runs one material's code:
// no divergence between materials and a much smaller instruction footprint.
// Sun NEE at a diffuse vertex (renderer.rs:495-518): the parked contribution
// with the occlusion test still to do.
// `gp`: the guide mixture of a guided bounce (its density replaces the cosine
// lobe's in the MIS weight), or null.
RT_D bool sun_nee_diffuse(const DevScene& S, float3 p, float3 nrm, float3 T_att, float3 sf,
                                             float r1, float r2, float3* dir, float3* c, const float4* gp = nullptr) {
    float3 sun_s = sample_sun_cone(S.sun_dir, r1, r2);
    float3 su = unit3(sun_s);
    float brdf = fmaxf(dot3(nrm, su) / PI_F, 0.0f);
    if (!(brdf > 0.0f)) return false;
    float3 sun_color = preetham_sky(sun_s, S.sun_dir, S.turbidity) * sf;
    float area_pdf = S.n_lights > 0 ? lights_pdf_value(S, p, sun_s) : 0.0f;
    float pb = gp ? rtg::guide_pdf(gp, nrm.x, nrm.y, nrm.z, su.x, su.y, su.z) : brdf;
    float mis_d = SUN_PDF * SUN_PDF + pb * pb + area_pdf * area_pdf;
    *c = T_att * brdf * SUN_PDF * sun_color / mis_d;
    *dir = sun_s;
    return true;
}

// Specular sun NEE at a rough conductor (renderer.rs:421-456) with the
// conductor's specular_brdf_cos / specular_sampling_pdf (material.rs:504-551),
// per hero wavelength; also the MIS weight of the sampled bounce against the sun.
RT_D bool sun_nee_conductor(const DevScene& S, const DevMaterial& m, float3 p, float3 nrm,
                                               float3 wo, float3 dir, float cos_o, float alpha, float3 T, float4 w,
                                               int tint, float lam0, int H, float r1, float r2, float3* sdir,
                                               float3* c, float* sun_w) {
    bool park = false;
    float3 sun_s = sample_sun_cone(S.sun_dir, r1, r2);
    float cos_i = dot3(sun_s, nrm);
    if (cos_i > 0.0f) {
        float3 hh = unit3(wo + sun_s);
        float wo_h = fmaxf(dot3(wo, hh), 0.0f), h_n = fmaxf(dot3(hh, nrm), 0.0f);
        float base = ggx_ndf(h_n, alpha) * (1.0f / (1.0f + smith_lambda(cos_o, alpha) + smith_lambda(cos_i, alpha)));
        float comp = fminf(1.0f / fmaxf(e_ss_lut(S, cos_o, alpha), 0.05f), 10.0f);
        float wv[4] = {w.x, w.y, w.z, w.w};
        for (int i = 0; i < H; i++) {
            if (wv[i] == 0.0f) continue;
            float nn, kk;
            metal_ior(m, lam_k(S, lam0, i, H), &nn, &kk);
            wv[i] *= base * fresnel_conductor(wo_h, nn, kk) / (4.0f * cos_o) * comp;
        }
        float3 brdf_cos = spec_factor(S, tint == TINT_NONE ? TINT_CMF : tint,
                                      make_float4(wv[0], wv[1], wv[2], wv[3]), lam0, H);
        if (brdf_cos.x > 0.0f || brdf_cos.y > 0.0f || brdf_cos.z > 0.0f) {
            float p_mat = ggx_ndf(h_n, alpha) * smith_g1(cos_o, alpha) / (4.0f * cos_o);
            float mis_d = SUN_PDF * SUN_PDF + p_mat * p_mat;
            if (mis_d > 0.0f) {
                *c = T * brdf_cos * preetham_sky(sun_s, S.sun_dir, S.turbidity) * SUN_PDF / mis_d;
                *sdir = sun_s;
                park = true;
            }
        }
    }
    float3 hb = unit3(wo + dir);
    float p_b = ggx_ndf(fmaxf(dot3(hb, nrm), 0.0f), alpha) * smith_g1(cos_o, alpha) / (4.0f * cos_o);
    *sun_w = p_b > 0.0f ? (p_b * p_b) / fmaxf(p_b * p_b + SUN_PDF * SUN_PDF, 1e-8f) : 1.0f;
    return park;
}

RT_D int material_class(uint32_t ref) {
    if (ref == RT_MISS_REF) return CLS_MISS;
    return hit_is_medium(ref) ? CLS_MEDIUM : CLS_EMIT + (int)RT_HIT_CODE(ref);
}

#define CLS_BLOCK 256
#define CLS_ITEMS 4
__global__ void __launch_bounds__(CLS_BLOCK) k_classify(const float4* __restrict__ hit, const uint32_t* cin,
                                                        ClassQueues Q, uint32_t* cls_count) {
    __shared__ BlockQ<CLS_N, CLS_BLOCK / 32> shq;
    uint32_t* qctr[CLS_N];
#pragma unroll
    for (int c = 0; c < CLS_N; c++) qctr[c] = cls_count + c;
    uint32_t n = *cin;
    const uint32_t tile = CLS_BLOCK * CLS_ITEMS;
    for (uint32_t t0 = blockIdx.x * tile; t0 < n; t0 += gridDim.x * tile) {
        // CLS_ITEMS consecutive paths per thread, so each class queue lists
        // neighbouring paths next to each other
        uint32_t i0 = t0 + threadIdx.x * CLS_ITEMS;
        int cls[CLS_ITEMS];
        uint32_t cnt[CLS_N], off[CLS_N];
#pragma unroll
        for (int c = 0; c < CLS_N; c++) cnt[c] = 0;
#pragma unroll
        for (int k = 0; k < CLS_ITEMS; k++) {
            uint32_t i = i0 + k;
            cls[k] = i < n ? material_class(__float_as_uint(__ldg(reinterpret_cast<const float*>(hit + i)))) : -1;
#pragma unroll
            for (int c = 0; c < CLS_N; c++) cnt[c] += cls[k] == c;
        }
        block_reserve(shq, qctr, cnt, off);
#pragma unroll
        for (int k = 0; k < CLS_ITEMS; k++) {
#pragma unroll
            for (int c = 0; c < CLS_N; c++)
                if (cls[k] == c) Q.q[c][off[c]++] = i0 + k;
        }
    }
}

// ── shade: one bounce of ray_color for the paths of one material class ───────
struct Surf { float3 p, nrm; float t; bool front; int mat; };

RT_D Surf surface(const DevScene& S, float4 hv, float3 o, float3 d) {
    Surf r;
    uint32_t ref = __float_as_uint(hv.x);
    r.t = hv.y;
    r.p = ray_at(o, d, r.t);
    uint32_t type = RT_HIT_TYPE(ref), idx = RT_HIT_INDEX(ref);
    float3 outward;
    if (type == RT_PRIM_TRI) {                                                      // triangle.rs:91-108
        const float4* g = S.tri + (size_t)idx * 3;
        float4 ga = __ldg(g), gb = __ldg(g + 1), gc = __ldg(g + 2);
        float3 e1 = mk(ga.w, gb.x, gb.y), e2 = mk(gb.z, gb.w, gc.x);
        r.mat = __float_as_int(gc.z);
        if (__float_as_int(gc.w)) {
            const float4* gn = S.tri_n + (size_t)idx * 3;
            float4 na = __ldg(gn), nb = __ldg(gn + 1), nc = __ldg(gn + 2);
            float b1 = hv.z, b2 = hv.w, b0 = 1.0f - b1 - b2;
            float3 sn = b0 * mk(na.x, na.y, na.z) + b1 * mk(na.w, nb.x, nb.y) + b2 * mk(nb.z, nb.w, nc.x);
            outward = len2(sn) > 1e-12f ? unit3(sn) : unit3(cross3(e1, e2));
        } else {
            outward = unit3(cross3(e1, e2));
        }
    } else if (type == RT_PRIM_QUAD) {                                              // quad.rs:53-56
        const float4* g = S.quad + (size_t)idx * 5;
        float4 g0 = __ldg(g);
        outward = mk(g0.x, g0.y, g0.z);
        r.mat = __float_as_int(__ldg(g + 4).y);
    } else if (type == RT_PRIM_SPHERE) {                                            // sphere.rs:62-68
        const float4* g = S.sphere + (size_t)idx * 2;
        float4 s0 = __ldg(g);
        outward = (r.p - mk(s0.x, s0.y, s0.z)) / s0.w;
        r.mat = __float_as_int(__ldg(g + 1).y);
    } else {                                                                        // diamond.rs:257-275
        float4 c0 = __ldg(S.cvx + (size_t)idx * 2);
        int cnt = __float_as_int(c0.y);
        if (cnt < 0) {                                                              // cylinder, cone, disk, plane
            r.mat = __float_as_int(c0.z);
            r.nrm = shape_normal(-1 - cnt, S.shape_par + __float_as_int(c0.x), o, d, r.t, __float_as_int(hv.z),
                                 &r.front);
            return r;
        }
        int pi = max(__float_as_int(hv.z), 0);
        int wp = __float_as_int(c0.x) + pi;
        float4 q = __ldg(S.cvx_planes + wp);
        outward = mk(q.x, q.y, q.z);
        r.mat = __float_as_int(c0.z);
        r.front = dot3(d, outward) < 0.0f;
        float4 sn = __ldg(S.cvx_shade + (size_t)wp * 2 + (r.front ? 0 : 1));   // polished facet normal, world space
        r.nrm = mk(sn.x, sn.y, sn.z);
        return r;
    }
    r.front = dot3(d, outward) < 0.0f;                                              // hittable.rs:89-93
    r.nrm = r.front ? outward : -outward;
    return r;
}

// SKY: the scene has a Physical sky (Preetham background, sun NEE); the other
// instantiation leaves that code out so env-map and plain scenes keep their
// registers.
// GUIDE (diffuse class only): bounces drawn from the guide mixture.
// Resident blocks per SM the shading kernels are compiled for: 8 (64
// registers).  Diffuse shading, the busiest class, spills some there and still
// measured fastest (icosphere shade 26.3 ms against 26.4 at 127 registers and
// 26.5 at 80; box frame 1.285 ms against 1.30 and 1.33); the conductor and
// miss classes fit without spilling (icosphere shade 24.5 ms against 26.1 at
// 4 blocks).  PBR, which would spill half a kilobyte per thread at 64, stays at
// 4 (≤ 128 registers).  An explicit bound of 1 lets ptxas take more registers
// than its plain heuristic and cost 15 % of the shading time.
#ifndef RT_SHADE_MINB
#define RT_SHADE_MINB 8
#endif
#ifndef RT_SHADE_PBR_MINB
#define RT_SHADE_PBR_MINB 4
#endif
template <int CLS, bool SKY, bool GUIDE>
__global__ void __launch_bounds__(RT_SHADE_BLOCK, CLS == CLS_PBR ? RT_SHADE_PBR_MINB : RT_SHADE_MINB)
k_shade(DevScene S, PathState A, PathState B, PathState Rt,
                                                          const RenderLaunch* __restrict__ Rp,
                                                          const uint32_t* __restrict__ qin, const uint32_t* cin,
                                                          uint32_t* cout, float4* __restrict__ sq, uint32_t* ctr) {
    const RenderLaunch& R = *Rp;
    // queues appended to: [next set, retire records, gather requests, shadow rays]
    constexpr int NQ = (CLS == CLS_DIFFUSE || CLS == CLS_METAL || CLS == CLS_PBR) ? 4
                     : (CLS == CLS_MISS || CLS == CLS_EMIT) ? 1 : 2;
    __shared__ BlockQ<NQ, RT_SHADE_BLOCK / 32> shq;
    uint32_t* qctr[NQ];
    if constexpr (NQ == 1) {
        qctr[0] = ctr + CTR_RETIRE_COUNT;
    } else {
        qctr[0] = cout;
        qctr[1] = ctr + CTR_RETIRE_COUNT;
        if constexpr (NQ == 4) { qctr[2] = ctr + CTR_GATHER_COUNT; qctr[3] = ctr + CTR_SHADOW_COUNT; }
    }
    uint32_t n = *cin;
    int H = (int)R.hero;
    bool have_lights = S.n_lights > 0;
    // static tiles of one path per thread (the cost per path of one class is even)
    for (uint32_t t0 = blockIdx.x * RT_SHADE_BLOCK; t0 < n; t0 += gridDim.x * RT_SHADE_BLOCK) {
        uint32_t qi = t0 + threadIdx.x;
        bool active = qi < n;
        uint32_t pid = active ? qin[qi] : 0u;
        bool cont = false, sh0 = false, sh1 = false, gath = false;
        float4 sh0a, sh0b, sh1a, sh1b, ga, gb;
        const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
        float4 np0 = zero4, np1 = zero4, npc = zero4;     // contributions parked this bounce
        float4 Lout = zero4, o_out = zero4, d_out = zero4, thr_out = zero4, w_out = zero4;
        uint4 meta = make_uint4(0u, 0u, 0u, 0u);
        uint32_t head = rtg::REC_NONE;   // newest guide record of the path
        if (active) {
            meta = A.meta[pid];
            float4 thr = A.thr[pid], w = A.wts[pid], L = A.L[pid];
            float4 p0 = A.pend0[pid], p1 = A.pend1[pid];
            // fold the previous bounce's parked contributions in the reference's
            // order: caustic injection, area-light NEE, env NEE (renderer.rs:461-540)
            if (R.photons) {
                float4 pc = A.pendC[pid];
                L.x += pc.x; L.y += pc.y; L.z += pc.z;
            }
            L.x += p0.x; L.y += p0.y; L.z += p0.z;
            L.x += p1.x; L.y += p1.y; L.z += p1.z;
            float4 ro = A.ray_o[pid], rdv = A.ray_d[pid];
            float3 o = mk(ro.x, ro.y, ro.z), d = mk(rdv.x, rdv.y, rdv.z);
            float3 T = mk(thr.x, thr.y, thr.z);
            float prev_mis = thr.w;
            uint32_t flags = meta.z;
            uint32_t depth = flags & PF_DEPTH_MASK;
            bool prev_spec = flags & PF_PREV_SPEC;
            int tint = (flags & PF_TINT_MASK) >> PF_TINT_SHIFT;
            float lam0 = __uint_as_float(meta.w);
            Rng rng = R.n_jobs ? make_rng(R.jobs[meta.z >> PF_JOB_SHIFT].seed, meta.x,
                                          R.jobs[meta.z >> PF_JOB_SHIFT].sample_idx + meta.y)
                               : make_rng(R.seed, meta.x, R.sample_idx + meta.y);
            uint32_t b = D_BOUNCE0 + depth * D_PER_BOUNCE;
            float3 Lc = mk(L.x, L.y, L.z);
            if (R.guide.mode == 2) {
                // the previous guided vertex's own estimates are folded: what the
                // path gathers from here on arrives along that vertex's bounce
                head = A.rec[pid];
                if (flags & PF_REC_OPEN) {
                    reinterpret_cast<float*>(R.guide.rec_b + head)[3] = L.x + L.y + L.z;
                    flags &= ~PF_REC_OPEN;
                }
            }
            if (CLS == CLS_MISS) {                                                  // renderer.rs:381-403
                float env_pdf = 0.0f;
                float3 bg;
                if (S.has_env) {
                    float u, v;
                    env_uv(S, d, &u, &v);
                    env_pdf = env_pdf_uv(S, u, v);
                    bg = (depth == 0 && S.vis_type >= 0) ? bg_type_eval(S.vis_type, S.vis_color, S.vis_top,
                                                                        S.vis_bottom, d)
                                                         : env_lookup_uv(S, u, v);
                } else {
                    bg = bg_eval(S, d);
                }
                // prev_mis holds the specular-bounce sun weight after a specular vertex
                float sun_pdf = 0.0f;
                if constexpr (SKY) {
                    sun_pdf = sun_pdf_value(S, d);
                    bg = preetham_sky(d, S.sun_dir, S.turbidity);
                }
                float emit_w = (sun_pdf + env_pdf == 0.0f) ? 1.0f : prev_mis;
                Lc = Lc + T * (bg * spec_factor(S, tint, w, lam0, H)) * R.bg_scale * emit_w;
            } else if (CLS == CLS_EMIT) {                                           // renderer.rs:415-419
                float4 hv = A.hit[pid];
                uint32_t ref = __float_as_uint(hv.x), type = RT_HIT_TYPE(ref), idx = RT_HIT_INDEX(ref);
                int mat = type == RT_PRIM_TRI ? __float_as_int(__ldg(S.tri + (size_t)idx * 3 + 2).z)
                        : type == RT_PRIM_QUAD ? __float_as_int(__ldg(S.quad + (size_t)idx * 5 + 4).y)
                                               : __float_as_int(__ldg(S.sphere + (size_t)idx * 2 + 1).y);
                float emit_w = (prev_spec || !have_lights) ? 1.0f : prev_mis;
                Lc = Lc + T * emission(S, S.mats[mat], tint, w, lam0, H) * emit_w;
            } else {
                bool alive = true;
                float3 sf = mk(1.f, 1.f, 1.f);
                if constexpr (CLS == CLS_MEDIUM) {
                    // medium scatter: HenyeyGreenstein::scatter (volume.rs:29-35), a
                    // skip_pdf bounce of the specular branch (renderer.rs:421-456)
                    float4 hv = A.hit[pid];
                    const DevMedium& M = S.media[RT_HIT_INDEX(__float_as_uint(hv.x))];
                    float3 p = ray_at(o, d, hv.y);
                    float3 dir = hg_sample(unit3(d), M.g, rnd(rng, b + B_SCATTER0), rnd(rng, b + B_SCATTER1));
                    T = T * M.color;
                    o = p; d = dir;
                    prev_spec = true; prev_mis = 1.0f;
                } else {
                float4 hv = A.hit[pid];
                Surf sf_ = surface(S, hv, o, d);
                float3 p = sf_.p, nrm = sf_.nrm;
                float t = sf_.t;
                bool front = sf_.front;
                const DevMaterial& m = S.mats[sf_.mat];
                float3 udir = unit3(d);
                if (CLS == CLS_DIELEC) {                                            // material.rs:133-149, 369-402
                    bool spectral = m.type == RT_MAT_SPECTRAL_DIELECTRIC;
                    float ior = spectral ? m.cauchy_b + m.cauchy_c / ((lam0 * 1e-3f) * (lam0 * 1e-3f)) : m.cauchy_b;
                    if (spectral && H > 1 && m.cauchy_c != 0.0f && (flags & PF_SEC_ALIVE)) {
                        w = make_float4(w.x * (float)H, 0.f, 0.f, 0.f);
                        flags &= ~PF_SEC_ALIVE;
                    }
                    float ratio = front ? 1.0f / ior : ior;
                    float ct = fminf(dot3(-udir, nrm), 1.0f);
                    float st = sqrtf(1.0f - ct * ct);
                    bool refl = ratio * st > 1.0f || fresnel_dielectric(ct, ratio) > rnd(rng, b + B_SCATTER0);
                    float3 dir;
                    if (refl) {
                        dir = reflect3(udir, nrm);
                    } else {
                        float c2 = fminf(dot3(-udir, nrm), 1.0f);
                        float3 perp = ratio * (udir + c2 * nrm);
                        float kk = 1.0f - len2(perp);
                        dir = kk < 0.0f ? reflect3(udir, nrm) : perp + (-sqrtf(kk) * nrm);
                    }
                    float3 att = mk(1.f, 1.f, 1.f);
                    if (spectral) {
                        if (tint == TINT_NONE && !refl) tint = TINT_FIRE;
                        if (!front) {
                            att.x *= expf(-m.absorption[0] * t);
                            att.y *= expf(-m.absorption[1] * t);
                            att.z *= expf(-m.absorption[2] * t);
                        }
                    }
                    T = T * att;
                    o = p; d = dir;
                    prev_spec = true; prev_mis = 1.0f;
                } else if (CLS == CLS_METAL) {                                      // material.rs:449-500
                    float3 wo = unit3(-d);
                    float cos_o = dot3(wo, nrm);
                    float alpha = fmaxf(m.roughness * m.roughness, 1e-4f);
                    float3 dir;
                    float cos_h;
                    if (cos_o <= 0.0f) {
                        alive = false;
                    } else if (m.roughness == 0.0f) {
                        dir = reflect3(udir, nrm);
                        cos_h = cos_o;
                    } else {
                        float3 up = fabsf(nrm.y) < 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
                        float3 tt = unit3(cross3(nrm, up));
                        float3 bb = cross3(nrm, tt);
                        float3 wo_ts = mk(dot3(wo, tt), dot3(wo, bb), cos_o);
                        float3 mts = vndf_sample(wo_ts, alpha, alpha, rnd(rng, b + B_SCATTER0), rnd(rng, b + B_SCATTER1));
                        float3 mm = unit3(tt * mts.x + bb * mts.y + nrm * mts.z);
                        float vo_h = fmaxf(dot3(wo, mm), 0.0f);
                        dir = unit3(2.0f * vo_h * mm - wo);
                        cos_h = vo_h;
                        if (dot3(dir, nrm) <= 0.0f) alive = false;
                    }
                    if (alive && dot3(dir, nrm) <= 0.0f) alive = false;
                    if (alive) {
                        float weight = 1.0f;
                        if (m.roughness != 0.0f) {
                            float lo = smith_lambda(cos_o, alpha);
                            float li = smith_lambda(fmaxf(dot3(dir, nrm), 0.0f), alpha);
                            float ec = fminf(1.0f / fmaxf(e_ss_lut(S, cos_o, alpha), 0.05f), 10.0f);
                            weight = ((1.0f + lo) / (1.0f + lo + li)) * ec;
                        }
                        float ws[4] = {w.x, w.y, w.z, w.w};
                        for (int i = 0; i < H; i++) {
                            if (ws[i] == 0.0f) continue;
                            float nn, kk;
                            metal_ior(m, lam_k(S, lam0, i, H), &nn, &kk);
                            ws[i] *= fresnel_conductor(cos_h, nn, kk);
                        }
                        // specular sun NEE (renderer.rs:421-456) with the conductor's
                        // specular_brdf_cos / specular_sampling_pdf (material.rs:504-551)
                        float sun_w = 1.0f;
                        if (SKY && S.has_sun && m.roughness != 0.0f) {
                            float3 sun_s, c;
                            if (sun_nee_conductor(S, m, p, nrm, wo, dir, cos_o, alpha, T, w, tint, lam0, H,
                                                  rnd(rng, b + B_SUN0), rnd(rng, b + B_SUN1), &sun_s, &c, &sun_w)) {
                                np0 = make_float4(c.x, c.y, c.z, 0.f);
                                sh0 = true;
                                sh0a = make_float4(p.x, p.y, p.z, INFINITY);
                                sh0b = make_float4(sun_s.x, sun_s.y, sun_s.z, 0.f);
                            }
                        }
                        w = make_float4(ws[0], ws[1], ws[2], ws[3]);
                        if (tint == TINT_NONE) tint = TINT_CMF;
                        T = T * weight;
                        o = p; d = dir;
                        prev_spec = true; prev_mis = sun_w;
                    }
                } else {                                                            // renderer.rs:405-572
                    sf = spec_factor(S, tint, w, lam0, H);
                    float3 att, hint;       // the scatter attenuation and the caustic albedo hint
                    float3 sn = nrm;        // the shading normal (a PBR normal map tilts it)
                    bool diffuse = true;
                    if constexpr (CLS == CLS_PBR) {
                        // PbrMaterial: its emission adds at the hit (renderer.rs:415-417),
                        // then one lobe scatters (material.rs:790-920)
                        float emit_w = (prev_spec || !have_lights) ? 1.0f : prev_mis;
                        Lc = Lc + T * (mk(m.emission[0], m.emission[1], m.emission[2]) * sf) * emit_w;
                        PbrHit ph = pbr_scalars(m);
                        if (pbr_textured(m))
                            ph = pbr_hit(S, m, hit_uv(S, hv, front ? nrm : -nrm), nrm, &sn);
                        float3 wo = unit3(-d), dir;
                        int lobe = pbr_scatter(S, m, ph, wo, sn, rnd(rng, b + B_LOBE0), rnd(rng, b + B_LOBE1),
                                               rnd(rng, b + B_SCATTER0), rnd(rng, b + B_SCATTER1), &att, &dir);
                        hint = ph.albedo;
                        if (lobe != PBR_DIFFUSE) diffuse = false;
                        if (lobe == PBR_NONE) alive = false;
                        if (lobe == PBR_SPECULAR) {
                            // specular sun NEE (renderer.rs:421-456) with the PBR lobes'
                            // specular_brdf_cos / specular_sampling_pdf
                            float sun_w = 1.0f;
                            if (SKY && S.has_sun) {
                                float3 sun_s = sample_sun_cone(S.sun_dir, rnd(rng, b + B_SUN0), rnd(rng, b + B_SUN1));
                                float p_mat;
                                float3 bc = pbr_spec_brdf_cos(S, m, ph, wo, sn, sun_s, &p_mat);
                                if (bc.x > 0.0f || bc.y > 0.0f || bc.z > 0.0f) {
                                    float mis_d = SUN_PDF * SUN_PDF + p_mat * p_mat;
                                    if (mis_d > 0.0f) {
                                        float3 c = T * bc * (preetham_sky(sun_s, S.sun_dir, S.turbidity) * sf) *
                                                   SUN_PDF / mis_d;
                                        np0 = make_float4(c.x, c.y, c.z, 0.f);
                                        sh0 = true;
                                        sh0a = make_float4(p.x, p.y, p.z, INFINITY);
                                        sh0b = make_float4(sun_s.x, sun_s.y, sun_s.z, 0.f);
                                    }
                                }
                                float p_b = pbr_spec_pdf(S, m, ph, wo, sn, dir);
                                if (p_b > 0.0f) sun_w = (p_b * p_b) / fmaxf(p_b * p_b + SUN_PDF * SUN_PDF, 1e-8f);
                            }
                            T = T * att;
                            o = p; d = dir;
                            prev_spec = true; prev_mis = sun_w;
                        }
                    } else {
                        att = mk(m.albedo[0], m.albedo[1], m.albedo[2]);
                        if (m.albedo_tex) {                                         // texture.rs Image / Mottle
                            HitUV uv = hit_uv(S, hv, front ? nrm : -nrm);
                            att = tex_value(S, m.albedo_tex, uv.u, uv.v, p);
                        }
                        if (m.type == RT_MAT_CHECKER) {
                            int xi = (int)floorf(m.checker_scale * p.x), yi = (int)floorf(m.checker_scale * p.y);
                            int zi = (int)floorf(m.checker_scale * p.z);
                            if ((xi + yi + zi) % 2 != 0) att = mk(m.odd[0], m.odd[1], m.odd[2]);
                        }
                        hint = att;
                    }
                    if (diffuse) {
                        const float4* gp = GUIDE ? R.guide.gpar + (size_t)pid * rtg::GP_F4 : nullptr;
                        // density of the bounce strategy at unit direction u, for the MIS weights
                        auto bounce_pdf = [&](float3 u, float cos_pdf) {
                            return GUIDE ? rtg::guide_pdf(gp, sn.x, sn.y, sn.z, u.x, u.y, u.z) : cos_pdf;
                        };
                        if (R.photons) {
                            // caustic injection: the gather kernel turns T·tint·albedo into × irradiance
                            float3 f = T * sf * hint;
                            npc = make_float4(f.x, f.y, f.z, 0.f);
                            gath = true;
                            ga = make_float4(p.x, p.y, p.z, 0.f);
                            gb = make_float4(nrm.x, nrm.y, nrm.z, 0.f);
                        }
                        if (have_lights) {
                            uint32_t pick = rnd_u32(rng, b + B_LPICK) % (uint32_t)S.n_lights;
                            float3 ldir = light_generate(S.lights[pick], p, rnd(rng, b + B_LPT0), rnd(rng, b + B_LPT1));
                            LRec lr;
                            if (lights_hit(S, p, ldir, &lr)) {
                                float l_pdf = lights_pdf_value(S, p, ldir);
                                float3 lu = unit3(ldir);
                                float brdf = fmaxf(dot3(sn, lu) / PI_F, 0.0f);
                                float sun_p = SKY ? sun_pdf_value(S, ldir) : 0.0f;
                                float env_p = env_dir_pdf(S, ldir);
                                float pb = bounce_pdf(lu, brdf);
                                float mis_d = l_pdf * l_pdf + pb * pb + sun_p * sun_p + env_p * env_p;
                                if (mis_d > 0.0f && brdf > 0.0f) {
                                    float3 nee = emission(S, S.mats[lr.mat], tint, w, lam0, H);
                                    float3 c = T * att * brdf * l_pdf * nee / mis_d;
                                    np0 = make_float4(c.x, c.y, c.z, 0.f);
                                    sh0 = true;
                                    sh0a = make_float4(p.x, p.y, p.z, lr.t * (1.0f - 1e-4f));
                                    sh0b = make_float4(ldir.x, ldir.y, ldir.z, 0.f);
                                }
                            }
                        }
                        if (SKY && S.has_sun) {                                         // renderer.rs:495-518
                            // the sun shares the env-NEE slot: a Physical sky has no env map
                            float3 sun_s, c;
                            if (sun_nee_diffuse(S, p, sn, T * att, sf, rnd(rng, b + B_SUN0), rnd(rng, b + B_SUN1),
                                                &sun_s, &c, gp)) {
                                np1 = make_float4(c.x, c.y, c.z, 0.f);
                                sh1 = true;
                                sh1a = make_float4(p.x, p.y, p.z, INFINITY);
                                sh1b = make_float4(sun_s.x, sun_s.y, sun_s.z, 0.f);
                            }
                        }
                        if (S.has_env) {
                            float epdf;
                            float3 edir = env_sample_dir(S, rnd(rng, b + B_ENV_ROW), rnd(rng, b + B_ENV_COL),
                                                         rnd(rng, b + B_ENV_JU), rnd(rng, b + B_ENV_JV), &epdf);
                            if (epdf > 0.0f) {
                                float3 eu = unit3(edir);
                                float brdf = fmaxf(dot3(sn, eu) / PI_F, 0.0f);
                                if (brdf > 0.0f) {
                                    float area_pdf = have_lights ? lights_pdf_value(S, p, edir) : 0.0f;
                                    float3 ec = env_lookup(S, edir) * sf;
                                    float pb = bounce_pdf(eu, brdf);
                                    float mis_d = epdf * epdf + pb * pb + area_pdf * area_pdf;
                                    float3 c = T * att * brdf * epdf * ec / mis_d;
                                    np1 = make_float4(c.x, c.y, c.z, 0.f);
                                    sh1 = true;
                                    sh1a = make_float4(p.x, p.y, p.z, INFINITY);
                                    sh1b = make_float4(edir.x, edir.y, edir.z, 0.f);
                                }
                            }
                        }
                        // cosine-weighted bounce (pdf.rs:12-41)
                        float r1 = rnd(rng, b + B_COS0), r2 = rnd(rng, b + B_COS1);
                        float sp_, cp_;
                        sincosf(2.0f * PI_F * r1, &sp_, &cp_);
                        float sq_ = sqrtf(r2);
                        float3 wn = unit3(sn);
                        float3 hh = fabsf(wn.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
                        float3 vv = unit3(cross3(wn, hh));
                        float3 uu = cross3(wn, vv);
                        float3 idir = (cp_ * sq_) * uu + (sp_ * sq_) * vv + sqrtf(1.0f - r2) * wn;
                        if (GUIDE && rnd(rng, b + B_LOBE0) < __ldg(gp + 10).x) {
                            // one-sample MIS: a vMF lobe of the guide instead of the cosine lobe
                            float gx, gy, gz;
                            rtg::vmf_mix_sample(gp, rnd(rng, b + B_LOBE1), rnd(rng, b + B_SCATTER0),
                                                rnd(rng, b + B_SCATTER1), &gx, &gy, &gz);
                            idir = mk(gx, gy, gz);
                        }
                        float3 iu = unit3(idir);
                        float pdf_val = GUIDE ? rtg::guide_pdf(gp, wn.x, wn.y, wn.z, iu.x, iu.y, iu.z)
                                              : fmaxf(dot3(iu, wn) / PI_F, 0.0f);
                        float scat = fmaxf(dot3(sn, iu) / PI_F, 0.0f);
                        if (pdf_val <= 0.0f || scat <= 0.0f || dot3(idir, nrm) <= 0.0f) {
                            alive = false;
                        } else {
                            if (GUIDE && R.guide.mode == 2) {
                                // training record: the radiance this path gathers after
                                // the vertex, over T·sf here, estimates f·L_i·cos / p
                                uint32_t r = atomicAdd(R.guide.rec_count, 1u);
                                if (r < R.guide.rec_cap) {
                                    float ts = T.x * sf.x + T.y * sf.y + T.z * sf.z;
                                    R.guide.rec_a[r] = make_float4(p.x, p.y, p.z, ts);
                                    R.guide.rec_b[r] = make_float4(wn.x, wn.y, wn.z, -1.0f);
                                    R.guide.rec_c[r] = make_float4(iu.x, iu.y, iu.z, __uint_as_float(head));
                                    float th_o, ph_o;
                                    rtg::blob_angles(unit3(mk(-d.x, -d.y, -d.z)), &th_o, &ph_o);
                                    R.guide.rec_o[r] = make_float2(th_o, ph_o);
                                    R.guide.rec_w[r] = 0.0f;
                                    head = r;
                                    flags |= PF_REC_OPEN;
                                }
                            }
                            float area = have_lights ? lights_pdf_value(S, p, idir) : 0.0f;
                            float sun = SKY ? sun_pdf_value(S, idir) : 0.0f;
                            float env = env_dir_pdf(S, idir);
                            prev_mis = (pdf_val * pdf_val) / fmaxf(pdf_val * pdf_val + (area * area + sun * sun + env * env), 1e-8f);
                            T = T * (att * (scat / pdf_val));
                            o = p; d = idir;
                            prev_spec = false;
                        }
                    }   // diffuse
                }
                }   // surface
                if (alive && depth >= 2) {                                          // renderer.rs:574-579
                    float3 eff = T * ((CLS == CLS_DIFFUSE || CLS == CLS_PBR) ? sf : spec_factor(S, tint, w, lam0, H));
                    float survive = fmaxf(fmaxf(eff.x, eff.y), eff.z);
                    float pr = fminf(survive, 1.0f);
                    if (survive <= 0.0f || rnd(rng, b + B_RR) >= pr) alive = false;
                    else T = T / pr;
                }
                cont = alive && depth + 1 < R.max_depth;
            }
            Lout = make_float4(Lc.x, Lc.y, Lc.z, 0.f);
            if (cont) {
                meta.z = (flags & ~(PF_DEPTH_MASK | PF_PREV_SPEC | PF_TINT_MASK)) | ((depth + 1) & PF_DEPTH_MASK)
                         | (prev_spec ? PF_PREV_SPEC : 0u) | ((uint32_t)tint << PF_TINT_SHIFT);
                o_out = make_float4(o.x, o.y, o.z, 0.f);
                d_out = make_float4(d.x, d.y, d.z, 0.f);
                thr_out = make_float4(T.x, T.y, T.z, prev_mis);
                w_out = w;
            }
        }
        // block-aggregated compaction: paths that go on into B, ended paths into
        // the retire records; parked contributions and shadow rays follow them
        bool ended = active && !cont;
        uint32_t cnt[NQ], off[NQ];
        uint32_t slot = 0, rs = 0;
        if constexpr (NQ == 1) {
            cnt[0] = ended;
            block_reserve(shq, qctr, cnt, off);
            rs = off[0];
        } else {
            cnt[0] = cont;
            cnt[1] = ended;
            if constexpr (NQ == 4) { cnt[2] = gath; cnt[3] = (uint32_t)sh0 + (uint32_t)sh1; }
            block_reserve(shq, qctr, cnt, off);
            slot = off[0];
            rs = off[1];
        }
        if (cont) {
            B.ray_o[slot] = o_out; B.ray_d[slot] = d_out; B.thr[slot] = thr_out; B.wts[slot] = w_out;
            B.meta[slot] = meta; B.L[slot] = Lout; B.pend0[slot] = np0; B.pend1[slot] = np1;
            if (R.photons) B.pendC[slot] = npc;
            if (R.guide.mode == 2) B.rec[slot] = head;
        } else if (ended) {
            Rt.meta[rs] = meta; Rt.L[rs] = Lout; Rt.pend0[rs] = np0; Rt.pend1[rs] = np1;
            if (R.photons) Rt.pendC[rs] = npc;
            if (R.guide.mode == 2) Rt.rec[rs] = head;
        }
        if constexpr (NQ == 4) {
            uint32_t tag = cont ? slot << 2 : (rs << 2) | PT_RETIRED;
            if (gath) {
                uint32_t g = off[2];
                ga.w = __uint_as_float(tag);
                A.gq[(size_t)g * 2] = ga; A.gq[(size_t)g * 2 + 1] = gb;
            }
            uint32_t s0 = off[3];
            if (sh0) { sh0b.w = __uint_as_float(tag); sq[(size_t)s0 * 2] = sh0a; sq[(size_t)s0 * 2 + 1] = sh0b; s0++; }
            if (sh1) { sh1b.w = __uint_as_float(tag | 1u); sq[(size_t)s0 * 2] = sh1a; sq[(size_t)s0 * 2 + 1] = sh1b; }
        }
    }
}

// ── accumulate_sample over the passes of one call, in sample order ──────────
__global__ void k_accumulate(const float* __restrict__ scratch, uint32_t nsamp, uint32_t npix, float* acc, float* m2,
                             uint32_t* cnt, const uint8_t* conv, float clamp, uint32_t min_samples, float floor_) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        if (conv && conv[i]) continue;
        float3 a = mk(acc[i * 3], acc[i * 3 + 1], acc[i * 3 + 2]);
        float3 q = mk(m2[i * 3], m2[i * 3 + 1], m2[i * 3 + 2]);
        uint32_t n = cnt[i];
        for (uint32_t k = 0; k < nsamp; k++) {
            const float* s = scratch + ((size_t)k * npix + i) * 3;
            float3 sc = mk(s[0], s[1], s[2]);
            if (!isfinite(sc.x) || !isfinite(sc.y) || !isfinite(sc.z)) continue;
            float3 old_mean = n > 0 ? a / (float)n : mk(0.f, 0.f, 0.f);
            if (clamp > 0.0f && n >= min_samples) {
                float l = lum3(sc), th = fmaxf(clamp * lum3(old_mean), floor_);
                if (l > th) sc = sc * (th / l);
            }
            a = a + sc;
            n += 1;
            float3 nm = a / (float)n;
            q = q + (sc - old_mean) * (sc - nm);
        }
        acc[i * 3] = a.x; acc[i * 3 + 1] = a.y; acc[i * 3 + 2] = a.z;
        m2[i * 3] = q.x; m2[i * 3 + 1] = q.y; m2[i * 3 + 2] = q.z;
        cnt[i] = n;
    }
}

// ── guide inference: the mixture of every diffuse-class path of the bounce ──
// Two kernels.  k_guide_encode, one thread per queue entry and no shared
// memory (so the hash-table gathers run at full occupancy), recomputes the hit
// as the shading kernel does and writes the 64 bf16 inputs (hash grid at the
// hit, one-blob of the outgoing direction) in queue order.  k_guide_infer runs the network on those rows,
// 32 per warp as two 16-row tensor-core tiles fed straight from global memory,
// and lanes 0..15 write the mixtures of the tile's paths.
#define GUIDE_WARPS 8
#define GUIDE_LDO 52
static size_t guide_infer_smem() {
    return (size_t)rtg::W_SMEM * 2 + (size_t)GUIDE_WARPS * 16 * GUIDE_LDO * 4;
}
__global__ void __launch_bounds__(256) k_guide_encode(DevScene S, PathState A, const RenderLaunch* __restrict__ Rp,
                                                      const uint32_t* __restrict__ qin, const uint32_t* cin) {
    const RenderLaunch& R = *Rp;
    uint32_t n = *cin;
    for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi < n; qi += gridDim.x * blockDim.x) {
        uint32_t pid = qin[qi];
        float4 hv = A.hit[pid], ro = A.ray_o[pid], rdv = A.ray_d[pid];
        Surf sf = surface(S, hv, mk(ro.x, ro.y, ro.z), mk(rdv.x, rdv.y, rdv.z));
        uint32_t v[32];
        float th, ph;
        rtg::blob_angles(unit3(mk(-rdv.x, -rdv.y, -rdv.z)), &th, &ph);      // ω_o
        rtg::encode_packed(R.guide, R.guide.tbf, sf.p, th, ph, v);
        uint4* dst = R.guide.enc + (size_t)qi * 8;
#pragma unroll
        for (int k = 0; k < 8; k++) dst[k] = make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    }
}
__global__ void __launch_bounds__(GUIDE_WARPS * 32) k_guide_infer(const RenderLaunch* __restrict__ Rp,
                                                                  const uint32_t* __restrict__ qin,
                                                                  const uint32_t* cin) {
    const RenderLaunch& R = *Rp;
    extern __shared__ __align__(16) unsigned char gsm[];
    __nv_bfloat16* Ws = reinterpret_cast<__nv_bfloat16*>(gsm);
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* S_o = reinterpret_cast<float*>(Ws + rtg::W_SMEM) + warp * 16 * GUIDE_LDO;
    rtg::load_weights(R.guide.wbf, Ws);
    __syncthreads();
    uint32_t n = *cin;
    const __nv_bfloat16* enc = reinterpret_cast<const __nv_bfloat16*>(R.guide.enc);
    int g = lane >> 2, t = lane & 3;
    for (uint32_t base = (blockIdx.x * GUIDE_WARPS + warp) * 32; base < n; base += gridDim.x * GUIDE_WARPS * 32) {
        for (int mt = 0; mt < 2; mt++) {
            uint32_t r0 = base + 16 * mt;
            if (r0 >= n) break;                                   // uniform across the warp
            // rows past n read as zeros (the queue holds at most the pool)
            uint32_t ra = r0 + g, rb = r0 + g + 8;
            uint32_t x0[4][4], h1[4][4], h2[4][4], h3[4][4];
#pragma unroll
            for (int kb = 0; kb < 4; kb++) {
                int c = 16 * kb + 2 * t;
                x0[kb][0] = ra < n ? rtg::ld_u32(enc + (size_t)ra * rtg::NIN + c) : 0u;
                x0[kb][1] = rb < n ? rtg::ld_u32(enc + (size_t)rb * rtg::NIN + c) : 0u;
                x0[kb][2] = ra < n ? rtg::ld_u32(enc + (size_t)ra * rtg::NIN + c + 8) : 0u;
                x0[kb][3] = rb < n ? rtg::ld_u32(enc + (size_t)rb * rtg::NIN + c + 8) : 0u;
            }
            float o[6][4];
            rtg::mlp_forward(Ws, x0, h1, h2, h3, o);
            rtg::store_out(o, S_o, GUIDE_LDO);
            __syncwarp();
            uint32_t qi = r0 + lane;
            if (lane < 16 && qi < n) {
                float4 gp[rtg::GP_F4];
                rtg::mixture_from_outputs(S_o + lane * GUIDE_LDO, gp, R.guide.amax, R.guide.lkmax);
                float4* dst = R.guide.gpar + (size_t)qin[qi] * rtg::GP_F4;
#pragma unroll
                for (int k = 0; k < rtg::GP_F4; k++) dst[k] = gp[k];
            }
            __syncwarp();
        }
    }
}

namespace rth {
void launch_guide_infer(const DevScene& S, const PathState& A, const RenderLaunch& R, const uint32_t* queue,
                        const uint32_t* count, int sms, cudaStream_t st) {
    cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)guide_infer_smem());
    k_guide_encode<<<sms * 8, 256, 0, st>>>(S, A, R.dev, queue, count);
    k_guide_infer<<<sms * 2, GUIDE_WARPS * 32, guide_infer_smem(), st>>>(R.dev, queue, count);
}
void launch_generate(const DevScene& S, const PathState& A, const RenderLaunch& R, uint32_t capacity,
                     uint32_t* count0, cudaStream_t st) {
    int grid = (int)std::max<uint32_t>(1u, std::min<uint32_t>((capacity + 255) / 256, 148u * 16u));
    k_generate<<<grid, 256, 0, st>>>(S, A, R.dev, count0);
}
void launch_shade(const DevScene& S, const PathState& A, const PathState& B, const PathState& Rt, const RenderLaunch& R,
                  uint32_t* ctr, const ClassQueues& Q, uint32_t* cout, float4* sq, int sms, cudaStream_t st,
                  const ShadeFork* fk) {
    // ctr: this iteration's counter block (see rt_internal.h for the slots)
    int grid = sms * (S.shade_per_sm > 0 ? S.shade_per_sm : RT_SHADE_BLOCKS_PER_SM);
    k_classify<<<sms * 4, CLS_BLOCK, 0, st>>>(A.hit, ctr + CTR_COUNT, Q, ctr + CTR_CLS_COUNT);
    // the classes but diffuse go to side streams, ordered after classification
    // only (not after the guide's inference, which only the diffuse class reads)
    int nside = 0;
    if (fk) cudaEventRecord(fk->fork, st);
    auto stream_of = [&](int C) -> cudaStream_t {
        if (!fk || C == CLS_DIFFUSE) return st;
        cudaStream_t s2 = fk->side[nside];
        cudaStreamWaitEvent(s2, fk->fork, 0);
        return s2;
    };
    if (R.guide.mode != 0)
        launch_guide_infer(S, A, R, Q.q[CLS_DIFFUSE], ctr + CTR_CLS_COUNT + CLS_DIFFUSE, sms, st);
#define RT_SHADE_CLASS_G(C, G)                                                                              \
    do {                                                                                                    \
        if (!((S.class_mask >> (C)) & 1u)) break;                                                           \
        cudaStream_t cs = stream_of(C);                                                                     \
        if (S.bg_type == RT_BG_PHYSICAL)                                                                    \
            k_shade<C, true, G><<<grid, RT_SHADE_BLOCK, 0, cs>>>(S, A, B, Rt, R.dev, Q.q[C], ctr + CTR_CLS_COUNT + C, cout, sq, ctr); \
        else                                                                                                \
            k_shade<C, false, G><<<grid, RT_SHADE_BLOCK, 0, cs>>>(S, A, B, Rt, R.dev, Q.q[C], ctr + CTR_CLS_COUNT + C, cout, sq, ctr); \
        if (cs != st) cudaEventRecord(fk->join[nside++], cs);                                              \
    } while (0)
#define RT_SHADE_CLASS(C) RT_SHADE_CLASS_G(C, false)
    RT_SHADE_CLASS(CLS_MISS);
    RT_SHADE_CLASS(CLS_EMIT);
    if (R.guide.mode != 0) { RT_SHADE_CLASS_G(CLS_DIFFUSE, true); }
    else { RT_SHADE_CLASS(CLS_DIFFUSE); }
    RT_SHADE_CLASS(CLS_METAL);
    RT_SHADE_CLASS(CLS_DIELEC);
    if (S.n_pbr > 0) { RT_SHADE_CLASS(CLS_PBR); }
    if (S.n_media > 0) { RT_SHADE_CLASS(CLS_MEDIUM); }
#undef RT_SHADE_CLASS
#undef RT_SHADE_CLASS_G
    for (int i = 0; i < nside; i++) cudaStreamWaitEvent(st, fk->join[i], 0);
}
void launch_retire(const DevScene& S, const PathState& B, const PathState& Rt, const RenderLaunch& R, uint32_t* ctr,
                   uint32_t* hdr, uint32_t* clear_block, uint32_t* cout, int sms, cudaStream_t st) {
    k_retire<<<sms * 8, RETIRE_BLOCK, 0, st>>>(S, B, Rt, R.dev, ctr, hdr, clear_block, cout);
}
void launch_active_list(const uint8_t* conv, uint32_t width, uint32_t height, uint32_t* list, uint32_t* count,
                        cudaStream_t st) {
    uint32_t npix = width * height;
    int grid = (int)std::max<uint32_t>(1u, std::min<uint32_t>((npix + 255) / 256, 148u * 16u));
    k_active_list<<<grid, 256, 0, st>>>(conv, width, height, list, count);
}
void launch_zero_converged(const uint8_t* conv, uint32_t npix, uint32_t nsamp, float* scratch, cudaStream_t st) {
    k_zero_converged<<<148 * 16, 256, 0, st>>>(conv, npix, nsamp, scratch);
}
void launch_accumulate(const float* scratch, uint32_t nsamp, uint32_t npix, float* acc, float* m2, uint32_t* cnt,
                       const uint8_t* conv, float clamp, uint32_t min_samples, float floor_, cudaStream_t st) {
    int grid = (int)std::min<uint32_t>((npix + 255) / 256, 148u * 16u);
    k_accumulate<<<grid, 256, 0, st>>>(scratch, nsamp, npix, acc, m2, cnt, conv, clamp, min_samples, floor_);
}
}  // namespace rth
