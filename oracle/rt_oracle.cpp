// rt_oracle.cpp — CPU ORACLE for the render hot path.  TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++ on the host CPU, the reference renderer's
// hot path (mcrepeau/rustracer, a pure-Rust CPU path tracer).  It is the
// checker the CUDA library is compared against and the timed CPU baseline.
// Nothing in the product (rustracer_b200/) links or calls it; only tests/,
// __graft_entry__.smoke() and bench.py's CPU legs load it.
//
// What it follows, by reference file:line:
//   math/ray ........ src/vec3.rs:14-116, src/ray.rs:25-42, src/aabb.rs:10-35, src/onb.rs:10-20
//   BVH build ....... src/bvh.rs:52-225   (binned SAH, 12 buckets, 3 binary levels per 8-wide node)
//   traversal ....... src/bvh.rs:229-288 (closest), :487-575 (any / transmittance), slab test :326-364
//   primitives ...... src/triangle.rs:75-140, src/quad.rs:21-96, src/sphere.rs:47-118
//   light list ...... src/hittable.rs:156-225 (linear hit scan, mean pdf, uniform pick)
//   materials ....... src/material.rs:14-149 (lights, Lambertian, Fresnel, dielectric boundary),
//                     :161-321 (GGX, Smith, E_ss LUT, VNDF), :323-403 (Dielectric, SpectralDielectric),
//                     :427-554 (SpectralMetal)
//   spectrum ........ src/spectrum.rs:64-277
//   background ...... src/renderer.rs:23-223 (EnvMapData CDF sampling, bilinear lookup, Solid/Gradient/Split)
//   path loop ....... src/renderer.rs:371-585 (ray_color), :655-730 (render_tiles)
//   camera .......... src/camera.rs:24-59
//   accumulation .... src/main.rs:603-677 (accumulate_sample, mark_converged)
//
// Deliberate, documented differences from the reference (both this oracle and
// the CUDA library implement them identically):
//   * Random numbers: the reference draws from rand 0.8's SmallRng seeded per
//     image row (renderer.rs:688-691); its stream cannot be consumed in the
//     same order by a parallel GPU path, so both sides use a counter-based hash
//     keyed on (seed, pixel, sample, dimension) — pcg3d of Jarzynski & Olano,
//     "Hash Functions for GPU Rendering", JCGT 2020.  Image-level parity is
//     statistical; ray-level parity (hit ids, t) is exact.
//   * Closest-hit ties: equal t goes to the smaller canonical prim id instead of
//     the last one visited (bvh.rs:250-253), so hit ids do not depend on the BVH
//     layout.  Box culling is made conservative (ray reciprocal directions are
//     kept finite and the slab exit is widened by 2^-16 relative) so that the
//     traversal returns exactly the brute-force minimum.
//   * Hero wavelengths: hero_count = 1 reproduces the reference's single λ per
//     path; hero_count = 4 carries 4 rotated wavelengths (Wilkie et al. 2014)
//     whose per-λ scalar weights generalise the reference's spectral_weighted
//     throughput; secondaries are terminated at dispersive boundaries.
//   * Lens sampling draws the unit disk by the polar map instead of rejection.
//   * Object transforms are applied to the primitives before the call
//     (world-space triangles), and meshes join the world BVH directly instead
//     of being nested BVH leaves (mesh.rs:91).
//
// Built by oracle/build.py with -O3 -mavx2 -mfma -ffp-contract=off: Rust never
// contracts a*b+c into an FMA, so the oracle must not either.

#include "../include/rt_api.h"
#include "../include/rt_spectral_tables.h"

#include <immintrin.h>
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace orc {

static const float PI_F = 3.14159265358979323846f;

// ── vec3.rs ──────────────────────────────────────────────────────────────────
struct V3 { float x, y, z; };
static inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
static inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 operator*(V3 a, float t) { return v3(a.x * t, a.y * t, a.z * t); }
static inline V3 operator*(float t, V3 a) { return a * t; }
static inline V3 operator/(V3 a, float t) { return v3(a.x / t, a.y / t, a.z / t); }   // exact division (vec3.rs:95-97)
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float len2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline float length(V3 a) { return std::sqrt(len2(a)); }
static inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline V3 unit(V3 a) { return a / length(a); }
static inline float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
static inline float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline float rmin(float a, float b) { return std::fmin(a, b); }   // f32::min drops one NaN
static inline float rmax(float a, float b) { return std::fmax(a, b); }
static inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline V3 reflect(V3 v, V3 n) { return v - 2.0f * dot(v, n) * n; }   // vec3.rs:49
// vec3.rs:55-61 — returns false when k < 0
static inline bool refract(V3 v, V3 n, float eta, V3* out) {
    float cos_t = rmin(dot(-v, n), 1.0f);
    V3 perp = eta * (v + cos_t * n);
    float k = 1.0f - len2(perp);
    if (k < 0.0f) return false;
    *out = perp + (-std::sqrt(k) * n);
    return true;
}
// vec3.rs:37-42
static inline void onb_vec(V3 n, V3* u, V3* v) {
    V3 up = std::fabs(n.y) < 0.9f ? v3(0, 1, 0) : v3(1, 0, 0);
    *u = unit(cross(n, up));
    *v = cross(n, *u);
}
// onb.rs:10-20
struct Onb { V3 u, v, w; };
static inline Onb onb_from_w(V3 n) {
    Onb o;
    o.w = unit(n);
    V3 a = std::fabs(o.w.x) > 0.9f ? v3(0, 1, 0) : v3(1, 0, 0);
    o.v = unit(cross(o.w, a));
    o.u = cross(o.w, o.v);
    return o;
}
static inline V3 onb_local(const Onb& o, V3 a) { return a.x * o.u + a.y * o.v + a.z * o.w; }

// ── counter-based RNG (pcg3d) ────────────────────────────────────────────────
static inline uint32_t mix32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}
static inline uint32_t pcg3d_x(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t x = a * 1664525u + 1013904223u;
    uint32_t y = b * 1664525u + 1013904223u;
    uint32_t z = c * 1664525u + 1013904223u;
    x += y * z; y += z * x; z += x * y;
    x ^= x >> 16; y ^= y >> 16; z ^= z >> 16;
    x += y * z; y += z * x; z += x * y;
    return x;
}
struct Rng { uint32_t a, b, c; };
static inline Rng make_rng(uint64_t seed, uint32_t pixel, uint32_t sample) {
    Rng r;
    r.a = pixel;
    r.b = sample ^ mix32((uint32_t)seed);
    r.c = mix32((uint32_t)(seed >> 32) + 0x9E3779B9u);
    return r;
}
static inline uint32_t rnd_u32(const Rng& r, uint32_t dim) { return pcg3d_x(r.a, r.b, dim ^ r.c); }
static inline float rnd(const Rng& r, uint32_t dim) { return (float)(rnd_u32(r, dim) >> 8) * (1.0f / 16777216.0f); }

// dimension layout of one path
enum {
    D_JIT_U = 0, D_JIT_V = 1, D_LENS_R = 2, D_LENS_P = 3, D_TIME = 4, D_LAMBDA = 5, D_LENS_K = 6,
    D_BOUNCE0 = 8, D_PER_BOUNCE = 16,
    B_SCATTER0 = 0, B_SCATTER1 = 1, B_LPICK = 2, B_LPT0 = 3, B_LPT1 = 4,
    B_SUN0 = 5, B_SUN1 = 6,
    B_ENV_ROW = 7, B_ENV_COL = 8, B_ENV_JU = 9, B_ENV_JV = 10, B_COS0 = 11, B_COS1 = 12, B_RR = 13,
    B_LOBE0 = 14, B_LOBE1 = 15,   // PBR lobe choice: clearcoat, then base specular
};

// ── spectrum.rs ──────────────────────────────────────────────────────────────
struct Spectrum {
    int n = RT_CIE_N;                 // entries on the 5 nm grid from 380 nm
    float xyz[RT_CIE_N + RT_CIE_EXT_N][3];
    float norms[3], fire_norms[3];
    float lam_lo = 380.0f, lam_range = 320.0f;
};
static inline void xyz_to_srgb_clamped(float x, float y, float z, float out[3]) {   // spectrum.rs:66-73
    out[0] = rmax(3.2406f * x - 1.5372f * y - 0.4986f * z, 0.0f);
    out[1] = rmax(-0.9689f * x + 1.8758f * y + 0.0415f * z, 0.0f);
    out[2] = rmax(0.0557f * x - 0.2040f * y + 1.0570f * z, 0.0f);
}
static const float FIRE_LUMA_POW = 0.5f, FIRE_LUMA_FLOOR = 0.08f, FIRE_DESAT = 0.5f;
static inline void fire_color(float x, float y, float z, float c[3]) {            // spectrum.rs:148-160
    float w = rmax(std::pow(y, FIRE_LUMA_POW), FIRE_LUMA_FLOOR);
    float rgb[3]; xyz_to_srgb_clamped(x, y, z, rgb);
    c[0] = rgb[0] * w; c[1] = rgb[1] * w; c[2] = rgb[2] * w;
    float d = FIRE_DESAT;
    if (d > 0.0f) {
        float lum = 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
        for (int i = 0; i < 3; i++) c[i] = c[i] * (1.0f - d) + lum * d;
    }
}
static void spectrum_init(Spectrum& s, int range_mode) {
    s.n = range_mode ? RT_CIE_N + RT_CIE_EXT_N : RT_CIE_N;
    for (int i = 0; i < s.n; i++)
        for (int k = 0; k < 3; k++)
            s.xyz[i][k] = i < RT_CIE_N ? RT_CIE_XYZ[i][k] : RT_CIE_XYZ_EXT[i - RT_CIE_N][k];
    float sum[3] = {0, 0, 0}, fsum[3] = {0, 0, 0};
    for (int i = 0; i < s.n; i++) {                                                 // spectrum.rs:80-95
        float rgb[3]; xyz_to_srgb_clamped(s.xyz[i][0], s.xyz[i][1], s.xyz[i][2], rgb);
        sum[0] += rgb[0]; sum[1] += rgb[1]; sum[2] += rgb[2];
        float c[3]; fire_color(s.xyz[i][0], s.xyz[i][1], s.xyz[i][2], c);           // spectrum.rs:162-177
        fsum[0] += c[0]; fsum[1] += c[1]; fsum[2] += c[2];
    }
    for (int k = 0; k < 3; k++) {
        s.norms[k] = (float)s.n / rmax(sum[k], 1e-6f);
        s.fire_norms[k] = (float)s.n / rmax(fsum[k], 1e-6f);
    }
    s.lam_lo = 380.0f;
    s.lam_range = range_mode ? 400.0f : 320.0f;
}
static inline void cmf_lerp(const Spectrum& s, float lambda, float xyz[3]) {       // spectrum.rs:105-110
    float t = clampf((lambda - RT_CIE_START) / RT_CIE_STEP, 0.0f, (float)(s.n - 1));
    int i = std::min((int)t, s.n - 2);
    float frac = t - (float)i;
    for (int k = 0; k < 3; k++) xyz[k] = s.xyz[i][k] + frac * (s.xyz[i + 1][k] - s.xyz[i][k]);
}
static inline V3 spectral_to_rgb(const Spectrum& s, float lambda) {               // spectrum.rs:104-114
    float xyz[3]; cmf_lerp(s, lambda, xyz);
    float rgb[3]; xyz_to_srgb_clamped(xyz[0], xyz[1], xyz[2], rgb);
    return v3(rgb[0] * s.norms[0], rgb[1] * s.norms[1], rgb[2] * s.norms[2]);
}
static inline V3 spectral_fire_rgb(const Spectrum& s, float lambda) {             // spectrum.rs:183-193
    float xyz[3]; cmf_lerp(s, lambda, xyz);
    float c[3]; fire_color(xyz[0], xyz[1], xyz[2], c);
    return v3(c[0] * s.fire_norms[0], c[1] * s.fire_norms[1], c[2] * s.fire_norms[2]);
}
static inline float planck_raw(float lambda_nm, float temp_k) {                    // spectrum.rs:204-208
    const float HC_OVER_K = 14388000.0f;
    float x = HC_OVER_K / (lambda_nm * temp_k);
    float l2 = lambda_nm * lambda_nm, l4 = l2 * l2;
    return 1.0f / (lambda_nm * l4 * rmax(std::exp(x) - 1.0f, 1e-30f));
}
static inline void metal_ior(const RtMaterial& m, float lambda, float* n, float* k) {   // spectrum.rs:227-233
    const float* ns; const float* ks; int cnt; float start, step;
    if (m.metal >= RT_METAL_GOLD && m.metal <= RT_METAL_SILVER) {
        ns = RT_METAL_NK[m.metal][0]; ks = RT_METAL_NK[m.metal][1];
        cnt = RT_METAL_NK_N; start = RT_METAL_NK_START; step = RT_METAL_NK_STEP;
    } else {
        ns = m.nk_n; ks = m.nk_k; cnt = m.nk_count; start = m.nk_start; step = m.nk_step;
    }
    float t = clampf((lambda - start) / step, 0.0f, (float)(cnt - 1));
    int i = std::min((int)t, cnt - 2);
    float f = t - (float)i;
    *n = ns[i] + f * (ns[i + 1] - ns[i]);
    *k = ks[i] + f * (ks[i + 1] - ks[i]);
}
static inline float fresnel_conductor(float cos_i, float n, float k) {             // spectrum.rs:247-262
    float cos2 = cos_i * cos_i;
    float sin2 = rmax(1.0f - cos2, 0.0f);
    float n2 = n * n, k2 = k * k;
    float t0 = n2 - k2 - sin2;
    float a2pb2 = std::sqrt(t0 * t0 + 4.0f * n2 * k2);
    float t1 = a2pb2 + cos2;
    float a = std::sqrt(rmax(0.5f * (a2pb2 + t0), 0.0f));
    float t2 = 2.0f * cos_i * a;
    float rs = (t1 - t2) / rmax(t1 + t2, 1e-12f);
    float t3 = cos2 * a2pb2 + sin2 * sin2;
    float t4 = t2 * sin2;
    float rp = rs * (t3 - t4) / rmax(t3 + t4, 1e-12f);
    return clampf(0.5f * (rp + rs), 0.0f, 1.0f);
}
static inline float cauchy_ior(float lambda_nm, float b, float c) {                // spectrum.rs:274-277
    float um = lambda_nm * 1e-3f;
    return b + c / (um * um);
}

// ── material.rs helpers ──────────────────────────────────────────────────────
static inline float fresnel_dielectric(float cos_i, float eta) {                   // material.rs:119-127
    float sin2_i = rmax(1.0f - cos_i * cos_i, 0.0f);
    float sin2_t = eta * eta * sin2_i;
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = std::sqrt(1.0f - sin2_t);
    float rs = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    float rp = (eta * cos_t - cos_i) / (eta * cos_t + cos_i);
    return (rs * rs + rp * rp) * 0.5f;
}
static inline float smith_g1(float c, float alpha) {                               // material.rs:163-167
    float a2 = alpha * alpha, c2 = c * c;
    return 2.0f * c / (c + std::sqrt(a2 + (1.0f - a2) * c2));
}
static inline float smith_lambda(float c, float alpha) {                           // material.rs:179-183
    float a2 = alpha * alpha, c2 = c * c;
    return (std::sqrt(a2 + (1.0f - a2) * c2) - c) / (2.0f * c);
}
static inline float ggx_ndf(float cos_h, float alpha) {                            // material.rs:308-312
    float a2 = alpha * alpha;
    float d = 1.0f + cos_h * cos_h * (a2 - 1.0f);
    return a2 / rmax(PI_F * d * d, 1e-12f);
}
static inline V3 vndf_sample(V3 wo, float ax, float ay, float xi1, float xi2) {   // material.rs:273-303
    V3 wh = unit(v3(ax * wo.x, ay * wo.y, wo.z));
    float len = std::sqrt(wh.x * wh.x + wh.y * wh.y);
    V3 t1 = len > 1e-6f ? v3(-wh.y / len, wh.x / len, 0.0f) : v3(1, 0, 0);
    V3 t2 = cross(wh, t1);
    float a = 1.0f / (1.0f + wh.z);
    float r = std::sqrt(xi1);
    float p1, p2;
    if (xi2 < a) {
        float phi = xi2 / a * PI_F;
        p1 = r * std::cos(phi); p2 = r * std::sin(phi);
    } else {
        float phi = PI_F + (xi2 - a) / (1.0f - a) * PI_F;
        p1 = r * std::cos(phi); p2 = r * std::sin(phi) * wh.z;
    }
    float p3 = std::sqrt(rmax(1.0f - p1 * p1 - p2 * p2, 0.0f));
    V3 nh = t1 * p1 + t2 * p2 + wh * p3;
    return unit(v3(ax * nh.x, ay * nh.y, rmax(nh.z, 0.0f)));
}

// E_ss(mu, alpha) LUT (material.rs:206-241): 64×64 texels, 64×64 stratified
// VNDF samples each.  Jitter comes from the counter hash (texel, sample) instead
// of SmallRng; the estimator is the reference's.
static const int E_N = 64;
static float g_elut[E_N][E_N];
static std::once_flag g_elut_once;
static void build_e_lut() {
    const int G = 64;
    for (int i = 0; i < E_N; i++) {
        float mu = ((float)i + 0.5f) / (float)E_N;
        for (int j = 0; j < E_N; j++) {
            float alpha = rmax(((float)j + 0.5f) / (float)E_N, 1e-3f);
            V3 wo = v3(0.0f, 0.0f, mu);
            float lam_o = smith_lambda(mu, alpha);
            double sum = 0.0;
            uint32_t texel = (uint32_t)(i * E_N + j);
            for (int k = 0; k < G; k++) {
                for (int l = 0; l < G; l++) {
                    uint32_t smp = (uint32_t)(k * G + l);
                    float r1 = (float)(pcg3d_x(texel, smp, 0xE55E0001u) >> 8) * (1.0f / 16777216.0f);
                    float r2 = (float)(pcg3d_x(texel, smp, 0xE55E0002u) >> 8) * (1.0f / 16777216.0f);
                    float xi1 = ((float)k + r1) / (float)G;
                    float xi2 = ((float)l + r2) / (float)G;
                    V3 m = vndf_sample(wo, alpha, alpha, xi1, xi2);
                    float vo_h = rmax(dot(wo, m), 0.0f);
                    V3 wi = 2.0f * vo_h * m - wo;
                    if (wi.z <= 0.0f) continue;
                    float lam_i = smith_lambda(wi.z, alpha);
                    sum += (double)((1.0f + lam_o) / (1.0f + lam_o + lam_i));
                }
            }
            g_elut[i][j] = (float)(sum / (double)(G * G));
        }
    }
}
static inline float e_ss_lut(float mu, float alpha) {                              // material.rs:246-260
    std::call_once(g_elut_once, build_e_lut);
    float x = clampf(clampf(mu, 0.0f, 1.0f) * (float)E_N - 0.5f, 0.0f, (float)(E_N - 1));
    float y = clampf(clampf(alpha, 0.0f, 1.0f) * (float)E_N - 0.5f, 0.0f, (float)(E_N - 1));
    int i0 = (int)x, j0 = (int)y;
    int i1 = std::min(i0 + 1, E_N - 1), j1 = std::min(j0 + 1, E_N - 1);
    float fx = x - (float)i0, fy = y - (float)j0;
    float e00 = g_elut[i0][j0], e10 = g_elut[i1][j0], e01 = g_elut[i0][j1], e11 = g_elut[i1][j1];
    return (e00 * (1.0f - fx) + e10 * fx) * (1.0f - fy) + (e01 * (1.0f - fx) + e11 * fx) * fy;
}
static inline float specular_energy_comp(float mu, float alpha) {                  // material.rs:265-267
    return rmin(1.0f / rmax(e_ss_lut(mu, alpha), 0.05f), 10.0f);
}

// ── PbrMaterial (material.rs:680-1050) ──────────────────────────────────────
static inline float smith_lambda_aniso(float c, float tx, float ty, float ax, float ay) {   // material.rs:187-190
    return (std::sqrt(c * c + ax * ax * tx * tx + ay * ay * ty * ty) - c) / (2.0f * c);
}
static inline float smith_g1_aniso(float c, float tx, float ty, float ax, float ay) {       // material.rs:172-175
    float denom = c + std::sqrt(c * c + ax * ax * tx * tx + ay * ay * ty * ty);
    return rmin(rmax(2.0f * c / rmax(denom, 1e-6f), 0.0f), 1.0f);
}
static inline float ggx_ndf_aniso(V3 h, float ax, float ay) {                      // material.rs:316-321
    float hx = h.x / ax, hy = h.y / ay;
    float d = hx * hx + hy * hy + h.z * h.z;
    return 1.0f / rmax(PI_F * ax * ay * d * d, 1e-12f);
}
static inline float schlick(float cosine, float ref_idx) {                         // material.rs:106-111
    float b = (1.0f - ref_idx) / (1.0f + ref_idx);
    float r0 = b * b, u = 1.0f - cosine;
    return r0 + (1.0f - r0) * (u * u * u * u * u);
}
static inline V3 schlick_color(float ct, V3 f0) {                                  // material.rs:155-160
    float u = rmax(1.0f - ct, 0.0f), t = u * u * u * u * u;
    return f0 + (v3(1, 1, 1) - f0) * t;
}
// NACRE_LUT (material.rs:1096-1118) from spectral_to_rgb over 380..700 nm
static V3 g_nacre[256];
static std::once_flag g_nacre_once;
static void nacre_init() {
    float sum[3] = {0, 0, 0};
    for (int i = 0; i < RT_CIE_N; i++) {
        float rgb[3];
        xyz_to_srgb_clamped(RT_CIE_XYZ[i][0], RT_CIE_XYZ[i][1], RT_CIE_XYZ[i][2], rgb);
        for (int k = 0; k < 3; k++) sum[k] += rgb[k];
    }
    float norm[3];
    for (int k = 0; k < 3; k++) norm[k] = (float)RT_CIE_N / rmax(sum[k], 1e-6f);
    for (int i = 0; i < 256; i++) {
        float opd = (float)i / 255.0f * 2500.0f;
        V3 c = v3(0, 0, 0);
        for (float lambda = 380.0f; lambda <= 700.01f; lambda += 5.0f) {
            float t = rmin(rmax((lambda - 380.0f) / 5.0f, 0.0f), (float)(RT_CIE_N - 1));
            int k = std::min((int)t, RT_CIE_N - 2);
            float f = t - (float)k, xyz[3], rgb[3];
            for (int q = 0; q < 3; q++) xyz[q] = RT_CIE_XYZ[k][q] + f * (RT_CIE_XYZ[k + 1][q] - RT_CIE_XYZ[k][q]);
            xyz_to_srgb_clamped(xyz[0], xyz[1], xyz[2], rgb);
            float irid = 0.5f * (1.0f + std::cos(2.0f * PI_F * opd / lambda));
            c = c + v3(rgb[0] * norm[0], rgb[1] * norm[1], rgb[2] * norm[2]) * irid;
        }
        g_nacre[i] = c / 65.0f;
    }
}
static V3 nacre_color(float ct, float film_ior, float thick) {                     // material.rs:1130-1146
    std::call_once(g_nacre_once, nacre_init);
    float sin_sq = rmax(1.0f - ct * ct, 0.0f);
    float cos_t = std::sqrt(rmax(1.0f - sin_sq / (film_ior * film_ior), 0.0f));
    float opd = 2.0f * film_ior * thick * cos_t;
    float t = rmin(rmax(opd / 2500.0f, 0.0f), 1.0f) * 255.0f;
    int lo = (int)t, hi = std::min(lo + 1, 255);
    V3 raw = g_nacre[lo] * (1.0f - (t - (float)lo)) + g_nacre[hi] * (t - (float)lo);
    float blend = std::pow(ct, 0.5f);
    return raw * blend + v3(0.5f, 0.5f, 0.5f) * (1.0f - blend);
}
struct PbrCommon { V3 albedo, f0; float alpha, p_coat, p_spec, ax, ay; };
static PbrCommon pbr_common(const RtMaterial& m, float cos_o) {
    PbrCommon c;
    c.albedo = v3(m.albedo[0], m.albedo[1], m.albedo[2]);
    c.alpha = rmax(m.roughness * m.roughness, 1e-4f);
    c.f0 = v3(0.04f, 0.04f, 0.04f) * (1.0f - m.metallic) + c.albedo * m.metallic;
    c.p_coat = m.clearcoat > 1e-3f ? rmax(schlick(cos_o, 1.0f / 1.5f) * m.clearcoat, 0.12f * m.clearcoat) : 0.0f;
    c.p_spec = m.metallic > 0.999f ? 1.0f : rmin(rmax(luminance(schlick_color(cos_o, c.f0)), 0.04f), 0.9f);
    // Disney aspect: ax (tangent) = α/aspect, ay (bitangent) = α·aspect
    float aspect = std::sqrt(rmax(1.0f - 0.9f * rmin(rmax(m.anisotropy, 0.0f), 1.0f), 0.001f));
    c.ax = c.alpha / aspect;
    c.ay = c.alpha * aspect;
    return c;
}
static void pbr_frame(const RtMaterial& m, V3 n, V3* t, V3* b) {
    V3 t0, b0;
    onb_vec(n, &t0, &b0);
    float ca = std::cos(m.anisotropy_angle), sa = std::sin(m.anisotropy_angle);
    *t = t0 * ca + b0 * sa;
    *b = b0 * ca - t0 * sa;
}
enum { PBR_NONE = 0, PBR_SPECULAR = 1, PBR_DIFFUSE = 2 };
// PbrMaterial::scatter (material.rs:790-920)
static int pbr_scatter(const RtMaterial& m, V3 wo, V3 n, float xi_coat, float xi_spec, float xi1, float xi2,
                       V3* att, V3* dir) {
    float cos_o = dot(wo, n);
    if (cos_o <= 0.0f) return PBR_NONE;
    PbrCommon c = pbr_common(m, cos_o);
    if (xi_coat < c.p_coat) {
        float ac = rmax(m.clearcoat_roughness * m.clearcoat_roughness, 1e-4f);
        V3 t, b;
        onb_vec(n, &t, &b);
        V3 ms = vndf_sample(v3(dot(wo, t), dot(wo, b), cos_o), ac, ac, xi1, xi2);
        V3 mm = unit(t * ms.x + b * ms.y + n * ms.z);
        float vo_h = rmax(dot(wo, mm), 0.0f);
        V3 wi = unit(2.0f * vo_h * mm - wo);
        float cos_i = dot(wi, n);
        if (cos_i <= 0.0f) return PBR_NONE;
        float f_coat = schlick(vo_h, 1.0f / 1.5f) * m.clearcoat;
        float lo = smith_lambda(cos_o, ac), li = smith_lambda(cos_i, ac);
        float w = ((1.0f + lo) / (1.0f + lo + li)) * specular_energy_comp(cos_o, ac);
        V3 film = m.film_thickness > 0.0f ? nacre_color(vo_h, m.film_ior, m.film_thickness) : v3(1, 1, 1);
        *att = film * (f_coat * w / c.p_coat);
        *dir = wi;
        return PBR_SPECULAR;
    }
    if (xi_spec < c.p_spec) {
        V3 t, b;
        pbr_frame(m, n, &t, &b);
        V3 wo_ts = v3(dot(wo, t), dot(wo, b), cos_o);
        V3 ms = vndf_sample(wo_ts, c.ax, c.ay, xi1, xi2);
        V3 mm = unit(t * ms.x + b * ms.y + n * ms.z);
        float vo_h = rmax(dot(wo, mm), 0.0f);
        V3 wi = unit(2.0f * vo_h * mm - wo);
        float cos_i = dot(wi, n);
        if (cos_i <= 0.0f) return PBR_NONE;
        V3 wi_ts = v3(dot(wi, t), dot(wi, b), cos_i);
        float lo = smith_lambda_aniso(cos_o, wo_ts.x, wo_ts.y, c.ax, c.ay);
        float li = smith_lambda_aniso(cos_i, wi_ts.x, wi_ts.y, c.ax, c.ay);
        float w = ((1.0f + lo) / (1.0f + lo + li)) * specular_energy_comp(cos_o, c.alpha);
        *att = schlick_color(vo_h, c.f0) * w / (c.p_spec * (1.0f - c.p_coat));
        *dir = wi;
        return PBR_SPECULAR;
    }
    V3 sheen = v3(0, 0, 0);
    if (m.sheen > 0.0f && m.metallic < 0.999f) {
        float luma = luminance(c.albedo);
        V3 c_tint = luma > 1e-6f ? c.albedo / luma : v3(1, 1, 1);
        V3 sc = v3(1, 1, 1) * (1.0f - m.sheen_tint) + c_tint * m.sheen_tint;
        float u = 1.0f - cos_o, f_h = u * u * u * u * u;
        sheen = sc * (m.sheen * (1.0f - m.metallic) * f_h * PI_F);
    }
    *att = (c.albedo * (1.0f - m.metallic) + sheen) / ((1.0f - c.p_spec) * (1.0f - c.p_coat));
    return PBR_DIFFUSE;
}
// PbrMaterial::specular_brdf_cos (material.rs:935-992)
static V3 pbr_specular_brdf_cos(const RtMaterial& m, V3 wo, V3 n, V3 wi) {
    float cos_o = dot(wo, n), cos_i = dot(wi, n);
    if (cos_o <= 0.0f || cos_i <= 0.0f) return v3(0, 0, 0);
    PbrCommon c = pbr_common(m, cos_o);
    V3 h = unit(wo + wi);
    float wo_h = rmax(dot(wo, h), 0.0f), h_n = rmax(dot(h, n), 0.0f);
    V3 res = v3(0, 0, 0);
    if (m.clearcoat > 1e-3f) {
        float ac = rmax(m.clearcoat_roughness * m.clearcoat_roughness, 1e-4f);
        float d = ggx_ndf(h_n, ac);
        float g2 = 1.0f / (1.0f + smith_lambda(cos_o, ac) + smith_lambda(cos_i, ac));
        float f_c = schlick(wo_h, 1.0f / 1.5f) * m.clearcoat;
        V3 film = m.film_thickness > 0.0f ? nacre_color(wo_h, m.film_ior, m.film_thickness) : v3(1, 1, 1);
        res = res + film * (d * f_c * g2 / (4.0f * cos_o) * specular_energy_comp(cos_o, ac));
    }
    V3 t, b;
    pbr_frame(m, n, &t, &b);
    V3 h_ts = v3(dot(h, t), dot(h, b), h_n);
    float d = ggx_ndf_aniso(h_ts, c.ax, c.ay);
    float g2 = 1.0f / (1.0f + smith_lambda_aniso(cos_o, dot(wo, t), dot(wo, b), c.ax, c.ay) +
                       smith_lambda_aniso(cos_i, dot(wi, t), dot(wi, b), c.ax, c.ay));
    return res + schlick_color(wo_h, c.f0) * (d * g2 / (4.0f * cos_o) * specular_energy_comp(cos_o, c.alpha));
}
// PbrMaterial::specular_sampling_pdf (material.rs:994-1045)
static float pbr_specular_pdf(const RtMaterial& m, V3 wo, V3 n, V3 wi) {
    float cos_o = dot(wo, n), cos_i = dot(wi, n);
    if (cos_o <= 0.0f || cos_i <= 0.0f) return 0.0f;
    PbrCommon c = pbr_common(m, cos_o);
    V3 h = unit(wo + wi);
    float h_n = rmax(dot(h, n), 0.0f);
    float pdf = 0.0f;
    if (m.clearcoat > 1e-3f) {
        float ac = rmax(m.clearcoat_roughness * m.clearcoat_roughness, 1e-4f);
        pdf += c.p_coat * ggx_ndf(h_n, ac) * smith_g1(cos_o, ac) / (4.0f * cos_o);
    }
    if ((1.0f - c.p_coat) * c.p_spec > 1e-6f) {
        V3 t, b;
        pbr_frame(m, n, &t, &b);
        float d = ggx_ndf_aniso(v3(dot(h, t), dot(h, b), h_n), c.ax, c.ay);
        pdf += (1.0f - c.p_coat) * c.p_spec * d * smith_g1_aniso(cos_o, dot(wo, t), dot(wo, b), c.ax, c.ay) /
               (4.0f * cos_o);
    }
    return pdf;
}

// ── scene ────────────────────────────────────────────────────────────────────
struct Aabb { V3 mn, mx; };
static inline Aabb surrounding(const Aabb& a, const Aabb& b) {                     // aabb.rs:10-15
    return Aabb{v3(rmin(a.mn.x, b.mn.x), rmin(a.mn.y, b.mn.y), rmin(a.mn.z, b.mn.z)),
                v3(rmax(a.mx.x, b.mx.x), rmax(a.mx.y, b.mx.y), rmax(a.mx.z, b.mx.z))};
}
static inline Aabb pad(Aabb b) {                                                    // aabb.rs:18-29
    const float D = 0.0001f;
    float px = b.mx.x - b.mn.x < D ? D : 0.0f;
    float py = b.mx.y - b.mn.y < D ? D : 0.0f;
    float pz = b.mx.z - b.mn.z < D ? D : 0.0f;
    return Aabb{v3(b.mn.x - px, b.mn.y - py, b.mn.z - pz), v3(b.mx.x + px, b.mx.y + py, b.mx.z + pz)};
}
static inline float surface_area(const Aabb& b) {                                  // bvh.rs:47-50
    V3 d = b.mx - b.mn;
    return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
}

struct Tri { V3 v0, e1, e2; V3 n0, n1, n2; bool has_n; int mat; float uv[6]; V3 t0, t1, t2; };
struct Quad { V3 q, u, v, normal, w; float d, area; int mat; };
struct Sphere { V3 c; float r; int mat; };

static const int W8 = 8;
struct Node { float mn[3][W8], mx[3][W8]; int32_t ch[W8]; };

struct EnvMap {
    int w = 0, h = 0;
    std::vector<float> img;           // h × w × 3
    std::vector<float> marginal, cond;
    float inv_total = 0.0f, rot_y = 0.0f, sin_r = 0.0f, cos_r = 1.0f;
};

struct Scene {
    std::vector<Tri> tris;
    std::vector<Quad> quads;
    std::vector<Sphere> spheres;
    std::vector<RtMaterial> mats;
    std::vector<int32_t> lights;      // canonical prim ids of the NEE light copies
    RtBackground bg;
    EnvMap env;
    bool has_env = false;
    Spectrum spec;
    // blackbody constants per material (material.rs:47-62)
    std::vector<float> bb_norm;
    std::vector<V3> bb_avg;
    // BVH
    std::vector<Node> nodes;
    std::vector<int32_t> leaf_prims;  // leaf slot → canonical prim id
    int64_t n_tris = 0, n_quads = 0, n_spheres = 0, n_convex = 0;
    // analytic convex solids (diamond.rs:198-253): outward half-spaces n·x ≤ d
    // placed in world space; `off` indexes the solid's own run of world planes
    struct Convex { int32_t off, n, mat; float polish; Aabb box; };
    std::vector<Convex> convex;
    std::vector<float> convex_planes;   // 4 floats per world plane
    std::vector<V3> convex_shade;       // per world plane: front-face and back-face shading normal
    // cylinders, cones, disks, infinite planes (cylinder.rs, cone.rs, disk.rs, plane.rs) in
    // object space with the objects' SRT placement; ids follow the convex solids
    struct Shape {
        int32_t type, mat;
        V3 c, n, u, v;          // centre / point; unit normal and its onb (disk, plane)
        float radius, height, wave_a, wave_s;
        bool placed;            // a non-identity placement
        float R[9], inv_scale;
        V3 t;
        Aabb box;
    };
    int64_t n_shapes = 0;
    std::vector<Shape> shapes;
    // textures (texture.rs)
    struct Texture { int32_t type, w, h; std::vector<uint8_t> px; float scale; V3 lo, hi; float vec[768]; int32_t perm[768]; };
    std::vector<Texture> textures;
    // caustic photon map (photon.rs:31-36): implicit kd-tree, kept in emission order too
    struct KdPhoton { float pos[3], power[3], nor[3]; uint8_t axis; int32_t idx; };
    std::vector<KdPhoton> photons;    // kd order
    std::vector<KdPhoton> photons_by_index;
    bool has_photons = false;
    float gather_r2 = 0.0f, gather_norm = 0.0f;
    uint32_t knn_k = 0;
    // participating media (volume.rs:78-263); a box boundary is its 6 quads
    std::vector<RtMedium> media;
    // grid media (no counterpart in the reference): voxels and per-brick majorants
    struct GridMed { std::vector<float> grid, major; int res[3] = {1, 1, 1}, nb[3] = {1, 1, 1}; V3 lo, inv_vox, bw, inv_bw; };
    std::vector<GridMed> media_grid;
    std::vector<std::vector<Quad>> media_quads;
};

static inline bool is_emissive_type(int t) { return t == RT_MAT_DIFFUSE_LIGHT || t == RT_MAT_BLACKBODY_LIGHT; }
static const int PRIM_SHAPE = 4;   // oracle-internal type of the other analytic shapes
static inline int prim_type(const Scene& s, int64_t gid) {
    if (gid < s.n_tris) return RT_PRIM_TRI;
    if (gid < s.n_tris + s.n_quads) return RT_PRIM_QUAD;
    if (gid < s.n_tris + s.n_quads + s.n_spheres) return RT_PRIM_SPHERE;
    return gid < s.n_tris + s.n_quads + s.n_spheres + s.n_convex ? RT_PRIM_CONVEX : PRIM_SHAPE;
}
static inline int64_t n_prims(const Scene& s) { return s.n_tris + s.n_quads + s.n_spheres + s.n_convex + s.n_shapes; }
static inline const Scene::Shape& shape_of(const Scene& s, int64_t gid) {
    return s.shapes[gid - s.n_tris - s.n_quads - s.n_spheres - s.n_convex];
}

static Aabb prim_box(const Scene& s, int64_t gid) {
    int t = prim_type(s, gid);
    if (t == RT_PRIM_TRI) {                                                         // triangle.rs:128-140
        const Tri& tr = s.tris[gid];
        V3 a = tr.v0, b = tr.v0 + tr.e1, c = tr.v0 + tr.e2;
        Aabb bb{v3(rmin(rmin(a.x, b.x), c.x), rmin(rmin(a.y, b.y), c.y), rmin(rmin(a.z, b.z), c.z)),
                v3(rmax(rmax(a.x, b.x), c.x), rmax(rmax(a.y, b.y), c.y), rmax(rmax(a.z, b.z), c.z))};
        return pad(bb);
    } else if (t == RT_PRIM_QUAD) {                                                 // quad.rs:71-80
        const Quad& q = s.quads[gid - s.n_tris];
        V3 c[4] = {q.q, q.q + q.u, q.q + q.v, q.q + q.u + q.v};
        V3 mn = c[0], mx = c[0];
        for (int i = 1; i < 4; i++) {
            mn = v3(rmin(mn.x, c[i].x), rmin(mn.y, c[i].y), rmin(mn.z, c[i].z));
            mx = v3(rmax(mx.x, c[i].x), rmax(mx.y, c[i].y), rmax(mx.z, c[i].z));
        }
        return pad(Aabb{mn, mx});
    } else if (t == RT_PRIM_SPHERE) {                                               // sphere.rs:111-118
        const Sphere& sp = s.spheres[gid - s.n_tris - s.n_quads];
        V3 r = v3(sp.r, sp.r, sp.r);
        return Aabb{sp.c - r, sp.c + r};
    }
    if (t == PRIM_SHAPE) return shape_of(s, gid).box;
    return s.convex[gid - s.n_tris - s.n_quads - s.n_spheres].box;                  // diamond.rs:172-186
}

// ── BVH build (bvh.rs:52-225) ────────────────────────────────────────────────
static const int NUM_BUCKETS = 12;

struct Builder {
    const std::vector<Aabb>* boxes;
    std::vector<Node>* nodes;
    std::vector<int32_t>* leaf_prims;
};

// sah_partition (bvh.rs:52-145) on the index list `objs`; returns the split point
// after reordering objs into (left, right) by a stable sort on bucket id.
static size_t sah_partition(const std::vector<Aabb>& boxes, std::vector<int32_t>& objs) {
    size_t span = objs.size();
    float c_min[3] = {INFINITY, INFINITY, INFINITY}, c_max[3] = {-INFINITY, -INFINITY, -INFINITY};
    Aabb node_bbox = boxes[objs[0]];
    for (size_t k = 0; k < span; k++) {
        const Aabb& b = boxes[objs[k]];
        for (int a = 0; a < 3; a++) {
            float c = (comp(b.mn, a) + comp(b.mx, a)) * 0.5f;
            c_min[a] = rmin(c_min[a], c);
            c_max[a] = rmax(c_max[a], c);
        }
        if (k > 0) node_bbox = surrounding(node_bbox, b);
    }
    float node_sa = surface_area(node_bbox);
    float best_cost = INFINITY;
    int best_axis = 0, best_split = 0;
    for (int axis = 0; axis < 3; axis++) {
        float extent = c_max[axis] - c_min[axis];
        if (extent < 1e-6f) continue;
        bool has[NUM_BUCKETS] = {};
        Aabb bb[NUM_BUCKETS];
        uint32_t cnt[NUM_BUCKETS] = {};
        for (size_t k = 0; k < span; k++) {
            const Aabb& b = boxes[objs[k]];
            float c = (comp(b.mn, axis) + comp(b.mx, axis)) * 0.5f;
            float t = (c - c_min[axis]) / extent;
            int bi = std::min((int)((float)NUM_BUCKETS * t), NUM_BUCKETS - 1);
            cnt[bi]++;
            bb[bi] = has[bi] ? surrounding(bb[bi], b) : b;
            has[bi] = true;
        }
        float left_sa[NUM_BUCKETS]; uint32_t left_n[NUM_BUCKETS];
        bool acc_has = false; Aabb acc; uint32_t acc_n = 0;
        for (int i = 0; i < NUM_BUCKETS; i++) {
            acc_n += cnt[i];
            if (has[i]) { acc = acc_has ? surrounding(acc, bb[i]) : bb[i]; acc_has = true; }
            left_n[i] = acc_n;
            left_sa[i] = acc_has ? surface_area(acc) : 0.0f;
        }
        acc_has = false; acc_n = 0;
        for (int split = NUM_BUCKETS - 2; split >= 0; split--) {
            acc_n += cnt[split + 1];
            if (has[split + 1]) { acc = acc_has ? surrounding(acc, bb[split + 1]) : bb[split + 1]; acc_has = true; }
            uint32_t nl = left_n[split], nr = acc_n;
            if (nl == 0 || nr == 0) continue;
            float right_sa = acc_has ? surface_area(acc) : 0.0f;
            float cost = 1.0f + (left_sa[split] * (float)nl + right_sa * (float)nr) / node_sa;
            if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = split; }
        }
    }
    float extent = c_max[best_axis] - c_min[best_axis];
    // stable counting sort by bucket id == order.sort_by_key(bid) (a stable sort)
    std::vector<int32_t> bucketed[NUM_BUCKETS];
    for (size_t k = 0; k < span; k++) {
        int bi = 0;
        if (!(extent < 1e-6f)) {
            const Aabb& b = boxes[objs[k]];
            float c = (comp(b.mn, best_axis) + comp(b.mx, best_axis)) * 0.5f;
            float t = (c - c_min[best_axis]) / extent;
            bi = std::min((int)((float)NUM_BUCKETS * t), NUM_BUCKETS - 1);
        }
        bucketed[bi].push_back(objs[k]);
    }
    size_t pos = 0, mid_off = 0;
    for (int bkt = 0; bkt < NUM_BUCKETS; bkt++) {
        for (int32_t o : bucketed[bkt]) objs[pos++] = o;
        if (bkt == best_split) mid_off = pos;
    }
    return (mid_off == 0 || mid_off == span) ? span / 2 : mid_off;
}

static void split_recursive(const std::vector<Aabb>& boxes, std::vector<int32_t> objs, int depth,
                            std::vector<std::vector<int32_t>>& out) {              // bvh.rs:148-162
    if (depth == 3 || objs.size() <= 1) { out.push_back(std::move(objs)); return; }
    size_t mid = sah_partition(boxes, objs);
    std::vector<int32_t> l(objs.begin(), objs.begin() + mid), r(objs.begin() + mid, objs.end());
    split_recursive(boxes, std::move(l), depth + 1, out);
    split_recursive(boxes, std::move(r), depth + 1, out);
}

static int32_t build_rec(Builder& B, const std::vector<int32_t>& objs, Aabb* out_box) {   // bvh.rs:290-323
    const std::vector<Aabb>& boxes = *B.boxes;
    if (objs.size() == 1) {
        int32_t idx = (int32_t)B.leaf_prims->size();
        B.leaf_prims->push_back(objs[0]);
        *out_box = boxes[objs[0]];
        return -(idx + 1);
    }
    std::vector<std::vector<int32_t>> groups;
    if (objs.size() <= (size_t)W8) {                                                // split_n, bvh.rs:165-174
        for (int32_t o : objs) groups.push_back(std::vector<int32_t>{o});
    } else {
        split_recursive(boxes, objs, 0, groups);
    }
    size_t my = B.nodes->size();
    Node sentinel;
    memset(&sentinel, 0, sizeof(sentinel));
    for (int c = 0; c < W8; c++) sentinel.ch[c] = INT32_MIN;
    B.nodes->push_back(sentinel);
    Node node = sentinel;
    Aabb nb{};
    for (size_t i = 0; i < groups.size(); i++) {
        Aabb cb;
        int32_t child = build_rec(B, groups[i], &cb);
        node.ch[i] = child;
        for (int a = 0; a < 3; a++) { node.mn[a][i] = comp(cb.mn, a); node.mx[a][i] = comp(cb.mx, a); }
        nb = i == 0 ? cb : surrounding(nb, cb);
    }
    (*B.nodes)[my] = node;
    *out_box = nb;
    return (int32_t)my;
}

static void build_bvh(Scene& s) {                                                   // bvh.rs:199-225
    int64_t n = n_prims(s);
    s.nodes.clear(); s.leaf_prims.clear();
    if (n == 0) return;
    std::vector<Aabb> boxes(n);
    for (int64_t i = 0; i < n; i++) boxes[i] = prim_box(s, i);
    std::vector<int32_t> objs(n);
    for (int64_t i = 0; i < n; i++) objs[i] = (int32_t)i;
    s.nodes.reserve(n / 4 + 1);
    Builder B{&boxes, &s.nodes, &s.leaf_prims};
    Aabb root_box;
    int32_t root = build_rec(B, objs, &root_box);
    if (root < 0) {
        Node nd;
        memset(&nd, 0, sizeof(nd));
        for (int c = 0; c < W8; c++) nd.ch[c] = INT32_MIN;
        nd.ch[0] = root;
        for (int a = 0; a < 3; a++) { nd.mn[a][0] = comp(boxes[0].mn, a); nd.mx[a][0] = comp(boxes[0].mx, a); }
        s.nodes.push_back(nd);
    }
}

// ── primitive tests ──────────────────────────────────────────────────────────
struct Ray { V3 o, d; };

// triangle.rs:75-89 (hit) — returns t, barycentrics
static inline bool tri_hit(const Tri& tr, const Ray& r, float tmin, float tmax, float* t_out, float* b1o, float* b2o) {
    V3 h = cross(r.d, tr.e2);
    float a = dot(tr.e1, h);
    if (std::fabs(a) < 1e-8f) return false;
    float f = 1.0f / a;
    V3 s = r.o - tr.v0;
    float b1 = f * dot(s, h);
    if (!(b1 >= 0.0f && b1 <= 1.0f)) return false;
    V3 q = cross(s, tr.e1);
    float b2 = f * dot(r.d, q);
    if (b2 < 0.0f || b1 + b2 > 1.0f) return false;
    float t = f * dot(tr.e2, q);
    if (t < tmin || t > tmax) return false;
    *t_out = t; *b1o = b1; *b2o = b2;
    return true;
}
// quad.rs:37-57
static inline bool quad_hit(const Quad& q, const Ray& r, float tmin, float tmax, float* t_out, float* al, float* be) {
    float denom = dot(q.normal, r.d);
    if (!(std::fabs(denom) >= 1e-8f)) return false;
    float t = (q.d - dot(q.normal, r.o)) / denom;
    if (t < tmin || t > tmax) return false;
    V3 p = r.o + t * r.d;
    V3 planar = p - q.q;
    float alpha = dot(q.w, cross(planar, q.v));
    float beta = dot(q.w, cross(q.u, planar));
    if (!(alpha >= 0.0f && alpha <= 1.0f) || !(beta >= 0.0f && beta <= 1.0f)) return false;
    *t_out = t; *al = alpha; *be = beta;
    return true;
}
// sphere.rs:47-61
static inline bool sphere_hit(const Sphere& sp, const Ray& r, float tmin, float tmax, float* t_out) {
    V3 oc = r.o - sp.c;
    float a = len2(r.d);
    if (!(a > 0.0f)) return false;
    float half_b = dot(oc, r.d);
    float c = len2(oc) - sp.r * sp.r;
    float disc = half_b * half_b - a * c;
    if (disc < 0.0f) return false;
    float sq = std::sqrt(disc);
    float root = (-half_b - sq) / a;
    if (root < tmin || root > tmax) {
        root = (-half_b + sq) / a;
        if (root < tmin || root > tmax) return false;
    }
    *t_out = root;
    return true;
}
// convex_hit (diamond.rs:202-253): the interval inside every half-space; the
// entry for outside rays, the exit for rays inside the solid.  *plane is the
// index of the crossing plane.
static bool convex_hit(const float* planes, int32_t n, const Ray& r, float tmin, float tmax, float* t_out,
                       int32_t* plane) {
    float t_enter = tmin, t_exit = tmax;
    int32_t enter_i = -1, exit_i = -1;
    bool entry_found = false;
    for (int32_t i = 0; i < n; i++) {
        V3 nv = v3(planes[i * 4], planes[i * 4 + 1], planes[i * 4 + 2]);
        float d = planes[i * 4 + 3];
        float nd = dot(nv, r.d);
        float t_face = (d - dot(nv, r.o)) / nd;
        if (std::fabs(nd) < 1e-8f) {
            if (dot(nv, r.o) > d) return false;
            continue;
        }
        if (nd < 0.0f) {
            if (t_face > t_enter) { t_enter = t_face; enter_i = i; entry_found = true; }
        } else {
            // an exit exactly at tmax still names its plane
            if (t_face < t_exit || (exit_i < 0 && t_face == t_exit)) { t_exit = t_face; exit_i = i; }
        }
        if (t_enter > t_exit) return false;
    }
    if (t_enter > t_exit) return false;
    if (t_enter == t_exit && t_enter < tmax) return false;
    if (entry_found) { *t_out = t_enter; *plane = enter_i; return true; }
    // An interior ray whose exit lies beyond tmax crosses no surface in
    // [tmin, tmax].  The reference returns t_max with a default normal here,
    // a phantom that its last-visited tie rule lets win against a real hit at
    // the same t, so the answer would depend on the traversal order.
    if (exit_i < 0 || t_exit > tmax) return false;
    *t_out = t_exit; *plane = exit_i;
    return true;
}

// ── cylinder, cone, disk, infinite plane ──────────────────────────────────────
// The ray in the shape's object space through the SRT wrappers, outermost
// first: Translate, Rotate (mat_apply_t), UniformScale (transform.rs:29-45,
// 158-164, 228-242).
static inline Ray shape_local(const Scene::Shape& sh, const Ray& r) {
    if (!sh.placed) return r;
    V3 o1 = r.o - sh.t;
    const float* m = sh.R;
    V3 o2 = v3(m[0] * o1.x + m[3] * o1.y + m[6] * o1.z, m[1] * o1.x + m[4] * o1.y + m[7] * o1.z,
               m[2] * o1.x + m[5] * o1.y + m[8] * o1.z);
    V3 d2 = v3(m[0] * r.d.x + m[3] * r.d.y + m[6] * r.d.z, m[1] * r.d.x + m[4] * r.d.y + m[7] * r.d.z,
               m[2] * r.d.x + m[5] * r.d.y + m[8] * r.d.z);
    return Ray{sh.inv_scale * o2, sh.inv_scale * d2};
}
// the closest crossing in [tmin, tmax] and which surface: 0 lateral (or the
// disk / plane), 1 bottom cap or cone base, 2 top cap
static bool shape_hit(const Scene::Shape& sh, const Ray& r, float tmin, float tmax, float* t_out, int32_t* part) {
    if (sh.type == RT_SHAPE_CYLINDER || sh.type == RT_SHAPE_CONE) {
        bool cone = sh.type == RT_SHAPE_CONE;
        V3 oc = r.o - sh.c;
        float dx = r.d.x, dy = r.d.y, dz = r.d.z, h = sh.height;
        float best_t = tmax;
        bool found = false;
        float a, half_b, c;
        if (cone) {                                                                  // cone.rs:19-63
            float k = (sh.radius / h) * (sh.radius / h), hy = h - oc.y;
            a = dx * dx + dz * dz - k * dy * dy;
            half_b = oc.x * dx + oc.z * dz + k * hy * dy;
            c = oc.x * oc.x + oc.z * oc.z - k * hy * hy;
        } else {                                                                     // cylinder.rs:132-167
            a = dx * dx + dz * dz;
            half_b = oc.x * dx + oc.z * dz;
            c = oc.x * oc.x + oc.z * oc.z - sh.radius * sh.radius;
        }
        if (cone ? std::fabs(a) > 1e-8f : a > 1e-8f) {
            float disc = half_b * half_b - a * c;
            if (disc >= 0.0f) {
                float sq = std::sqrt(disc);
                float roots[2] = {(-half_b - sq) / a, (-half_b + sq) / a};
                for (float root : roots) {
                    if (root < tmin || root > best_t) continue;
                    float ly = (r.o + root * r.d).y - sh.c.y;
                    if (ly < 0.0f || ly > h) continue;
                    best_t = root; *part = 0; found = true;
                }
            }
        }
        if (std::fabs(dy) > 1e-8f) {                                                // caps / base disk
            int ncap = cone ? 1 : 2;
            for (int k = 0; k < ncap; k++) {
                float cap_y = k == 0 ? 0.0f : h;
                float t = cone ? -oc.y / dy : (cap_y - oc.y) / dy;
                if (cone ? !(t >= tmin && t <= best_t) : (t < tmin || t > best_t)) continue;
                V3 p = r.o + t * r.d;
                float lx = p.x - sh.c.x, lz = p.z - sh.c.z;
                if (lx * lx + lz * lz > sh.radius * sh.radius) continue;
                best_t = t; *part = 1 + k; found = true;
            }
        }
        if (found) *t_out = best_t;
        return found;
    }
    float denom = dot(sh.n, r.d);                                                   // disk.rs:146-157, plane.rs:37-42
    if (!(std::fabs(denom) >= 1e-8f)) return false;
    float t = dot(sh.n, sh.c - r.o) / denom;
    if (t < tmin || t > tmax) return false;
    if (sh.type == RT_SHAPE_DISK) {
        V3 off = (r.o + t * r.d) - sh.c;
        if (len2(off) > sh.radius * sh.radius) return false;
    }
    *t_out = t; *part = 0;
    return true;
}
// object-space outward normal of a crossing (cylinder.rs:155-159, cone.rs:50-54,
// the caps, disk.rs:153, plane.rs:46-66 with the wave bump)
static V3 shape_outward(const Scene::Shape& sh, V3 p, int32_t part) {
    if (sh.type == RT_SHAPE_CYLINDER) {
        if (part == 0) return v3((p.x - sh.c.x) / sh.radius, 0.0f, (p.z - sh.c.z) / sh.radius);
        return v3(0.0f, part == 1 ? -1.0f : 1.0f, 0.0f);
    }
    if (sh.type == RT_SHAPE_CONE) {
        if (part != 0) return v3(0.0f, -1.0f, 0.0f);
        float h = sh.height, k = (sh.radius / h) * (sh.radius / h);
        float ly = p.y - sh.c.y;
        V3 g = v3(p.x - sh.c.x, k * (h - ly), p.z - sh.c.z);
        return len2(g) > 1e-12f ? unit(g) : v3(0.0f, 1.0f, 0.0f);
    }
    if (sh.type == RT_SHAPE_PLANE && sh.wave_a > 1e-6f) {
        V3 off = p - sh.c;
        float u = dot(off, sh.u), v = dot(off, sh.v), sc = sh.wave_s, a = sh.wave_a;
        float phi1 = sc * u + 0.7f * sc * v, phi2 = 1.3f * sc * v - 0.5f * sc * u;
        float dh_du = a * sc * std::cos(phi1) - 0.25f * a * sc * std::cos(phi2);
        float dh_dv = 0.7f * a * sc * std::cos(phi1) + 0.65f * a * sc * std::cos(phi2);
        return unit(sh.n - dh_du * sh.u - dh_dv * sh.v);
    }
    return sh.n;
}

static inline bool prim_hit(const Scene& s, int64_t gid, const Ray& r, float tmin, float tmax,
                            float* t, float* b1, float* b2) {
    if (gid < s.n_tris) return tri_hit(s.tris[gid], r, tmin, tmax, t, b1, b2);
    if (gid < s.n_tris + s.n_quads) return quad_hit(s.quads[gid - s.n_tris], r, tmin, tmax, t, b1, b2);
    *b1 = 0.0f; *b2 = 0.0f;
    if (gid < s.n_tris + s.n_quads + s.n_spheres) return sphere_hit(s.spheres[gid - s.n_tris - s.n_quads], r, tmin, tmax, t);
    if (prim_type(s, gid) == PRIM_SHAPE) {
        const Scene::Shape& sh = shape_of(s, gid);
        int32_t part = 0;
        if (!shape_hit(sh, shape_local(sh, r), tmin, tmax, t, &part)) return false;
        memcpy(b1, &part, 4);
        return true;
    }
    const Scene::Convex& c = s.convex[gid - s.n_tris - s.n_quads - s.n_spheres];
    int32_t pi = -1;
    if (!convex_hit(s.convex_planes.data() + (size_t)c.off * 4, c.n, r, tmin, tmax, t, &pi)) return false;
    // the crossing plane's index rides in b1 (an exit with no exit plane keeps -1)
    int32_t bits = pi;
    memcpy(b1, &bits, 4);
    return true;
}

// ── traversal (bvh.rs:229-288, slab test :326-364) ───────────────────────────
static const float SLAB_WIDEN = 1.52587890625e-05f;   // 2^-16

// Reciprocal direction for the slab test.  A zero (or denormal) component gives
// ±inf and, for a ray lying exactly in a box face plane, (bound − o)·inv = 0·∞
// = NaN; that slab is then taken as the whole line (the ray is inside the
// closed slab), so culling stays conservative (the AVX2 path of the reference,
// bvh.rs:326-364, drops such boxes — bvh.rs:450-456 documents the asymmetry).
static inline float safe_inv(float d) { return 1.0f / d; }

struct TraceStats { int64_t nodes = 0, tris = 0, quads = 0, spheres = 0; };

// 8-wide AVX2 slab test; returns the hit mask and t_near per child.
static inline uint32_t slab8(const Node& nd, const float ro[3], const float id[3], float tmin, float tmax, float tnear[8]) {
    __m256i ch = _mm256_loadu_si256((const __m256i*)nd.ch);
    __m256i sent = _mm256_set1_epi32(INT32_MIN);
    uint32_t invalid = (uint32_t)_mm256_movemask_ps(_mm256_castsi256_ps(_mm256_cmpeq_epi32(ch, sent)));
    __m256 t0 = _mm256_set1_ps(tmin), t1 = _mm256_set1_ps(tmax);
    const __m256 ninf = _mm256_set1_ps(-INFINITY), pinf = _mm256_set1_ps(INFINITY);
    for (int a = 0; a < 3; a++) {
        __m256 o = _mm256_set1_ps(ro[a]), iv = _mm256_set1_ps(id[a]);
        __m256 da = _mm256_mul_ps(_mm256_sub_ps(_mm256_loadu_ps(nd.mn[a]), o), iv);
        __m256 db = _mm256_mul_ps(_mm256_sub_ps(_mm256_loadu_ps(nd.mx[a]), o), iv);
        __m256 nan = _mm256_cmp_ps(da, db, _CMP_UNORD_Q);
        __m256 lo = _mm256_blendv_ps(_mm256_min_ps(da, db), ninf, nan);
        __m256 hi = _mm256_blendv_ps(_mm256_max_ps(da, db), pinf, nan);
        t0 = _mm256_max_ps(t0, lo);
        t1 = _mm256_min_ps(t1, hi);
    }
    // widened exit: t1 + |t1|·2^-16 (conservative culling)
    __m256 absmask = _mm256_castsi256_ps(_mm256_set1_epi32(0x7fffffff));
    __m256 t1w = _mm256_add_ps(t1, _mm256_mul_ps(_mm256_and_ps(t1, absmask), _mm256_set1_ps(SLAB_WIDEN)));
    uint32_t mask = (uint32_t)_mm256_movemask_ps(_mm256_cmp_ps(t0, t1w, _CMP_LE_OQ));
    _mm256_storeu_ps(tnear, t0);
    return mask & (~invalid) & 0xffu;
}

struct HitRes { int32_t gid; float t, b1, b2; };

// A ray with a NaN coordinate or bound hits nothing (the reference would let a
// NaN sphere root through its range check, sphere.rs:57-61).
static inline bool ray_has_nan(const Ray& r, float tmin, float tmax) {
    return std::isnan(r.o.x) || std::isnan(r.o.y) || std::isnan(r.o.z) || std::isnan(r.d.x) || std::isnan(r.d.y) ||
           std::isnan(r.d.z) || std::isnan(tmin) || std::isnan(tmax);
}

template <bool STATS>
static HitRes closest_hit(const Scene& s, const Ray& r, float tmin, float tmax, TraceStats* st) {
    HitRes best{-1, tmax, 0.0f, 0.0f};
    if (s.nodes.empty() || ray_has_nan(r, tmin, tmax)) return best;
    int32_t stack[128];
    std::vector<int32_t> overflow;
    int top = 0;
    stack[top++] = 0;
    float ro[3] = {r.o.x, r.o.y, r.o.z};
    float id[3] = {safe_inv(r.d.x), safe_inv(r.d.y), safe_inv(r.d.z)};
    float closest = tmax;
    while (top > 0 || !overflow.empty()) {
        int32_t e;
        if (top > 0) e = stack[--top]; else { e = overflow.back(); overflow.pop_back(); }
        if (e < 0) {
            int32_t gid = s.leaf_prims[-e - 1];
            if (STATS) {
                int t = prim_type(s, gid);
                if (t == RT_PRIM_TRI) st->tris++; else if (t == RT_PRIM_QUAD) st->quads++; else st->spheres++;
            }
            float t, b1, b2;
            if (prim_hit(s, gid, r, tmin, closest, &t, &b1, &b2)) {
                if (t < closest || best.gid < 0 || gid < best.gid) {
                    closest = t;
                    best = HitRes{gid, t, b1, b2};
                }
            }
            continue;
        }
        const Node& nd = s.nodes[e];
        if (STATS) st->nodes++;
        float tn[8];
        uint32_t mask = slab8(nd, ro, id, tmin, closest, tn);
        if (!mask) continue;
        float ht[8]; int32_t hc[8]; int n = 0;
        for (int c = 0; c < 8; c++) if (mask & (1u << c)) { ht[n] = tn[c]; hc[n] = nd.ch[c]; n++; }
        // sort far-to-near so the nearest is popped first (bvh.rs:271-284)
        for (int i = 1; i < n; i++) {
            float tv = ht[i]; int32_t cv = hc[i]; int j = i - 1;
            while (j >= 0 && ht[j] < tv) { ht[j + 1] = ht[j]; hc[j + 1] = hc[j]; j--; }
            ht[j + 1] = tv; hc[j + 1] = cv;
        }
        for (int i = 0; i < n; i++) {
            if (top < 128) stack[top++] = hc[i]; else overflow.push_back(hc[i]);
        }
    }
    return best;
}

static HitRes closest_hit_brute(const Scene& s, const Ray& r, float tmin, float tmax) {
    HitRes best{-1, tmax, 0.0f, 0.0f};
    if (ray_has_nan(r, tmin, tmax)) return best;
    int64_t n = n_prims(s);
    float closest = tmax;
    for (int64_t g = 0; g < n; g++) {
        float t, b1, b2;
        if (prim_hit(s, g, r, tmin, closest, &t, &b1, &b2)) {
            if (t < closest || best.gid < 0) { closest = t; best = HitRes{(int32_t)g, t, b1, b2}; }
        }
    }
    return best;
}

// any_hit / opaque transmittance (bvh.rs:487-575)
static bool any_hit(const Scene& s, const Ray& r, float tmin, float tmax) {
    if (s.nodes.empty() || ray_has_nan(r, tmin, tmax)) return false;
    int32_t stack[128];
    std::vector<int32_t> overflow;
    int top = 0;
    stack[top++] = 0;
    float ro[3] = {r.o.x, r.o.y, r.o.z};
    float id[3] = {safe_inv(r.d.x), safe_inv(r.d.y), safe_inv(r.d.z)};
    while (top > 0 || !overflow.empty()) {
        int32_t e;
        if (top > 0) e = stack[--top]; else { e = overflow.back(); overflow.pop_back(); }
        if (e < 0) {
            float t, b1, b2;
            if (prim_hit(s, s.leaf_prims[-e - 1], r, tmin, tmax, &t, &b1, &b2)) return true;
            continue;
        }
        float tn[8];
        uint32_t mask = slab8(s.nodes[e], ro, id, tmin, tmax, tn);
        for (int c = 0; c < 8; c++)
            if (mask & (1u << c)) { if (top < 128) stack[top++] = s.nodes[e].ch[c]; else overflow.push_back(s.nodes[e].ch[c]); }
    }
    return false;
}

// ── participating media (volume.rs:39-263, perlin.rs:35-91) ──────────────────
// A medium's random stream is keyed on the ray's bits, as the reference seeds
// a SmallRng from origin xyz, direction x and wavelength (volume.rs:114-120):
// here a pcg3d stream of those bits, identical on the CPU and the GPU.
struct MedRng { uint32_t a, b, c; };
static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline MedRng medium_rng(V3 o, V3 d, float lam) {
    MedRng r;
    r.a = fbits(o.x) ^ mix32(fbits(d.x) + 0x9E3779B9u);
    r.b = fbits(o.y) ^ mix32(fbits(lam) + 0x7F4A7C15u);
    r.c = mix32(fbits(o.z) + 0x4D454449u);
    return r;
}
static inline float medium_rnd(const MedRng& r, uint32_t i) {
    return (float)(pcg3d_x(r.a, r.b, r.c ^ (i * 0x9E3779B9u)) >> 8) * (1.0f / 16777216.0f);
}

// Perlin::noise / turb (perlin.rs:35-91)
static float perlin_noise(const float* perlin_vec, const int32_t* perlin_perm, V3 p) {
    float fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
    float u = p.x - fx, v = p.y - fy, w = p.z - fz;
    u = u * u * (3.0f - 2.0f * u);
    v = v * v * (3.0f - 2.0f * v);
    w = w * w * (3.0f - 2.0f * w);
    int i = (int)fx, j = (int)fy, k = (int)fz;
    float accum = 0.0f;
    for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++)
            for (int dk = 0; dk < 2; dk++) {
                int idx = perlin_perm[(i + di) & 255] ^ perlin_perm[256 + ((j + dj) & 255)] ^
                          perlin_perm[512 + ((k + dk) & 255)];
                V3 c = v3(perlin_vec[idx * 3], perlin_vec[idx * 3 + 1], perlin_vec[idx * 3 + 2]);
                float fi = (float)di, fj = (float)dj, fk = (float)dk;
                V3 wt = v3(u - fi, v - fj, w - fk);
                accum += (fi * u + (1.0f - fi) * (1.0f - u)) * (fj * v + (1.0f - fj) * (1.0f - v)) *
                         (fk * w + (1.0f - fk) * (1.0f - w)) * dot(c, wt);
            }
    return accum;
}
static float perlin_turb(const float* perlin_vec, const int32_t* perlin_perm, V3 p, int depth) {
    float accum = 0.0f, weight = 1.0f;
    for (int i = 0; i < depth; i++) {
        accum += weight * perlin_noise(perlin_vec, perlin_perm, p);
        weight *= 0.5f;
        p = v3(p.x * 2.0f, p.y * 2.0f, p.z * 2.0f);
    }
    return std::fabs(accum);
}
// NoiseMedium::density_at (volume.rs:188-191); density holds max(density, ε)
// and threshold is clamped to [0, 0.99] at scene creation (volume.rs:180-184)
static float medium_density_at(const RtMedium& m, V3 p) {
    float n = perlin_turb(m.perlin_vec, m.perlin_perm, p * m.noise_scale, 7) * 0.5f;
    return rmax(n - m.threshold, 0.0f) * m.density;
}

// First boundary hit in [tmin, tmax]: the sphere's near-then-far root, or the
// nearest of the box's 6 quads (the BvhTree over make_box, quad.rs:201-215).
static bool bound_hit(const Scene& s, int mi, const Ray& r, float tmin, float tmax, float* t) {
    const RtMedium& m = s.media[mi];
    if (m.boundary == RT_BOUND_SPHERE)
        return sphere_hit(Sphere{v3(m.center[0], m.center[1], m.center[2]), m.radius, 0}, r, tmin, tmax, t);
    bool any = false;
    float closest = tmax;
    for (const Quad& q : s.media_quads[mi]) {
        float tq, a, b;
        if (quad_hit(q, r, tmin, closest, &tq, &a, &b)) { closest = tq; any = true; }
    }
    *t = closest;
    return any;
}

// ── grid medium (no counterpart in the reference) ────────────────────────────
// σ_t(x) = density × trilinear interpolation of the voxels between voxel
// centres, clamped at the box faces; majorants per brick of 8³ voxels, each the
// largest voxel its lookups read (one voxel of apron) enlarged by 2^-20.
static const int GRID_BRICK = 8;
static const uint32_t GRID_MAX_STEPS = 4096;
static float grid_density_at(const RtMedium& m, const Scene::GridMed& G, V3 p) {
    const float c[3] = {(p.x - G.lo.x) * G.inv_vox.x - 0.5f, (p.y - G.lo.y) * G.inv_vox.y - 0.5f,
                        (p.z - G.lo.z) * G.inv_vox.z - 0.5f};
    int i0[3], i1[3];
    float f[3];
    for (int a = 0; a < 3; a++) {
        float u = rmin(rmax(c[a], 0.0f), (float)(G.res[a] - 1));
        int i = std::min((int)u, std::max(G.res[a] - 2, 0));
        i0[a] = i;
        i1[a] = std::min(i + 1, G.res[a] - 1);
        f[a] = u - (float)i;
    }
    auto at = [&](int i, int j, int k) { return G.grid[((size_t)k * G.res[1] + j) * G.res[0] + i]; };
    float c00 = at(i0[0], i0[1], i0[2]) * (1.0f - f[0]) + at(i1[0], i0[1], i0[2]) * f[0];
    float c10 = at(i0[0], i1[1], i0[2]) * (1.0f - f[0]) + at(i1[0], i1[1], i0[2]) * f[0];
    float c01 = at(i0[0], i0[1], i1[2]) * (1.0f - f[0]) + at(i1[0], i0[1], i1[2]) * f[0];
    float c11 = at(i0[0], i1[1], i1[2]) * (1.0f - f[0]) + at(i1[0], i1[1], i1[2]) * f[0];
    float c0 = c00 * (1.0f - f[1]) + c10 * f[1], c1 = c01 * (1.0f - f[1]) + c11 * f[1];
    return m.density * (c0 * (1.0f - f[2]) + c1 * f[2]);
}

// 3-D DDA over the majorant bricks (Amanatides & Woo 1987) from the point at t0
struct BrickWalk { int b[3], step[3]; float tnext[3], dt[3]; };
static void brick_walk_init(const Scene::GridMed& G, const Ray& r, float t0, BrickWalk& w) {
    V3 p = r.o + t0 * r.d;
    const float pc[3] = {p.x, p.y, p.z}, oc[3] = {r.o.x, r.o.y, r.o.z}, dc[3] = {r.d.x, r.d.y, r.d.z};
    const float lo[3] = {G.lo.x, G.lo.y, G.lo.z}, bw[3] = {G.bw.x, G.bw.y, G.bw.z};
    const float ib[3] = {G.inv_bw.x, G.inv_bw.y, G.inv_bw.z};
    for (int a = 0; a < 3; a++) {
        int b = (int)std::floor((pc[a] - lo[a]) * ib[a]);
        b = std::min(std::max(b, 0), G.nb[a] - 1);
        w.b[a] = b;
        if (dc[a] > 0.0f) {
            w.step[a] = 1;
            w.tnext[a] = (lo[a] + (float)(b + 1) * bw[a] - oc[a]) / dc[a];
            w.dt[a] = bw[a] / dc[a];
        } else if (dc[a] < 0.0f) {
            w.step[a] = -1;
            w.tnext[a] = (lo[a] + (float)b * bw[a] - oc[a]) / dc[a];
            w.dt[a] = -bw[a] / dc[a];
        } else {
            w.step[a] = 0;
            w.tnext[a] = INFINITY;
            w.dt[a] = INFINITY;
        }
    }
}
static bool brick_walk_next(const Scene::GridMed& G, BrickWalk& w) {
    int a = w.tnext[0] <= w.tnext[1] ? (w.tnext[0] <= w.tnext[2] ? 0 : 2) : (w.tnext[1] <= w.tnext[2] ? 1 : 2);
    w.b[a] += w.step[a];
    w.tnext[a] += w.dt[a];
    return w.b[a] >= 0 && w.b[a] < G.nb[a];
}
static float brick_major(const RtMedium& m, const Scene::GridMed& G, const BrickWalk& w) {
    return m.density * G.major[((size_t)w.b[2] * G.nb[1] + w.b[1]) * G.nb[0] + w.b[0]];
}
static const int GRID_MAX_SEGMENTS = 3 * RT_GRID_MAX_RES / GRID_BRICK + 4;

// delta tracking (Woodcock) in [t1, t2] against each brick's majorant
static float grid_sample(const RtMedium& m, const Scene::GridMed& G, const Ray& r, float lam, float t1, float t2) {
    MedRng g = medium_rng(r.o, r.d, lam);
    float len = length(r.d);
    BrickWalk w;
    brick_walk_init(G, r, t1, w);
    float t = t1;
    uint32_t k = 0;
    for (int seg = 0; seg < GRID_MAX_SEGMENTS; seg++) {
        float tb = rmin(rmin(w.tnext[0], w.tnext[1]), rmin(w.tnext[2], t2));
        float mu = brick_major(m, G, w);
        if (mu > 0.0f) {
            float inv = 1.0f / (mu * len);
            while (k < GRID_MAX_STEPS) {
                float tt = t - inv * std::log(rmax(medium_rnd(g, 2 * k), FLT_EPSILON));
                float xi = medium_rnd(g, 2 * k + 1);
                k++;
                if (tt >= tb) break;
                t = tt;
                if (xi * mu < grid_density_at(m, G, r.o + t * r.d)) return t;
            }
            if (k >= GRID_MAX_STEPS) return INFINITY;
        }
        if (tb >= t2) return INFINITY;
        t = rmax(t, tb);
        if (!brick_walk_next(G, w)) return INFINITY;
    }
    return INFINITY;
}

// ratio tracking (Cramer 1978; Novák et al. 2014) over [a, b]: the product of
// (1 − σ_t/μ) at tentative collisions, an unbiased estimate of exp(−∫σ_t)
static float grid_transmittance(const RtMedium& m, const Scene::GridMed& G, const Ray& r, float a, float b, float tmax) {
    MedRng g = medium_rng(r.o, r.d, tmax);
    float len = length(r.d);
    BrickWalk w;
    brick_walk_init(G, r, a, w);
    float t = a, T = 1.0f;
    uint32_t k = 0;
    for (int seg = 0; seg < GRID_MAX_SEGMENTS; seg++) {
        float tb = rmin(rmin(w.tnext[0], w.tnext[1]), rmin(w.tnext[2], b));
        float mu = brick_major(m, G, w);
        if (mu > 0.0f) {
            float inv = 1.0f / (mu * len);
            while (k < GRID_MAX_STEPS) {
                float tt = t - inv * std::log(rmax(medium_rnd(g, 0x40000u + k), FLT_EPSILON));
                k++;
                if (tt >= tb) break;
                t = tt;
                T *= rmax(1.0f - grid_density_at(m, G, r.o + t * r.d) / mu, 0.0f);
                if (T <= 0.0f) return 0.0f;
            }
            if (k >= GRID_MAX_STEPS) return T;
        }
        if (tb >= b) return T;
        t = rmax(t, tb);
        if (!brick_walk_next(G, w)) return T;
    }
    return T;
}

// Scatter distance of ConstantMedium::hit (volume.rs:97-138) / NoiseMedium::hit
// (:195-235) for t_max = ∞; INFINITY when the ray leaves the medium first.  The
// candidate depends on the ray alone, so "nearest of surface and medium" gives
// the reference's closest hit for any traversal order.  Delta tracking is
// bounded at 4096 steps (the reference loops until exit).
static float medium_sample(const Scene& s, int mi, const Ray& r, float lam, float tmin) {
    const RtMedium& m = s.media[mi];
    float t1, t2;
    if (!bound_hit(s, mi, r, -INFINITY, INFINITY, &t1)) return INFINITY;
    if (!bound_hit(s, mi, r, t1 + 0.0001f, INFINITY, &t2)) return INFINITY;
    if (t1 < tmin) t1 = tmin;
    if (t1 >= t2) return INFINITY;
    if (t1 < 0.0f) t1 = 0.0f;
    if (m.type == RT_MEDIUM_GRID) return grid_sample(m, s.media_grid[mi], r, lam, t1, t2);
    float len = length(r.d);
    MedRng g = medium_rng(r.o, r.d, lam);
    if (m.type == RT_MEDIUM_CONSTANT) {
        float dist_inside = (t2 - t1) * len;
        float xi = rmax(medium_rnd(g, 0), FLT_EPSILON);
        float hit_dist = (-1.0f / m.density) * std::log(xi);
        if (hit_dist > dist_inside) return INFINITY;
        return t1 + hit_dist / len;
    }
    float inv_maj = 1.0f / (m.density * len);
    float t = t1;
    for (uint32_t k = 0; k < 4096; k++) {
        t -= inv_maj * std::log(rmax(medium_rnd(g, 2 * k), FLT_EPSILON));
        if (t >= t2) return INFINITY;
        float dens = medium_density_at(m, r.o + t * r.d);
        if (medium_rnd(g, 2 * k + 1) < dens / m.density) return t;
    }
    return INFINITY;
}

// Nearest medium event before `tsurf` (medium ids follow all primitives, so an
// exact tie goes to the surface); returns the medium index or -1.
static int media_event(const Scene& s, const Ray& r, float lam, float tmin, float tsurf, float* t_out) {
    int best = -1;
    float bt = tsurf;
    for (int mi = 0; mi < (int)s.media.size(); mi++) {
        float t = medium_sample(s, mi, r, lam, tmin);
        if (t < bt) { bt = t; best = mi; }
    }
    *t_out = bt;
    return best;
}

// Medium::transmittance (volume.rs:68-76, 140-146, 237-252)
static float medium_transmittance(const Scene& s, int mi, const Ray& r, float tmin, float tmax) {
    const RtMedium& m = s.media[mi];
    float t1, t2;
    if (!bound_hit(s, mi, r, -INFINITY, INFINITY, &t1)) return 1.0f;
    if (!bound_hit(s, mi, r, t1 + 0.0001f, INFINITY, &t2)) return 1.0f;
    float a = rmax(rmax(t1, 0.0f), tmin), b = rmin(t2, tmax);
    if (a >= b) return 1.0f;
    if (m.type == RT_MEDIUM_GRID) return grid_transmittance(m, s.media_grid[mi], r, a, b, tmax);
    float len = length(r.d);
    float l = (b - a) * len;
    if (m.type == RT_MEDIUM_CONSTANT) return std::exp(-m.density * l);
    const int K = 16;
    float seg_t = l / len, sum = 0.0f;
    for (int i = 0; i < K; i++) {
        float t = a + seg_t * ((float)i + 0.5f) / (float)K;
        sum += medium_density_at(m, r.o + t * r.d);
    }
    return std::exp(-sum / (float)K * l);
}

// world.transmittance (bvh.rs:532-575): 0 behind an opaque primitive, else
// the product of the media's transmittances
static float scene_transmittance(const Scene& s, const Ray& r, float tmin, float tmax) {
    if (any_hit(s, r, tmin, tmax)) return 0.0f;
    float tr = 1.0f;
    for (int mi = 0; mi < (int)s.media.size(); mi++) {
        tr *= medium_transmittance(s, mi, r, tmin, tmax);
        if (tr <= 0.0f) return 0.0f;
    }
    return tr;
}

// hg_sample (volume.rs:39-62)
static V3 hg_sample(V3 w, float g, float xi1, float xi2) {
    float cos_t;
    if (std::fabs(g) < 1e-3f) {
        cos_t = 1.0f - 2.0f * xi1;
    } else {
        float sq = (1.0f - g * g) / rmax(1.0f - g + 2.0f * g * xi1, 1e-12f);
        cos_t = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    float sin_t = std::sqrt(rmax(1.0f - cos_t * cos_t, 0.0f));
    float phi = 2.0f * PI_F * xi2;
    V3 helper = std::fabs(w.x) > 0.9f ? v3(0, 1, 0) : v3(1, 0, 0);
    V3 u = unit(cross(w, helper));
    V3 v = cross(w, u);
    return u * (sin_t * std::cos(phi)) + v * (sin_t * std::sin(phi)) + w * cos_t;
}

// ── hit record (hittable.rs:73-94) ───────────────────────────────────────────
struct Rec { V3 p, normal, tangent; float t, u, v; bool front; int mat; int32_t gid; };

static inline V3 sphere_uv_calc(V3 p, float* u, float* v) {                         // sphere.rs:11-15
    float theta = std::acos(clampf(-p.y, -1.0f, 1.0f));
    float phi = std::atan2(-p.z, p.x) + PI_F;
    *u = phi / (2.0f * PI_F); *v = theta / PI_F;
    return p;
}

// micro_tilt (hittable.rs:261-270): a fixed per-facet tilt of the normal
static V3 micro_tilt(uint64_t idx, float amp, V3 n) {
    if (amp <= 0.0f) return n;
    uint64_t h = (idx * 0x9E3779B97F4A7C15ull) ^ 0xD1B54A32D192ED03ull;
    float a = (float)(uint32_t)(h >> 32) / (float)UINT32_MAX * 2.0f - 1.0f;
    float b = (float)(uint32_t)h / (float)UINT32_MAX * 2.0f - 1.0f;
    V3 up = std::fabs(n.x) < 0.9f ? v3(1, 0, 0) : v3(0, 1, 0);
    V3 t = unit(cross(n, up));
    V3 b2 = cross(n, t);
    return unit(n + t * (a * amp) + b2 * (b * amp));
}

// Gem placement (scene_file.rs:924-930): UniformScale about the origin
// (transform.rs:15-27), Rotate::euler_about the gem's center
// (transform.rs:218-224), Translate.  The reference moves the ray into object
// space; here the planes move to world space instead (the same half-spaces):
// x_w = R(s x − p) + p + t, so n·x ≤ d becomes (R n)·x_w ≤ (R n)·(p + t) + s d − n·p.
static V3 rot_apply(const float* R, V3 v) {                                         // transform.rs:150-156
    return v3(R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z,
              R[6] * v.x + R[7] * v.y + R[8] * v.z);
}
static void place_planes(const RtConvex& c, const float* pl, std::vector<float>& out, std::vector<V3>& shade) {
    V3 p = v3(c.pivot[0], c.pivot[1], c.pivot[2]);
    V3 pt = v3(c.pivot[0] + c.translate[0], c.pivot[1] + c.translate[1], c.pivot[2] + c.translate[2]);
    for (int j = 0; j < c.n_planes; j++) {
        V3 n = v3(pl[j * 4], pl[j * 4 + 1], pl[j * 4 + 2]);
        V3 nw = rot_apply(c.rot, n);
        float dw = dot(nw, pt) + (c.scale * pl[j * 4 + 3] - dot(n, p));
        out.insert(out.end(), {nw.x, nw.y, nw.z, dw});
        // Diamond::hit tilts the object-space face normal of the first plane
        // whose normal matches (diamond.rs:266-270); Rotate then turns it.
        int f = 0;
        while (f < j && !(std::fabs(pl[f * 4] - n.x) < 1e-6f && std::fabs(pl[f * 4 + 1] - n.y) < 1e-6f &&
                          std::fabs(pl[f * 4 + 2] - n.z) < 1e-6f)) f++;
        shade.push_back(rot_apply(c.rot, micro_tilt((uint64_t)f, c.polish, n)));
        shade.push_back(rot_apply(c.rot, micro_tilt((uint64_t)f, c.polish, -n)));
    }
}
static Aabb placed_box(const RtConvex& c) {                                         // transform.rs:180-200
    V3 mn = v3(INFINITY, INFINITY, INFINITY), mx = v3(-INFINITY, -INFINITY, -INFINITY);
    V3 p = v3(c.pivot[0], c.pivot[1], c.pivot[2]), t = v3(c.translate[0], c.translate[1], c.translate[2]);
    for (int k = 0; k < 8; k++) {
        V3 x = v3(k & 1 ? c.box_hi[0] : c.box_lo[0], k & 2 ? c.box_hi[1] : c.box_lo[1], k & 4 ? c.box_hi[2] : c.box_lo[2]);
        V3 w = rot_apply(c.rot, x * c.scale - p) + p + t;
        mn = v3(std::fmin(mn.x, w.x), std::fmin(mn.y, w.y), std::fmin(mn.z, w.z));
        mx = v3(std::fmax(mx.x, w.x), std::fmax(mx.y, w.y), std::fmax(mx.z, w.z));
    }
    float e = 1e-5f * std::fmax(std::fmax(std::fmax(std::fabs(mn.x), std::fabs(mx.x)), std::fmax(std::fabs(mn.y), std::fabs(mx.y))),
                                std::fmax(std::fabs(mn.z), std::fabs(mx.z))) + 1e-6f;
    return Aabb{mn - v3(e, e, e), mx + v3(e, e, e)};
}

static Rec make_rec(const Scene& s, const Ray& r, const HitRes& h) {
    Rec rec;
    rec.tangent = v3(0, 0, 0);
    rec.gid = h.gid; rec.t = h.t;
    rec.p = r.o + h.t * r.d;
    V3 outward;
    int t = prim_type(s, h.gid);
    if (t == RT_PRIM_TRI) {                                                         // triangle.rs:91-108
        const Tri& tr = s.tris[h.gid];
        float b0 = 1.0f - h.b1 - h.b2;
        if (tr.has_n) {
            V3 sn = b0 * tr.n0 + h.b1 * tr.n1 + h.b2 * tr.n2;
            outward = len2(sn) > 1e-12f ? unit(sn) : unit(cross(tr.e1, tr.e2));
        } else {
            outward = unit(cross(tr.e1, tr.e2));
        }
        rec.u = b0 * tr.uv[0] + h.b1 * tr.uv[2] + h.b2 * tr.uv[4];
        rec.v = b0 * tr.uv[1] + h.b1 * tr.uv[3] + h.b2 * tr.uv[5];
        // Gram-Schmidt against the shading normal, onb fallback
        V3 rt = b0 * tr.t0 + h.b1 * tr.t1 + h.b2 * tr.t2;
        rt = rt - outward * dot(rt, outward);
        if (len2(rt) > 1e-8f) {
            rec.tangent = unit(rt);
        } else {
            V3 ou, ov;
            onb_vec(outward, &ou, &ov);
            rec.tangent = ou;
        }
        rec.mat = tr.mat;
    } else if (t == RT_PRIM_QUAD) {
        const Quad& q = s.quads[h.gid - s.n_tris];
        outward = q.normal;
        rec.u = h.b1; rec.v = h.b2;
        rec.mat = q.mat;
    } else if (t == RT_PRIM_SPHERE) {
        const Sphere& sp = s.spheres[h.gid - s.n_tris - s.n_quads];
        outward = (rec.p - sp.c) / sp.r;
        sphere_uv_calc(outward, &rec.u, &rec.v);
        rec.mat = sp.mat;
    } else if (t == PRIM_SHAPE) {
        const Scene::Shape& sh = shape_of(s, h.gid);
        int32_t part;
        memcpy(&part, &h.b1, 4);
        Ray lr = shape_local(sh, r);
        V3 ow = shape_outward(sh, lr.o + h.t * lr.d, part);
        rec.u = 0.0f; rec.v = 0.0f;
        rec.mat = sh.mat;
        // HitRecord::new in object space, then Rotate turns the normal (transform.rs:236-241)
        rec.front = dot(lr.d, ow) < 0.0f;
        V3 nn = rec.front ? ow : -ow;
        if (sh.placed) {
            const float* m = sh.R;
            nn = v3(m[0] * nn.x + m[1] * nn.y + m[2] * nn.z, m[3] * nn.x + m[4] * nn.y + m[5] * nn.z,
                    m[6] * nn.x + m[7] * nn.y + m[8] * nn.z);
        }
        rec.normal = nn;
        return rec;
    } else {                                                                        // diamond.rs:257-275
        const Scene::Convex& c = s.convex[h.gid - s.n_tris - s.n_quads - s.n_spheres];
        int32_t pi;
        memcpy(&pi, &h.b1, 4);
        if (pi < 0) pi = 0;                         // (1,0,0)·… fallback of an unbounded exit: plane 0's normal
        const float* pl = s.convex_planes.data() + (size_t)(c.off + pi) * 4;
        outward = v3(pl[0], pl[1], pl[2]);
        rec.u = 0.0f; rec.v = 0.0f;
        rec.mat = c.mat;
        rec.front = dot(r.d, outward) < 0.0f;
        rec.normal = s.convex_shade[(size_t)(c.off + pi) * 2 + (rec.front ? 0 : 1)];
        return rec;
    }
    rec.front = dot(r.d, outward) < 0.0f;
    rec.normal = rec.front ? outward : -outward;
    return rec;
}

// ── light list (hittable.rs:156-225, quad.rs:82-96, sphere.rs:87-109) ───────
static bool light_hit(const Scene& s, int32_t gid, const Ray& r, float tmin, float tmax, Rec* rec) {
    float t, b1, b2;
    if (!prim_hit(s, gid, r, tmin, tmax, &t, &b1, &b2)) return false;
    *rec = make_rec(s, r, HitRes{gid, t, b1, b2});
    return true;
}
static bool lights_hit(const Scene& s, const Ray& r, float tmin, float tmax, Rec* out) {
    float closest = tmax; bool any = false;
    for (int32_t g : s.lights) {
        Rec rec;
        if (light_hit(s, g, r, tmin, closest, &rec)) { closest = rec.t; *out = rec; any = true; }
    }
    return any;
}
static float prim_pdf_value(const Scene& s, int32_t gid, V3 origin, V3 dir) {
    int t = prim_type(s, gid);
    if (t == RT_PRIM_SPHERE) {
        const Sphere& sp = s.spheres[gid - s.n_tris - s.n_quads];
        V3 tc = sp.c - origin;
        float d2 = len2(tc), r2 = sp.r * sp.r;
        if (d2 <= r2) return 0.0f;
        float ctm = std::sqrt(1.0f - r2 / d2);
        return 1.0f / (2.0f * PI_F * (1.0f - ctm));
    }
    Ray r{origin, dir};
    Rec rec;
    if (!light_hit(s, gid, r, 0.001f, INFINITY, &rec)) return 0.0f;
    float dist2 = len2(rec.p - origin);
    float cos_t = std::fabs(dot(unit(dir), rec.normal));
    if (t == RT_PRIM_QUAD) {
        if (cos_t < 1e-8f) return 0.0f;
        return dist2 / (cos_t * s.quads[gid - s.n_tris].area);
    }
    const Tri& tr = s.tris[gid];
    float area = 0.5f * length(cross(tr.e1, tr.e2));
    if (cos_t < 1e-8f || area <= 0.0f) return 0.0f;
    return dist2 / (cos_t * area);
}
static float lights_pdf_value(const Scene& s, V3 origin, V3 dir) {
    if (s.lights.empty()) return 0.0f;
    float w = 1.0f / (float)s.lights.size();
    float sum = 0.0f;
    for (int32_t g : s.lights) sum += w * prim_pdf_value(s, g, origin, dir);
    return sum;
}
static V3 prim_pdf_generate(const Scene& s, int32_t gid, V3 origin, float r1, float r2) {
    int t = prim_type(s, gid);
    if (t == RT_PRIM_QUAD) {
        const Quad& q = s.quads[gid - s.n_tris];
        V3 point = q.q + r1 * q.u + r2 * q.v;
        return unit(point - origin);
    }
    if (t == RT_PRIM_TRI) {
        const Tri& tr = s.tris[gid];
        if (r1 + r2 > 1.0f) { r1 = 1.0f - r1; r2 = 1.0f - r2; }
        V3 p = tr.v0 + r1 * tr.e1 + r2 * tr.e2;
        return unit(p - origin);
    }
    const Sphere& sp = s.spheres[gid - s.n_tris - s.n_quads];
    V3 tc = sp.c - origin;
    float d2 = len2(tc), rr = sp.r * sp.r;
    if (d2 <= rr) return unit(tc);
    float ctm = std::sqrt(1.0f - rr / d2);
    float phi = 2.0f * PI_F * r1;
    float ct = 1.0f - r2 * (1.0f - ctm);
    float st = std::sqrt(rmax(1.0f - ct * ct, 0.0f));
    return onb_local(onb_from_w(unit(tc)), v3(std::cos(phi) * st, std::sin(phi) * st, ct));
}

// ── environment map (renderer.rs:23-180) ─────────────────────────────────────
static void env_build(EnvMap& e, const RtBackground& bg) {
    e.w = bg.env_w; e.h = bg.env_h;
    size_t n = (size_t)e.w * e.h;
    e.img.assign(bg.env_rgb, bg.env_rgb + n * 3);
    e.cond.assign(n, 0.0f);
    e.marginal.assign(e.h, 0.0f);
    std::vector<float> row_w(e.h, 0.0f);
    for (int j = 0; j < e.h; j++) {
        float sin_j = std::sin(PI_F * ((float)j + 0.5f) / (float)e.h);
        float sum = 0.0f;
        for (int i = 0; i < e.w; i++) {
            const float* px = &e.img[((size_t)j * e.w + i) * 3];
            sum += luminance(v3(px[0], px[1], px[2])) * sin_j;
            e.cond[(size_t)j * e.w + i] = sum;
        }
        if (sum > 0.0f) { for (int i = 0; i < e.w; i++) e.cond[(size_t)j * e.w + i] /= sum; }
        else { for (int i = 0; i < e.w; i++) e.cond[(size_t)j * e.w + i] = (float)(i + 1) / (float)e.w; }
        row_w[j] = sum;
    }
    float total = 0.0f;
    for (int j = 0; j < e.h; j++) total += row_w[j];
    float cum = 0.0f;
    for (int j = 0; j < e.h; j++) {
        cum += row_w[j];
        e.marginal[j] = total > 0.0f ? cum / total : (float)(j + 1) / (float)e.h;
    }
    e.inv_total = total > 0.0f ? 1.0f / total : 0.0f;
    e.rot_y = bg.env_rot_y_deg * (PI_F / 180.0f);
    e.sin_r = std::sin(e.rot_y); e.cos_r = std::cos(e.rot_y);
}
static inline V3 env_rot(const EnvMap& e, V3 d) { return v3(d.x * e.cos_r + d.z * e.sin_r, d.y, -d.x * e.sin_r + d.z * e.cos_r); }
static inline V3 env_unrot(const EnvMap& e, V3 d) { return v3(d.x * e.cos_r - d.z * e.sin_r, d.y, d.x * e.sin_r + d.z * e.cos_r); }
static inline float rem_euclid1(float a) { float r = std::fmod(a, 1.0f); return r < 0.0f ? r + 1.0f : r; }
static inline int rem_euclid_i(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }
static V3 env_sample(const EnvMap& e, V3 dir) {                                    // renderer.rs:97-121
    V3 d = env_unrot(e, unit(dir));
    float u = rem_euclid1(0.5f + std::atan2(d.x, d.z) / (2.0f * PI_F));
    float v = std::acos(clampf(d.y, -1.0f, 1.0f)) / PI_F;
    float x = u * (float)e.w - 0.5f, y = v * (float)e.h - 0.5f;
    int x0 = (int)std::floor(x), y0 = (int)std::floor(y);
    float fx = x - (float)x0, fy = y - (float)y0;
    auto get = [&](int ix, int iy) {
        int xx = rem_euclid_i(ix, e.w), yy = std::min(std::max(iy, 0), e.h - 1);
        const float* p = &e.img[((size_t)yy * e.w + xx) * 3];
        return v3(p[0], p[1], p[2]);
    };
    V3 c00 = get(x0, y0), c10 = get(x0 + 1, y0), c01 = get(x0, y0 + 1), c11 = get(x0 + 1, y0 + 1);
    return (c00 * (1.0f - fx) + c10 * fx) * (1.0f - fy) + (c01 * (1.0f - fx) + c11 * fx) * fy;
}
static float env_pdf_at(const EnvMap& e, int i, int j) {                            // renderer.rs:169-179
    const float* p = &e.img[((size_t)j * e.w + i) * 3];
    float lum = luminance(v3(p[0], p[1], p[2]));
    return lum * (float)((size_t)e.w * e.h) * e.inv_total / (2.0f * PI_F * PI_F);
}
static float env_dir_pdf(const EnvMap& e, V3 dir) {                                  // renderer.rs:157-167
    V3 d = env_unrot(e, unit(dir));
    float u = rem_euclid1(0.5f + std::atan2(d.x, d.z) / (2.0f * PI_F));
    float v = std::acos(clampf(d.y, -1.0f, 1.0f)) / PI_F;
    int i = std::min((int)(u * (float)e.w), e.w - 1);
    int j = std::min((int)(v * (float)e.h), e.h - 1);
    i = std::max(i, 0);
    j = std::max(j, 0);
    return env_pdf_at(e, i, j);
}
static V3 env_sample_dir(const EnvMap& e, float x1, float x2, float x3, float x4, float* pdf) {   // renderer.rs:126-154
    int j = (int)(std::lower_bound(e.marginal.begin(), e.marginal.end(), x1) - e.marginal.begin());
    j = std::min(j, e.h - 1);
    const float* row = &e.cond[(size_t)j * e.w];
    int i = (int)(std::lower_bound(row, row + e.w, x2) - row);
    i = std::min(i, e.w - 1);
    float u = ((float)i + x3) / (float)e.w;
    float v = ((float)j + x4) / (float)e.h;
    float phi = 2.0f * PI_F * (u - 0.5f);
    float theta = PI_F * v;
    float st = std::sin(theta);
    V3 dir = env_rot(e, v3(st * std::sin(phi), std::cos(theta), st * std::cos(phi)));
    *pdf = env_pdf_at(e, i, j);
    return dir;
}
// ── Physical sky (renderer.rs:18, 231-362) ──────────────────────────────────
static const float COS_SUN_MAX = 0.9999892f;
static inline float perez(float a, float b, float c, float dp, float e, float ct, float g, float cg) {
    return (1.0f + a * std::exp(b / ct)) * (1.0f + c * std::exp(dp * g) + e * cg * cg);
}
// preetham_sky (renderer.rs:231-337)
static V3 preetham_sky(V3 dir, V3 sun_dir, float turbidity) {
    V3 d = unit(dir), sun = unit(sun_dir);
    float cos_gamma = clampf(dot(d, sun), -1.0f, 1.0f);
    float gamma = std::acos(cos_gamma);
    float t = clampf(turbidity, 1.7f, 20.0f);
    float cos_theta_s = rmax(sun.y, 0.0175f);
    float theta_s = std::acos(cos_theta_s);
    float ay = 0.1787f * t - 1.4630f, by = -0.3554f * t + 0.4275f, cy = 0.0227f * t + 5.3251f,
          dy = 0.1206f * t - 2.5771f, ey = -0.0670f * t + 0.3703f;
    float ax = -0.0193f * t - 0.2592f, bx = -0.0665f * t + 0.0008f, cx = -0.0004f * t + 0.2125f,
          dx = -0.0641f * t - 0.8989f, ex = -0.0033f * t + 0.0452f;
    float acy = -0.0167f * t - 0.2608f, bcy = -0.0950f * t + 0.0092f, ccy = -0.0079f * t + 0.2102f,
          dcy = -0.0441f * t - 1.6537f, ecy = -0.0109f * t + 0.0529f;
    float fn_y = perez(ay, by, cy, dy, ey, 1.0f, theta_s, cos_theta_s);
    float fn_x = perez(ax, bx, cx, dx, ex, 1.0f, theta_s, cos_theta_s);
    float fn_cy = perez(acy, bcy, ccy, dcy, ecy, 1.0f, theta_s, cos_theta_s);
    float yz = rmax((4.0453f * t - 4.9710f) * std::tan((4.0f / 9.0f - t / 120.0f) * (PI_F - 2.0f * theta_s))
                    - 0.2155f * t + 2.4192f, 0.0f);
    if (cos_gamma > COS_SUN_MAX && sun.y > 0.0f && d.y > 0.0f) {
        float disc = yz * 111.0f;
        return v3(disc, disc * 0.95f, disc * 0.85f);
    }
    float ts = theta_s, ts2 = ts * ts, ts3 = ts2 * ts;
    float xz = t * t * (0.00166f * ts3 - 0.00375f * ts2 + 0.00209f * ts)
             + t * (-0.02903f * ts3 + 0.06377f * ts2 - 0.03202f * ts + 0.00394f)
             + (0.11693f * ts3 - 0.21196f * ts2 + 0.06052f * ts + 0.25886f);
    float yzc = t * t * (0.00275f * ts3 - 0.00610f * ts2 + 0.00317f * ts)
              + t * (-0.04214f * ts3 + 0.08970f * ts2 - 0.04153f * ts + 0.00516f)
              + (0.15346f * ts3 - 0.26756f * ts2 + 0.06670f * ts + 0.26688f);
    float ct = rmax(d.y, 0.001f);
    float fy = perez(ay, by, cy, dy, ey, ct, gamma, cos_gamma);
    float fx = perez(ax, bx, cx, dx, ex, ct, gamma, cos_gamma);
    float fcy = perez(acy, bcy, ccy, dcy, ecy, ct, gamma, cos_gamma);
    float cap_y = rmax(yz * fy / fn_y, 0.0f);
    float cap_x = clampf(xz * fx / fn_x, 0.001f, 0.998f);
    float cap_yc = clampf(yzc * fcy / fn_cy, 0.001f, 0.998f);
    float lum = cap_y * 0.05f;
    float big_x = cap_x / cap_yc * lum, big_y = lum;
    float big_z = rmax((1.0f - cap_x - cap_yc) / cap_yc * lum, 0.0f);
    V3 sky = v3(rmax(3.2406f * big_x - 1.5372f * big_y - 0.4986f * big_z, 0.0f),
                rmax(-0.9689f * big_x + 1.8758f * big_y + 0.0415f * big_z, 0.0f),
                rmax(0.0557f * big_x - 0.2040f * big_y + 1.0570f * big_z, 0.0f));
    if (d.y < 0.0f) {
        float tt = rmin(-d.y * 8.0f, 1.0f);
        return sky * (1.0f - tt) + v3(0.07f, 0.06f, 0.05f) * tt;
    }
    return sky;
}
static inline bool has_sun(const Scene& s) { return s.bg.type == RT_BG_PHYSICAL && s.bg.sun_dir[1] > 0.0f; }
static inline V3 sun_vec(const Scene& s) { return v3(s.bg.sun_dir[0], s.bg.sun_dir[1], s.bg.sun_dir[2]); }
// sun_pdf_value (renderer.rs:340-348)
static float sun_pdf_value(const Scene& s, V3 dir) {
    if (has_sun(s) && dot(unit(dir), unit(sun_vec(s))) > COS_SUN_MAX) return 1.0f / (2.0f * PI_F * (1.0f - COS_SUN_MAX));
    return 0.0f;
}
// sample_sun_cone (renderer.rs:351-362)
static V3 sample_sun_cone(V3 axis, float cos_max, float r1, float r2) {
    float cos_t = 1.0f - r1 * (1.0f - cos_max);
    float sin_t = std::sqrt(rmax(1.0f - cos_t * cos_t, 0.0f));
    float phi = 2.0f * PI_F * r2;
    V3 up = std::fabs(axis.x) < 0.999f ? v3(1, 0, 0) : v3(0, 1, 0);
    V3 t = unit(cross(axis, up));
    V3 b = cross(axis, t);
    return t * (sin_t * std::cos(phi)) + b * (sin_t * std::sin(phi)) + axis * cos_t;
}

static V3 bg_eval_type(int type, const float* color, const float* top, const float* bottom, V3 dir) {
    if (type == RT_BG_SOLID) return v3(color[0], color[1], color[2]);
    float t = (clampf(dir.y, -1.0f, 1.0f) + 1.0f) * 0.5f;                           // renderer.rs:200-203
    return v3(bottom[0], bottom[1], bottom[2]) * (1.0f - t) + v3(top[0], top[1], top[2]) * t;
}
static V3 bg_eval(const Scene& s, V3 dir) {                                          // renderer.rs:197-208
    const RtBackground& b = s.bg;
    if (b.type == RT_BG_ENVMAP) {
        if (b.visible_type >= 0) return bg_eval_type(b.visible_type, b.visible_color, b.visible_top, b.visible_bottom, dir);
        return env_sample(s.env, dir);
    }
    if (b.type == RT_BG_PHYSICAL) return preetham_sky(dir, v3(b.sun_dir[0], b.sun_dir[1], b.sun_dir[2]), b.turbidity);
    return bg_eval_type(b.type, b.color, b.top, b.bottom, dir);
}
static V3 env_eval(const Scene& s, V3 dir) { return s.has_env ? env_sample(s.env, dir) : v3(0, 0, 0); }
static float env_pdf_value(const Scene& s, V3 dir) { return s.has_env ? env_dir_pdf(s.env, dir) : 0.0f; }

// ── caustic photon map (photon.rs) ───────────────────────────────────────────
typedef Scene::KdPhoton KdPhoton;

// kd_build (photon.rs:165-191): median on the widest axis, implicit tree whose
// root is the middle element of the slice.
static void kd_build(KdPhoton* nodes, size_t n) {
    if (n == 0) return;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) { mn[k] = std::min(mn[k], nodes[i].pos[k]); mx[k] = std::max(mx[k], nodes[i].pos[k]); }
    int axis = 0;
    for (int k = 1; k < 3; k++) if (mx[k] - mn[k] > mx[axis] - mn[axis]) axis = k;
    size_t mid = n / 2;
    std::nth_element(nodes, nodes + mid, nodes + n,
                     [axis](const KdPhoton& a, const KdPhoton& b) { return a.pos[axis] < b.pos[axis]; });
    nodes[mid].axis = (uint8_t)axis;
    kd_build(nodes, mid);
    kd_build(nodes + mid + 1, n - mid - 1);
}

// kd_gather (photon.rs:195-228): Σ power·(1 − d²/r²) over d² < r², n_p·n > 0.
static void kd_gather(const KdPhoton* nodes, size_t n, const float p[3], float r2, const float nrm[3], V3& acc) {
    if (n == 0) return;
    size_t mid = n / 2;
    const KdPhoton& nd = nodes[mid];
    float dx = nd.pos[0] - p[0], dy = nd.pos[1] - p[1], dz = nd.pos[2] - p[2];
    float d2 = dx * dx + dy * dy + dz * dz;
    if (d2 < r2) {
        float dt = nd.nor[0] * nrm[0] + nd.nor[1] * nrm[1] + nd.nor[2] * nrm[2];
        if (dt > 0.0f) acc = acc + v3(nd.power[0], nd.power[1], nd.power[2]) * (1.0f - d2 / r2);
    }
    int axis = nd.axis;
    float sq = p[axis] - nd.pos[axis];
    if (sq <= 0.0f) {
        kd_gather(nodes, mid, p, r2, nrm, acc);
        if (sq * sq < r2) kd_gather(nodes + mid + 1, n - mid - 1, p, r2, nrm, acc);
    } else {
        kd_gather(nodes + mid + 1, n - mid - 1, p, r2, nrm, acc);
        if (sq * sq < r2) kd_gather(nodes, mid, p, r2, nrm, acc);
    }
}

// every photon with d² ≤ r2 (or < r2 when `strict`), optionally on the normal's side
static void kd_collect(const KdPhoton* nodes, size_t n, const float p[3], float r2, bool strict, const float* nrm,
                       std::vector<std::pair<float, const KdPhoton*>>& out) {
    if (n == 0) return;
    size_t mid = n / 2;
    const KdPhoton& nd = nodes[mid];
    float dx = nd.pos[0] - p[0], dy = nd.pos[1] - p[1], dz = nd.pos[2] - p[2];
    float d2 = dx * dx + dy * dy + dz * dz;
    if (strict ? d2 < r2 : d2 <= r2) {
        bool ok = true;
        if (nrm) ok = nd.nor[0] * nrm[0] + nd.nor[1] * nrm[1] + nd.nor[2] * nrm[2] > 0.0f;
        if (ok) out.emplace_back(d2, &nd);
    }
    int axis = nd.axis;
    float sq = p[axis] - nd.pos[axis];
    if (sq <= 0.0f) {
        kd_collect(nodes, mid, p, r2, strict, nrm, out);
        if (sq * sq <= r2) kd_collect(nodes + mid + 1, n - mid - 1, p, r2, strict, nrm, out);
    } else {
        kd_collect(nodes + mid + 1, n - mid - 1, p, r2, strict, nrm, out);
        if (sq * sq <= r2) kd_collect(nodes, mid, p, r2, strict, nrm, out);
    }
}

// Irradiance estimate at (p, n).  knn_k = 0: the reference's fixed-radius
// Epanechnikov estimate × 2/(π² r²) (photon.rs:137-157).  knn_k > 0: the same
// kernel with the radius r_k = distance of the k-th nearest photon on the
// normal's side within the maximum radius (the maximum radius when fewer than
// k exist); the k-th photon itself gets weight 0, so the estimate equals the
// fixed-radius gather at r_k.
static V3 photon_irradiance(const Scene& s, V3 p, V3 n) {
    V3 acc = v3(0, 0, 0);
    if (!s.has_photons || s.photons.empty()) return acc;
    float pp[3] = {p.x, p.y, p.z}, nn[3] = {n.x, n.y, n.z};
    float r2 = s.gather_r2;
    if (s.knn_k > 0) {
        std::vector<std::pair<float, const KdPhoton*>> c;
        kd_collect(s.photons.data(), s.photons.size(), pp, r2, true, nn, c);
        if (c.size() >= s.knn_k) {
            std::nth_element(c.begin(), c.begin() + (s.knn_k - 1), c.end(),
                             [](const std::pair<float, const KdPhoton*>& a, const std::pair<float, const KdPhoton*>& b) {
                                 return a.first < b.first;
                             });
            r2 = c[s.knn_k - 1].first;
        }
        if (!(r2 > 0.0f)) return acc;
    }
    kd_gather(s.photons.data(), s.photons.size(), pp, r2, nn, acc);
    return acc * (2.0f / (PI_F * PI_F * r2));
}

// ── textures (texture.rs:25-57, material.rs:633-786) ──────────────────────────
static float srgb_decode(uint8_t c) {                                               // output.rs:90-96
    float v = (float)c / 255.0f;
    return v <= 0.04045f ? v / 12.92f : std::pow((v + 0.055f) / 1.055f, 2.4f);
}
// Texture::value: the nearest texel sRGB-decoded, or the Perlin mottle
static V3 tex_value(const Scene& s, int id, float u, float v, V3 p) {
    const Scene::Texture& t = s.textures[id - 1];
    if (t.type == RT_TEX_MOTTLE) {
        float m = clampf(2.0f * perlin_turb(t.vec, t.perm, v3(p.x * t.scale, p.y * t.scale, p.z * t.scale), 7), 0.0f, 1.0f);
        return t.lo * (1.0f - m) + t.hi * m;
    }
    float uu = clampf(u, 0.0f, 1.0f), vv = 1.0f - clampf(v, 0.0f, 1.0f);
    uint32_t x = std::min((uint32_t)(uu * (float)t.w), (uint32_t)t.w - 1u);
    uint32_t y = std::min((uint32_t)(vv * (float)t.h), (uint32_t)t.h - 1u);
    const uint8_t* q = t.px.data() + ((size_t)y * t.w + x) * 3;
    return v3(srgb_decode(q[0]), srgb_decode(q[1]), srgb_decode(q[2]));
}
// bilinear_coords + sample_srgb (mode 0) / sample_rgb (1) / sample_linear (2)
static V3 tex_bilinear(const Scene& s, int id, float u, float v, int mode) {
    const Scene::Texture& t = s.textures[id - 1];
    float uu = clampf(u, 0.0f, 1.0f), vv = 1.0f - clampf(v, 0.0f, 1.0f);
    float fx = clampf(uu * (float)t.w - 0.5f, 0.0f, (float)(t.w - 1));
    float fy = clampf(vv * (float)t.h - 0.5f, 0.0f, (float)(t.h - 1));
    uint32_t x0 = (uint32_t)fx, y0 = (uint32_t)fy;
    uint32_t x1 = std::min(x0 + 1u, (uint32_t)t.w - 1u), y1 = std::min(y0 + 1u, (uint32_t)t.h - 1u);
    float tx = fx - (float)x0, ty = fy - (float)y0;
    auto px = [&](uint32_t x, uint32_t y) {
        const uint8_t* q = t.px.data() + ((size_t)y * t.w + x) * 3;
        if (mode == 0) return v3(srgb_decode(q[0]), srgb_decode(q[1]), srgb_decode(q[2]));
        if (mode == 1) return v3((float)q[0] / 255.0f, (float)q[1] / 255.0f, (float)q[2] / 255.0f);
        float r = (float)q[0] / 255.0f;
        return v3(r, r, r);
    };
    V3 c0 = px(x0, y0) * (1.0f - tx) + px(x1, y0) * tx;
    V3 c1 = px(x0, y1) * (1.0f - tx) + px(x1, y1) * tx;
    return c0 * (1.0f - ty) + c1 * ty;
}
// PbrMaterial::params (material.rs:758-786) as a copy of the material with the
// mapped albedo (× ao), roughness and metallic; *sn the normal-mapped normal
static RtMaterial pbr_params(const Scene& s, const RtMaterial& m, const Rec& rec, V3* sn) {
    RtMaterial h = m;
    *sn = rec.normal;
    if (m.normal_tex && len2(rec.tangent) > 1e-6f) {                                // tbn_normal
        V3 raw = tex_bilinear(s, m.normal_tex, rec.u, rec.v, 1);
        V3 ts = v3(raw.x * 2.0f - 1.0f, raw.y * 2.0f - 1.0f, raw.z * 2.0f - 1.0f);
        V3 ng = rec.normal, t = rec.tangent, b = cross(ng, t);
        V3 pert = t * ts.x + b * ts.y + ng * ts.z;
        if (len2(pert) > 1e-12f) *sn = unit(pert);
    }
    V3 a = m.albedo_tex ? tex_bilinear(s, m.albedo_tex, rec.u, rec.v, 0) : v3(m.albedo[0], m.albedo[1], m.albedo[2]);
    if (m.ao_tex) a = a * tex_bilinear(s, m.ao_tex, rec.u, rec.v, 2).x;
    h.albedo[0] = a.x; h.albedo[1] = a.y; h.albedo[2] = a.z;
    if (m.roughness_tex) h.roughness = tex_bilinear(s, m.roughness_tex, rec.u, rec.v, 2).x;
    if (m.metallic_tex) h.metallic = tex_bilinear(s, m.metallic_tex, rec.u, rec.v, 2).x;
    return h;
}

// trace_photon (photon.rs:232-277): one wavelength per photon, at most 12
// bounces; stored at the first diffuse hit after ≥ 1 specular bounce.  Each new
// segment is a fresh ray (spectral_weighted = false), so every refraction of a
// spectral dielectric and every conductor bounce applies its colour tint.
enum { P_EMIT0 = 0, P_EMIT1 = 1, P_EMIT2 = 2, P_EMIT3 = 3, P_LAMBDA = 4, P_BOUNCE0 = 8, P_PER_BOUNCE = 4 };
static const int PHOTON_MAX_DEPTH = 12;

static bool trace_photon(const Scene& s, V3 pos, V3 dir, float lum_clamp, V3 power, const Rng& rng, KdPhoton* out) {
    float lam = s.spec.lam_lo + s.spec.lam_range * rnd(rng, P_LAMBDA);
    if (lam >= s.spec.lam_lo + s.spec.lam_range) lam = std::nextafter(s.spec.lam_lo + s.spec.lam_range, 0.0f);
    uint32_t spec_depth = 0;
    // storage at a diffuse surface, spectral spikes clamped once (photon.rs:260-271)
    auto store = [&](const Rec& rec) {
        float lum = luminance(power);
        if (lum > lum_clamp) power = power * (lum_clamp / lum);
        KdPhoton k;
        k.pos[0] = rec.p.x; k.pos[1] = rec.p.y; k.pos[2] = rec.p.z;
        k.power[0] = power.x; k.power[1] = power.y; k.power[2] = power.z;
        k.nor[0] = rec.normal.x; k.nor[1] = rec.normal.y; k.nor[2] = rec.normal.z;
        k.axis = 0;
        *out = k;
        return true;
    };
    for (int bounce = 0; bounce < PHOTON_MAX_DEPTH; bounce++) {
        uint32_t base = P_BOUNCE0 + bounce * P_PER_BOUNCE;
        Ray ray{pos, dir};
        HitRes h = closest_hit<false>(s, ray, 0.001f, INFINITY, nullptr);
        float tmed;
        int med = s.media.empty() ? -1 : media_event(s, ray, lam, 0.001f, h.gid < 0 ? INFINITY : h.t, &tmed);
        if (med >= 0) {
            // a medium scatter is a skip_pdf bounce of the caustic path (photon.rs:252-260)
            const RtMedium& M = s.media[med];
            power = power * v3(M.color[0], M.color[1], M.color[2]);
            V3 np = ray.o + tmed * ray.d;
            dir = hg_sample(unit(ray.d), M.g, rnd(rng, base + 0), rnd(rng, base + 1));
            pos = np;
            spec_depth++;
            continue;
        }
        if (h.gid < 0) return false;
        Rec rec = make_rec(s, ray, h);
        const RtMaterial& m = s.mats[rec.mat];
        if (m.type == RT_MAT_DIFFUSE_LIGHT || m.type == RT_MAT_BLACKBODY_LIGHT) return false;   // scatter → None
        V3 unit_dir = unit(ray.d);
        if (m.type == RT_MAT_DIELECTRIC || m.type == RT_MAT_SPECTRAL_DIELECTRIC) {
            bool spectral = m.type == RT_MAT_SPECTRAL_DIELECTRIC;
            float ior = spectral ? cauchy_ior(lam, m.cauchy_b, m.cauchy_c) : m.cauchy_b;
            float ratio = rec.front ? 1.0f / ior : ior;
            float cos_t = rmin(dot(-unit_dir, rec.normal), 1.0f);
            float sin_t = std::sqrt(1.0f - cos_t * cos_t);
            bool reflected = ratio * sin_t > 1.0f || fresnel_dielectric(cos_t, ratio) > rnd(rng, base + 0);
            V3 nd;
            if (reflected) nd = reflect(unit_dir, rec.normal);
            else if (!refract(unit_dir, rec.normal, ratio, &nd)) nd = reflect(unit_dir, rec.normal);
            V3 att = v3(1, 1, 1);
            if (spectral) {
                if (!reflected) att = spectral_fire_rgb(s.spec, lam);
                if (!rec.front) {
                    att.x *= std::exp(-m.absorption[0] * rec.t);
                    att.y *= std::exp(-m.absorption[1] * rec.t);
                    att.z *= std::exp(-m.absorption[2] * rec.t);
                }
            }
            power = power * att;
            pos = rec.p; dir = nd;
            spec_depth++;
        } else if (m.type == RT_MAT_SPECTRAL_METAL) {
            V3 n = rec.normal;
            V3 wo = unit(-ray.d);
            float cos_o = dot(wo, n);
            if (cos_o <= 0.0f) return false;
            float alpha = rmax(m.roughness * m.roughness, 1e-4f);
            V3 nd; float cos_h;
            if (m.roughness == 0.0f) { nd = reflect(unit_dir, n); cos_h = cos_o; }
            else {
                V3 t, b;
                onb_vec(n, &t, &b);
                V3 wo_ts = v3(dot(wo, t), dot(wo, b), cos_o);
                V3 m_ts = vndf_sample(wo_ts, alpha, alpha, rnd(rng, base + 0), rnd(rng, base + 1));
                V3 mm = unit(t * m_ts.x + b * m_ts.y + n * m_ts.z);
                float vo_h = rmax(dot(wo, mm), 0.0f);
                V3 wi = unit(2.0f * vo_h * mm - wo);
                if (dot(wi, n) <= 0.0f) return false;
                nd = wi; cos_h = vo_h;
            }
            if (dot(nd, n) <= 0.0f) return false;
            float weight = 1.0f;
            if (m.roughness != 0.0f) {
                float lam_o = smith_lambda(cos_o, alpha);
                float lam_i = smith_lambda(rmax(dot(nd, n), 0.0f), alpha);
                weight = ((1.0f + lam_o) / (1.0f + lam_o + lam_i)) * specular_energy_comp(cos_o, alpha);
            }
            float nn, kk;
            metal_ior(m, lam, &nn, &kk);
            power = power * (spectral_to_rgb(s.spec, lam) * (fresnel_conductor(cos_h, nn, kk) * weight));
            pos = rec.p; dir = nd;
            spec_depth++;
        } else if (m.type == RT_MAT_PBR) {
            // PbrMaterial::scatter: a specular lobe carries the photon on, the
            // diffuse lobe stores it where can_receive_caustics (material.rs:1049)
            V3 att, nd, sn;
            RtMaterial mh = pbr_params(s, m, rec, &sn);
            int lobe = pbr_scatter(mh, unit(-ray.d), sn, rnd(rng, base + 2), rnd(rng, base + 3),
                                   rnd(rng, base + 0), rnd(rng, base + 1), &att, &nd);
            if (lobe == PBR_NONE) return false;
            if (lobe == PBR_SPECULAR) {
                power = power * att;
                pos = rec.p; dir = nd;
                spec_depth++;
                continue;
            }
            if (!(m.metallic < 0.999f) || spec_depth == 0) return false;
            return store(rec);
        } else {
            // diffuse (Lambertian / checker): can_receive_caustics (material.rs:101)
            if (spec_depth == 0) return false;
            return store(rec);
        }
    }
    return false;
}

static inline Rng photon_rng(uint64_t seed, uint32_t gid) {
    Rng r;
    r.a = gid;
    r.b = mix32((uint32_t)seed) ^ 0x50484F54u;
    r.c = mix32((uint32_t)(seed >> 32) + 0x9E3779B9u);
    return r;
}

// photon_bounds of the world (hittable.rs:199-212): union of the primitive boxes
static Aabb world_bounds(const Scene& s) {
    // photon_bounds: infinite planes stay out (plane.rs:97-102)
    bool any = false;
    Aabb b{v3(0, 0, 0), v3(0, 0, 0)};
    for (int64_t i = 0; i < n_prims(s); i++) {
        if (prim_type(s, i) == PRIM_SHAPE && shape_of(s, i).type == RT_SHAPE_PLANE) continue;
        b = any ? surrounding(b, prim_box(s, i)) : prim_box(s, i);
        any = true;
    }
    for (const RtMedium& m : s.media) {                                            // volume.rs:152-154
        Aabb mb;
        if (m.boundary == RT_BOUND_BOX)
            mb = Aabb{v3(rmin(m.p_min[0], m.p_max[0]), rmin(m.p_min[1], m.p_max[1]), rmin(m.p_min[2], m.p_max[2])),
                      v3(rmax(m.p_min[0], m.p_max[0]), rmax(m.p_min[1], m.p_max[1]), rmax(m.p_min[2], m.p_max[2]))};
        else
            mb = Aabb{v3(m.center[0] - m.radius, m.center[1] - m.radius, m.center[2] - m.radius),
                      v3(m.center[0] + m.radius, m.center[1] + m.radius, m.center[2] + m.radius)};
        b = any ? surrounding(b, mb) : mb;
        any = true;
    }
    return b;
}

// Emitter geometry for photon `i` of emitter `e` (photon.rs:41-94, 97-135).
struct EmitterSetup {
    V3 t, b, center, dir, power, normal, corner, u, v, ta, ba;
    float radius, lum_clamp;
    int type;
    V3 target;        // projection sphere of a quad source (target_r 0: the whole hemisphere)
    float target_r;
};
static EmitterSetup setup_emitter(const Scene& s, const RtPhotonEmitter& e0) {
    RtPhotonEmitter e = e0;
    if (e.type == RT_EMIT_LIGHT) {
        // a quad of the light list as PhotonMap::build_from_quad's source
        // (photon.rs:97-135), coloured by the emission of its material: a diffuse
        // light's colour, a blackbody's time-averaged RGB × intensity (material.rs:53-59)
        const Quad& q = s.quads[s.lights[e.light] - s.n_tris];
        const RtMaterial& m = s.mats[q.mat];
        V3 col = m.type == RT_MAT_BLACKBODY_LIGHT ? s.bb_avg[q.mat]
               : m.type == RT_MAT_PBR ? v3(m.emission[0], m.emission[1], m.emission[2]) * m.emission_strength
               : v3(m.albedo[0], m.albedo[1], m.albedo[2]);
        e.type = RT_EMIT_QUAD;
        e.corner[0] = q.q.x; e.corner[1] = q.q.y; e.corner[2] = q.q.z;
        e.u[0] = q.u.x; e.u[1] = q.u.y; e.u[2] = q.u.z;
        e.v[0] = q.v.x; e.v[1] = q.v.y; e.v[2] = q.v.z;
        e.color[0] = col.x; e.color[1] = col.y; e.color[2] = col.z;
    }
    if (e.type == RT_EMIT_SUN) {
        // rebuild_caustics with a Physical sky (scene.rs:40-52): the sun as a disk
        // emitter, coloured by the sky radiance 0.04 off the sun direction, ×π
        V3 sun = sun_vec(s);
        V3 perp = std::fabs(sun.x) < 0.9f ? unit(v3(0.0f, -sun.z, sun.y)) : unit(v3(-sun.z, 0.0f, sun.x));
        V3 power_dir = unit(sun + perp * 0.04f);
        V3 col = bg_eval(s, power_dir) * PI_F;
        e.type = RT_EMIT_DISK;
        e.dir[0] = sun.x; e.dir[1] = sun.y; e.dir[2] = sun.z;
        e.color[0] = col.x; e.color[1] = col.y; e.color[2] = col.z;
    }
    EmitterSetup E{};
    E.type = e.type;
    if (e.type == RT_EMIT_DISK) {
        V3 sun = v3(e.dir[0], e.dir[1], e.dir[2]);
        V3 sun_down = unit(-sun);
        V3 up = std::fabs(sun_down.x) < 0.999f ? v3(1, 0, 0) : v3(0, 1, 0);
        E.t = unit(cross(sun_down, up));
        E.b = cross(sun_down, E.t);
        const float CLIP = 1.0e3f;
        Aabb bb = world_bounds(s);
        auto clip = [&](float x) { return clampf(x, -CLIP, CLIP); };
        V3 mn = v3(clip(bb.mn.x), clip(bb.mn.y), clip(bb.mn.z)), mx = v3(clip(bb.mx.x), clip(bb.mx.y), clip(bb.mx.z));
        V3 c = (mn + mx) * 0.5f;
        float r = rmax(length(mx - mn) * 0.5f, 1.0e-3f);
        E.center = c + unit(sun) * r;
        E.radius = r;
        float disk_area = PI_F * r * r;
        E.power = v3(e.color[0], e.color[1], e.color[2]) * (disk_area / ((float)e.n_photons * PI_F));
        E.lum_clamp = 15.0f * disk_area / (PI_F * 20.0f * 20.0f);
        E.dir = sun_down;
    } else {
        E.corner = v3(e.corner[0], e.corner[1], e.corner[2]);
        E.u = v3(e.u[0], e.u[1], e.u[2]);
        E.v = v3(e.v[0], e.v[1], e.v[2]);
        V3 cr = cross(E.u, E.v);
        float area = length(cr);
        E.normal = cr / area;
        onb_vec(E.normal, &E.ta, &E.ba);
        E.power = v3(e.color[0], e.color[1], e.color[2]) * (area * PI_F / (float)e.n_photons);
        E.lum_clamp = 15.0f;
        E.target = v3(e.target[0], e.target[1], e.target[2]);
        E.target_r = e.target[3] > 0.0f ? e.target[3] : 0.0f;
    }
    return E;
}

// One photon of an emitter; returns the factor on the emitter's photon power
// (1, or for a quad aimed at its projection sphere the ratio of the cosine
// density to the cone's uniform density, 0: not traced).
static float emit_photon(const EmitterSetup& E, const Rng& rng, V3* pos, V3* dir) {
    if (E.type == RT_EMIT_DISK) {
        float r = E.radius * std::sqrt(rnd(rng, P_EMIT0));
        float phi = 2.0f * PI_F * rnd(rng, P_EMIT1);
        *pos = E.center + E.t * (r * std::cos(phi)) + E.b * (r * std::sin(phi));
        *dir = E.dir;
        return 1.0f;
    }
    float ss = rnd(rng, P_EMIT0), tt = rnd(rng, P_EMIT1);
    *pos = E.corner + E.u * ss + E.v * tt;
    if (E.target_r > 0.0f) {
        // uniform in the cone toward the projection sphere (the sphere-light
        // sampling of sphere.rs:111-118)
        V3 tc = E.target - *pos;
        float d2 = len2(tc), rr = E.target_r * E.target_r;
        if (d2 > rr) {
            float ctm = std::sqrt(1.0f - rr / d2);
            float phi = 2.0f * PI_F * rnd(rng, P_EMIT3);
            float ct = 1.0f - rnd(rng, P_EMIT2) * (1.0f - ctm);
            float st = std::sqrt(rmax(1.0f - ct * ct, 0.0f));
            *dir = onb_local(onb_from_w(unit(tc)), v3(std::cos(phi) * st, std::sin(phi) * st, ct));
            float cl = dot(*dir, E.normal);
            return cl > 0.0f ? 2.0f * cl * (1.0f - ctm) : 0.0f;
        }
    }
    float ct = std::sqrt(rnd(rng, P_EMIT2));
    float st = std::sqrt(1.0f - ct * ct);
    float phi = 2.0f * PI_F * rnd(rng, P_EMIT3);
    *dir = st * std::cos(phi) * E.ta + st * std::sin(phi) * E.ba + ct * E.normal;
    return 1.0f;
}

// ── hero-wavelength state ────────────────────────────────────────────────────
// The reference path carries an RGB throughput that, after the first spectral
// event, includes the CMF tint of its single wavelength (material.rs:384-400,
// :491-497).  Here throughput T holds every achromatic/RGB factor and each of
// H wavelengths λ_i carries a scalar weight w_i; the path's effective RGB
// throughput is T ⊙ (1/H) Σ_i w_i · tint(λ_i), tint = (1,1,1) before the first
// spectral event, spectral_to_rgb (metal) or spectral_fire_rgb (dispersive
// refraction) after it.  H = 1 is the reference exactly.
enum { TINT_NONE = 0, TINT_CMF = 1, TINT_FIRE = 2 };
struct SpecState { int H; float lam[4]; float w[4]; int tint; };
static inline V3 tint_rgb(const Spectrum& sp, int tint, float lam) {
    return tint == TINT_CMF ? spectral_to_rgb(sp, lam) : spectral_fire_rgb(sp, lam);
}
static V3 spec_factor(const Spectrum& sp, const SpecState& ss) {
    if (ss.tint == TINT_NONE) {
        float m = 0.0f;
        for (int i = 0; i < ss.H; i++) m += ss.w[i];
        float v = m / (float)ss.H;
        return v3(v, v, v);
    }
    V3 acc = v3(0, 0, 0);
    for (int i = 0; i < ss.H; i++) if (ss.w[i] != 0.0f) acc = acc + tint_rgb(sp, ss.tint, ss.lam[i]) * ss.w[i];
    return acc / (float)ss.H;
}
// emitted_at (material.rs:64-81) folded with the spectral factor
static V3 emission(const Scene& s, int mat, const SpecState& ss) {
    const RtMaterial& m = s.mats[mat];
    if (m.type == RT_MAT_DIFFUSE_LIGHT) return v3(m.albedo[0], m.albedo[1], m.albedo[2]) * spec_factor(s.spec, ss);
    if (m.type == RT_MAT_PBR)                                                       // material.rs:922-924
        return v3(m.emission[0], m.emission[1], m.emission[2]) * m.emission_strength * spec_factor(s.spec, ss);
    if (m.type == RT_MAT_BLACKBODY_LIGHT) {
        if (ss.tint == TINT_NONE) return s.bb_avg[mat] * spec_factor(s.spec, ss);
        V3 acc = v3(0, 0, 0);
        for (int i = 0; i < ss.H; i++) {
            if (ss.w[i] == 0.0f) continue;
            float sc = planck_raw(ss.lam[i], m.temp_k) * s.bb_norm[mat] * m.intensity;
            acc = acc + tint_rgb(s.spec, ss.tint, ss.lam[i]) * (ss.w[i] * sc);
        }
        return acc / (float)ss.H;
    }
    return v3(0, 0, 0);
}
static inline bool is_emissive_mat(const RtMaterial& m) {
    return m.type == RT_MAT_DIFFUSE_LIGHT || m.type == RT_MAT_BLACKBODY_LIGHT;
}
static inline V3 lambert_albedo(const Scene& s, const RtMaterial& m, const Rec& rec) {   // texture.rs:28-57
    if (m.albedo_tex) return tex_value(s, m.albedo_tex, rec.u, rec.v, rec.p);
    V3 p = rec.p;
    if (m.type == RT_MAT_CHECKER) {
        int x = (int)std::floor(m.checker_scale * p.x);
        int y = (int)std::floor(m.checker_scale * p.y);
        int z = (int)std::floor(m.checker_scale * p.z);
        if ((x + y + z) % 2 == 0) return v3(m.albedo[0], m.albedo[1], m.albedo[2]);
        return v3(m.odd[0], m.odd[1], m.odd[2]);
    }
    return v3(m.albedo[0], m.albedo[1], m.albedo[2]);
}

// ── ray_color (renderer.rs:371-585) ──────────────────────────────────────────
struct PassCtx {
    const Scene* s;
    RtPassParams p;
    RtCamera cam;
};

static V3 ray_color(const Scene& s, Ray ray, const Rng& rng, SpecState ss, uint32_t max_depth, float bg_scale,
                    int64_t* n_ext, int64_t* n_shadow) {
    V3 T = v3(1, 1, 1);
    V3 color = v3(0, 0, 0);
    bool prev_specular = true;
    float prev_mis_w_brdf = 1.0f;
    float prev_spec_sun_weight = 1.0f;
    bool have_lights = !s.lights.empty();
    for (uint32_t depth = 0; depth < max_depth; depth++) {
        uint32_t base = D_BOUNCE0 + depth * D_PER_BOUNCE;
        (*n_ext)++;
        HitRes h = closest_hit<false>(s, ray, 0.001f, INFINITY, nullptr);
        float tmed;
        int med = s.media.empty() ? -1 : media_event(s, ray, ss.lam[0], 0.001f, h.gid < 0 ? INFINITY : h.t, &tmed);
        if (med >= 0) {
            // medium scatter: HenyeyGreenstein::scatter (volume.rs:29-35), skip_pdf →
            // the specular branch (renderer.rs:421-456) with no emission
            const RtMedium& M = s.media[med];
            V3 p = ray.o + tmed * ray.d;
            V3 dir = hg_sample(unit(ray.d), M.g, rnd(rng, base + B_SCATTER0), rnd(rng, base + B_SCATTER1));
            prev_spec_sun_weight = 1.0f;
            T = T * v3(M.color[0], M.color[1], M.color[2]);
            ray = Ray{p, dir};
            prev_specular = true;
            prev_mis_w_brdf = 1.0f;
        } else if (h.gid < 0) {
            float sun_pdf = sun_pdf_value(s, ray.d);
            float env_pdf = env_pdf_value(s, ray.d);
            float emit_w = (sun_pdf + env_pdf == 0.0f) ? 1.0f : (prev_specular ? prev_spec_sun_weight : prev_mis_w_brdf);
            V3 bg = (depth == 0 || !s.has_env) ? bg_eval(s, ray.d) : env_eval(s, ray.d);
            color = color + T * (bg * spec_factor(s.spec, ss)) * bg_scale * emit_w;
            break;
        } else {
        Rec rec = make_rec(s, ray, h);
        const RtMaterial& m = s.mats[rec.mat];
        float emit_w = (prev_specular || !have_lights) ? 1.0f : prev_mis_w_brdf;
        if (is_emissive_mat(m)) {
            color = color + T * emission(s, rec.mat, ss) * emit_w;
            break;   // lights do not scatter (material.rs:19,65)
        }
        V3 unit_dir = unit(ray.d);
        if (m.type == RT_MAT_DIELECTRIC || m.type == RT_MAT_SPECTRAL_DIELECTRIC) {
            // dielectric_boundary (material.rs:133-149) + SpectralDielectric (:369-402)
            bool spectral = m.type == RT_MAT_SPECTRAL_DIELECTRIC;
            float ior = spectral ? cauchy_ior(ss.lam[0], m.cauchy_b, m.cauchy_c) : m.cauchy_b;
            if (spectral && ss.H > 1 && m.cauchy_c != 0.0f && ss.lam[1] != 0.0f) {
                // dispersion: only the hero wavelength follows this direction;
                // the secondaries end here (once — lam[1] = 0 marks them gone)
                float w0 = ss.w[0] * (float)ss.H;
                for (int i = 0; i < ss.H; i++) { ss.w[i] = 0.0f; if (i) ss.lam[i] = 0.0f; }
                ss.w[0] = w0;
            }
            float ratio = rec.front ? 1.0f / ior : ior;
            float cos_t = rmin(dot(-unit_dir, rec.normal), 1.0f);
            float sin_t = std::sqrt(1.0f - cos_t * cos_t);
            bool reflected = ratio * sin_t > 1.0f || fresnel_dielectric(cos_t, ratio) > rnd(rng, base + B_SCATTER0);
            V3 dir;
            if (reflected) dir = reflect(unit_dir, rec.normal);
            else if (!refract(unit_dir, rec.normal, ratio, &dir)) dir = reflect(unit_dir, rec.normal);
            V3 att = v3(1, 1, 1);
            if (spectral) {
                if (ss.tint == TINT_NONE && !reflected) ss.tint = TINT_FIRE;
                if (!rec.front) {
                    float d = rec.t;
                    att.x *= std::exp(-m.absorption[0] * d);
                    att.y *= std::exp(-m.absorption[1] * d);
                    att.z *= std::exp(-m.absorption[2] * d);
                }
            }
            prev_spec_sun_weight = 1.0f;
            T = T * att;
            ray = Ray{rec.p, dir};
            prev_specular = true;
            prev_mis_w_brdf = 1.0f;
        } else if (m.type == RT_MAT_SPECTRAL_METAL) {
            // SpectralMetal::scatter (material.rs:449-500)
            V3 n = rec.normal;
            V3 wo = unit(-ray.d);
            float cos_o = dot(wo, n);
            if (cos_o <= 0.0f) break;
            V3 dir; float cos_h;
            float alpha = rmax(m.roughness * m.roughness, 1e-4f);
            if (m.roughness == 0.0f) {
                dir = reflect(unit_dir, n);
                cos_h = cos_o;
            } else {
                V3 t, b;
                onb_vec(n, &t, &b);
                V3 wo_ts = v3(dot(wo, t), dot(wo, b), cos_o);
                V3 m_ts = vndf_sample(wo_ts, alpha, alpha, rnd(rng, base + B_SCATTER0), rnd(rng, base + B_SCATTER1));
                V3 mm = unit(t * m_ts.x + b * m_ts.y + n * m_ts.z);
                float vo_h = rmax(dot(wo, mm), 0.0f);
                V3 wi = unit(2.0f * vo_h * mm - wo);
                if (dot(wi, n) <= 0.0f) break;
                dir = wi; cos_h = vo_h;
            }
            if (dot(dir, n) <= 0.0f) break;
            float weight = 1.0f;
            if (m.roughness != 0.0f) {
                float lam_o = smith_lambda(cos_o, alpha);
                float lam_i = smith_lambda(rmax(dot(dir, n), 0.0f), alpha);
                weight = ((1.0f + lam_o) / (1.0f + lam_o + lam_i)) * specular_energy_comp(cos_o, alpha);
            }
            // specular sun NEE (renderer.rs:421-456) with SpectralMetal::specular_brdf_cos /
            // specular_sampling_pdf (material.rs:504-551); zero for a smooth conductor
            prev_spec_sun_weight = 1.0f;
            if (has_sun(s) && m.roughness != 0.0f) {
                const float p_sun = 1.0f / (2.0f * PI_F * (1.0f - COS_SUN_MAX));
                V3 sun_s = sample_sun_cone(unit(sun_vec(s)), COS_SUN_MAX, rnd(rng, base + B_SUN0), rnd(rng, base + B_SUN1));
                float cos_i = dot(sun_s, n);
                if (cos_o > 0.0f && cos_i > 0.0f) {
                    V3 hh = unit(wo + sun_s);
                    float wo_h = rmax(dot(wo, hh), 0.0f), h_n = rmax(dot(hh, n), 0.0f);
                    float D = ggx_ndf(h_n, alpha);
                    float g2 = 1.0f / (1.0f + smith_lambda(cos_o, alpha) + smith_lambda(cos_i, alpha));
                    float comp = specular_energy_comp(cos_o, alpha);
                    SpecState sv = ss;
                    for (int i = 0; i < ss.H; i++) {
                        if (ss.w[i] == 0.0f) continue;
                        float nn, kk;
                        metal_ior(m, ss.lam[i], &nn, &kk);
                        sv.w[i] = ss.w[i] * (D * fresnel_conductor(wo_h, nn, kk) * g2 / (4.0f * cos_o) * comp);
                    }
                    if (sv.tint == TINT_NONE) sv.tint = TINT_CMF;
                    V3 brdf_cos = spec_factor(s.spec, sv);
                    (*n_shadow)++;
                    float tr = scene_transmittance(s, Ray{rec.p, sun_s}, 0.001f, INFINITY);
                    if (tr > 0.0f && (brdf_cos.x > 0.0f || brdf_cos.y > 0.0f || brdf_cos.z > 0.0f)) {
                        float p_mat = ggx_ndf(h_n, alpha) * smith_g1(cos_o, alpha) / (4.0f * cos_o);
                        V3 sun_color = bg_eval(s, sun_s);
                        float mis_d = p_sun * p_sun + p_mat * p_mat;
                        if (mis_d > 0.0f) color = color + T * tr * brdf_cos * sun_color * p_sun / mis_d;
                    }
                }
                V3 hb = unit(wo + dir);
                float p_b = (dot(dir, n) > 0.0f) ? ggx_ndf(rmax(dot(hb, n), 0.0f), alpha) * smith_g1(cos_o, alpha) / (4.0f * cos_o) : 0.0f;
                if (p_b > 0.0f) prev_spec_sun_weight = (p_b * p_b) / rmax(p_b * p_b + p_sun * p_sun, 1e-8f);
            }
            for (int i = 0; i < ss.H; i++) {
                if (ss.w[i] == 0.0f) continue;
                float nn, kk;
                metal_ior(m, ss.lam[i], &nn, &kk);
                ss.w[i] *= fresnel_conductor(cos_h, nn, kk);
            }
            if (ss.tint == TINT_NONE) ss.tint = TINT_CMF;
            T = T * weight;
            ray = Ray{rec.p, dir};
            prev_specular = true;
            prev_mis_w_brdf = 1.0f;
        } else {
            // Lambertian / checker (material.rs:85-102) or PbrMaterial
            // (material.rs:790-920): diffuse branch renderer.rs:457-572
            V3 att, hint;   // scatter attenuation; albedo_hint for the caustic term
            V3 sn = rec.normal;   // the shading normal (a PBR normal map tilts it)
            bool diffuse = true;
            if (m.type == RT_MAT_PBR) {
                // the emission adds at the hit (renderer.rs:415-417), then one lobe scatters
                color = color + T * emission(s, rec.mat, ss) * emit_w;
                RtMaterial mh = pbr_params(s, m, rec, &sn);
                V3 wo = unit(-ray.d), dir;
                int lobe = pbr_scatter(mh, wo, sn, rnd(rng, base + B_LOBE0), rnd(rng, base + B_LOBE1),
                                       rnd(rng, base + B_SCATTER0), rnd(rng, base + B_SCATTER1), &att, &dir);
                if (lobe == PBR_NONE) break;
                hint = v3(mh.albedo[0], mh.albedo[1], mh.albedo[2]);
                if (lobe == PBR_SPECULAR) {
                    // specular sun NEE (renderer.rs:421-456)
                    prev_spec_sun_weight = 1.0f;
                    if (has_sun(s)) {
                        const float p_sun = 1.0f / (2.0f * PI_F * (1.0f - COS_SUN_MAX));
                        V3 sun_s = sample_sun_cone(unit(sun_vec(s)), COS_SUN_MAX, rnd(rng, base + B_SUN0),
                                                   rnd(rng, base + B_SUN1));
                        (*n_shadow)++;
                        float tr = scene_transmittance(s, Ray{rec.p, sun_s}, 0.001f, INFINITY);
                        if (tr > 0.0f) {
                            V3 bc = pbr_specular_brdf_cos(mh, wo, sn, sun_s);
                            if (bc.x > 0.0f || bc.y > 0.0f || bc.z > 0.0f) {
                                float p_mat = pbr_specular_pdf(mh, wo, sn, sun_s);
                                V3 sun_color = bg_eval(s, sun_s) * spec_factor(s.spec, ss);
                                float mis_d = p_sun * p_sun + p_mat * p_mat;
                                if (mis_d > 0.0f) color = color + T * tr * bc * sun_color * p_sun / mis_d;
                            }
                        }
                        float p_b = pbr_specular_pdf(mh, wo, sn, dir);
                        if (p_b > 0.0f) prev_spec_sun_weight = (p_b * p_b) / rmax(p_b * p_b + p_sun * p_sun, 1e-8f);
                    }
                    T = T * att;
                    ray = Ray{rec.p, dir};
                    prev_specular = true;
                    prev_mis_w_brdf = 1.0f;
                    diffuse = false;
                }
            } else {
                att = lambert_albedo(s, m, rec);
                hint = att;
            }
            if (diffuse) {
                if (s.has_photons) {                                                    // renderer.rs:461-467
                    V3 irr = photon_irradiance(s, rec.p, rec.normal);
                    if (irr.x > 0.0f || irr.y > 0.0f || irr.z > 0.0f)
                        color = color + (T * spec_factor(s.spec, ss)) * hint * irr;
                }
                if (have_lights) {
                    uint32_t pick = rnd_u32(rng, base + B_LPICK) % (uint32_t)s.lights.size();
                    V3 light_dir = prim_pdf_generate(s, s.lights[pick], rec.p, rnd(rng, base + B_LPT0), rnd(rng, base + B_LPT1));
                    Ray shadow{rec.p, light_dir};
                    Rec lrec;
                    if (lights_hit(s, shadow, 0.001f, INFINITY, &lrec)) {
                        (*n_shadow)++;
                        float tr = scene_transmittance(s, shadow, 0.001f, lrec.t * (1.0f - 1e-4f));
                        if (tr > 0.0f) {
                            float l_pdf = lights_pdf_value(s, rec.p, light_dir);
                            float brdf = rmax(dot(sn, unit(light_dir)) / PI_F, 0.0f);
                            float sun_p = sun_pdf_value(s, light_dir);
                            float env_p = env_pdf_value(s, light_dir);
                            float mis_d = l_pdf * l_pdf + brdf * brdf + sun_p * sun_p + env_p * env_p;
                            if (mis_d > 0.0f && brdf > 0.0f) {
                                V3 nee = emission(s, lrec.mat, ss);
                                color = color + T * tr * att * brdf * l_pdf * nee / mis_d;
                            }
                        }
                    }
                }
                if (has_sun(s)) {                                                       // renderer.rs:495-518
                    V3 sun_s = sample_sun_cone(unit(sun_vec(s)), COS_SUN_MAX, rnd(rng, base + B_SUN0), rnd(rng, base + B_SUN1));
                    (*n_shadow)++;
                    float tr = scene_transmittance(s, Ray{rec.p, sun_s}, 0.001f, INFINITY);
                    if (tr > 0.0f) {
                        float brdf = rmax(dot(sn, unit(sun_s)) / PI_F, 0.0f);
                        if (brdf > 0.0f) {
                            float sun_pdf = 1.0f / (2.0f * PI_F * (1.0f - COS_SUN_MAX));
                            V3 sun_color = bg_eval(s, sun_s) * spec_factor(s.spec, ss);
                            float area_pdf = have_lights ? lights_pdf_value(s, rec.p, sun_s) : 0.0f;
                            float mis_d = sun_pdf * sun_pdf + brdf * brdf + area_pdf * area_pdf;
                            color = color + T * tr * att * brdf * sun_pdf * sun_color / mis_d;
                        }
                    }
                }
                if (s.has_env) {
                    float env_pdf;
                    V3 env_dir = env_sample_dir(s.env, rnd(rng, base + B_ENV_ROW), rnd(rng, base + B_ENV_COL),
                                                rnd(rng, base + B_ENV_JU), rnd(rng, base + B_ENV_JV), &env_pdf);
                    if (env_pdf > 0.0f) {
                        Ray shadow{rec.p, env_dir};
                        (*n_shadow)++;
                        float tr = scene_transmittance(s, shadow, 0.001f, INFINITY);
                        if (tr > 0.0f) {
                            float brdf = rmax(dot(sn, unit(env_dir)) / PI_F, 0.0f);
                            if (brdf > 0.0f) {
                                float area_pdf = have_lights ? lights_pdf_value(s, rec.p, env_dir) : 0.0f;
                                V3 env_color = env_eval(s, env_dir) * spec_factor(s.spec, ss);
                                float mis_d = env_pdf * env_pdf + brdf * brdf + area_pdf * area_pdf;
                                color = color + T * tr * att * brdf * env_pdf * env_color / mis_d;
                            }
                        }
                    }
                }
                // indirect: cosine-weighted sample (pdf.rs:12-41)
                Onb uvw = onb_from_w(sn);
                float r1 = rnd(rng, base + B_COS0), r2 = rnd(rng, base + B_COS1);
                float phi = 2.0f * PI_F * r1;
                float sq = std::sqrt(r2);
                V3 ind_dir = onb_local(uvw, v3(std::cos(phi) * sq, std::sin(phi) * sq, std::sqrt(1.0f - r2)));
                float pdf_val = rmax(dot(unit(ind_dir), uvw.w) / PI_F, 0.0f);
                if (pdf_val <= 0.0f) break;
                float scat_pdf = rmax(dot(sn, unit(ind_dir)) / PI_F, 0.0f);
                if (scat_pdf <= 0.0f) break;
                if (dot(ind_dir, rec.normal) <= 0.0f) break;
                float area = have_lights ? lights_pdf_value(s, rec.p, ind_dir) : 0.0f;
                float sun = sun_pdf_value(s, ind_dir);
                float env = env_pdf_value(s, ind_dir);
                float nee_sq = area * area + sun * sun + env * env;
                prev_mis_w_brdf = (pdf_val * pdf_val) / rmax(pdf_val * pdf_val + nee_sq, 1e-8f);
                T = T * (att * (scat_pdf / pdf_val));
                ray = Ray{rec.p, ind_dir};
                prev_specular = false;
            }   // diffuse
        }
        }   // surface hit
        if (depth >= 2) {                                                           // renderer.rs:574-579
            V3 eff = T * spec_factor(s.spec, ss);
            float survive = rmax(rmax(eff.x, eff.y), eff.z);
            float p = rmin(survive, 1.0f);
            if (survive <= 0.0f || rnd(rng, base + B_RR) >= p) break;
            T = T / p;
        }
    }
    return color;
}

// ── camera + render_tiles (camera.rs:47-59, renderer.rs:655-730) ─────────────
static void render_pixel(const Scene& s, const RtCamera& cam, const RtPassParams& p, uint32_t sample_idx,
                         uint32_t row, uint32_t col, float out[3], int64_t* n_ext, int64_t* n_sh) {
    uint32_t w = p.width, h = p.height;
    uint32_t i = row * w + col;
    Rng rng = make_rng(p.seed, i, sample_idx);
    float w_denom = (float)std::max<uint32_t>(w - 1, 1), h_denom = (float)std::max<uint32_t>(h - 1, 1);
    uint32_t strata = p.strata, strata2 = strata * strata;
    uint32_t ray_y = h - 1 - row;
    float uj, vj;
    if (strata2 > 0) {
        uint32_t offset = (i * 0x9E3779B9u) % strata2;
        uint32_t sidx = (sample_idx + offset) % strata2;
        uint32_t sx = sidx % strata, sy = sidx / strata;
        uj = ((float)sx + rnd(rng, D_JIT_U)) / (float)strata;
        vj = ((float)sy + rnd(rng, D_JIT_V)) / (float)strata;
    } else {
        uj = rnd(rng, D_JIT_U); vj = rnd(rng, D_JIT_V);
    }
    float u = ((float)col + uj) / w_denom;
    float v = ((float)ray_y + vj) / h_denom;
    V3 cu = v3(cam.u[0], cam.u[1], cam.u[2]), cv = v3(cam.v[0], cam.v[1], cam.v[2]);
    V3 origin = v3(cam.origin[0], cam.origin[1], cam.origin[2]);
    V3 rd;
    if (cam.aperture_blades >= 3) {
        // sample_polygon (camera.rs:66-79): a fan wedge of the N-gon, then a folded
        // uniform triangle sample
        float nb = (float)cam.aperture_blades, rot = PI_F / nb;
        float k = (float)(rnd_u32(rng, D_LENS_K) % (uint32_t)cam.aperture_blades);
        float a1 = 2.0f * PI_F * k / nb + rot, a2 = 2.0f * PI_F * (k + 1.0f) / nb + rot;
        float r1 = rnd(rng, D_LENS_R), r2 = rnd(rng, D_LENS_P);
        if (r1 + r2 > 1.0f) { r1 = 1.0f - r1; r2 = 1.0f - r2; }
        rd = cam.lens_radius * (v3(std::cos(a1), std::sin(a1), 0.0f) * r1 + v3(std::cos(a2), std::sin(a2), 0.0f) * r2);
    } else {
        float lr = std::sqrt(rnd(rng, D_LENS_R)), lp = 2.0f * PI_F * rnd(rng, D_LENS_P);
        rd = cam.lens_radius * v3(lr * std::cos(lp), lr * std::sin(lp), 0.0f);
    }
    V3 offset = cu * rd.x + cv * rd.y;
    V3 ll = v3(cam.lower_left[0], cam.lower_left[1], cam.lower_left[2]);
    V3 hz = v3(cam.horizontal[0], cam.horizontal[1], cam.horizontal[2]);
    V3 vt = v3(cam.vertical[0], cam.vertical[1], cam.vertical[2]);
    Ray r{origin + offset, ll + u * hz + v * vt - origin - offset};
    (void)rnd(rng, D_TIME);   // ray time: no moving geometry in the flat description
    SpecState ss;
    ss.H = (int)std::max<uint32_t>(1, std::min<uint32_t>(p.hero_count, 4));
    float lam0 = s.spec.lam_lo + s.spec.lam_range * rnd(rng, D_LAMBDA);
    if (lam0 >= s.spec.lam_lo + s.spec.lam_range) lam0 = std::nextafter(s.spec.lam_lo + s.spec.lam_range, 0.0f);
    for (int k = 0; k < ss.H; k++) {
        float off = std::fmod(lam0 - s.spec.lam_lo + (float)k * (s.spec.lam_range / (float)ss.H), s.spec.lam_range);
        ss.lam[k] = s.spec.lam_lo + off;
        ss.w[k] = 1.0f;
    }
    ss.tint = TINT_NONE;
    V3 c = ray_color(s, r, rng, ss, p.max_depth, p.bg_scale, n_ext, n_sh);
    out[0] = c.x; out[1] = c.y; out[2] = c.z;
}

// ── photon-free scene construction ───────────────────────────────────────────
static std::string g_err;

static int scene_create(const RtSceneDesc* d, Scene** out) {
    if (!d || !out) { g_err = "null argument"; return RT_ERR_INVALID; }
    Scene* s = new Scene();
    s->n_tris = d->n_tris; s->n_quads = d->n_quads; s->n_spheres = d->n_spheres;
    s->mats.assign(d->mats, d->mats + d->n_mats);
    s->tris.resize(d->n_tris);
    for (int64_t i = 0; i < d->n_tris; i++) {
        const float* v = d->tri_v + i * 9;
        Tri& t = s->tris[i];
        t.v0 = v3(v[0], v[1], v[2]);
        V3 v1 = v3(v[3], v[4], v[5]), v2 = v3(v[6], v[7], v[8]);
        t.e1 = v1 - t.v0; t.e2 = v2 - t.v0;
        t.has_n = d->tri_n != nullptr;
        if (t.has_n) {
            const float* n = d->tri_n + i * 9;
            t.n0 = v3(n[0], n[1], n[2]); t.n1 = v3(n[3], n[4], n[5]); t.n2 = v3(n[6], n[7], n[8]);
        }
        t.mat = d->tri_mat[i];
        // texture coordinates and tangents, or mesh.rs:75-81's defaults
        static const float duv[6] = {0.0f, 0.0f, 1.0f, 0.0f, 0.5f, 1.0f};
        const float* uv = d->tri_uv ? d->tri_uv + i * 6 : duv;
        for (int k = 0; k < 6; k++) t.uv[k] = uv[k];
        if (d->tri_uv && d->tri_tangent) {
            const float* g = d->tri_tangent + i * 9;
            t.t0 = v3(g[0], g[1], g[2]); t.t1 = v3(g[3], g[4], g[5]); t.t2 = v3(g[6], g[7], g[8]);
        } else {
            t.t0 = t.t1 = t.t2 = v3(1, 0, 0);
        }
    }
    // textures (texture.rs): image texels, or a mottle's Perlin tables
    for (int32_t i = 0; i < d->n_textures; i++) {
        const RtTexture& t = d->textures[i];
        Scene::Texture x;
        x.type = t.type; x.w = t.width; x.h = t.height; x.scale = t.scale;
        x.lo = v3(t.lo[0], t.lo[1], t.lo[2]); x.hi = v3(t.hi[0], t.hi[1], t.hi[2]);
        if (t.type == RT_TEX_IMAGE) x.px.assign(t.rgb8, t.rgb8 + (size_t)t.width * t.height * 3);
        else { memcpy(x.vec, t.perlin_vec, sizeof(x.vec)); memcpy(x.perm, t.perlin_perm, sizeof(x.perm)); }
        s->textures.push_back(std::move(x));
    }
    s->quads.resize(d->n_quads);
    for (int64_t i = 0; i < d->n_quads; i++) {                                      // quad.rs:21-33
        const float* q = d->quad_quv + i * 9;
        Quad& Q = s->quads[i];
        Q.q = v3(q[0], q[1], q[2]); Q.u = v3(q[3], q[4], q[5]); Q.v = v3(q[6], q[7], q[8]);
        V3 n = cross(Q.u, Q.v);
        Q.area = length(n);
        if (!(Q.area > 1e-6f * length(Q.u) * length(Q.v))) {
            delete s; g_err = "degenerate quad " + std::to_string(i); return RT_ERR_INVALID;
        }
        Q.normal = n / Q.area;
        Q.d = dot(Q.normal, Q.q);
        Q.w = n / dot(n, n);
        Q.mat = d->quad_mat[i];
    }
    s->spheres.resize(d->n_spheres);
    for (int64_t i = 0; i < d->n_spheres; i++) {
        const float* p = d->sphere + i * 4;
        s->spheres[i] = Sphere{v3(p[0], p[1], p[2]), p[3], d->sphere_mat[i]};
    }
    // participating media (scene_file.rs:962-983, volume.rs:88-97, 170-186)
    if (d->n_media < 0 || (d->n_media > 0 && !d->media)) { delete s; g_err = "bad media list"; return RT_ERR_INVALID; }
    for (int32_t i = 0; i < d->n_media; i++) {
        RtMedium m = d->media[i];
        bool ok = (m.type == RT_MEDIUM_CONSTANT || m.type == RT_MEDIUM_NOISE || m.type == RT_MEDIUM_GRID) &&
                  (m.boundary == RT_BOUND_SPHERE || m.boundary == RT_BOUND_BOX) && std::isfinite(m.density) &&
                  m.density >= 0.0f;
        if (m.boundary == RT_BOUND_SPHERE) ok = ok && m.radius > 0.0f;
        if (!ok) { delete s; g_err = "invalid medium " + std::to_string(i); return RT_ERR_INVALID; }
        if (m.type == RT_MEDIUM_NOISE) {
            m.density = rmax(m.density, FLT_EPSILON);
            m.threshold = rmin(rmax(m.threshold, 0.0f), 0.99f);
        }
        std::vector<Quad> qs;
        if (m.boundary == RT_BOUND_BOX) {                                            // quad.rs:201-215
            V3 mn = v3(rmin(m.p_min[0], m.p_max[0]), rmin(m.p_min[1], m.p_max[1]), rmin(m.p_min[2], m.p_max[2]));
            V3 mx = v3(rmax(m.p_min[0], m.p_max[0]), rmax(m.p_min[1], m.p_max[1]), rmax(m.p_min[2], m.p_max[2]));
            V3 dx = v3(mx.x - mn.x, 0, 0), dy = v3(0, mx.y - mn.y, 0), dz = v3(0, 0, mx.z - mn.z);
            V3 qq[6][3] = {{v3(mn.x, mn.y, mx.z), dx, dy}, {v3(mx.x, mn.y, mx.z), -dz, dy},
                           {v3(mx.x, mn.y, mn.z), -dx, dy}, {v3(mn.x, mn.y, mn.z), dz, dy},
                           {v3(mn.x, mx.y, mx.z), dx, -dz}, {v3(mn.x, mn.y, mn.z), dx, dz}};
            for (auto& f : qq) {
                Quad Q;
                Q.q = f[0]; Q.u = f[1]; Q.v = f[2];
                V3 n = cross(Q.u, Q.v);
                Q.area = length(n);
                if (!(Q.area > 0.0f)) { delete s; g_err = "degenerate medium box " + std::to_string(i); return RT_ERR_INVALID; }
                Q.normal = n / Q.area;
                Q.d = dot(Q.normal, Q.q);
                Q.w = n / dot(n, n);
                Q.mat = 0;
                qs.push_back(Q);
            }
        }
        Scene::GridMed G;
        if (m.type == RT_MEDIUM_GRID) {
            bool gok = m.boundary == RT_BOUND_BOX && m.grid != nullptr;
            for (int a = 0; a < 3; a++) gok = gok && m.grid_res[a] >= 1 && m.grid_res[a] <= RT_GRID_MAX_RES;
            if (!gok) { delete s; g_err = "invalid grid medium " + std::to_string(i); return RT_ERR_INVALID; }
            size_t nv = (size_t)m.grid_res[0] * m.grid_res[1] * m.grid_res[2];
            G.grid.assign(m.grid, m.grid + nv);
            for (float v : G.grid)
                if (!(v >= 0.0f) || !std::isfinite(v)) { delete s; g_err = "grid voxel values must be finite and >= 0"; return RT_ERR_INVALID; }
            for (int a = 0; a < 3; a++) { G.res[a] = m.grid_res[a]; G.nb[a] = (G.res[a] + GRID_BRICK - 1) / GRID_BRICK; }
            G.major.assign((size_t)G.nb[0] * G.nb[1] * G.nb[2], 0.0f);
            for (int bz = 0; bz < G.nb[2]; bz++)
                for (int by = 0; by < G.nb[1]; by++)
                    for (int bx = 0; bx < G.nb[0]; bx++) {
                        const int b[3] = {bx, by, bz};
                        int lo[3], hi[3];
                        for (int a = 0; a < 3; a++) {
                            lo[a] = std::max(b[a] * GRID_BRICK - 1, 0);
                            hi[a] = std::min(b[a] * GRID_BRICK + GRID_BRICK, G.res[a] - 1);
                        }
                        float mx = 0.0f;
                        for (int z = lo[2]; z <= hi[2]; z++)
                            for (int y = lo[1]; y <= hi[1]; y++)
                                for (int x = lo[0]; x <= hi[0]; x++)
                                    mx = rmax(mx, G.grid[((size_t)z * G.res[1] + y) * G.res[0] + x]);
                        G.major[((size_t)bz * G.nb[1] + by) * G.nb[0] + bx] = mx * 1.00000095367431640625f;
                    }
            V3 mn = v3(rmin(m.p_min[0], m.p_max[0]), rmin(m.p_min[1], m.p_max[1]), rmin(m.p_min[2], m.p_max[2]));
            V3 mx = v3(rmax(m.p_min[0], m.p_max[0]), rmax(m.p_min[1], m.p_max[1]), rmax(m.p_min[2], m.p_max[2]));
            V3 ext = mx - mn;
            G.lo = mn;
            G.inv_vox = v3((float)G.res[0] / ext.x, (float)G.res[1] / ext.y, (float)G.res[2] / ext.z);
            G.bw = v3(ext.x / (float)G.res[0] * GRID_BRICK, ext.y / (float)G.res[1] * GRID_BRICK,
                      ext.z / (float)G.res[2] * GRID_BRICK);
            G.inv_bw = v3(1.0f / G.bw.x, 1.0f / G.bw.y, 1.0f / G.bw.z);
            m.grid = nullptr;                 // the scene keeps its own copy
        }
        s->media.push_back(m);
        s->media_quads.push_back(qs);
        s->media_grid.push_back(std::move(G));
    }
    // analytic convex solids (diamond.rs:93-195)
    if (d->n_convex < 0 || (d->n_convex > 0 && (!d->convex || !d->convex_planes))) {
        delete s; g_err = "bad convex list"; return RT_ERR_INVALID;
    }
    s->n_convex = d->n_convex;
    for (int64_t i = 0; i < d->n_convex; i++) {
        const RtConvex& c = d->convex[i];
        bool ok = c.n_planes >= 4 && c.n_planes <= 1024 && c.plane_offset >= 0 && c.mat >= 0 && c.mat < d->n_mats &&
                  !is_emissive_type(d->mats[c.mat].type) && c.scale > 0.0f && c.polish >= 0.0f && c.polish <= 0.25f;
        if (!ok) { delete s; g_err = "invalid convex solid " + std::to_string(i); return RT_ERR_INVALID; }
        int32_t off = (int32_t)(s->convex_planes.size() / 4);
        place_planes(c, d->convex_planes + (size_t)c.plane_offset * 4, s->convex_planes, s->convex_shade);
        s->convex.push_back(Scene::Convex{off, c.n_planes, c.mat, c.polish, placed_box(c)});
    }
    // cylinders, cones, disks, infinite planes
    if (d->n_shapes < 0 || (d->n_shapes > 0 && !d->shapes)) { delete s; g_err = "bad shape list"; return RT_ERR_INVALID; }
    s->n_shapes = d->n_shapes;
    for (int64_t i = 0; i < d->n_shapes; i++) {
        const RtShape& q = d->shapes[i];
        Scene::Shape sh;
        sh.type = q.type; sh.mat = q.mat;
        sh.c = v3(q.center[0], q.center[1], q.center[2]);
        V3 nraw = v3(q.normal[0], q.normal[1], q.normal[2]);
        bool planar = q.type == RT_SHAPE_DISK || q.type == RT_SHAPE_PLANE;
        bool ok = q.type >= RT_SHAPE_CYLINDER && q.type <= RT_SHAPE_PLANE && q.mat >= 0 && q.mat < d->n_mats &&
                  q.scale > 0.0f && !(planar && !(len2(nraw) > 1e-12f)) &&
                  !(q.type != RT_SHAPE_PLANE && !(q.radius > 0.0f)) &&
                  !((q.type == RT_SHAPE_CYLINDER || q.type == RT_SHAPE_CONE) && !(q.height > 0.0f));
        if (!ok) { delete s; g_err = "invalid shape " + std::to_string(i); return RT_ERR_INVALID; }
        sh.n = planar ? unit(nraw) : v3(0, 1, 0);
        onb_vec(sh.n, &sh.u, &sh.v);                                               // disk.rs:118-119, plane.rs:31-32
        sh.radius = q.radius; sh.height = q.height; sh.wave_a = q.wave_amplitude; sh.wave_s = q.wave_scale;
        memcpy(sh.R, q.rot, sizeof(sh.R));
        sh.inv_scale = 1.0f / q.scale;
        sh.t = v3(q.translate[0], q.translate[1], q.translate[2]);
        bool ident_r = q.rot[0] == 1.0f && q.rot[4] == 1.0f && q.rot[8] == 1.0f && q.rot[1] == 0.0f && q.rot[2] == 0.0f &&
                       q.rot[3] == 0.0f && q.rot[5] == 0.0f && q.rot[6] == 0.0f && q.rot[7] == 0.0f;
        sh.placed = !(ident_r && q.scale == 1.0f && sh.t.x == 0.0f && sh.t.y == 0.0f && sh.t.z == 0.0f);
        // object-space box (cylinder.rs:226-232, cone.rs:126-132, disk.rs:166-175, plane.rs:80-95)
        Aabb ob;
        if (q.type == RT_SHAPE_CYLINDER || q.type == RT_SHAPE_CONE) {
            V3 rr = v3(sh.radius, 0.0f, sh.radius);
            ob = Aabb{sh.c - rr, sh.c + rr + v3(0.0f, sh.height, 0.0f)};
        } else if (q.type == RT_SHAPE_DISK) {
            V3 ext = v3(sh.radius * std::sqrt(rmax(1.0f - sh.n.x * sh.n.x, 0.0f)),
                        sh.radius * std::sqrt(rmax(1.0f - sh.n.y * sh.n.y, 0.0f)),
                        sh.radius * std::sqrt(rmax(1.0f - sh.n.z * sh.n.z, 0.0f)));
            ob = pad(Aabb{sh.c - ext, sh.c + ext});
        } else {
            const float B = 1e5f, E = 1e-3f;
            float lo[3], hi[3], nn[3] = {sh.n.x, sh.n.y, sh.n.z}, pp[3] = {sh.c.x, sh.c.y, sh.c.z};
            for (int a = 0; a < 3; a++) {
                if (std::fabs(nn[a]) > 0.999f) { lo[a] = pp[a] - E; hi[a] = pp[a] + E; }
                else { lo[a] = -B; hi[a] = B; }
            }
            ob = Aabb{v3(lo[0], lo[1], lo[2]), v3(hi[0], hi[1], hi[2])};
        }
        if (sh.placed) {                                                            // the corners, placed
            V3 mn = v3(INFINITY, INFINITY, INFINITY), mx = v3(-INFINITY, -INFINITY, -INFINITY);
            for (int k = 0; k < 8; k++) {
                V3 x = v3(k & 1 ? ob.mx.x : ob.mn.x, k & 2 ? ob.mx.y : ob.mn.y, k & 4 ? ob.mx.z : ob.mn.z) * q.scale;
                V3 w = v3(q.rot[0] * x.x + q.rot[1] * x.y + q.rot[2] * x.z, q.rot[3] * x.x + q.rot[4] * x.y + q.rot[5] * x.z,
                          q.rot[6] * x.x + q.rot[7] * x.y + q.rot[8] * x.z) + sh.t;
                mn = v3(rmin(mn.x, w.x), rmin(mn.y, w.y), rmin(mn.z, w.z));
                mx = v3(rmax(mx.x, w.x), rmax(mx.y, w.y), rmax(mx.z, w.z));
            }
            float e = 1e-5f * rmax(rmax(rmax(std::fabs(mn.x), std::fabs(mx.x)), rmax(std::fabs(mn.y), std::fabs(mx.y))),
                                   rmax(std::fabs(mn.z), std::fabs(mx.z))) + 1e-6f;
            ob = Aabb{mn - v3(e, e, e), mx + v3(e, e, e)};
        }
        sh.box = ob;
        s->shapes.push_back(sh);
    }
    s->lights.assign(d->light_prims, d->light_prims + d->n_lights);
    s->bg = d->bg;
    s->has_env = d->bg.type == RT_BG_ENVMAP && d->bg.env_rgb && d->bg.env_w > 0 && d->bg.env_h > 0;
    if (s->has_env) env_build(s->env, d->bg);
    s->bg.env_rgb = nullptr;
    spectrum_init(s->spec, d->spectral_range);
    s->bb_norm.assign(s->mats.size(), 0.0f);
    s->bb_avg.assign(s->mats.size(), v3(0, 0, 0));
    for (size_t mi = 0; mi < s->mats.size(); mi++) {                                // material.rs:47-62
        const RtMaterial& m = s->mats[mi];
        if (m.type != RT_MAT_BLACKBODY_LIGHT) continue;
        int N = s->spec.n;
        std::vector<float> raw(N);
        float sum = 0.0f;
        for (int i = 0; i < N; i++) { raw[i] = planck_raw(380.0f + (float)i * 5.0f, m.temp_k); sum += raw[i]; }
        float mean = sum / (float)N;
        float norm = 1.0f / rmax(mean, 1e-30f);
        V3 acc = v3(0, 0, 0);
        for (int i = 0; i < N; i++) acc = acc + spectral_to_rgb(s->spec, 380.0f + (float)i * 5.0f) * (raw[i] * norm);
        s->bb_norm[mi] = norm;
        s->bb_avg[mi] = acc / (float)N * m.intensity;
    }
    std::call_once(g_elut_once, build_e_lut);   // build the E_ss LUT outside any timed render
    build_bvh(*s);
    *out = s;
    return RT_OK;
}

// ── thread pool helper (rows handed out dynamically, like Rayon's row tasks) ──
template <class F>
static void parallel_rows(uint32_t n_rows, int n_threads, F f) {
    if (n_threads <= 1) { for (uint32_t r = 0; r < n_rows; r++) f(r, 0); return; }
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < n_threads; t++)
        th.emplace_back([&, t]() { for (;;) { uint32_t r = next.fetch_add(1); if (r >= n_rows) break; f(r, t); } });
    for (auto& x : th) x.join();
}

}  // namespace orc

using namespace orc;

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

int32_t orc_scene_create(const RtSceneDesc* d, void** out) {
    Scene* s = nullptr;
    int rc = scene_create(d, &s);
    *out = s;
    return rc;
}
int32_t orc_scene_destroy(void* s) { delete (Scene*)s; return RT_OK; }

int32_t orc_bvh_export(void* sp, float* nodes, int64_t* n_nodes, int32_t* leaf, int64_t* n_leaves) {
    Scene* s = (Scene*)sp;
    if (n_nodes) *n_nodes = (int64_t)s->nodes.size();
    if (n_leaves) *n_leaves = (int64_t)s->leaf_prims.size();
    if (nodes) memcpy(nodes, s->nodes.data(), s->nodes.size() * sizeof(Node));
    if (leaf) memcpy(leaf, s->leaf_prims.data(), s->leaf_prims.size() * sizeof(int32_t));
    return RT_OK;
}

// rays: n × 8 (o, d, tmin, tmax); mode 0 = BVH, 1 = brute force
int32_t orc_trace_closest(void* sp, const float* rays, int64_t n, RtHit* hits, int32_t mode, int32_t threads) {
    Scene* s = (Scene*)sp;
    int64_t chunk = 4096, nch = (n + chunk - 1) / chunk;
    parallel_rows((uint32_t)nch, threads, [&](uint32_t c, int) {
        for (int64_t i = c * chunk; i < std::min(n, (int64_t)(c + 1) * chunk); i++) {
            const float* r = rays + i * 8;
            Ray ray{v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5])};
            HitRes h = mode == 1 ? closest_hit_brute(*s, ray, r[6], r[7]) : closest_hit<false>(*s, ray, r[6], r[7], nullptr);
            float tm;
            int med = s->media.empty() ? -1 : media_event(*s, ray, 550.0f, r[6], h.gid < 0 ? r[7] : h.t, &tm);
            if (med >= 0) h = HitRes{(int32_t)(n_prims(*s) + med), tm, 0.0f, 0.0f};
            hits[i].prim = h.gid; hits[i].t = h.gid >= 0 ? h.t : 0.0f;
            hits[i].b1 = h.gid >= 0 ? h.b1 : 0.0f; hits[i].b2 = h.gid >= 0 ? h.b2 : 0.0f;
        }
    });
    return RT_OK;
}

int32_t orc_trace_any(void* sp, const float* rays, int64_t n, uint8_t* occ, int32_t threads) {
    Scene* s = (Scene*)sp;
    int64_t chunk = 4096, nch = (n + chunk - 1) / chunk;
    parallel_rows((uint32_t)nch, threads, [&](uint32_t c, int) {
        for (int64_t i = c * chunk; i < std::min(n, (int64_t)(c + 1) * chunk); i++) {
            const float* r = rays + i * 8;
            occ[i] = any_hit(*s, Ray{v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5])}, r[6], r[7]) ? 1 : 0;
        }
    });
    return RT_OK;
}

int32_t orc_trace_transmittance(void* sp, const float* rays, int64_t n, float* tr, int32_t threads) {
    Scene* s = (Scene*)sp;
    int64_t chunk = 1024, nch = (n + chunk - 1) / chunk;
    parallel_rows((uint32_t)nch, threads, [&](uint32_t c, int) {
        for (int64_t i = c * chunk; i < std::min(n, (int64_t)(c + 1) * chunk); i++) {
            const float* r = rays + i * 8;
            tr[i] = scene_transmittance(*s, Ray{v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5])}, r[6], r[7]);
        }
    });
    return RT_OK;
}

// Background::eval for n directions (renderer.rs:196-208), and the sun pdf
int32_t orc_bg_eval_n(void* sp, const float* dirs, int64_t n, float* rgb, float* sun_pdf) {
    Scene* s = (Scene*)sp;
    for (int64_t i = 0; i < n; i++) {
        V3 d = v3(dirs[i * 3], dirs[i * 3 + 1], dirs[i * 3 + 2]);
        V3 c = bg_eval(*s, d);
        rgb[i * 3] = c.x; rgb[i * 3 + 1] = c.y; rgb[i * 3 + 2] = c.z;
        if (sun_pdf) sun_pdf[i] = sun_pdf_value(*s, d);
    }
    return RT_OK;
}
// sample_sun_cone around the scene's sun for n (r1, r2) pairs
int32_t orc_sun_sample(void* sp, const float* r, int64_t n, float* dirs) {
    Scene* s = (Scene*)sp;
    for (int64_t i = 0; i < n; i++) {
        V3 d = sample_sun_cone(unit(sun_vec(*s)), COS_SUN_MAX, r[i * 2], r[i * 2 + 1]);
        dirs[i * 3] = d.x; dirs[i * 3 + 1] = d.y; dirs[i * 3 + 2] = d.z;
    }
    return RT_OK;
}

// hg_sample for n (w, g, xi1, xi2) rows of 6 floats → n × 3 directions
int32_t orc_hg_sample(const float* in, int64_t n, float* out) {
    for (int64_t i = 0; i < n; i++) {
        const float* a = in + i * 6;
        V3 d = hg_sample(v3(a[0], a[1], a[2]), a[3], a[4], a[5]);
        out[i * 3] = d.x; out[i * 3 + 1] = d.y; out[i * 3 + 2] = d.z;
    }
    return RT_OK;
}

// PbrMaterial::scatter for n rows of 10 floats (wo xyz, n xyz, xi_coat, xi_spec,
// xi1, xi2) → per row lobe (PBR_NONE / PBR_SPECULAR / PBR_DIFFUSE), attenuation
// and direction; plus specular_brdf_cos and specular_sampling_pdf at an
// explicit wi (the row's direction when spec_wi is NULL)
int32_t orc_pbr_scatter(const RtMaterial* m, const float* in, int64_t n, int32_t* lobe, float* att, float* dir,
                        const float* spec_wi, float* brdf_cos, float* pdf) {
    for (int64_t i = 0; i < n; i++) {
        const float* a = in + i * 10;
        V3 wo = v3(a[0], a[1], a[2]), nn = v3(a[3], a[4], a[5]), at = v3(0, 0, 0), d = v3(0, 0, 0);
        lobe[i] = pbr_scatter(*m, wo, nn, a[6], a[7], a[8], a[9], &at, &d);
        att[i * 3] = at.x; att[i * 3 + 1] = at.y; att[i * 3 + 2] = at.z;
        dir[i * 3] = d.x; dir[i * 3 + 1] = d.y; dir[i * 3 + 2] = d.z;
        if (brdf_cos && pdf) {
            V3 wi = spec_wi ? v3(spec_wi[i * 3], spec_wi[i * 3 + 1], spec_wi[i * 3 + 2]) : d;
            V3 bc = pbr_specular_brdf_cos(*m, wo, nn, wi);
            brdf_cos[i * 3] = bc.x; brdf_cos[i * 3 + 1] = bc.y; brdf_cos[i * 3 + 2] = bc.z;
            pdf[i] = pbr_specular_pdf(*m, wo, nn, wi);
        }
    }
    return RT_OK;
}

// ── output (output.rs:7-190, main.rs:571-583) ──────────────────────────────
static inline float aces_curve(float x) {                                          // output.rs:12-15
    x = rmax(x, 0.0f);
    return (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
}
static V3 aces_tonemap(V3 c) {                                                     // output.rs:17-31
    float r = aces_curve(c.x * 0.59719f + c.y * 0.35458f + c.z * 0.04823f);
    float g = aces_curve(c.x * 0.07600f + c.y * 0.90834f + c.z * 0.01566f);
    float b = aces_curve(c.x * 0.02840f + c.y * 0.13383f + c.z * 0.83777f);
    return v3(r * 1.60475f + g * -0.53108f + b * -0.07367f, r * -0.10208f + g * 1.10813f + b * -0.00605f,
              r * -0.00327f + g * -0.07276f + b * 1.07602f);
}
static inline float agx_curve(float x) {                                           // output.rs:39-43
    float x2 = x * x, x4 = x2 * x2;
    return 15.5f * x4 * x2 - 40.14f * x4 * x + 31.96f * x4 - 6.868f * x2 * x + 0.4298f * x2 + 0.1191f * x - 0.00232f;
}
static V3 agx_tonemap(V3 c) {                                                      // output.rs:45-80
    float in[3] = {c.x * 0.842479062253094f + c.y * 0.0784335999999992f + c.z * 0.0792237451477643f,
                   c.x * 0.0423282422610123f + c.y * 0.878468636469772f + c.z * 0.0791661274605434f,
                   c.x * 0.0423756549057051f + c.y * 0.0784336f + c.z * 0.879142973793104f};
    float k[3];
    for (int i = 0; i < 3; i++) {
        float e = (std::log2(rmax(in[i], 1e-10f)) - -12.47393f) / 16.5f;
        k[i] = agx_curve(rmin(rmax(e, 0.0f), 1.0f));
    }
    float luma = luminance(v3(k[0], k[1], k[2]));
    for (int i = 0; i < 3; i++) k[i] = luma + 1.4f * (std::pow(k[i], 1.35f) - luma);
    return v3(k[0] * 1.19687900512017f + k[1] * -0.0980208811401368f + k[2] * -0.0990297440797205f,
              k[0] * -0.0528968517574562f + k[1] * 1.15190312990417f + k[2] * -0.0989611768448433f,
              k[0] * -0.0529716355144234f + k[1] * -0.0980434501171241f + k[2] * 1.15107567775604f);
}
static inline uint8_t encode8(float x) {                                           // output.rs:84-86, 104
    x = rmax(x, 0.0f);
    float e = x <= 0.0031308f ? 12.92f * x : 1.055f * std::pow(x, 1.0f / 2.4f) - 0.055f;
    return (uint8_t)(rmin(rmax(e, 0.0f), 0.999f) * 256.0f);
}
// apply_optics + tone_map over an image: `lin` per-sample means, or sum / max(count, 1)
int32_t orc_develop(const float* lin, const float* sum, const uint32_t* cnt, const RtDevelopParams* p,
                    uint8_t* out) {
    uint32_t w = p->width, h = p->height;
    auto fetch = [&](size_t i) {
        if (lin) return v3(lin[i * 3], lin[i * 3 + 1], lin[i * 3 + 2]);
        float n = (float)std::max<uint32_t>(cnt[i], 1u);
        return v3(sum[i * 3] / n, sum[i * 3 + 1] / n, sum[i * 3 + 2] / n);
    };
    float cx = ((float)w - 1.0f) * 0.5f, cy = ((float)h - 1.0f) * 0.5f;
    float rcorner = rmax(std::sqrt(cx * cx + cy * cy), 1e-6f);
    for (uint32_t y = 0; y < h; y++)
        for (uint32_t x = 0; x < w; x++) {
            size_t i = (size_t)y * w + x;
            V3 c;
            if (p->vignette == 0.0f && p->distortion == 0.0f) {
                c = fetch(i);
            } else {                                                                // output.rs:159-190
                float dx = ((float)x - cx) / rcorner, dy = ((float)y - cy) / rcorner;
                float r2 = dx * dx + dy * dy;
                float s = 1.0f - p->distortion * r2;
                float sx = rmin(rmax(cx + dx * rcorner * s, 0.0f), (float)w - 1.0f);
                float sy = rmin(rmax(cy + dy * rcorner * s, 0.0f), (float)h - 1.0f);
                size_t x0 = (size_t)sx, y0 = (size_t)sy;
                size_t x1 = std::min<size_t>(x0 + 1, w - 1), y1 = std::min<size_t>(y0 + 1, h - 1);
                float fx = sx - (float)x0, fy = sy - (float)y0;
                V3 c00 = fetch(y0 * w + x0), c10 = fetch(y0 * w + x1), c01 = fetch(y1 * w + x0), c11 = fetch(y1 * w + x1);
                c = (c00 * (1.0f - fx) + c10 * fx) * (1.0f - fy) + (c01 * (1.0f - fx) + c11 * fx) * fy;
                c = c * rmax(1.0f - p->vignette * r2, 0.0f);
            }
            c = c * p->exposure;
            V3 m = p->tonemapper == RT_TONEMAP_ACES ? aces_tonemap(c) : agx_tonemap(c);
            out[i * 3] = encode8(m.x);
            out[i * 3 + 1] = encode8(m.y);
            out[i * 3 + 2] = encode8(m.z);
        }
    return RT_OK;
}
// apply_optics alone (output.rs:159-190) on a linear image, for its tests
int32_t orc_apply_optics(const float* img, uint32_t w, uint32_t h, float vignette, float distortion, float* out) {
    float cx = ((float)w - 1.0f) * 0.5f, cy = ((float)h - 1.0f) * 0.5f;
    float rcorner = rmax(std::sqrt(cx * cx + cy * cy), 1e-6f);
    auto at = [&](size_t i) { return v3(img[i * 3], img[i * 3 + 1], img[i * 3 + 2]); };
    for (uint32_t y = 0; y < h; y++)
        for (uint32_t x = 0; x < w; x++) {
            size_t i = (size_t)y * w + x;
            V3 c = at(i);
            if (vignette != 0.0f || distortion != 0.0f) {
                float dx = ((float)x - cx) / rcorner, dy = ((float)y - cy) / rcorner;
                float r2 = dx * dx + dy * dy, s = 1.0f - distortion * r2;
                float sx = rmin(rmax(cx + dx * rcorner * s, 0.0f), (float)w - 1.0f);
                float sy = rmin(rmax(cy + dy * rcorner * s, 0.0f), (float)h - 1.0f);
                size_t x0 = (size_t)sx, y0 = (size_t)sy;
                size_t x1 = std::min<size_t>(x0 + 1, w - 1), y1 = std::min<size_t>(y0 + 1, h - 1);
                float fx = sx - (float)x0, fy = sy - (float)y0;
                c = (at(y0 * w + x0) * (1.0f - fx) + at(y0 * w + x1) * fx) * (1.0f - fy) +
                    (at(y1 * w + x0) * (1.0f - fx) + at(y1 * w + x1) * fx) * fy;
                c = c * rmax(1.0f - vignette * r2, 0.0f);
            }
            out[i * 3] = c.x; out[i * 3 + 1] = c.y; out[i * 3 + 2] = c.z;
        }
    return RT_OK;
}

// Texture lookups for tests: rows of (u, v, px, py, pz) → RGB; mode −1 is
// Texture::value, 0/1/2 the PBR bilinear samplers (sRGB, raw, red channel)
int32_t orc_tex_sample(void* sp, int32_t id, int32_t mode, const float* in, int64_t n, float* out) {
    Scene* s = (Scene*)sp;
    if (id < 1 || id > (int32_t)s->textures.size()) return RT_ERR_INVALID;
    for (int64_t i = 0; i < n; i++) {
        const float* a = in + i * 5;
        V3 c = mode < 0 ? tex_value(*s, id, a[0], a[1], v3(a[2], a[3], a[4])) : tex_bilinear(*s, id, a[0], a[1], mode);
        out[i * 3] = c.x; out[i * 3 + 1] = c.y; out[i * 3 + 2] = c.z;
    }
    return RT_OK;
}
// The hit record's (u, v) and tangent for rays: n × 8 rays → n × 5 (u, v, tangent)
int32_t orc_hit_uv(void* sp, const float* rays, int64_t n, float* out) {
    Scene* s = (Scene*)sp;
    for (int64_t i = 0; i < n; i++) {
        const float* r = rays + i * 8;
        Ray ray{v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5])};
        HitRes h = closest_hit<false>(*s, ray, r[6], r[7], nullptr);
        float* o = out + i * 5;
        if (h.gid < 0) { for (int k = 0; k < 5; k++) o[k] = 0.0f; continue; }
        Rec rec = make_rec(*s, ray, h);
        o[0] = rec.u; o[1] = rec.v; o[2] = rec.tangent.x; o[3] = rec.tangent.y; o[4] = rec.tangent.z;
    }
    return RT_OK;
}

// Per-ray traversal counters for the algorithmic-bytes roofline:
// out[i*4 + {0,1,2,3}] = nodes visited, triangle, sphere, quad tests.
int32_t orc_trace_stats(void* sp, const float* rays, int64_t n, int64_t* out, int32_t threads) {
    Scene* s = (Scene*)sp;
    int64_t chunk = 4096, nch = (n + chunk - 1) / chunk;
    parallel_rows((uint32_t)nch, threads, [&](uint32_t c, int) {
        for (int64_t i = c * chunk; i < std::min(n, (int64_t)(c + 1) * chunk); i++) {
            const float* r = rays + i * 8;
            TraceStats st;
            closest_hit<true>(*s, Ray{v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5])}, r[6], r[7], &st);
            out[i * 4 + 0] = st.nodes; out[i * 4 + 1] = st.tris; out[i * 4 + 2] = st.spheres; out[i * 4 + 3] = st.quads;
        }
    });
    return RT_OK;
}

// render_tiles for params->n_samples consecutive passes; scratch n_samples×h×w×3.
// row_begin/row_end bound the rows rendered (a CPU-baseline sample may render a
// band of rows); rows outside are left untouched.
int32_t orc_render_pass(void* sp, const RtCamera* cam, const RtPassParams* p, float* scratch,
                        const uint8_t* converged, int32_t threads, uint32_t row_begin, uint32_t row_end,
                        int64_t* counters) {
    Scene* s = (Scene*)sp;
    uint32_t w = p->width, h = p->height;
    if (row_end == 0 || row_end > h) row_end = h;
    std::vector<int64_t> ext(std::max(threads, 1), 0), sh(std::max(threads, 1), 0);
    for (uint32_t k = 0; k < std::max<uint32_t>(p->n_samples, 1); k++) {
        uint32_t sidx = p->sample_idx + k;
        float* out = scratch + (size_t)k * w * h * 3;
        parallel_rows(row_end - row_begin, threads, [&](uint32_t rr, int tid) {
            uint32_t row = rr + row_begin;
            for (uint32_t col = 0; col < w; col++) {
                size_t i = (size_t)row * w + col;
                if (converged && converged[i]) { out[i * 3] = out[i * 3 + 1] = out[i * 3 + 2] = 0.0f; continue; }
                render_pixel(*s, *cam, *p, sidx, row, col, out + i * 3, &ext[tid], &sh[tid]);
            }
        });
    }
    if (counters) {
        counters[0] = counters[1] = 0;
        for (size_t t = 0; t < ext.size(); t++) { counters[0] += ext[t]; counters[1] += sh[t]; }
    }
    return RT_OK;
}

// accumulate_sample (main.rs:603-643) for one pass over npix pixels
int32_t orc_accumulate(float* acc, const float* scratch, uint32_t* n, float* m2, const uint8_t* conv,
                       int64_t npix, float clamp, uint32_t min_samples, float floor_) {
    for (int64_t i = 0; i < npix; i++) {
        if (conv && conv[i]) continue;
        V3 sc = v3(scratch[i * 3], scratch[i * 3 + 1], scratch[i * 3 + 2]);
        if (!std::isfinite(sc.x) || !std::isfinite(sc.y) || !std::isfinite(sc.z)) continue;
        uint32_t old_n = n[i];
        V3 a = v3(acc[i * 3], acc[i * 3 + 1], acc[i * 3 + 2]);
        V3 old_mean = old_n > 0 ? a / (float)old_n : v3(0, 0, 0);
        float old_lum = luminance(old_mean);
        if (clamp > 0.0f && old_n >= min_samples) {
            float l = luminance(sc);
            float thresh = rmax(clamp * old_lum, floor_);
            if (l > thresh) sc = sc * (thresh / l);
        }
        a = a + sc;
        n[i] = old_n + 1;
        V3 new_mean = a / (float)n[i];
        V3 mm = v3(m2[i * 3], m2[i * 3 + 1], m2[i * 3 + 2]) + (sc - old_mean) * (sc - new_mean);
        acc[i * 3] = a.x; acc[i * 3 + 1] = a.y; acc[i * 3 + 2] = a.z;
        m2[i * 3] = mm.x; m2[i * 3 + 1] = mm.y; m2[i * 3 + 2] = mm.z;
    }
    return RT_OK;
}

// mark_converged (main.rs:646-677) with ADAPTIVE_THRESHOLD as a parameter
int64_t orc_mark_converged(uint8_t* conv, const uint32_t* n, const float* m2, const float* acc, int64_t npix, float thresh) {
    int64_t cnt = 0;
    for (int64_t i = 0; i < npix; i++) {
        if (!conv[i] && n[i] > 0) {
            bool ok = true;
            for (int c = 0; c < 3; c++) {
                float mean = acc[i * 3 + c] / (float)std::max<uint32_t>(n[i], 1);
                if (mean < 1e-4f) continue;
                float var = m2[i * 3 + c] / (float)std::max<uint32_t>(n[i] - 1, 1);
                float se = std::sqrt(var / (float)n[i]);
                if (se / mean >= thresh) { ok = false; break; }
            }
            if (ok) conv[i] = 1;
        }
        cnt += conv[i] ? 1 : 0;
    }
    return cnt;
}

// ── scalar functions pinned by the reference's unit tests ────────────────────
float orc_fresnel_dielectric(float c, float eta) { return fresnel_dielectric(c, eta); }
float orc_fresnel_conductor(float c, float n, float k) { return fresnel_conductor(c, n, k); }
float orc_cauchy_ior(float l, float b, float c) { return cauchy_ior(l, b, c); }
float orc_planck_raw(float l, float t) { return planck_raw(l, t); }
float orc_ggx_ndf(float c, float a) { return ggx_ndf(c, a); }
float orc_smith_g1(float c, float a) { return smith_g1(c, a); }
float orc_smith_lambda(float c, float a) { return smith_lambda(c, a); }
float orc_e_ss(float mu, float a) { return e_ss_lut(mu, a); }
float orc_energy_comp(float mu, float a) { return specular_energy_comp(mu, a); }
void orc_elut_export(float* out) { e_ss_lut(0.5f, 0.5f); memcpy(out, g_elut, sizeof(g_elut)); }
void orc_spectral_to_rgb(float l, int32_t range_mode, float* out) {
    static Spectrum sp[2]; static std::once_flag f[2];
    int m = range_mode ? 1 : 0;
    std::call_once(f[m], [&]() { spectrum_init(sp[m], m); });
    V3 c = spectral_to_rgb(sp[m], l); out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
void orc_spectral_fire_rgb(float l, int32_t range_mode, float* out) {
    static Spectrum sp[2]; static std::once_flag f[2];
    int m = range_mode ? 1 : 0;
    std::call_once(f[m], [&]() { spectrum_init(sp[m], m); });
    V3 c = spectral_fire_rgb(sp[m], l); out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
void orc_metal_ior(int32_t metal, float l, float* n, float* k) {
    RtMaterial m; memset(&m, 0, sizeof(m)); m.metal = metal;
    metal_ior(m, l, n, k);
}
void orc_vndf_sample(const float* wo, float ax, float ay, float x1, float x2, float* out) {
    V3 m = vndf_sample(v3(wo[0], wo[1], wo[2]), ax, ay, x1, x2); out[0] = m.x; out[1] = m.y; out[2] = m.z;
}
// quad/triangle/sphere hit against a one-prim scene is covered by orc_trace_closest;
// env map queries for the renderer.rs env tests:
void orc_env_sample(void* sp, const float* dir, float* out) {
    Scene* s = (Scene*)sp; V3 c = env_sample(s->env, v3(dir[0], dir[1], dir[2])); out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
float orc_env_pdf(void* sp, const float* dir) { return env_pdf_value(*(Scene*)sp, v3(dir[0], dir[1], dir[2])); }
void orc_env_sample_dir(void* sp, const float* xi, float* dir, float* pdf) {
    Scene* s = (Scene*)sp; V3 d = env_sample_dir(s->env, xi[0], xi[1], xi[2], xi[3], pdf); dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
}
void orc_bg_eval(void* sp, const float* dir, float* out) {
    Scene* s = (Scene*)sp; V3 c = bg_eval(*s, v3(dir[0], dir[1], dir[2])); out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
void orc_env_eval(void* sp, const float* dir, float* out) {
    Scene* s = (Scene*)sp; V3 c = env_eval(*s, v3(dir[0], dir[1], dir[2])); out[0] = c.x; out[1] = c.y; out[2] = c.z;
}
float orc_lights_pdf_value(void* sp, const float* o, const float* d) {
    return lights_pdf_value(*(Scene*)sp, v3(o[0], o[1], o[2]), v3(d[0], d[1], d[2]));
}
void orc_rng(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t dim, uint32_t* u, float* f) {
    Rng r = make_rng(seed, pixel, sample);
    *u = rnd_u32(r, dim); *f = rnd(r, dim);
}

}  // extern "C"

// ── photon map entry points ───────────────────────────────────────────────────
extern "C" {

static void photon_finish(Scene* s, std::vector<KdPhoton>&& ph, float radius, uint32_t k) {
    s->photons_by_index = ph;
    s->photons = std::move(ph);
    kd_build(s->photons.data(), s->photons.size());
    s->has_photons = true;
    s->gather_r2 = radius * radius;
    s->gather_norm = 2.0f / (PI_F * PI_F * radius * radius);
    s->knn_k = k;
}

int32_t orc_photon_build(void* sp, const RtPhotonParams* p, int64_t* n_stored, int32_t threads) {
    Scene* s = (Scene*)sp;
    if (!p || p->n_emitters < 0 || p->n_emitters > RT_MAX_EMITTERS || !(p->gather_radius > 0.0f)) return RT_ERR_INVALID;
    uint32_t total = 0;
    for (int e = 0; e < p->n_emitters; e++) {
        const RtPhotonEmitter& em = p->emitters[e];
        if (em.type == RT_EMIT_SUN && s->bg.type != RT_BG_PHYSICAL) return RT_ERR_INVALID;
        if (em.type == RT_EMIT_LIGHT &&
            (em.light < 0 || em.light >= (int32_t)s->lights.size() || prim_type(*s, s->lights[em.light]) != RT_PRIM_QUAD))
            return RT_ERR_INVALID;
        total += em.n_photons;
    }
    // a shard of the emission order: photons first .. first + count − 1
    uint32_t first = p->first_photon, count = p->shard_photons ? p->shard_photons : total - first;
    if ((uint64_t)first + count > total) return RT_ERR_INVALID;
    std::vector<KdPhoton> slot(total);
    std::vector<uint8_t> ok(total, 0);
    uint32_t off = 0;
    for (int e = 0; e < p->n_emitters; e++) {
        const RtPhotonEmitter& em = p->emitters[e];
        if (em.n_photons == 0) continue;
        EmitterSetup E = setup_emitter(*s, em);
        uint32_t n = em.n_photons, base = off;
        uint32_t chunk = 4096, nch = (n + chunk - 1) / chunk;
        parallel_rows(nch, threads, [&](uint32_t c, int) {
            for (uint32_t i = c * chunk; i < std::min(n, (c + 1) * chunk); i++) {
                uint32_t gid = base + i;
                if (gid < first || gid - first >= count) continue;
                Rng rng = photon_rng(p->seed, gid);
                V3 pos, dir;
                float wgt = emit_photon(E, rng, &pos, &dir);
                if (!(wgt > 0.0f)) continue;
                KdPhoton k;
                if (trace_photon(*s, pos, dir, E.lum_clamp, E.power * wgt, rng, &k)) {
                    k.idx = (int32_t)gid;
                    slot[gid] = k;
                    ok[gid] = 1;
                }
            }
        });
        off += n;
    }
    std::vector<KdPhoton> ph;
    for (uint32_t i = 0; i < total; i++) if (ok[i]) ph.push_back(slot[i]);
    if (n_stored) *n_stored = (int64_t)ph.size();
    photon_finish(s, std::move(ph), p->gather_radius, p->knn_k);
    return RT_OK;
}

int32_t orc_photon_set(void* sp, const float* pos, const float* power, const float* nor, const int32_t* idx, int64_t n,
                       float radius, uint32_t k) {
    Scene* s = (Scene*)sp;
    std::vector<KdPhoton> ph(n);
    for (int64_t i = 0; i < n; i++) {
        for (int c = 0; c < 3; c++) { ph[i].pos[c] = pos[i * 3 + c]; ph[i].power[c] = power[i * 3 + c]; ph[i].nor[c] = nor[i * 3 + c]; }
        ph[i].axis = 0;
        ph[i].idx = idx ? idx[i] : (int32_t)i;
    }
    photon_finish(s, std::move(ph), radius, k);
    return RT_OK;
}

int32_t orc_photon_export(void* sp, float* pos, float* power, float* nor, int32_t* idx, int64_t* n) {
    Scene* s = (Scene*)sp;
    if (n) *n = (int64_t)s->photons_by_index.size();
    for (size_t i = 0; pos && i < s->photons_by_index.size(); i++) {
        const KdPhoton& k = s->photons_by_index[i];
        for (int c = 0; c < 3; c++) { pos[i * 3 + c] = k.pos[c]; power[i * 3 + c] = k.power[c]; nor[i * 3 + c] = k.nor[c]; }
        idx[i] = k.idx;
    }
    return RT_OK;
}

// queries n × 6 (p, n) → irradiance n × 3
int32_t orc_photon_gather(void* sp, const float* q, int64_t n, float* irr, int32_t threads) {
    Scene* s = (Scene*)sp;
    int64_t chunk = 1024, nch = (n + chunk - 1) / chunk;
    parallel_rows((uint32_t)nch, threads, [&](uint32_t c, int) {
        for (int64_t i = c * chunk; i < std::min(n, (int64_t)(c + 1) * chunk); i++) {
            V3 r = photon_irradiance(*s, v3(q[i * 6], q[i * 6 + 1], q[i * 6 + 2]), v3(q[i * 6 + 3], q[i * 6 + 4], q[i * 6 + 5]));
            irr[i * 3] = r.x; irr[i * 3 + 1] = r.y; irr[i * 3 + 2] = r.z;
        }
    });
    return RT_OK;
}

// k nearest photons with d² ≤ rmax², sorted by (d², emission index)
int32_t orc_knn(void* sp, const float* q, int64_t n, int32_t k, float rmax, int32_t* out_idx, float* out_d2, int32_t threads) {
    Scene* s = (Scene*)sp;
    float r2 = rmax * rmax;
    int64_t chunk = 256, nch = (n + chunk - 1) / chunk;
    parallel_rows((uint32_t)nch, threads, [&](uint32_t c, int) {
        std::vector<std::pair<float, const KdPhoton*>> cand;
        for (int64_t i = c * chunk; i < std::min(n, (int64_t)(c + 1) * chunk); i++) {
            cand.clear();
            kd_collect(s->photons.data(), s->photons.size(), q + i * 3, r2, false, nullptr, cand);
            std::sort(cand.begin(), cand.end(), [](const std::pair<float, const KdPhoton*>& a,
                                                   const std::pair<float, const KdPhoton*>& b) {
                return a.first < b.first || (a.first == b.first && a.second->idx < b.second->idx);
            });
            for (int j = 0; j < k; j++) {
                bool have = j < (int)cand.size();
                out_idx[i * k + j] = have ? cand[j].second->idx : -1;
                out_d2[i * k + j] = have ? cand[j].first : INFINITY;
            }
        }
    });
    return RT_OK;
}

}  // extern "C"
