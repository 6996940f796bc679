// rt_device.cuh — device data layouts and per-thread math shared by the
// traversal (rt_trace.cu) and shading (rt_shade.cu) kernels.
//
// HBM layout (all arrays 16-byte aligned, read through the read-only path):
//   nodes  : 8-wide BVH nodes, 14 float4 = 224 B each, the reference layout of
//            src/bvh.rs:25-32 (min[3][8], max[3][8], children[8]) so one node is
//            fetched with 14 128-bit loads.  child ≥ 0 → inner node, child with
//            the top bit set → leaf (type in bits 28-30, index in bits 0-27),
//            0xFFFFFFFF → empty slot.
//   tri    : 3 float4 per triangle, leaf order: (v0.xyz, e1.x) (e1.yz, e2.xy)
//            (e2.z, gid, mat, has_normals).  e1 = v1 - v0 and e2 = v2 - v0 are
//            the exact f32 differences the reference forms per hit
//            (triangle.rs:76-77), so the hit arithmetic is unchanged.
//   tri_n  : 3 float4 per triangle: (n0.xyz, n1.x) (n1.yz, n2.xy) (n2.z, -, -, -)
//   quad   : 5 float4: (normal.xyz, d) (Q.xyz, u.x) (u.yz, v.xy) (v.z, w.xyz) (gid, mat, area, -)
//   sphere : 2 float4: (centre.xyz, r) (gid, mat, -, -)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define RT_HD __host__ __device__ __forceinline__
#define RT_D __device__ __forceinline__

#define RT_LEAF_BIT   0x80000000u
#define RT_EMPTY_REF  0xFFFFFFFFu
#define RT_MISS_REF   0xFFFFFFFFu
// Hit records written by the extend kernel: bits 31:29 = material class code
// (0 emitter, 1 diffuse, 2 conductor, 3 dielectric, 4 PBR), 28:27 = primitive
// type, 26:0 = typed index (so at most 2^27 primitives of one type).
// RT_MISS_REF (code 7) is never a hit.
#define RT_HIT_TYPE(ref)  (((ref) >> 27) & 3u)
#define RT_HIT_INDEX(ref) ((ref) & 0x07FFFFFFu)
#define RT_HIT_CODE(ref)  ((ref) >> 29)
#define RT_HIT_MAX_INDEX  0x07FFFFFFu
// the hit record of a leaf reference (type in 30:28, index in 27:0) and a class code
#define RT_HIT_MAKE(leaf_ref, code) (((uint32_t)(code) << 29) | ((((leaf_ref) >> 28) & 3u) << 27) | ((leaf_ref) & 0x07FFFFFFu))

namespace rtd {

static constexpr float PI_F = 3.14159265358979323846f;
static constexpr float SLAB_WIDEN = 1.52587890625e-05f;   // 2^-16: conservative slab exit

// ── device material record ──────────────────────────────────────────────────
struct DevMaterial {
    int   type;
    int   metal;        // 0-2 builtin tables, 3 custom
    float albedo[3];
    float odd[3];
    float checker_scale;
    float cauchy_b, cauchy_c;
    float absorption[3];
    float roughness;
    float temp_k, intensity;
    float bb_norm;      // 1 / mean(planck) over the sampled grid (material.rs:47-52)
    float bb_avg[3];    // time-averaged RGB of the blackbody (material.rs:53-59)
    int   nk_count;
    float nk_start, nk_step;
    float nk_n[16], nk_k[16];
    // PBR (material.rs:680-1050); the anisotropy frame rotation and aspect are
    // precomputed: aniso_c/s = cos/sin(anisotropy_angle), aspect = sqrt(max(1 − 0.9·a, 0.001))
    float metallic, aniso_c, aniso_s, aspect;
    float clearcoat, clearcoat_roughness, film_thickness, film_ior, sheen, sheen_tint;
    float emission[3];   // emission × emission_strength
    int albedo_tex, roughness_tex, metallic_tex, ao_tex, normal_tex;   // 1-based, 0 = none
};

struct DevLight {        // one entry of the NEE light list (hittable.rs:138-225)
    int    type;         // RT_PRIM_QUAD / RT_PRIM_SPHERE
    int    mat;
    float4 g[5];         // quad record or sphere record (same packing as above)
};

// A participating medium (volume.rs:78-263): boundary sphere or box faces (the
// quad record of make_box, quad.rs:201-215, without the id row), HG albedo and
// asymmetry, and for the noise medium its Perlin tables (perlin.rs:4-33).
struct DevFace { float4 g[4]; };
struct DevMedium {
    int type, boundary;          // RT_MEDIUM_*, RT_BOUND_*
    float4 sphere;               // centre, radius
    DevFace face[6];
    float density;               // σ, or the noise medium's density scale max(density, ε)
    float g, noise_scale, threshold;
    float3 color;
    const float4* vec;           // 256 Perlin vectors
    const int32_t* perm;         // 3 × 256 permutations
    // grid medium: σ_t = density × trilinear(grid) over the box [lo, lo + 1/inv_vox·res];
    // major holds per brick of RT_GRID_BRICK³ voxels the largest voxel value the
    // brick's trilinear lookups read (one voxel of apron), slightly enlarged
    const float* grid;
    const float* major;
    int res[3], nb[3];
    float3 lo, inv_vox, bw, inv_bw;   // box corner, voxels per unit, brick width, bricks per unit
};
#define RT_GRID_BRICK 8

// A texture (texture.rs): an 8-bit RGB image, or a Perlin mottle between two colours
struct DevTexture {
    int type, w, h;              // RT_TEX_*
    const uint8_t* px;           // IMAGE: h × w × 3
    float scale;
    float3 lo, hi;
    const float4* vec;           // MOTTLE: 256 Perlin vectors
    const int32_t* perm;         // 3 × 256 permutations
};

struct DevScene {
    const float4* nodes;
    // the same nodes with 8-bit child boxes, 8 float4 each (see encode_qnode),
    // and which copy the traversal reads (RT_NODES_*)
    const float4* qnodes;
    // 4-wide nodes of the same binary tree, 7 float4 each (lower x, y, z and
    // upper x, y, z planes of 4 children, then their references)
    const float4* nodes4;
    int node_format;
    const float4* tri;
    const float4* tri_n;
    const float4* quad;
    const float4* sphere;
    const DevLight* lights;
    const DevMaterial* mats;
    const uint8_t* mat_code;    // class code per material (see RT_HIT_CODE)
    int n_lights, n_mats;
    const DevMedium* media;
    int n_media;
    int n_pbr;                  // PBR materials in the scene (their shading kernel runs only if > 0)
    uint32_t class_mask;        // bit per shading class some material of the scene can produce (host side)
    // analytic convex solids in leaf order: 2 float4 each, (plane offset, count,
    // material, polish) (canonical id, -, -, -); their world-space planes
    // (n.xyz, d); per plane the world-space shading normals of a front-face and
    // a back-face hit, micro-tilted in object space (diamond.rs:267-270)
    const float4* cvx;
    const float4* cvx_planes;
    const float4* cvx_shade;
    // cylinders, cones, disks and infinite planes share the convex leaf type:
    // their count field is −1 − RT_SHAPE_*, their offset indexes 8 float4 here
    // (see shape_test)
    const float4* shape_par;
    int n_analytic;             // convex solids + shapes (the traversal compiles their tests in only if > 0)
    int trace_per_sm, shade_per_sm;   // launch tuning (host side; 0 = the built-in grids)
    // traversal stack beyond the shared-memory ring: entry e ≥ RT_SHORT_STACK
    // of global thread g at stack_spill[(e − RT_SHORT_STACK) · threads + g];
    // stack_cap entries in all (7 per tree level; lowered only by rt_set_tuning)
    uint32_t* stack_spill;
    int stack_cap;
    int stack_ring;             // shared-memory ring slots: RT_SHORT_STACK unless tuned (a power of two)
    // textures; per triangle 2 float4 of (u, v) at the corners and 3 float4 of
    // corner tangents (NULL: the reference's default UVs and (1, 0, 0) tangents)
    const DevTexture* tex;
    const float* srgb_lut;      // 256 sRGB → linear values (output.rs:90-96)
    const float4* tri_uv;
    const float4* tri_tan;
    // spectral tables: CIE x̄ȳz̄ on the 5 nm grid from 380 nm and the per-channel
    // normalisations of spectral_to_rgb / spectral_fire_rgb (spectrum.rs:78-177)
    const float4* cmf;          // n_spec entries (x, y, z, -)
    int   n_spec;
    float norms[3], fire_norms[3];
    float lam_lo, lam_range;
    const float* elut;          // 64×64 E_ss(mu, alpha)
    const float4* nacre;        // 256 thin-film colours over OPD 0..2500 nm (material.rs:1096-1118)
    // environment map
    int   has_env;
    int   env_w, env_h;
    const float4* env;          // rgb + luminance per texel
    const float2* env_alias;    // (probability, alias index bits) per texel
    float env_inv_total;
    float env_sin_r, env_cos_r;
    // background
    int   bg_type;
    float bg_color[3], bg_top[3], bg_bottom[3];
    int   vis_type;
    float vis_color[3], vis_top[3], vis_bottom[3];
    // Physical sky (renderer.rs:231-362): unit sun direction, turbidity, and
    // whether the sun is above the horizon (sun NEE and the sun pdf need it)
    float3 sun_dir;
    float  turbidity;
    int    has_sun;
};

// ── float3 helpers ──────────────────────────────────────────────────────────
RT_HD float3 mk(float x, float y, float z) { return make_float3(x, y, z); }
RT_HD float3 operator+(float3 a, float3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
RT_HD float3 operator-(float3 a, float3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
RT_HD float3 operator-(float3 a) { return mk(-a.x, -a.y, -a.z); }
RT_HD float3 operator*(float3 a, float3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
RT_HD float3 operator*(float3 a, float t) { return mk(a.x * t, a.y * t, a.z * t); }
RT_HD float3 operator*(float t, float3 a) { return mk(a.x * t, a.y * t, a.z * t); }
// r.at(t) (ray.rs): o + t·d with the product rounded before the sum, as on the
// CPU; a fused multiply-add would move points off a plane by a different
// rounding, which flips floor-based lookups (the checker) at y = 0
RT_HD float3 ray_at(float3 o, float3 d, float t) {
#ifdef __CUDA_ARCH__
    return mk(__fadd_rn(o.x, __fmul_rn(t, d.x)), __fadd_rn(o.y, __fmul_rn(t, d.y)), __fadd_rn(o.z, __fmul_rn(t, d.z)));
#else
    return mk(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
#endif
}
RT_HD float3 operator/(float3 a, float t) { return mk(a.x / t, a.y / t, a.z / t); }
RT_HD float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RT_HD float len2(float3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
RT_HD float3 cross3(float3 a, float3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
RT_D float3 unit3(float3 a) { return a / sqrtf(len2(a)); }
RT_HD float lum3(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
RT_HD float clampf_(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
RT_D float3 reflect3(float3 v, float3 n) { return v - 2.0f * dot3(v, n) * n; }
// a in the frame of Onb::from_w(n) (onb.rs:10-20)
RT_D float3 onb_local_w(float3 n, float3 a) {
    float3 w = unit3(n);
    float3 h = fabsf(w.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
    float3 v = unit3(cross3(w, h));
    float3 u = cross3(w, v);
    return a.x * u + a.y * v + a.z * w;
}

// ── counter-based RNG: pcg3d (Jarzynski & Olano, JCGT 2020) ──────────────────
RT_HD uint32_t mix32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
    return x;
}
RT_HD uint32_t pcg3d_x(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t x = a * 1664525u + 1013904223u;
    uint32_t y = b * 1664525u + 1013904223u;
    uint32_t z = c * 1664525u + 1013904223u;
    x += y * z; y += z * x; z += x * y;
    x ^= x >> 16; y ^= y >> 16; z ^= z >> 16;
    x += y * z; y += z * x; z += x * y;
    return x;
}
struct Rng { uint32_t a, b, c; };
RT_HD Rng make_rng(uint64_t seed, uint32_t pixel, uint32_t sample) {
    Rng r;
    r.a = pixel;
    r.b = sample ^ mix32((uint32_t)seed);
    r.c = mix32((uint32_t)(seed >> 32) + 0x9E3779B9u);
    return r;
}
RT_HD uint32_t rnd_u32(const Rng& r, uint32_t dim) { return pcg3d_x(r.a, r.b, dim ^ r.c); }
RT_HD float rnd(const Rng& r, uint32_t dim) { return (float)(rnd_u32(r, dim) >> 8) * (1.0f / 16777216.0f); }

enum {
    D_JIT_U = 0, D_JIT_V = 1, D_LENS_R = 2, D_LENS_P = 3, D_TIME = 4, D_LAMBDA = 5, D_LENS_K = 6,
    D_BOUNCE0 = 8, D_PER_BOUNCE = 16,
    B_SCATTER0 = 0, B_SCATTER1 = 1, B_LPICK = 2, B_LPT0 = 3, B_LPT1 = 4,
    B_SUN0 = 5, B_SUN1 = 6,
    B_ENV_ROW = 7, B_ENV_COL = 8, B_ENV_JU = 9, B_ENV_JV = 10, B_COS0 = 11, B_COS1 = 12, B_RR = 13,
    B_LOBE0 = 14, B_LOBE1 = 15,   // PBR lobe choice: clearcoat, then base specular
};

// Slab reciprocal: plain 1/d.  A ray with an infinite reciprocal component can
// produce (bound − o)·inv = 0·∞ = NaN when it lies exactly in a box face plane;
// the traversal then takes the NaN-aware slab path, where such a slab spans the
// whole line (the ray is inside the closed slab) so culling stays conservative.

// ── primitive hit tests: same f32 operation sequence as the reference ────────
// convex_hit (diamond.rs:202-253): the interval inside every half-space; the
// entry for outside rays, the exit for rays inside; *plane = crossing plane.
RT_D bool convex_test(const float4* pl, int n, float3 o, float3 d, float tmin, float tmax, float* t_out,
                      int* plane) {
    float t_enter = tmin, t_exit = tmax;
    int enter_i = -1, exit_i = -1;
    bool entry_found = false;
    for (int i = 0; i < n; i++) {
        float4 q = __ldg(pl + i);
        float3 nv = make_float3(q.x, q.y, q.z);
        float nd = nv.x * d.x + nv.y * d.y + nv.z * d.z;
        float no = nv.x * o.x + nv.y * o.y + nv.z * o.z;
        float t_face = (q.w - no) / nd;
        if (fabsf(nd) < 1e-8f) {
            if (no > q.w) return false;
            continue;
        }
        if (nd < 0.0f) {
            if (t_face > t_enter) { t_enter = t_face; enter_i = i; entry_found = true; }
        } else {
            if (t_face < t_exit || (exit_i < 0 && t_face == t_exit)) { t_exit = t_face; exit_i = i; }
        }
        if (t_enter > t_exit) return false;
    }
    if (t_enter > t_exit) return false;
    if (t_enter == t_exit && t_enter < tmax) return false;
    if (entry_found) { *t_out = t_enter; *plane = enter_i; return true; }
    // an interior ray whose exit lies beyond tmax crosses nothing in [tmin, tmax]
    if (exit_i < 0 || t_exit > tmax) return false;
    *t_out = t_exit; *plane = exit_i;
    return true;
}

// ── cylinder, cone, disk, infinite plane (cylinder.rs, cone.rs, disk.rs, plane.rs)
// Record P[0..7]: (centre, radius) (unit normal, height) (u axis, wave amplitude)
// (v axis, wave scale) (rotation row 0, scale) (row 1, 1/scale) (row 2, placed)
// (translation, 0).  The ray goes to object space through the SRT wrappers,
// outermost first: Translate, Rotate (transpose), UniformScale (transform.rs).
RT_D void shape_local(const float4* P, float3 o, float3 d, float3* lo, float3* ld) {
    float4 r0 = __ldg(P + 4), r1 = __ldg(P + 5), r2 = __ldg(P + 6);
    if (r2.w == 0.0f) { *lo = o; *ld = d; return; }
    float4 tr = __ldg(P + 7);
    float3 o1 = mk(o.x - tr.x, o.y - tr.y, o.z - tr.z);
    float3 o2 = mk(r0.x * o1.x + r1.x * o1.y + r2.x * o1.z, r0.y * o1.x + r1.y * o1.y + r2.y * o1.z,
                   r0.z * o1.x + r1.z * o1.y + r2.z * o1.z);
    float3 d2 = mk(r0.x * d.x + r1.x * d.y + r2.x * d.z, r0.y * d.x + r1.y * d.y + r2.y * d.z,
                   r0.z * d.x + r1.z * d.y + r2.z * d.z);
    float inv = r1.w;
    *lo = mk(inv * o2.x, inv * o2.y, inv * o2.z);
    *ld = mk(inv * d2.x, inv * d2.y, inv * d2.z);
}
// the closest crossing in [tmin, tmax] of an object-space ray; *part = 0 lateral
// surface (or the disk / plane), 1 bottom cap or cone base, 2 top cap
RT_D bool shape_test(int type, const float4* P, float3 o, float3 d, float tmin, float tmax, float* t_out, int* part) {
    float4 p0 = __ldg(P), p1 = __ldg(P + 1);
    float3 c = mk(p0.x, p0.y, p0.z);
    float radius = p0.w;
    if (type == RT_SHAPE_CYLINDER || type == RT_SHAPE_CONE) {                      // cylinder.rs:132-187, cone.rs:19-82
        bool cone = type == RT_SHAPE_CONE;
        float h = p1.w;
        float3 oc = o - c;
        float a, half_b, cc;
        if (cone) {
            float k = (radius / h) * (radius / h), hy = h - oc.y;
            a = d.x * d.x + d.z * d.z - k * d.y * d.y;
            half_b = oc.x * d.x + oc.z * d.z + k * hy * d.y;
            cc = oc.x * oc.x + oc.z * oc.z - k * hy * hy;
        } else {
            a = d.x * d.x + d.z * d.z;
            half_b = oc.x * d.x + oc.z * d.z;
            cc = oc.x * oc.x + oc.z * oc.z - radius * radius;
        }
        float best_t = tmax;
        bool found = false;
        if (cone ? fabsf(a) > 1e-8f : a > 1e-8f) {
            float disc = half_b * half_b - a * cc;
            if (disc >= 0.0f) {
                float sq = sqrtf(disc);
                float roots[2] = {(-half_b - sq) / a, (-half_b + sq) / a};
                for (int k = 0; k < 2; k++) {
                    float root = roots[k];
                    if (root < tmin || root > best_t) continue;
                    float ly = ray_at(o, d, root).y - c.y;
                    if (ly < 0.0f || ly > h) continue;
                    best_t = root; *part = 0; found = true;
                }
            }
        }
        if (fabsf(d.y) > 1e-8f) {
            for (int k = 0; k < (cone ? 1 : 2); k++) {
                float cap_y = k == 0 ? 0.0f : h;
                float t = cone ? -oc.y / d.y : (cap_y - oc.y) / d.y;
                if (cone ? !(t >= tmin && t <= best_t) : (t < tmin || t > best_t)) continue;
                float3 p = ray_at(o, d, t);
                float lx = p.x - c.x, lz = p.z - c.z;
                if (lx * lx + lz * lz > radius * radius) continue;
                best_t = t; *part = 1 + k; found = true;
            }
        }
        if (found) *t_out = best_t;
        return found;
    }
    float3 n = mk(p1.x, p1.y, p1.z);                                                // disk.rs:146-157, plane.rs:37-42
    float denom = dot3(n, d);
    if (!(fabsf(denom) >= 1e-8f)) return false;
    float t = dot3(n, c - o) / denom;
    if (t < tmin || t > tmax) return false;
    if (type == RT_SHAPE_DISK && len2(ray_at(o, d, t) - c) > radius * radius) return false;
    *t_out = t; *part = 0;
    return true;
}
// object-space outward normal of a crossing at p (cylinder.rs:155-159,
// cone.rs:50-54, the caps, disk.rs:153, plane.rs:46-66 with the wave bump)
RT_D float3 shape_outward(int type, const float4* P, float3 p, int part) {
    float4 p0 = __ldg(P), p1 = __ldg(P + 1);
    float3 c = mk(p0.x, p0.y, p0.z);
    if (type == RT_SHAPE_CYLINDER) {
        if (part == 0) return mk((p.x - c.x) / p0.w, 0.0f, (p.z - c.z) / p0.w);
        return mk(0.0f, part == 1 ? -1.0f : 1.0f, 0.0f);
    }
    if (type == RT_SHAPE_CONE) {
        if (part != 0) return mk(0.0f, -1.0f, 0.0f);
        float h = p1.w, k = (p0.w / h) * (p0.w / h), ly = p.y - c.y;
        float3 g = mk(p.x - c.x, k * (h - ly), p.z - c.z);
        return len2(g) > 1e-12f ? unit3(g) : mk(0.0f, 1.0f, 0.0f);
    }
    float3 n = mk(p1.x, p1.y, p1.z);
    float4 pu = __ldg(P + 2), pv = __ldg(P + 3);
    if (type == RT_SHAPE_PLANE && pu.w > 1e-6f) {
        float3 ua = mk(pu.x, pu.y, pu.z), va = mk(pv.x, pv.y, pv.z), off = p - c;
        float u = dot3(off, ua), v = dot3(off, va), sc = pv.w, a = pu.w;
        float phi1 = sc * u + 0.7f * sc * v, phi2 = 1.3f * sc * v - 0.5f * sc * u;
        float c1 = cosf(phi1), c2 = cosf(phi2);
        float dh_du = a * sc * c1 - 0.25f * a * sc * c2;
        float dh_dv = 0.7f * a * sc * c1 + 0.65f * a * sc * c2;
        return unit3(n - dh_du * ua - dh_dv * va);
    }
    return n;
}
// the world-space shading normal of a shape crossing: face-forward in object
// space (HitRecord::new), then turned by the rotation (transform.rs:236-241)
RT_D float3 shape_normal(int type, const float4* P, float3 o, float3 d, float t, int part, bool* front) {
    float3 lo, ld;
    shape_local(P, o, d, &lo, &ld);
    float3 ow = shape_outward(type, P, ray_at(lo, ld, t), part);
    *front = dot3(ld, ow) < 0.0f;
    float3 n = *front ? ow : -ow;
    float4 r0 = __ldg(P + 4), r1 = __ldg(P + 5), r2 = __ldg(P + 6);
    if (r2.w == 0.0f) return n;
    return mk(r0.x * n.x + r0.y * n.y + r0.z * n.z, r1.x * n.x + r1.y * n.y + r1.z * n.z,
              r2.x * n.x + r2.y * n.y + r2.z * n.z);
}

// triangle.rs:75-89
RT_D bool tri_test(float4 a, float4 b, float4 c, float3 o, float3 d, float tmin, float tmax,
                   float* t_out, float* b1o, float* b2o) {
    float3 v0 = mk(a.x, a.y, a.z), e1 = mk(a.w, b.x, b.y), e2 = mk(b.z, b.w, c.x);
    float3 h = cross3(d, e2);
    float aa = dot3(e1, h);
    if (fabsf(aa) < 1e-8f) return false;
    float f = 1.0f / aa;
    float3 s = o - v0;
    float b1 = f * dot3(s, h);
    if (!(b1 >= 0.0f && b1 <= 1.0f)) return false;
    float3 q = cross3(s, e1);
    float b2 = f * dot3(d, q);
    if (b2 < 0.0f || b1 + b2 > 1.0f) return false;
    float t = f * dot3(e2, q);
    if (t < tmin || t > tmax) return false;
    *t_out = t; *b1o = b1; *b2o = b2;
    return true;
}
// quad.rs:37-57
RT_D bool quad_test(const float4* g, float3 o, float3 d, float tmin, float tmax, float* t_out, float* al, float* be) {
    float4 g0 = g[0];
    float3 n = mk(g0.x, g0.y, g0.z);
    float denom = dot3(n, d);
    if (!(fabsf(denom) >= 1e-8f)) return false;
    float t = (g0.w - dot3(n, o)) / denom;
    if (t < tmin || t > tmax) return false;
    float4 g1 = g[1], g2 = g[2], g3 = g[3];
    float3 Q = mk(g1.x, g1.y, g1.z), u = mk(g1.w, g2.x, g2.y), v = mk(g2.z, g2.w, g3.x), w = mk(g3.y, g3.z, g3.w);
    float3 p = ray_at(o, d, t);
    float3 planar = p - Q;
    float alpha = dot3(w, cross3(planar, v));
    float beta = dot3(w, cross3(u, planar));
    if (!(alpha >= 0.0f && alpha <= 1.0f) || !(beta >= 0.0f && beta <= 1.0f)) return false;
    *t_out = t; *al = alpha; *be = beta;
    return true;
}
// sphere.rs:47-61
RT_D bool sphere_test(float4 s0, float3 o, float3 d, float tmin, float tmax, float* t_out) {
    float3 oc = o - mk(s0.x, s0.y, s0.z);
    float a = len2(d);
    if (!(a > 0.0f)) return false;
    float half_b = dot3(oc, d);
    float c = len2(oc) - s0.w * s0.w;
    float disc = half_b * half_b - a * c;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float root = (-half_b - sq) / a;
    if (root < tmin || root > tmax) {
        root = (-half_b + sq) / a;
        if (root < tmin || root > tmax) return false;
    }
    *t_out = root;
    return true;
}

}  // namespace rtd
