// rt_media.cuh — participating media on the device (volume.rs:39-263,
// perlin.rs:35-91): the ray-keyed random stream, Perlin turbulence, boundary
// intervals, free-flight sampling (constant: exponential; noise: delta
// tracking to the density scale; grid: delta tracking against per-brick
// majorants), shadow transmittance (grid: ratio tracking) and the HG phase
// function.  The CPU oracle restates the same functions (oracle/rt_oracle.cpp).
#pragma once
#include "../../include/rt_api.h"
#include "rt_device.cuh"

namespace rtd {

// A hit record of a medium event: class code 0 with type 3, the medium index
// in the index bits.  Convex solids share type 3 but are never emissive, so
// their code is non-zero; RT_MISS_REF has code 7.
#define RT_HIT_MEDIUM_BASE (3u << 27)
RT_HD bool hit_is_medium(uint32_t ref) { return (ref >> 27) == 3u; }

// random stream keyed on the ray's bits (origin xyz, direction x, wavelength;
// the reference seeds its medium RNG from these, volume.rs:114-120)
struct MedRng { uint32_t a, b, c; };
RT_D MedRng medium_rng(float3 o, float3 d, float lam) {
    MedRng r;
    r.a = __float_as_uint(o.x) ^ mix32(__float_as_uint(d.x) + 0x9E3779B9u);
    r.b = __float_as_uint(o.y) ^ mix32(__float_as_uint(lam) + 0x7F4A7C15u);
    r.c = mix32(__float_as_uint(o.z) + 0x4D454449u);
    return r;
}
RT_D float medium_rnd(const MedRng& r, uint32_t i) {
    return (float)(pcg3d_x(r.a, r.b, r.c ^ (i * 0x9E3779B9u)) >> 8) * (1.0f / 16777216.0f);
}

RT_D float perlin_noise(const float4* vec, const int32_t* perm, float3 p) {
    float fx = floorf(p.x), fy = floorf(p.y), fz = floorf(p.z);
    float u = p.x - fx, v = p.y - fy, w = p.z - fz;
    u = u * u * (3.0f - 2.0f * u);
    v = v * v * (3.0f - 2.0f * v);
    w = w * w * (3.0f - 2.0f * w);
    int i = (int)fx, j = (int)fy, k = (int)fz;
    float accum = 0.0f;
#pragma unroll
    for (int di = 0; di < 2; di++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++)
#pragma unroll
            for (int dk = 0; dk < 2; dk++) {
                int idx = (int)__ldg(perm + ((i + di) & 255)) ^ (int)__ldg(perm + 256 + ((j + dj) & 255)) ^
                          (int)__ldg(perm + 512 + ((k + dk) & 255));
                float4 c = __ldg(vec + idx);
                float fi = (float)di, fj = (float)dj, fk = (float)dk;
                float dt = c.x * (u - fi) + c.y * (v - fj) + c.z * (w - fk);
                accum += (fi * u + (1.0f - fi) * (1.0f - u)) * (fj * v + (1.0f - fj) * (1.0f - v)) *
                         (fk * w + (1.0f - fk) * (1.0f - w)) * dt;
            }
    return accum;
}
RT_D float medium_density_at(const DevMedium& m, float3 p) {
    float accum = 0.0f, weight = 1.0f;
    float3 q = p * m.noise_scale;
    for (int i = 0; i < 7; i++) {
        accum += weight * perlin_noise(m.vec, m.perm, q);
        weight *= 0.5f;
        q = mk(q.x * 2.0f, q.y * 2.0f, q.z * 2.0f);
    }
    float n = fabsf(accum) * 0.5f;
    return fmaxf(n - m.threshold, 0.0f) * m.density;
}

// first boundary hit in [tmin, tmax]
RT_D bool bound_hit(const DevMedium& m, float3 o, float3 d, float tmin, float tmax, float* t) {
    if (m.boundary == RT_BOUND_SPHERE) return sphere_test(m.sphere, o, d, tmin, tmax, t);
    bool any = false;
    float closest = tmax;
    for (int f = 0; f < 6; f++) {
        float tq, a, b;
        if (quad_test(m.face[f].g, o, d, tmin, closest, &tq, &a, &b)) { closest = tq; any = true; }
    }
    *t = closest;
    return any;
}

// ── grid medium (no counterpart in the reference) ────────────────────────────
// σ_t(x) = density × trilinear interpolation of the voxel values between voxel
// centres, clamped at the box faces.
RT_D float grid_density_at(const DevMedium& m, float3 p) {
    const float c[3] = {(p.x - m.lo.x) * m.inv_vox.x - 0.5f, (p.y - m.lo.y) * m.inv_vox.y - 0.5f,
                        (p.z - m.lo.z) * m.inv_vox.z - 0.5f};
    int i0[3], i1[3];
    float f[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float u = fminf(fmaxf(c[a], 0.0f), (float)(m.res[a] - 1));
        int i = min((int)u, max(m.res[a] - 2, 0));
        i0[a] = i;
        i1[a] = min(i + 1, m.res[a] - 1);
        f[a] = u - (float)i;
    }
    auto at = [&](int i, int j, int k) { return __ldg(m.grid + ((size_t)k * m.res[1] + j) * m.res[0] + i); };
    float c00 = at(i0[0], i0[1], i0[2]) * (1.0f - f[0]) + at(i1[0], i0[1], i0[2]) * f[0];
    float c10 = at(i0[0], i1[1], i0[2]) * (1.0f - f[0]) + at(i1[0], i1[1], i0[2]) * f[0];
    float c01 = at(i0[0], i0[1], i1[2]) * (1.0f - f[0]) + at(i1[0], i0[1], i1[2]) * f[0];
    float c11 = at(i0[0], i1[1], i1[2]) * (1.0f - f[0]) + at(i1[0], i1[1], i1[2]) * f[0];
    float c0 = c00 * (1.0f - f[1]) + c10 * f[1], c1 = c01 * (1.0f - f[1]) + c11 * f[1];
    return m.density * (c0 * (1.0f - f[2]) + c1 * f[2]);
}

// 3-D DDA over the majorant bricks (Amanatides & Woo 1987) from the point at t0
struct BrickWalk { int b[3], step[3]; float tnext[3], dt[3]; };
RT_D void brick_walk_init(const DevMedium& m, float3 o, float3 d, float t0, BrickWalk& w) {
    float3 p = ray_at(o, d, t0);
    const float pc[3] = {p.x, p.y, p.z}, oc[3] = {o.x, o.y, o.z}, dc[3] = {d.x, d.y, d.z};
    const float lo[3] = {m.lo.x, m.lo.y, m.lo.z}, bw[3] = {m.bw.x, m.bw.y, m.bw.z};
    const float ib[3] = {m.inv_bw.x, m.inv_bw.y, m.inv_bw.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        int b = (int)floorf((pc[a] - lo[a]) * ib[a]);
        b = min(max(b, 0), m.nb[a] - 1);
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
// end of the current brick's segment; false when the walk left the grid
RT_D bool brick_walk_next(const DevMedium& m, BrickWalk& w) {
    int a = w.tnext[0] <= w.tnext[1] ? (w.tnext[0] <= w.tnext[2] ? 0 : 2) : (w.tnext[1] <= w.tnext[2] ? 1 : 2);
    w.b[a] += w.step[a];
    w.tnext[a] += w.dt[a];
    return w.b[a] >= 0 && w.b[a] < m.nb[a];
}
RT_D float brick_major(const DevMedium& m, const BrickWalk& w) {
    return m.density * __ldg(m.major + ((size_t)w.b[2] * m.nb[1] + w.b[1]) * m.nb[0] + w.b[0]);
}
#define RT_GRID_MAX_STEPS 4096u   // tentative collisions per ray (bounded device loop)

// Delta tracking (Woodcock) in [t1, t2] against each brick's majorant: the
// scatter distance, or INFINITY when the ray leaves the box first.
RT_D float grid_sample(const DevMedium& m, float3 o, float3 d, float lam, float t1, float t2) {
    MedRng g = medium_rng(o, d, lam);
    float len = sqrtf(dot3(d, d));
    BrickWalk w;
    brick_walk_init(m, o, d, t1, w);
    float t = t1;
    uint32_t k = 0;
    for (int seg = 0; seg < 3 * RT_GRID_MAX_RES / RT_GRID_BRICK + 4; seg++) {
        float tb = fminf(fminf(w.tnext[0], w.tnext[1]), fminf(w.tnext[2], t2));
        float mu = brick_major(m, w);
        if (mu > 0.0f) {
            float inv = 1.0f / (mu * len);
            while (k < RT_GRID_MAX_STEPS) {
                float tt = t - inv * logf(fmaxf(medium_rnd(g, 2u * k), 1.1920928955078125e-07f));
                float xi = medium_rnd(g, 2u * k + 1u);
                k++;
                if (tt >= tb) break;
                t = tt;
                if (xi * mu < grid_density_at(m, ray_at(o, d, t))) return t;
            }
            if (k >= RT_GRID_MAX_STEPS) return INFINITY;
        }
        if (tb >= t2) return INFINITY;
        t = fmaxf(t, tb);
        if (!brick_walk_next(m, w)) return INFINITY;
    }
    return INFINITY;
}

// Ratio tracking (Cramer 1978; Novák et al. 2014) over [a, b]: the product of
// (1 − σ_t/μ) at tentative collisions, an unbiased estimate of exp(−∫σ_t).
// Its random stream is keyed on the shadow ray's bits and t_max.
RT_D float grid_transmittance(const DevMedium& m, float3 o, float3 d, float a, float b, float tmax) {
    MedRng g = medium_rng(o, d, tmax);
    float len = sqrtf(dot3(d, d));
    BrickWalk w;
    brick_walk_init(m, o, d, a, w);
    float t = a, T = 1.0f;
    uint32_t k = 0;
    for (int seg = 0; seg < 3 * RT_GRID_MAX_RES / RT_GRID_BRICK + 4; seg++) {
        float tb = fminf(fminf(w.tnext[0], w.tnext[1]), fminf(w.tnext[2], b));
        float mu = brick_major(m, w);
        if (mu > 0.0f) {
            float inv = 1.0f / (mu * len);
            while (k < RT_GRID_MAX_STEPS) {
                float tt = t - inv * logf(fmaxf(medium_rnd(g, 0x40000u + k), 1.1920928955078125e-07f));
                k++;
                if (tt >= tb) break;
                t = tt;
                T *= fmaxf(1.0f - grid_density_at(m, ray_at(o, d, t)) / mu, 0.0f);
                if (T <= 0.0f) return 0.0f;
            }
            if (k >= RT_GRID_MAX_STEPS) return T;
        }
        if (tb >= b) return T;
        t = fmaxf(t, tb);
        if (!brick_walk_next(m, w)) return T;
    }
    return T;
}

// scatter distance for t_max = ∞ (INFINITY when the ray leaves first);
// delta tracking is bounded at 4096 steps
RT_D float medium_sample(const DevMedium& m, float3 o, float3 d, float lam, float tmin) {
    float t1, t2;
    if (!bound_hit(m, o, d, -INFINITY, INFINITY, &t1)) return INFINITY;
    if (!bound_hit(m, o, d, t1 + 0.0001f, INFINITY, &t2)) return INFINITY;
    if (t1 < tmin) t1 = tmin;
    if (t1 >= t2) return INFINITY;
    if (t1 < 0.0f) t1 = 0.0f;
    if (m.type == RT_MEDIUM_GRID) return grid_sample(m, o, d, lam, t1, t2);
    float len = sqrtf(dot3(d, d));
    MedRng g = medium_rng(o, d, lam);
    if (m.type == RT_MEDIUM_CONSTANT) {
        float dist_inside = (t2 - t1) * len;
        float hit_dist = (-1.0f / m.density) * logf(fmaxf(medium_rnd(g, 0), 1.1920928955078125e-07f));
        if (hit_dist > dist_inside) return INFINITY;
        return t1 + hit_dist / len;
    }
    float inv_maj = 1.0f / (m.density * len);
    float t = t1;
    for (uint32_t k = 0; k < 4096u; k++) {
        t -= inv_maj * logf(fmaxf(medium_rnd(g, 2u * k), 1.1920928955078125e-07f));
        if (t >= t2) return INFINITY;
        float dens = medium_density_at(m, ray_at(o, d, t));
        if (medium_rnd(g, 2u * k + 1u) < dens / m.density) return t;
    }
    return INFINITY;
}

// nearest medium event before tsurf: medium index or -1
RT_D int media_event(const DevScene& S, float3 o, float3 d, float lam, float tmin, float tsurf, float* t_out) {
    int best = -1;
    float bt = tsurf;
    for (int mi = 0; mi < S.n_media; mi++) {
        float t = medium_sample(S.media[mi], o, d, lam, tmin);
        if (t < bt) { bt = t; best = mi; }
    }
    *t_out = bt;
    return best;
}

RT_D float medium_transmittance(const DevMedium& m, float3 o, float3 d, float tmin, float tmax) {
    float t1, t2;
    if (!bound_hit(m, o, d, -INFINITY, INFINITY, &t1)) return 1.0f;
    if (!bound_hit(m, o, d, t1 + 0.0001f, INFINITY, &t2)) return 1.0f;
    float a = fmaxf(fmaxf(t1, 0.0f), tmin), b = fminf(t2, tmax);
    if (a >= b) return 1.0f;
    if (m.type == RT_MEDIUM_GRID) return grid_transmittance(m, o, d, a, b, tmax);
    float len = sqrtf(dot3(d, d));
    float l = (b - a) * len;
    if (m.type == RT_MEDIUM_CONSTANT) return expf(-m.density * l);
    float seg_t = l / len, sum = 0.0f;
    for (int i = 0; i < 16; i++) {
        float t = a + seg_t * ((float)i + 0.5f) / 16.0f;
        sum += medium_density_at(m, ray_at(o, d, t));
    }
    return expf(-sum / 16.0f * l);
}

RT_D float media_transmittance(const DevScene& S, float3 o, float3 d, float tmin, float tmax) {
    float tr = 1.0f;
    for (int mi = 0; mi < S.n_media; mi++) {
        tr *= medium_transmittance(S.media[mi], o, d, tmin, tmax);
        if (tr <= 0.0f) return 0.0f;
    }
    return tr;
}

RT_D float3 hg_sample(float3 w, float g, float xi1, float xi2) {
    float cos_t;
    if (fabsf(g) < 1e-3f) {
        cos_t = 1.0f - 2.0f * xi1;
    } else {
        float sq = (1.0f - g * g) / fmaxf(1.0f - g + 2.0f * g * xi1, 1e-12f);
        cos_t = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    float sin_t = sqrtf(fmaxf(1.0f - cos_t * cos_t, 0.0f));
    float sp, cp;
    sincosf(2.0f * PI_F * xi2, &sp, &cp);
    float3 helper = fabsf(w.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
    float3 u = unit3(cross3(w, helper));
    float3 v = cross3(w, u);
    return u * (sin_t * cp) + v * (sin_t * sp) + w * cos_t;
}

}  // namespace rtd
