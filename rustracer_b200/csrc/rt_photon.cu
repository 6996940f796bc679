// rt_photon.cu — caustic photon map on the device (src/photon.rs).
//
// Build (rt_photon_build):
//   emit      one thread per photon: disk or cosine quad source (photon.rs:41-135)
//   trace     ≤ 12 bounces, reusing the closest-hit traversal kernel; k_photon_shade
//             continues specular photons and stores the first diffuse hit after a
//             specular bounce (trace_photon, photon.rs:232-277) into its emission slot
//   compact   stored photons in emission order (exclusive scan of the flags)
//   sort      key = grid cell (Morton code of its 10-bit coordinates) above the
//             30-bit Morton code of the position; stable radix sort
//   grid      [start, end) of every cell of a uniform grid (cells ≥ 2 × radius)
//   tree      implicit complete binary tree of boxes over 32-photon leaves of the
//             same order (node i has children 2i+1, 2i+2)
// Gather (one warp per query): the photons of the ≤ 2 × 2 × 2 cells that a ball
// of the map's radius meets, joined into one list that the lanes read 32 at a
// time (the box heap for a larger radius, or when those cells hold very many):
//   radius    Σ power·(1 − d²/r²) over d² < r², n_p·n > 0, × 2/(π²r²) (photon.rs:195-228)
//   k-NN      the k-th smallest d² among those photons within the maximum radius:
//             one traversal collects them into shared memory, a radix select
//             finds the k-th, the sum runs over the collected photons (more
//             than PH_CAND_CAP of them: histogram refinement over re-traversals)
//   rt_knn    exact k nearest (d² ≤ rmax²) sorted by (d², emission index)
#include <cub/cub.cuh>

#include "rt_internal.h"
#include "rt_media.cuh"
#include "rt_ggx.cuh"
#include "rt_texture.cuh"

using namespace rtd;

#define PH_LEAF 32
#define PH_STACK 64
#define PH_SEL_CAP 256

namespace {

RT_D float box_d2(float4 lo, float4 hi, float3 p) {
    float dx = fmaxf(fmaxf(lo.x - p.x, 0.0f), p.x - hi.x);
    float dy = fmaxf(fmaxf(lo.y - p.y, 0.0f), p.y - hi.y);
    float dz = fmaxf(fmaxf(lo.z - p.z, 0.0f), p.z - hi.z);
    // rounded like the photon distances (no fused multiply-add), so a box is
    // never farther than a photon on its boundary
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// ── emission ────────────────────────────────────────────────────────────────
struct EmitSetup {
    int type;
    float3 t, b, center, dir, normal, corner, u, v, ta, ba, power;
    float radius, lum_clamp;
    uint32_t first, count;
    float3 target;       // projection sphere of a quad source (target_r 0: the whole hemisphere)
    float target_r;
};
struct EmitSet { EmitSetup e[RT_MAX_EMITTERS]; int n; float lam_lo, lam_range; uint64_t seed; };

RT_D Rng photon_rng(uint64_t seed, uint32_t gid) {
    Rng r;
    r.a = gid;
    r.b = mix32((uint32_t)seed) ^ 0x50484F54u;
    r.c = mix32((uint32_t)(seed >> 32) + 0x9E3779B9u);
    return r;
}
enum { P_EMIT0 = 0, P_EMIT1 = 1, P_EMIT2 = 2, P_EMIT3 = 3, P_LAMBDA = 4, P_BOUNCE0 = 8, P_PER_BOUNCE = 4 };

// Photon slot i traces emission index first + i (its random stream and the
// index stored with it); the emitter is the one whose range holds that index.
__global__ void k_photon_emit(PathState P, EmitSet E, uint32_t first, uint32_t total, uint32_t* queue0,
                              uint32_t* count0, uint8_t* flags) {
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < total; slot += gridDim.x * blockDim.x) {
        uint32_t gid = first + slot;
        int ei = 0;
        for (int k = 1; k < E.n; k++) if (gid >= E.e[k].first) ei = k;
        const EmitSetup& em = E.e[ei];
        Rng rng = photon_rng(E.seed, gid);
        float3 o, d;
        float wgt = 1.0f;
        if (em.type == RT_EMIT_DISK) {
            float r = em.radius * sqrtf(rnd(rng, P_EMIT0));
            float sp, cp;
            sincosf(2.0f * PI_F * rnd(rng, P_EMIT1), &sp, &cp);
            o = em.center + em.t * (r * cp) + em.b * (r * sp);
            d = em.dir;
        } else {
            float ss = rnd(rng, P_EMIT0), tt = rnd(rng, P_EMIT1);
            o = em.corner + em.u * ss + em.v * tt;
            float3 tc = em.target - o;
            float d2 = len2(tc), rr = em.target_r * em.target_r;
            if (em.target_r > 0.0f && d2 > rr) {
                // projection map: uniform in the cone toward the target sphere,
                // power × cosine density / cone density (0: below the light's plane)
                float ctm = sqrtf(1.0f - rr / d2);
                float sp, cp;
                sincosf(2.0f * PI_F * rnd(rng, P_EMIT3), &sp, &cp);
                float ct = 1.0f - rnd(rng, P_EMIT2) * (1.0f - ctm);
                float st = sqrtf(fmaxf(1.0f - ct * ct, 0.0f));
                d = onb_local_w(unit3(tc), mk(cp * st, sp * st, ct));
                float cl = dot3(d, em.normal);
                wgt = cl > 0.0f ? 2.0f * cl * (1.0f - ctm) : 0.0f;
            } else {
                float ct = sqrtf(rnd(rng, P_EMIT2));
                float st = sqrtf(1.0f - ct * ct);
                float sp, cp;
                sincosf(2.0f * PI_F * rnd(rng, P_EMIT3), &sp, &cp);
                d = st * cp * em.ta + st * sp * em.ba + ct * em.normal;
            }
        }
        // a photon with no power is not traced: a NaN origin makes the
        // traversal report a miss, which ends it
        if (!(wgt > 0.0f)) o = mk(__int_as_float(0x7fc00000), 0.0f, 0.0f);
        float lam = E.lam_lo + E.lam_range * rnd(rng, P_LAMBDA);
        if (lam >= E.lam_lo + E.lam_range) lam = nextafterf(E.lam_lo + E.lam_range, 0.0f);
        P.ray_o[slot] = make_float4(o.x, o.y, o.z, em.lum_clamp);
        P.ray_d[slot] = make_float4(d.x, d.y, d.z, lam);
        P.thr[slot] = make_float4(em.power.x * wgt, em.power.y * wgt, em.power.z * wgt, 0.0f);
        P.meta[slot] = make_uint4(gid, 0u, 0u, 0u);
        flags[slot] = 0;
        queue0[slot] = slot;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *count0 = total;
}

// spectrum helpers (spectrum.rs); duplicated from the shading TU as device
// functions local to this file
RT_D float3 cmf_rgb(const DevScene& S, float lambda, bool fire) {
    float t = clampf_((lambda - 380.0f) / 5.0f, 0.0f, (float)(S.n_spec - 1));
    int i = min((int)t, S.n_spec - 2);
    float frac = t - (float)i;
    float4 a = __ldg(S.cmf + i), bb = __ldg(S.cmf + i + 1);
    float x = a.x + frac * (bb.x - a.x), y = a.y + frac * (bb.y - a.y), z = a.z + frac * (bb.z - a.z);
    float c[3] = {fmaxf(3.2406f * x - 1.5372f * y - 0.4986f * z, 0.0f),
                  fmaxf(-0.9689f * x + 1.8758f * y + 0.0415f * z, 0.0f),
                  fmaxf(0.0557f * x - 0.2040f * y + 1.0570f * z, 0.0f)};
    if (!fire) return mk(c[0] * S.norms[0], c[1] * S.norms[1], c[2] * S.norms[2]);
    float w = fmaxf(powf(y, 0.5f), 0.08f);
    for (int k = 0; k < 3; k++) c[k] *= w;
    float lum = 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
    for (int k = 0; k < 3; k++) c[k] = c[k] * 0.5f + lum * 0.5f;
    return mk(c[0] * S.fire_norms[0], c[1] * S.fire_norms[1], c[2] * S.fire_norms[2]);
}
RT_D float fresnel_diel(float ci, float eta) {
    float sin2_i = fmaxf(1.0f - ci * ci, 0.0f), sin2_t = eta * eta * sin2_i;
    if (sin2_t >= 1.0f) return 1.0f;
    float ct = sqrtf(1.0f - sin2_t);
    float rs = (eta * ci - ct) / (eta * ci + ct), rp = (eta * ct - ci) / (eta * ct + ci);
    return (rs * rs + rp * rp) * 0.5f;
}
RT_D float fresnel_cond(float ci, float n, float k) {
    float cos2 = ci * ci, sin2 = fmaxf(1.0f - cos2, 0.0f), n2 = n * n, k2 = k * k;
    float t0 = n2 - k2 - sin2, ab = sqrtf(t0 * t0 + 4.0f * n2 * k2), t1 = ab + cos2;
    float a = sqrtf(fmaxf(0.5f * (ab + t0), 0.0f)), t2 = 2.0f * ci * a;
    float rs = (t1 - t2) / fmaxf(t1 + t2, 1e-12f);
    float t3 = cos2 * ab + sin2 * sin2, t4 = t2 * sin2;
    float rp = rs * (t3 - t4) / fmaxf(t3 + t4, 1e-12f);
    return clampf_(0.5f * (rp + rs), 0.0f, 1.0f);
}
// One bounce of trace_photon for every queued photon.
__global__ void k_photon_shade(DevScene S, PathState P, uint32_t bounce, const uint32_t* __restrict__ qin,
                               const uint32_t* cin, uint32_t* qout, uint32_t* cout, float4* st_pos, float4* st_pow,
                               float4* st_nor, uint8_t* flags, uint64_t seed) {
    uint32_t n = *cin;
    for (uint32_t qi0 = blockIdx.x * blockDim.x; qi0 < n; qi0 += gridDim.x * blockDim.x) {
        uint32_t qi = qi0 + threadIdx.x;
        bool cont = false;
        uint32_t slot = 0;
        if (qi < n) {
            slot = qin[qi];
            const uint32_t eidx = P.meta[slot].x;      // emission index: the photon's random stream
            float4 hv = P.hit[slot], ro = P.ray_o[slot], rdv = P.ray_d[slot], th = P.thr[slot];
            uint32_t ref = __float_as_uint(hv.x);
            if (hit_is_medium(ref)) {
                // a medium scatter is a skip_pdf bounce of the caustic path (photon.rs:252-260)
                float3 o = mk(ro.x, ro.y, ro.z), d = mk(rdv.x, rdv.y, rdv.z);
                const DevMedium& M = S.media[RT_HIT_INDEX(ref)];
                Rng rng = photon_rng(seed, eidx);
                uint32_t base = P_BOUNCE0 + bounce * P_PER_BOUNCE;
                float3 p = ray_at(o, d, hv.y);
                float3 nd = hg_sample(unit3(d), M.g, rnd(rng, base + 0), rnd(rng, base + 1));
                P.ray_o[slot] = make_float4(p.x, p.y, p.z, ro.w);
                P.ray_d[slot] = make_float4(nd.x, nd.y, nd.z, rdv.w);
                P.thr[slot] = make_float4(th.x * M.color.x, th.y * M.color.y, th.z * M.color.z,
                                         __uint_as_float(__float_as_uint(th.w) + 1u));
                cont = true;
            } else if (ref != RT_MISS_REF) {
                float3 o = mk(ro.x, ro.y, ro.z), d = mk(rdv.x, rdv.y, rdv.z), power = mk(th.x, th.y, th.z);
                float lam = rdv.w, lum_clamp = ro.w;
                uint32_t spec_depth = __float_as_uint(th.w);
                float t = hv.y;
                float3 p = ray_at(o, d, t);
                uint32_t type = RT_HIT_TYPE(ref), idx = RT_HIT_INDEX(ref);
                float3 outward;
                int mat, cvx_wp = 0, shape = -1;
                if (type == RT_PRIM_TRI) {
                    const float4* g = S.tri + (size_t)idx * 3;
                    float4 ga = __ldg(g), gb = __ldg(g + 1), gc = __ldg(g + 2);
                    float3 e1 = mk(ga.w, gb.x, gb.y), e2 = mk(gb.z, gb.w, gc.x);
                    mat = __float_as_int(gc.z);
                    if (__float_as_int(gc.w)) {
                        const float4* gn = S.tri_n + (size_t)idx * 3;
                        float4 na = __ldg(gn), nb = __ldg(gn + 1), nc = __ldg(gn + 2);
                        float b1 = hv.z, b2 = hv.w, b0 = 1.0f - b1 - b2;
                        float3 sn = b0 * mk(na.x, na.y, na.z) + b1 * mk(na.w, nb.x, nb.y) + b2 * mk(nb.z, nb.w, nc.x);
                        outward = len2(sn) > 1e-12f ? unit3(sn) : unit3(cross3(e1, e2));
                    } else {
                        outward = unit3(cross3(e1, e2));
                    }
                } else if (type == RT_PRIM_QUAD) {
                    const float4* g = S.quad + (size_t)idx * 5;
                    float4 g0 = __ldg(g);
                    outward = mk(g0.x, g0.y, g0.z);
                    mat = __float_as_int(__ldg(g + 4).y);
                } else if (type == RT_PRIM_SPHERE) {
                    const float4* g = S.sphere + (size_t)idx * 2;
                    float4 s0 = __ldg(g);
                    outward = (p - mk(s0.x, s0.y, s0.z)) / s0.w;
                    mat = __float_as_int(__ldg(g + 1).y);
                } else {                                    // convex solid: the crossing plane's normal
                    float4 c0 = __ldg(S.cvx + (size_t)idx * 2);
                    shape = __float_as_int(c0.y) < 0 ? -1 - __float_as_int(c0.y) : -1;
                    cvx_wp = __float_as_int(c0.x) + (shape < 0 ? max(__float_as_int(hv.z), 0) : 0);
                    if (shape < 0) {
                        float4 q = __ldg(S.cvx_planes + cvx_wp);
                        outward = mk(q.x, q.y, q.z);
                    }
                    mat = __float_as_int(c0.z);
                }
                bool front;
                float3 nrm;
                if (shape >= 0) {                           // cylinder, cone, disk, plane
                    nrm = shape_normal(shape, S.shape_par + cvx_wp, o, d, hv.y, __float_as_int(hv.z), &front);
                } else {
                    front = dot3(d, outward) < 0.0f;
                    nrm = front ? outward : -outward;
                    if (type == RT_PRIM_CONVEX) {           // polished facet normal, world space
                        float4 sn = __ldg(S.cvx_shade + (size_t)cvx_wp * 2 + (front ? 0 : 1));
                        nrm = mk(sn.x, sn.y, sn.z);
                    }
                }
                const DevMaterial& m = S.mats[mat];
                bool store = false;
                Rng rng = photon_rng(seed, eidx);
                uint32_t base = P_BOUNCE0 + bounce * P_PER_BOUNCE;
                float3 udir = unit3(d);
                if (m.type == RT_MAT_DIELECTRIC || m.type == RT_MAT_SPECTRAL_DIELECTRIC) {
                    bool spectral = m.type == RT_MAT_SPECTRAL_DIELECTRIC;
                    float ior = spectral ? m.cauchy_b + m.cauchy_c / ((lam * 1e-3f) * (lam * 1e-3f)) : m.cauchy_b;
                    float ratio = front ? 1.0f / ior : ior;
                    float ct = fminf(dot3(-udir, nrm), 1.0f), st = sqrtf(1.0f - ct * ct);
                    bool refl = ratio * st > 1.0f || fresnel_diel(ct, ratio) > rnd(rng, base + 0);
                    float3 nd;
                    if (refl) nd = reflect3(udir, nrm);
                    else {
                        float3 perp = ratio * (udir + ct * nrm);
                        float kk = 1.0f - len2(perp);
                        nd = kk < 0.0f ? reflect3(udir, nrm) : perp + (-sqrtf(kk) * nrm);
                    }
                    float3 att = mk(1.f, 1.f, 1.f);
                    if (spectral) {
                        if (!refl) att = cmf_rgb(S, lam, true);
                        if (!front) {
                            att.x *= expf(-m.absorption[0] * t);
                            att.y *= expf(-m.absorption[1] * t);
                            att.z *= expf(-m.absorption[2] * t);
                        }
                    }
                    power = power * att;
                    o = p; d = nd; spec_depth++; cont = true;
                } else if (m.type == RT_MAT_SPECTRAL_METAL) {
                    float3 wo = unit3(-d);
                    float cos_o = dot3(wo, nrm);
                    if (cos_o > 0.0f) {
                        float alpha = fmaxf(m.roughness * m.roughness, 1e-4f);
                        float3 nd;
                        float cos_h;
                        bool ok = true;
                        if (m.roughness == 0.0f) { nd = reflect3(udir, nrm); cos_h = cos_o; }
                        else {
                            float3 up = fabsf(nrm.y) < 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
                            float3 tt = unit3(cross3(nrm, up)), bb = cross3(nrm, tt);
                            float3 mts = vndf_sample(mk(dot3(wo, tt), dot3(wo, bb), cos_o), alpha, alpha, rnd(rng, base + 0),
                                              rnd(rng, base + 1));
                            float3 mm = unit3(tt * mts.x + bb * mts.y + nrm * mts.z);
                            float voh = fmaxf(dot3(wo, mm), 0.0f);
                            nd = unit3(2.0f * voh * mm - wo);
                            cos_h = voh;
                            ok = dot3(nd, nrm) > 0.0f;
                        }
                        if (ok && dot3(nd, nrm) > 0.0f) {
                            float weight = 1.0f;
                            if (m.roughness != 0.0f) {
                                float lo = smith_lambda(cos_o, alpha), li = smith_lambda(fmaxf(dot3(nd, nrm), 0.0f), alpha);
                                weight = ((1.0f + lo) / (1.0f + lo + li)) * fminf(1.0f / fmaxf(e_ss_lut(S, cos_o, alpha), 0.05f), 10.0f);
                            }
                            float tn = clampf_((lam - m.nk_start) / m.nk_step, 0.0f, (float)(m.nk_count - 1));
                            int i = min((int)tn, m.nk_count - 2);
                            float f = tn - (float)i;
                            float nn = m.nk_n[i] + f * (m.nk_n[i + 1] - m.nk_n[i]);
                            float kk = m.nk_k[i] + f * (m.nk_k[i + 1] - m.nk_k[i]);
                            power = power * (cmf_rgb(S, lam, false) * (fresnel_cond(cos_h, nn, kk) * weight));
                            o = p; d = nd; spec_depth++; cont = true;
                        }
                    }
                } else if (m.type == RT_MAT_PBR) {
                    // PbrMaterial::scatter: a specular lobe carries the photon on, the
                    // diffuse lobe stores it where can_receive_caustics (material.rs:1049)
                    float3 att, nd, sn = nrm;
                    PbrHit ph = pbr_scalars(m);
                    if (pbr_textured(m)) ph = pbr_hit(S, m, hit_uv(S, hv, front ? nrm : -nrm), nrm, &sn);
                    int lobe = pbr_scatter(S, m, ph, unit3(-d), sn, rnd(rng, base + 2), rnd(rng, base + 3),
                                           rnd(rng, base + 0), rnd(rng, base + 1), &att, &nd);
                    if (lobe == PBR_SPECULAR) {
                        power = power * att;
                        o = p; d = nd; spec_depth++; cont = true;
                    }
                    store = lobe == PBR_DIFFUSE && m.metallic < 0.999f;   // can_receive_caustics: the scalar
                } else if (m.type == RT_MAT_LAMBERTIAN || m.type == RT_MAT_CHECKER) {
                    store = true;
                }
                if (store) {                                // photon.rs:260-271
                    if (spec_depth > 0) {
                        float lum = lum3(power);
                        if (lum > lum_clamp) power = power * (lum_clamp / lum);
                        st_pos[slot] = make_float4(p.x, p.y, p.z, __uint_as_float(eidx));
                        st_pow[slot] = make_float4(power.x, power.y, power.z, 0.f);
                        st_nor[slot] = make_float4(nrm.x, nrm.y, nrm.z, 0.f);
                        flags[slot] = 1;
                    }
                }
                if (cont) {
                    P.ray_o[slot] = make_float4(o.x, o.y, o.z, lum_clamp);
                    P.ray_d[slot] = make_float4(d.x, d.y, d.z, lam);
                    P.thr[slot] = make_float4(power.x, power.y, power.z, __uint_as_float(spec_depth));
                }
            }
        }
        uint32_t m = __ballot_sync(__activemask(), cont);
        if (m) {
            uint32_t lane = threadIdx.x & 31u;
            int leader = __ffs(m) - 1;
            uint32_t b = 0;
            if ((int)lane == leader) b = atomicAdd(cout, __popc(m));
            b = __shfl_sync(__activemask(), b, leader);
            if (cont) qout[b + __popc(m & ((1u << lane) - 1u))] = slot;
        }
    }
}

__global__ void k_flags_to_u32(const uint8_t* f, uint32_t* o, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) o[i] = f[i];
}
__global__ void k_compact(const uint8_t* f, const uint32_t* scan, uint32_t n, const float4* sp, const float4* sw,
                          const float4* sn, float4* dp, float4* dw, float4* dn) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!f[i]) continue;
        uint32_t j = scan[i];
        dp[j] = sp[i]; dw[j] = sw[i]; dn[j] = sn[i];
    }
}

// ── Morton codes over the stored photons' box ────────────────────────────────
__global__ void k_bounds(const float4* p, uint32_t n, float* lo, float* hi) {
    float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 q = p[i];
        l[0] = fminf(l[0], q.x); l[1] = fminf(l[1], q.y); l[2] = fminf(l[2], q.z);
        h[0] = fmaxf(h[0], q.x); h[1] = fmaxf(h[1], q.y); h[2] = fmaxf(h[2], q.z);
    }
    for (int k = 0; k < 3; k++) {
        for (int o = 16; o > 0; o >>= 1) {
            l[k] = fminf(l[k], __shfl_xor_sync(0xFFFFFFFFu, l[k], o));
            h[k] = fmaxf(h[k], __shfl_xor_sync(0xFFFFFFFFu, h[k], o));
        }
    }
    if ((threadIdx.x & 31u) == 0) {
        // float min/max through ordered integer atomics (values are finite)
        for (int k = 0; k < 3; k++) {
            int li = __float_as_int(l[k]), hi_ = __float_as_int(h[k]);
            if (li >= 0) atomicMin((int*)&lo[k], li); else atomicMax((unsigned*)&lo[k], (unsigned)li);
            if (hi_ >= 0) atomicMax((int*)&hi[k], hi_); else atomicMin((unsigned*)&hi[k], (unsigned)hi_);
        }
    }
}
RT_D uint32_t expand10(uint32_t v) {
    v &= 1023u;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
// One cubic cell size for all three axes: caustic photons often lie on one
// plane, and stretching that plane's near-zero extent to 1024 cells would put
// rounding noise into every third bit of the code (leaves of 32 photons
// scattered across the whole map).
// Cell of coordinate x along one axis: the same float arithmetic for photons
// and for query bounds, clamped into the grid — monotone in x, so a photon
// between two bounds lies in a cell between theirs.
RT_D int grid_cell(float x, float lo, float inv, int n) {
    float f = floorf((x - lo) * inv);
    return (int)fminf(fmaxf(f, 0.0f), (float)(n - 1));
}
RT_D uint32_t cell_linear(const PhotonGrid& G, float4 q) {
    uint32_t x = grid_cell(q.x, G.lo[0], G.inv, G.n[0]), y = grid_cell(q.y, G.lo[1], G.inv, G.n[1]);
    uint32_t z = grid_cell(q.z, G.lo[2], G.inv, G.n[2]);
    return x + (uint32_t)G.n[0] * (y + (uint32_t)G.n[1] * z);
}
__global__ void k_morton(const float4* p, uint32_t n, const float* lo, const float* hi, PhotonGrid G, uint64_t* key,
                         uint32_t* val) {
    float3 l = mk(lo[0], lo[1], lo[2]);
    float ext = fmaxf(fmaxf(fmaxf(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]), 1e-30f);
    float3 e = mk(ext, ext, ext);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 q = p[i];
        uint32_t x = (uint32_t)fminf(fmaxf((q.x - l.x) / e.x * 1024.0f, 0.0f), 1023.0f);
        uint32_t y = (uint32_t)fminf(fmaxf((q.y - l.y) / e.y * 1024.0f, 0.0f), 1023.0f);
        uint32_t z = (uint32_t)fminf(fmaxf((q.z - l.z) / e.z * 1024.0f, 0.0f), 1023.0f);
        uint32_t cx = grid_cell(q.x, G.lo[0], G.inv, G.n[0]), cy = grid_cell(q.y, G.lo[1], G.inv, G.n[1]);
        uint32_t cz = grid_cell(q.z, G.lo[2], G.inv, G.n[2]);
        uint64_t cell = (expand10(cx) << 2) | (expand10(cy) << 1) | expand10(cz);
        key[i] = cell << 30 | ((expand10(x) << 2) | (expand10(y) << 1) | expand10(z));
        val[i] = i;
    }
}
// [start, end) of every non-empty cell (the table is zeroed first: empty = [0, 0))
__global__ void k_cell_ranges(const float4* p, uint32_t n, PhotonGrid G, uint2* cells) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t c = cell_linear(G, p[i]);
        if (i == 0 || cell_linear(G, p[i - 1]) != c) cells[c].x = i;
        if (i + 1 == n || cell_linear(G, p[i + 1]) != c) cells[c].y = i + 1;
    }
}
__global__ void k_gather_sorted(const uint32_t* order, uint32_t n, const float4* sp, const float4* sw, const float4* sn,
                                float4* dp, float4* dw, float4* dn) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t j = order[i];
        dp[i] = sp[j]; dw[i] = sw[j]; dn[i] = sn[j];
    }
}
// leaf boxes (level `leaves` of the heap), then each internal level bottom-up
__global__ void k_leaf_boxes(const float4* p, uint32_t n, uint32_t nleaf_pow2, float4* blo, float4* bhi) {
    uint32_t first = nleaf_pow2 - 1;
    for (uint32_t L = blockIdx.x * blockDim.x + threadIdx.x; L < nleaf_pow2; L += gridDim.x * blockDim.x) {
        float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
        for (uint32_t k = L * PH_LEAF; k < min(n, (L + 1) * PH_LEAF); k++) {
            float4 q = p[k];
            lo.x = fminf(lo.x, q.x); lo.y = fminf(lo.y, q.y); lo.z = fminf(lo.z, q.z);
            hi.x = fmaxf(hi.x, q.x); hi.y = fmaxf(hi.y, q.y); hi.z = fmaxf(hi.z, q.z);
        }
        blo[first + L] = lo;
        bhi[first + L] = hi;
    }
}
__global__ void k_level_boxes(uint32_t first, uint32_t count, float4* blo, float4* bhi) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        uint32_t nd = first + i, a = 2 * nd + 1, b = 2 * nd + 2;
        float4 la = blo[a], lb = blo[b], ha = bhi[a], hb = bhi[b];
        blo[nd] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.f);
        bhi[nd] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.f);
    }
}

}  // namespace

// ── warp-cooperative queries (used by the render path and the API) ─────────
namespace rtph {

struct Map {
    const float4 *pos, *pow, *nor;   // (cell, Morton) order; pos.w = emission index bits
    const float4 *blo, *bhi;         // heap of boxes
    const uint2* cells;              // [start, end) per grid cell
    PhotonGrid G;
    uint32_t n, nleaf_pow2;
    float r2;                        // radius (or k-NN maximum radius) squared
    uint32_t knn_k;
};

// Cells a ball of squared radius r2 around p may reach.  The bounds are
// widened by 2^-10 of the radius plus 2^-20 of the coordinates' magnitude —
// far more than the rounding of p ± r and of the photons' float distances —
// so every photon with d² < r2 lies in one of the cells.
struct CellSpan { int i0[3], i1[3]; };
RT_D CellSpan cell_span(const Map& M, float3 p, float r2) {
    float r = sqrtf(r2);
    float q[3] = {p.x, p.y, p.z};
    CellSpan s;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float m = r * (1.0f + 0x1p-10f) + (fabsf(q[a]) + r) * 0x1p-20f;
        s.i0[a] = grid_cell(q[a] - m, M.G.lo[a], M.G.inv, M.G.n[a]);
        s.i1[a] = grid_cell(q[a] + m, M.G.lo[a], M.G.inv, M.G.n[a]);
    }
    return s;
}
RT_D uint2 cell_run(const Map& M, int x, int y, int z) {
    return __ldg(M.cells + x + M.G.n[0] * (y + M.G.n[1] * z));
}
// photons in the cells of a span (an upper bound of the work of enumerating them)
RT_D uint32_t span_photons(const Map& M, const CellSpan& s) {
    uint32_t t = 0;
    for (int z = s.i0[2]; z <= s.i1[2]; z++)
        for (int y = s.i0[1]; y <= s.i1[1]; y++)
            for (int x = s.i0[0]; x <= s.i1[0]; x++) {
                uint2 r = cell_run(M, x, y, z);
                t += r.y - r.x;
            }
    return t;
}
// the grid serves balls no larger than the map's radius, while the cells hold
// at most this many photons (else the box heap prunes better)
#define PH_GRID_WARP_MAX 4096u

// Visit every leaf whose box is within r2 of p; for each, lane j gets photon j
// of the leaf (or nothing).  `f(lane_photon_index_or_-1)` is called warp-wide.
template <class F>
RT_D void for_leaves(const Map& M, float3 p, float r2, F f) {
    uint32_t stack[PH_STACK];
    int sp = 0;
    uint32_t node = 0;
    uint32_t lane = threadIdx.x & 31u;
    uint32_t first_leaf = M.nleaf_pow2 - 1;
    while (true) {
        float4 lo = __ldg(M.blo + node), hi = __ldg(M.bhi + node);
        bool near = box_d2(lo, hi, p) <= r2 && lo.x <= hi.x;
        if (near) {
            if (node >= first_leaf) {
                uint32_t k = (node - first_leaf) * PH_LEAF + lane;
                f(k < M.n ? (int)k : -1);
            } else if (sp + 2 <= PH_STACK) {
                stack[sp++] = 2 * node + 2;
                stack[sp++] = 2 * node + 1;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
}

// Every photon within r2 of p (and others), each once, warp-wide: from the grid
// cells the ball meets when the grid serves r2 and they hold at most
// PH_GRID_WARP_MAX photons, else from the heap's leaves.
template <class F>
RT_D void for_near(const Map& M, float3 p, float r2, F f) {
    if (r2 <= M.G.r2) {
        CellSpan s = cell_span(M, p, r2);
        if (span_photons(M, s) <= PH_GRID_WARP_MAX) {
            uint32_t lane = threadIdx.x & 31u;
            for (int z = s.i0[2]; z <= s.i1[2]; z++)
                for (int y = s.i0[1]; y <= s.i1[1]; y++)
                    for (int x = s.i0[0]; x <= s.i1[0]; x++) {
                        uint2 r = cell_run(M, x, y, z);
                        for (uint32_t b = r.x; b < r.y; b += 32) {
                            uint32_t k = b + lane;
                            f(k < r.y ? (int)k : -1);
                        }
                    }
            return;
        }
    }
    for_leaves(M, p, r2, f);
}

RT_D float warp_sum(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Squared distance and dot product with separately rounded products and sums
// (no fused multiply-add), so the values equal the oracle's bit for bit.
RT_D float pdist2(float4 q, float3 p) {
    float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}
RT_D float pdot(float4 a, float3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}

// Candidate test shared by every pass: d² in [lo, hi) (or [lo, hi]) and, when
// a normal is given, the photon faces it.
struct KthRange {
    float lo, hi;
    bool hi_inclusive;
    RT_D bool in(float d2) const { return d2 >= lo && (hi_inclusive ? d2 <= hi : d2 < hi); }
};

RT_D bool kth_candidate(const Map& M, int i, float3 p, const float3* nrm, const KthRange& R, float& d2) {
    if (i < 0) return false;
    d2 = pdist2(__ldg(M.pos + i), p);
    if (!R.in(d2)) return false;
    return !nrm || pdot(__ldg(M.nor + i), *nrm) > 0.0f;
}

// k-th smallest d² among photons with d² < r2max (strict) or ≤ r2max, [and
// n_p·n > 0 when `nrm` is given]; returns r2max when fewer than k exist.
// Histogram refinement: 32 bins per pass over the current range; a bin's
// edges are the same floats in the counting pass and the next pass's range
// test, so no candidate is lost or counted twice.  Once the bin holding the
// k-th has at most PH_SEL_CAP candidates they are selected exactly in shared
// memory; if the range stops shrinking (many equal distances) the remaining
// distinct values are peeled off smallest first.
RT_D float warp_kth_d2(const Map& M, float3 p, const float3* nrm, float r2max, uint32_t k, bool strict,
                       uint32_t* hist /*32*/, float* sel /*PH_SEL_CAP*/) {
    uint32_t lane = threadIdx.x & 31u;
    KthRange R{0.0f, r2max, !strict};
    uint32_t need = k;        // rank of the k-th within the range
    for (int pass = 0; pass < 8; pass++) {
        hist[lane] = 0;
        __syncwarp();
        float w = (R.hi - R.lo) / 32.0f;
        if (!(w > 0.0f)) break;
        // edge j = lo + w·j for j < 32, edge 32 = hi; bin = last edge ≤ d2
        float my_edge = R.lo + w * (float)lane;
        uint32_t total = 0;
        for_near(M, p, R.hi, [&](int i) {
            float d2 = 0.0f;
            bool c = kth_candidate(M, i, p, nrm, R, d2);
            if (c) {
                int bin = w > 0.0f ? min(max((int)((d2 - R.lo) / w), 0), 31) : 0;
                while (bin > 0 && d2 < R.lo + w * (float)bin) bin--;
                while (bin < 31 && d2 >= R.lo + w * (float)(bin + 1)) bin++;
                atomicAdd(&hist[bin], 1u);
            }
            total += __popc(__ballot_sync(0xFFFFFFFFu, c));
        });
        __syncwarp();
        if (total < need) return pass == 0 ? r2max : R.hi;   // fewer than k in the whole range
        if (total <= PH_SEL_CAP) {
            // exact select: collect the candidates of the range and rank them
            uint32_t cnt = 0;
            for_near(M, p, R.hi, [&](int i) {
                float d2 = 0.0f;
                bool c = kth_candidate(M, i, p, nrm, R, d2);
                uint32_t m = __ballot_sync(0xFFFFFFFFu, c);
                if (c) sel[cnt + __popc(m & ((1u << lane) - 1u))] = d2;
                cnt += __popc(m);
            });
            __syncwarp();
            float found = R.hi;
            for (uint32_t j = lane; j < cnt; j += 32) {
                float v = sel[j];
                uint32_t less = 0, eq_before = 0;
                for (uint32_t t = 0; t < cnt; t++) {
                    float u = sel[t];
                    less += u < v;
                    eq_before += (u == v && t < j);
                }
                if (less + eq_before == need - 1) found = v;
            }
            for (int o = 16; o > 0; o >>= 1) found = fminf(found, __shfl_xor_sync(0xFFFFFFFFu, found, o));
            __syncwarp();
            return found;
        }
        // narrow to the bin that holds the need-th candidate
        uint32_t cum = 0, b = 31;
        for (int j = 0; j < 32; j++) {
            uint32_t h = hist[j];
            if (cum + h >= need) { b = j; break; }
            cum += h;
        }
        __syncwarp();
        float nlo = __shfl_sync(0xFFFFFFFFu, my_edge, b);
        float nhi = b == 31 ? R.hi : __shfl_sync(0xFFFFFFFFu, my_edge, (b + 1) & 31);
        if (b == 0) nlo = R.lo;
        bool same = nlo == R.lo && nhi == R.hi;
        need -= cum;
        R.hi_inclusive = b == 31 ? R.hi_inclusive : false;
        R.lo = nlo;
        R.hi = nhi;
        if (same) break;
    }
    // peel distinct values, smallest first (bounded)
    for (int it = 0; it < 64; it++) {
        float mn = INFINITY;
        for_near(M, p, R.hi, [&](int i) {
            float d2 = 0.0f;
            if (kth_candidate(M, i, p, nrm, R, d2)) mn = fminf(mn, d2);
        });
        for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
        if (!(mn < INFINITY)) return R.hi;
        uint32_t eq = 0;
        for_near(M, p, R.hi, [&](int i) {
            float d2 = 0.0f;
            bool c = kth_candidate(M, i, p, nrm, R, d2) && d2 == mn;
            eq += __popc(__ballot_sync(0xFFFFFFFFu, c));
        });
        if (eq >= need) return mn;
        need -= eq;
        R.lo = nextafterf(mn, INFINITY);
    }
    return R.hi;
}

// Irradiance estimate at (p, n) by one warp (all lanes call with the same query).
RT_D float3 warp_irradiance(const Map& M, float3 p, float3 n, uint32_t* hist, float* sel) {
    float r2 = M.r2;
    if (M.knn_k > 0) {
        r2 = warp_kth_d2(M, p, &n, M.r2, M.knn_k, true, hist, sel);
        if (!(r2 > 0.0f)) return mk(0.f, 0.f, 0.f);
    }
    float3 acc = mk(0.f, 0.f, 0.f);
    for_near(M, p, r2, [&](int i) {
        if (i < 0) return;
        float d2 = pdist2(__ldg(M.pos + i), p);
        if (d2 < r2) {
            if (pdot(__ldg(M.nor + i), n) > 0.0f) {
                float4 pw = __ldg(M.pow + i);
                float wgt = 1.0f - d2 / r2;
                acc = acc + mk(pw.x, pw.y, pw.z) * wgt;
            }
        }
    });
    float s = 2.0f / (PI_F * PI_F * r2);
    return mk(warp_sum(acc.x) * s, warp_sum(acc.y) * s, warp_sum(acc.z) * s);
}

// Shared-memory workspace of one warp for the single-pass k-NN gather.
#define PH_CAND_CAP 512
struct WarpScratch {
    float d2[PH_CAND_CAP];
    uint32_t id[PH_CAND_CAP];
    uint32_t hist[256];
};

// k-th smallest (1-based) of the cnt ≥ k non-negative floats v[] by a 4-pass
// radix select on their bits (non-negative floats order as unsigned integers),
// one warp, exact.
RT_D float warp_radix_select(const float* v, uint32_t cnt, uint32_t k, uint32_t* hist) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t prefix = 0, mask = 0, need = k;
#pragma unroll 1
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = lane; b < 256; b += 32) hist[b] = 0;
        __syncwarp();
        for (uint32_t j = lane; j < cnt; j += 32) {
            uint32_t key = __float_as_uint(v[j]);
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncwarp();
        // lane l owns bins 8l .. 8l + 7; an exclusive scan over the lanes finds the
        // bin holding the need-th key
        uint32_t h[8], tot = 0;
#pragma unroll
        for (int b = 0; b < 8; b++) { h[b] = hist[lane * 8 + b]; tot += h[b]; }
        uint32_t inc = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t x = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if (lane >= (uint32_t)o) inc += x;
        }
        uint32_t exc = inc - tot;
        bool mine = exc < need && need <= inc;
        uint32_t digit = 0, before = 0;
        if (mine) {
            uint32_t c = exc;
#pragma unroll
            for (int b = 0; b < 8; b++) {
                if (c + h[b] >= need) { digit = lane * 8 + b; before = c; break; }
                c += h[b];
            }
        }
        uint32_t who = __ffs(__ballot_sync(0xFFFFFFFFu, mine)) - 1;
        digit = __shfl_sync(0xFFFFFFFFu, digit, who);
        before = __shfl_sync(0xFFFFFFFFu, before, who);
        need -= before;
        prefix |= digit << shift;
        mask |= 255u << shift;
        __syncwarp();
    }
    return __uint_as_float(prefix);
}

// Irradiance at (p, n) by one warp in one traversal: the photons within the
// gather radius that face n are collected into shared memory, the k-th
// smallest d² is selected there (k-NN mode), and the Epanechnikov sum runs
// over the collected photons.  More candidates than PH_CAND_CAP: the
// histogram-refinement path (warp_irradiance) instead.  Same estimate as
// warp_irradiance; the terms are summed in another order.
// An upper bound of the k-NN search's k-th distance: descend the box heap
// toward p (the nearer child at every level) to a subtree of PH_SEED_LEAVES
// leaves, and take the k-th smallest d² of its facing photons (the maximum
// radius's r2 when it holds fewer than k or that is nearer).  The true k
// nearest are at least as near, so every one of them lies within the bound.
#define PH_SEED_LEAVES 4
RT_D float seed_bound(const Map& M, float3 p, float3 n, WarpScratch& W) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t node = 0, pos = 0, span = M.nleaf_pow2;
    while (span > PH_SEED_LEAVES) {
        uint32_t l = 2 * node + 1, r = l + 1;
        float dl = box_d2(__ldg(M.blo + l), __ldg(M.bhi + l), p), dr = box_d2(__ldg(M.blo + r), __ldg(M.bhi + r), p);
        bool right = dr < dl;
        node = right ? r : l;
        pos = 2 * pos + (right ? 1u : 0u);
        span >>= 1;
    }
    uint32_t first = pos * span * PH_LEAF, last = min(first + span * PH_LEAF, M.n);
    uint32_t c = 0;
    for (uint32_t i = first + lane; i < first + span * PH_LEAF; i += 32) {
        float d2 = INFINITY;
        if (i < last) {
            float v = pdist2(__ldg(M.pos + i), p);
            if (pdot(__ldg(M.nor + i), n) > 0.0f) d2 = v;
        }
        W.d2[i - first] = d2;
        c += d2 < INFINITY;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    __syncwarp();
    if (c < M.knn_k) return M.r2;
    return fminf(warp_radix_select(W.d2, span * PH_LEAF, M.knn_k, W.hist), M.r2);
}

RT_D float3 warp_irradiance_1pass(const Map& M, float3 p, float3 n, WarpScratch& W, uint32_t* hist, float* sel) {
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
    // the ball to collect: within the maximum radius and, in k-NN mode, within
    // the seed subtree's k-th distance (inclusive, so ties at it are kept)
    // (the grid's cells hold a few times the photons in range: no seed there)
    bool grid = M.r2 <= M.G.r2 && span_photons(M, cell_span(M, p, M.r2)) <= PH_GRID_WARP_MAX;
    float bound = !grid && M.knn_k > 0 && M.knn_k <= PH_SEED_LEAVES * PH_LEAF ? seed_bound(M, p, n, W) : M.r2;
    uint32_t cnt = 0;
    for_near(M, p, bound, [&](int i) {
        bool c = false;
        float d2 = 0.0f;
        if (i >= 0) {
            d2 = pdist2(__ldg(M.pos + i), p);
            c = d2 < M.r2 && d2 <= bound && pdot(__ldg(M.nor + i), n) > 0.0f;
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, c);
        uint32_t slot = cnt + __popc(m & lt);
        if (c && slot < PH_CAND_CAP) { W.d2[slot] = d2; W.id[slot] = (uint32_t)i; }
        cnt += __popc(m);
    });
    __syncwarp();
    if (cnt > PH_CAND_CAP) return warp_irradiance(M, p, n, hist, sel);
    float r2 = M.r2;
    if (M.knn_k > 0 && cnt >= M.knn_k) {
        r2 = warp_radix_select(W.d2, cnt, M.knn_k, W.hist);
        if (!(r2 > 0.0f)) return mk(0.f, 0.f, 0.f);
    }
    float3 acc = mk(0.f, 0.f, 0.f);
    for (uint32_t j = lane; j < cnt; j += 32) {
        float d2 = W.d2[j];
        if (d2 < r2) {
            float4 pw = __ldg(M.pow + W.id[j]);
            acc = acc + mk(pw.x, pw.y, pw.z) * (1.0f - d2 / r2);
        }
    }
    __syncwarp();
    float s = 2.0f / (PI_F * PI_F * r2);
    return mk(warp_sum(acc.x) * s, warp_sum(acc.y) * s, warp_sum(acc.z) * s);
}

// Irradiance at (p, n) by one warp from the grid: the ≤ 2 × 2 × 2 cells the
// ball of the map's radius meets are read by lanes 0-7, their runs are joined
// into one list (an inclusive scan of the lengths), and lane j tests entries
// j, j + 32, … of the list — every load coalesced, no lane idle while another
// works through a longer cell.  The facing photons within the radius go to
// shared memory; in k-NN mode with more than k of them the k-th d² is selected
// there.  Spans of more cells, crowded cells and maps without a grid take
// warp_irradiance_1pass.  Same estimate as warp_irradiance; the terms are
// summed in another order.
RT_D float3 warp_gather(const Map& M, float3 p, float3 n, WarpScratch& W, uint32_t* hist, float* sel) {
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
    if (!(M.r2 <= M.G.r2)) return warp_irradiance_1pass(M, p, n, W, hist, sel);
    CellSpan s = cell_span(M, p, M.r2);
    if (s.i1[0] - s.i0[0] > 1 || s.i1[1] - s.i0[1] > 1 || s.i1[2] - s.i0[2] > 1)
        return warp_irradiance_1pass(M, p, n, W, hist, sel);
    uint32_t st = 0, len = 0;
    if (lane < 8) {
        int x = s.i0[0] + (int)(lane & 1u), y = s.i0[1] + (int)((lane >> 1) & 1u), z = s.i0[2] + (int)(lane >> 2);
        if (x <= s.i1[0] && y <= s.i1[1] && z <= s.i1[2]) {
            uint2 r = cell_run(M, x, y, z);
            st = r.x;
            len = r.y - r.x;
        }
    }
    uint32_t inc = len;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= (uint32_t)o) inc += v;
    }
    const uint32_t T = __shfl_sync(0xFFFFFFFFu, inc, 7);
    if (T > PH_GRID_WARP_MAX) return warp_irradiance_1pass(M, p, n, W, hist, sel);
    uint32_t ex[8], sv[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
        ex[r] = __shfl_sync(0xFFFFFFFFu, inc - len, r);
        sv[r] = __shfl_sync(0xFFFFFFFFu, st, r);
    }
    uint32_t cnt = 0;
    // the radius-r_max sum, gathered in the same pass: the estimate whenever
    // fewer than k photons are in range (and always in radius mode)
    float3 acc0 = mk(0.f, 0.f, 0.f);
    for (uint32_t base = 0; base < T; base += 32) {
        uint32_t f = base + lane;
        bool c = false;
        float d2 = 0.0f;
        uint32_t k = 0;
        if (f < T) {
            // the run holding entry f: the last one starting at or before it
            // (an empty run starts where the next begins and is passed over)
            uint32_t e0 = ex[0], s0 = sv[0];
#pragma unroll
            for (int r = 1; r < 8; r++)
                if (ex[r] <= f) { e0 = ex[r]; s0 = sv[r]; }
            k = s0 + (f - e0);
            // position, normal and power in one round trip (the map is L2-resident)
            float4 q = __ldg(M.pos + k), nv = __ldg(M.nor + k), pw = __ldg(M.pow + k);
            d2 = pdist2(q, p);
            c = d2 < M.r2 && pdot(nv, n) > 0.0f;
            if (c) acc0 = acc0 + mk(pw.x, pw.y, pw.z) * (1.0f - d2 / M.r2);
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, c);
        uint32_t slot = cnt + __popc(m & lt);
        if (c && slot < PH_CAND_CAP) { W.d2[slot] = d2; W.id[slot] = k; }
        cnt += __popc(m);
    }
    __syncwarp();
    if (cnt > PH_CAND_CAP) return warp_irradiance(M, p, n, hist, sel);
    float r2 = M.r2;
    if (!(M.knn_k > 0 && cnt >= M.knn_k)) {
        float sc = 2.0f / (PI_F * PI_F * r2);
        return mk(warp_sum(acc0.x) * sc, warp_sum(acc0.y) * sc, warp_sum(acc0.z) * sc);
    }
    r2 = warp_radix_select(W.d2, cnt, M.knn_k, W.hist);
    if (!(r2 > 0.0f)) return mk(0.f, 0.f, 0.f);
    float3 acc = mk(0.f, 0.f, 0.f);
    for (uint32_t j = lane; j < cnt; j += 32) {
        float d2 = W.d2[j];
        if (d2 < r2) {
            float4 pw = __ldg(M.pow + W.id[j]);
            acc = acc + mk(pw.x, pw.y, pw.z) * (1.0f - d2 / r2);
        }
    }
    __syncwarp();
    float sc = 2.0f / (PI_F * PI_F * r2);
    return mk(warp_sum(acc.x) * sc, warp_sum(acc.y) * sc, warp_sum(acc.z) * sc);
}

}  // namespace rtph

// queries n × 6 → irradiance n × 3; one warp per query
__global__ void k_photon_gather_api(rtph::Map M, const float* q, uint32_t n, float* out) {
    __shared__ uint32_t hist[RT_SHADE_BLOCK / 32][32];
    __shared__ float sel[RT_SHADE_BLOCK / 32][PH_SEL_CAP];
    __shared__ rtph::WarpScratch ws[RT_SHADE_BLOCK / 32];
    uint32_t w = threadIdx.x >> 5, gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = gw; i < n; i += nw) {
        float3 p = mk(q[i * 6], q[i * 6 + 1], q[i * 6 + 2]), nn = mk(q[i * 6 + 3], q[i * 6 + 4], q[i * 6 + 5]);
        float3 r = rtph::warp_gather(M, p, nn, ws[w], hist[w], sel[w]);
        if ((threadIdx.x & 31u) == 0) { out[i * 3] = r.x; out[i * 3 + 1] = r.y; out[i * 3 + 2] = r.z; }
    }
}

// exact k nearest with d² ≤ rmax², sorted by (d², emission index)
__global__ void k_knn_api(rtph::Map M, const float* q, uint32_t n, int k, float rmax2, int* out_idx, float* out_d2,
                          int* err) {
    __shared__ uint32_t hist[RT_SHADE_BLOCK / 32][32];
    __shared__ float sel[RT_SHADE_BLOCK / 32][PH_SEL_CAP];
    __shared__ uint32_t cid[RT_SHADE_BLOCK / 32][PH_SEL_CAP];
    __shared__ float cd2[RT_SHADE_BLOCK / 32][PH_SEL_CAP];
    uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = gw; i < n; i += nw) {
        float3 p = mk(q[i * 3], q[i * 3 + 1], q[i * 3 + 2]);
        float rk = rtph::warp_kth_d2(M, p, nullptr, rmax2, (uint32_t)k, false, hist[w], sel[w]);
        // every photon with d² ≤ r_k² (k plus ties at r_k)
        uint32_t cnt = 0;
        rtph::for_near(M, p, rk, [&](int j) {
            bool c = false;
            float d2 = 0.0f;
            uint32_t id = 0;
            if (j >= 0) {
                float4 qq = __ldg(M.pos + j);
                d2 = rtph::pdist2(qq, p);
                c = d2 <= rk;
                id = __float_as_uint(qq.w);
            }
            uint32_t m = __ballot_sync(0xFFFFFFFFu, c);
            uint32_t slot = cnt + __popc(m & ((1u << lane) - 1u));
            if (c && slot < PH_SEL_CAP) { cid[w][slot] = id; cd2[w][slot] = d2; }
            cnt += __popc(m);
        });
        __syncwarp();
        if (cnt > PH_SEL_CAP) { if (lane == 0) atomicExch(err, RT_ERR_CAPACITY); cnt = PH_SEL_CAP; }
        // rank sort by (d², index)
        for (uint32_t j = lane; j < cnt; j += 32) {
            float v = cd2[w][j];
            uint32_t id = cid[w][j], r = 0;
            for (uint32_t t = 0; t < cnt; t++) {
                float u = cd2[w][t];
                r += (u < v) || (u == v && cid[w][t] < id);
            }
            if (r < (uint32_t)k) { out_idx[(size_t)i * k + r] = (int)id; out_d2[(size_t)i * k + r] = v; }
        }
        for (uint32_t r = cnt + lane; r < (uint32_t)k; r += 32) {
            out_idx[(size_t)i * k + r] = -1;
            out_d2[(size_t)i * k + r] = INFINITY;
        }
        __syncwarp();
    }
}

// render path: caustic injection at queued diffuse vertices (renderer.rs:461-467);
// pendC[pid] holds T·tint·albedo and becomes that × irradiance
__global__ void __launch_bounds__(RT_SHADE_BLOCK) k_photon_gather_paths(rtph::Map M, PendTargets T,
                                                                        const float4* __restrict__ gq,
                                                                        const uint32_t* count) {
    __shared__ uint32_t hist[RT_SHADE_BLOCK / 32][32];
    __shared__ float sel[RT_SHADE_BLOCK / 32][PH_SEL_CAP];
    __shared__ rtph::WarpScratch ws[RT_SHADE_BLOCK / 32];
    uint32_t n = *count;
    uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    // one warp per request (its cells' photons are few, and coalesced); the
    // next request is loaded while this one is gathered
    float4 na = make_float4(0.f, 0.f, 0.f, 0.f), nb = na;
    if (gw < n) { na = gq[(size_t)gw * 2]; nb = gq[(size_t)gw * 2 + 1]; }
    for (uint32_t i = gw; i < n; i += nw) {
        float4 qa = na, qb = nb;
        if (i + nw < n) { na = gq[(size_t)(i + nw) * 2]; nb = gq[(size_t)(i + nw) * 2 + 1]; }
        float3 r = rtph::warp_gather(M, mk(qa.x, qa.y, qa.z), mk(qb.x, qb.y, qb.z), ws[w], hist[w], sel[w]);
        if (lane == 0) {
            uint32_t tag = __float_as_uint(qa.w);
            float4* pc = T.pendC[(tag >> 1) & 1u] + (tag >> 2);
            float4 f = *pc;
            bool any = r.x > 0.0f || r.y > 0.0f || r.z > 0.0f;
            *pc = any ? make_float4(f.x * r.x, f.y * r.y, f.z * r.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

// ── host side ───────────────────────────────────────────────────────────────
PhotonMapDev::~PhotonMapDev() { free_all(); }
void PhotonMapDev::release() {
    n = 0;
    present = false;
    generation++;
    grid = PhotonGrid{{0.f, 0.f, 0.f}, 0.f, {1, 1, 1}, -1.f};
}
void PhotonMapDev::free_all() {
    void* ps[] = {pos, pow, nor, blo, bhi, exp_pos, exp_pow, exp_nor, flags, st_pos, st_pow, st_nor,
                  fl32, scan, key, val, key2, val2, bounds, tmp, cells};
    for (void* p : ps) if (p) cudaFree(p);
    pos = pow = nor = blo = bhi = exp_pos = exp_pow = exp_nor = st_pos = st_pow = st_nor = nullptr;
    flags = nullptr;
    fl32 = scan = val = val2 = nullptr;
    key = key2 = nullptr;
    bounds = nullptr;
    tmp = nullptr;
    cells = nullptr;
    cap_map = cap_heap = cap_cells = cap_work = cap_tmp = 0;
    release();
}

rtph::Map PhotonMapDev::view() const {
    rtph::Map M;
    M.pos = pos; M.pow = pow; M.nor = nor; M.blo = blo; M.bhi = bhi;
    M.cells = cells; M.G = grid;
    M.n = n; M.nleaf_pow2 = nleaf_pow2; M.r2 = r2; M.knn_k = knn_k;
    return M;
}


namespace rth {

// grow a device array to at least `n` elements of `bytes` (contents not kept)
template <class T>
static cudaError_t grow(T*& p, size_t n, size_t bytes) {
    if (p) cudaFree(p);
    p = nullptr;
    return cudaMalloc((void**)&p, std::max<size_t>(n, 1) * bytes);
}

// map arrays (emission-order copy, Morton-ordered copy, sort keys) for n photons
static cudaError_t ensure_map(PhotonMapDev& map, size_t n) {
    if (n <= map.cap_map && map.pos) return cudaSuccess;
    size_t c = std::max<size_t>(n, map.cap_map * 5 / 4);
    cudaError_t e;
    float4** f4[] = {&map.pos, &map.pow, &map.nor, &map.exp_pos, &map.exp_pow, &map.exp_nor};
    for (float4** q : f4) if ((e = grow(*q, c, sizeof(float4)))) return e;
    uint32_t** u4[] = {&map.val, &map.val2};
    for (uint32_t** q : u4) if ((e = grow(*q, c, sizeof(uint32_t)))) return e;
    if ((e = grow(map.key, c, sizeof(uint64_t))) || (e = grow(map.key2, c, sizeof(uint64_t)))) return e;
    if (!map.bounds && (e = grow(map.bounds, 6, sizeof(float)))) return e;
    map.cap_map = c;
    return cudaSuccess;
}

static cudaError_t ensure_tmp(PhotonMapDev& map, size_t bytes) {
    if (bytes <= map.cap_tmp && map.tmp) return cudaSuccess;
    size_t c = std::max<size_t>(bytes, map.cap_tmp * 5 / 4);
    cudaError_t e = grow(map.tmp, c, 1);
    if (!e) map.cap_tmp = c;
    return e;
}

// The cell grid for photons in the box [lo, hi] and gather radius² r2: cubic
// cells of 2r·(1 + 2^-9) — a ball of radius r (widened as cell_span widens it)
// meets at most 2 cells per axis — or larger, to keep ≤ 1000 cells per axis
// and ≤ RT_PH_GRID_MAX_CELLS cells in all.  No grid (one cell, r2 < 0) for a
// zero radius.
static PhotonGrid make_grid(const float lo[3], const float hi[3], float r2) {
    PhotonGrid G{{lo[0], lo[1], lo[2]}, 0.0f, {1, 1, 1}, -1.0f};
    if (!(r2 > 0.0f) || !std::isfinite(r2)) return G;
    double ext = 0.0;
    for (int a = 0; a < 3; a++) ext = std::max(ext, (double)hi[a] - (double)lo[a]);
    double c = std::max(2.0 * std::sqrt((double)r2) * (1.0 + 1.0 / 512.0), ext / 1000.0);
    if (!(c > 0.0)) return G;
    for (;;) {
        double cells = 1.0;
        for (int a = 0; a < 3; a++) {
            double na = std::floor(((double)hi[a] - (double)lo[a]) / c) + 1.0;
            G.n[a] = (int)std::min(na, 1024.0);
            cells *= G.n[a];
        }
        if (cells <= RT_PH_GRID_MAX_CELLS) break;
        c *= 1.25;
    }
    G.inv = (float)(1.0 / c);
    G.r2 = r2;
    return G;
}

// Sort the emission-order photons (exp_*, n of them) by (grid cell, Morton
// code) into pos/pow/nor, then the cell table and the box heap over
// PH_LEAF-photon leaves
static cudaError_t build_tree(PhotonMapDev& map, uint32_t n, cudaStream_t st) {
    cudaError_t e;
    float init[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    if ((e = cudaMemcpyAsync(map.bounds, init, sizeof(init), cudaMemcpyHostToDevice, st))) return e;
    k_bounds<<<std::min<uint32_t>((n + 255) / 256, 2048), 256, 0, st>>>(map.exp_pos, n, map.bounds, map.bounds + 3);
    float b[6];
    if ((e = cudaMemcpyAsync(b, map.bounds, sizeof(b), cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    map.grid = make_grid(b, b + 3, map.r2);
    size_t ncell = (size_t)map.grid.n[0] * map.grid.n[1] * map.grid.n[2];
    if (ncell > map.cap_cells || !map.cells) {
        if ((e = grow(map.cells, ncell, sizeof(uint2)))) return e;
        map.cap_cells = ncell;
    }
    if ((e = cudaMemsetAsync(map.cells, 0, ncell * sizeof(uint2), st))) return e;
    k_morton<<<std::min<uint32_t>((n + 255) / 256, 4096), 256, 0, st>>>(map.exp_pos, n, map.bounds, map.bounds + 3,
                                                                        map.grid, map.key, map.val);
    // stable radix sort: emission order among equal keys
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, map.key, map.key2, map.val, map.val2, (int)n, 0, 60, st);
    if ((e = ensure_tmp(map, tb))) return e;
    cub::DeviceRadixSort::SortPairs(map.tmp, tb, map.key, map.key2, map.val, map.val2, (int)n, 0, 60, st);
    uint32_t nleaf = (n + PH_LEAF - 1) / PH_LEAF, p2 = 1;
    while (p2 < nleaf) p2 <<= 1;
    map.nleaf_pow2 = p2;
    if ((size_t)(2 * p2 - 1) > map.cap_heap || !map.blo) {
        size_t c = 2 * (size_t)p2 - 1;
        if ((e = grow(map.blo, c, sizeof(float4))) || (e = grow(map.bhi, c, sizeof(float4)))) return e;
        map.cap_heap = c;
    }
    k_gather_sorted<<<std::min<uint32_t>((n + 255) / 256, 4096), 256, 0, st>>>(map.val2, n, map.exp_pos, map.exp_pow,
                                                                               map.exp_nor, map.pos, map.pow, map.nor);
    k_cell_ranges<<<std::min<uint32_t>((n + 255) / 256, 4096), 256, 0, st>>>(map.pos, n, map.grid, map.cells);
    k_leaf_boxes<<<std::min<uint32_t>((p2 + 255) / 256, 4096), 256, 0, st>>>(map.pos, n, p2, map.blo, map.bhi);
    for (uint32_t cnt = p2 / 2; cnt >= 1; cnt /= 2)
        k_level_boxes<<<std::min<uint32_t>((cnt + 255) / 256, 4096), 256, 0, st>>>(cnt - 1, cnt, map.blo, map.bhi);
    return cudaGetLastError();
}

cudaError_t photon_build(const DevScene& S, PhotonMapDev& map, const PathState& P, uint32_t* qa, uint32_t* qb,
                         uint32_t* counters, const RtPhotonParams& prm, const float* emit_setup, uint32_t first,
                         uint32_t count, int sms, cudaStream_t st, int64_t* n_stored, float stage_ms[3]) {
    map.release();
    EmitSet E{};
    E.n = prm.n_emitters;
    E.lam_lo = S.lam_lo;
    E.lam_range = S.lam_range;
    E.seed = prm.seed;
    uint32_t off = 0;
    for (int i = 0; i < prm.n_emitters; i++) {
        const float* f = emit_setup + i * 40;
        EmitSetup& x = E.e[i];
        int ty = prm.emitters[i].type;
        x.type = (ty == RT_EMIT_QUAD || ty == RT_EMIT_LIGHT) ? RT_EMIT_QUAD : RT_EMIT_DISK;   // the sun is a disk source
        x.t = mk(f[0], f[1], f[2]); x.b = mk(f[3], f[4], f[5]); x.center = mk(f[6], f[7], f[8]);
        x.dir = mk(f[9], f[10], f[11]); x.normal = mk(f[12], f[13], f[14]); x.corner = mk(f[15], f[16], f[17]);
        x.u = mk(f[18], f[19], f[20]); x.v = mk(f[21], f[22], f[23]); x.ta = mk(f[24], f[25], f[26]);
        x.ba = mk(f[27], f[28], f[29]); x.power = mk(f[30], f[31], f[32]);
        x.radius = f[33]; x.lum_clamp = f[34];
        x.target = mk(f[35], f[36], f[37]); x.target_r = f[38];
        x.first = off; x.count = prm.emitters[i].n_photons;
        off += x.count;
    }
    const uint32_t total = count;          // photons traced by this build (slots 0 .. total − 1)
    cudaError_t e;
    if (total > map.cap_work || !map.flags) {
        size_t c = std::max<size_t>(total, map.cap_work * 5 / 4);
        if ((e = grow(map.flags, c, 1)) || (e = grow(map.st_pos, c, sizeof(float4))) ||
            (e = grow(map.st_pow, c, sizeof(float4))) || (e = grow(map.st_nor, c, sizeof(float4))) ||
            (e = grow(map.fl32, c, sizeof(uint32_t))) || (e = grow(map.scan, c, sizeof(uint32_t))))
            return e;
        map.cap_work = c;
    }
    cudaEvent_t ev[4];
    for (auto& x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0], st);
    cudaMemsetAsync(counters, 0, sizeof(uint32_t) * 14 * RT_CTR_STRIDE, st);
    int grid = std::min<uint32_t>((total + 255) / 256, 148u * 16u);
    k_photon_emit<<<std::max(grid, 1), 256, 0, st>>>(P, E, first, total, qa, counters, map.flags);
    uint32_t* q[2] = {qa, qb};
    for (uint32_t b = 0; b < 12; b++) {
        uint32_t* c = counters + b * RT_CTR_STRIDE;
        uint32_t* cn = counters + (b + 1) * RT_CTR_STRIDE;
        launch_extend(S, P, q[b & 1], c + CTR_COUNT, c + CTR_EXTEND_NEXT, (int*)(counters + 13 * RT_CTR_STRIDE), sms, st);
        if (S.n_media > 0) launch_media(S, P, q[b & 1], c + CTR_COUNT, sms, st);
        k_photon_shade<<<sms * 8, 128, 0, st>>>(S, P, b, q[b & 1], c + CTR_COUNT, q[(b + 1) & 1], cn + CTR_COUNT,
                                                map.st_pos, map.st_pow, map.st_nor, map.flags, prm.seed);
    }
    cudaEventRecord(ev[1], st);
    // compact in emission order
    k_flags_to_u32<<<std::max(grid, 1), 256, 0, st>>>(map.flags, map.fl32, total);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, map.fl32, map.scan, (int)total, st);
    if ((e = ensure_tmp(map, tb))) return e;
    cub::DeviceScan::ExclusiveSum(map.tmp, tb, map.fl32, map.scan, (int)total, st);
    uint32_t last[2] = {0, 0};
    if (total) {
        cudaMemcpyAsync(&last[0], map.scan + total - 1, 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&last[1], map.fl32 + total - 1, 4, cudaMemcpyDeviceToHost, st);
    }
    if ((e = cudaStreamSynchronize(st))) return e;
    uint32_t n = total ? last[0] + last[1] : 0;
    if ((e = ensure_map(map, n))) return e;
    k_compact<<<std::max(grid, 1), 256, 0, st>>>(map.flags, map.scan, total, map.st_pos, map.st_pow, map.st_nor,
                                                 map.exp_pos, map.exp_pow, map.exp_nor);
    cudaEventRecord(ev[2], st);
    map.n = n;
    map.r2 = prm.gather_radius * prm.gather_radius;
    map.knn_k = prm.knn_k;
    if (n_stored) *n_stored = n;
    e = n ? build_tree(map, n, st) : cudaSuccess;
    cudaEventRecord(ev[3], st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (stage_ms)
        for (int k = 0; k < 3; k++) cudaEventElapsedTime(&stage_ms[k], ev[k], ev[k + 1]);
    for (auto& x : ev) cudaEventDestroy(x);
    if (e || e2) return e ? e : e2;
    map.present = true;
    return cudaSuccess;
}

cudaError_t photon_set(PhotonMapDev& map, const float4* cp, const float4* cw, const float4* cn, uint32_t n, float radius,
                       uint32_t k, cudaStream_t st) {
    map.release();
    cudaError_t e = ensure_map(map, n);
    if (e) return e;
    cudaMemcpyAsync(map.exp_pos, cp, (size_t)n * 16, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(map.exp_pow, cw, (size_t)n * 16, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(map.exp_nor, cn, (size_t)n * 16, cudaMemcpyHostToDevice, st);
    map.n = n;
    map.r2 = radius * radius;
    map.knn_k = k;
    if (n && (e = build_tree(map, n, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    map.present = true;
    return cudaSuccess;
}

void launch_photon_gather_api(const PhotonMapDev& map, const float* q, uint32_t n, float* out, int sms, cudaStream_t st) {
    k_photon_gather_api<<<sms * 4, RT_SHADE_BLOCK, 0, st>>>(map.view(), q, n, out);
}
void launch_knn_api(const PhotonMapDev& map, const float* q, uint32_t n, int k, float rmax2, int* idx, float* d2,
                    int* err, int sms, cudaStream_t st) {
    k_knn_api<<<sms * 4, RT_SHADE_BLOCK, 0, st>>>(map.view(), q, n, k, rmax2, idx, d2, err);
}
void launch_photon_gather_paths(const PhotonMapDev& map, const PendTargets& T, const float4* gq, const uint32_t* count,
                                int sms, cudaStream_t st) {
    k_photon_gather_paths<<<sms * 8, RT_SHADE_BLOCK, 0, st>>>(map.view(), T, gq, count);
}

}  // namespace rth
