// rt_texture.cuh — texture coordinates and texture lookups on the device
// (texture.rs, material.rs:633-786, triangle.rs:91-107, quad.rs:53-56,
// sphere.rs:11-15).  The CPU oracle restates the same functions
// (oracle/rt_oracle.cpp).
#pragma once
#include "rt_device.cuh"
#include "rt_media.cuh"
#include "rt_ggx.cuh"

namespace rtd {

struct HitUV { float u, v; float3 tan; };   // tan = 0 where the reference has no tangent

// (u, v) and tangent of a hit; `outward` is the unflipped (shading) normal
RT_D HitUV hit_uv(const DevScene& S, float4 hv, float3 outward) {
    HitUV r;
    r.u = 0.0f; r.v = 0.0f; r.tan = mk(0.f, 0.f, 0.f);
    uint32_t ref = __float_as_uint(hv.x), type = RT_HIT_TYPE(ref), idx = RT_HIT_INDEX(ref);
    if (type == RT_PRIM_TRI) {                                                      // triangle.rs:91-107
        float b1 = hv.z, b2 = hv.w, b0 = 1.0f - b1 - b2;
        float3 t0 = mk(1.f, 0.f, 0.f), t1 = t0, t2 = t0;
        if (S.tri_uv) {
            float4 a = __ldg(S.tri_uv + (size_t)idx * 2), b = __ldg(S.tri_uv + (size_t)idx * 2 + 1);
            r.u = b0 * a.x + b1 * a.z + b2 * b.x;
            r.v = b0 * a.y + b1 * a.w + b2 * b.y;
            float4 g0 = __ldg(S.tri_tan + (size_t)idx * 3), g1 = __ldg(S.tri_tan + (size_t)idx * 3 + 1),
                   g2 = __ldg(S.tri_tan + (size_t)idx * 3 + 2);
            t0 = mk(g0.x, g0.y, g0.z); t1 = mk(g0.w, g1.x, g1.y); t2 = mk(g1.z, g1.w, g2.x);
        } else {                                                                    // mesh.rs:75-77 defaults
            r.u = b0 * 0.0f + b1 * 1.0f + b2 * 0.5f;
            r.v = b0 * 0.0f + b1 * 0.0f + b2 * 1.0f;
        }
        float3 rt = b0 * t0 + b1 * t1 + b2 * t2;
        rt = rt - outward * dot3(rt, outward);
        if (len2(rt) > 1e-8f) {
            r.tan = unit3(rt);
        } else {
            float3 up = fabsf(outward.y) < 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);   // vec3.rs:37-42
            r.tan = unit3(cross3(outward, up));
        }
    } else if (type == RT_PRIM_QUAD) {                                              // quad.rs:53-56
        r.u = hv.z; r.v = hv.w;
    } else if (type == RT_PRIM_SPHERE) {                                            // sphere.rs:11-15
        float theta = acosf(clampf_(-outward.y, -1.0f, 1.0f));
        float phi = atan2f(-outward.z, outward.x) + PI_F;
        r.u = phi / (2.0f * PI_F);
        r.v = theta / PI_F;
    }
    return r;
}

// Texture::value for a Lambertian albedo (texture.rs:25-57): the nearest
// texel sRGB-decoded, or the Perlin mottle
RT_D float3 tex_value(const DevScene& S, int id, float u, float v, float3 p) {
    const DevTexture& t = S.tex[id - 1];
    if (t.type == RT_TEX_MOTTLE) {
        float acc = 0.0f, wgt = 1.0f;
        float3 q = mk(p.x * t.scale, p.y * t.scale, p.z * t.scale);
        for (int i = 0; i < 7; i++) {                                               // perlin.rs:61-71
            acc += wgt * perlin_noise(t.vec, t.perm, q);
            wgt *= 0.5f;
            q = mk(q.x * 2.0f, q.y * 2.0f, q.z * 2.0f);
        }
        float m = clampf_(2.0f * fabsf(acc), 0.0f, 1.0f);
        return t.lo * (1.0f - m) + t.hi * m;
    }
    float uu = clampf_(u, 0.0f, 1.0f), vv = 1.0f - clampf_(v, 0.0f, 1.0f);
    uint32_t x = min((uint32_t)(uu * (float)t.w), (uint32_t)t.w - 1u);
    uint32_t y = min((uint32_t)(vv * (float)t.h), (uint32_t)t.h - 1u);
    const uint8_t* q = t.px + ((size_t)y * t.w + x) * 3;
    return mk(__ldg(S.srgb_lut + q[0]), __ldg(S.srgb_lut + q[1]), __ldg(S.srgb_lut + q[2]));
}

// bilinear_coords (material.rs:633-646) and the three PBR samplers (:648-671);
// mode 0 sRGB colour, 1 raw colour / 255, 2 red channel / 255
RT_D float3 tex_bilinear(const DevScene& S, int id, float u, float v, int mode) {
    const DevTexture& t = S.tex[id - 1];
    float uu = clampf_(u, 0.0f, 1.0f), vv = 1.0f - clampf_(v, 0.0f, 1.0f);
    float fx = clampf_(uu * (float)t.w - 0.5f, 0.0f, (float)(t.w - 1));
    float fy = clampf_(vv * (float)t.h - 0.5f, 0.0f, (float)(t.h - 1));
    uint32_t x0 = (uint32_t)fx, y0 = (uint32_t)fy;
    uint32_t x1 = min(x0 + 1u, (uint32_t)t.w - 1u), y1 = min(y0 + 1u, (uint32_t)t.h - 1u);
    float tx = fx - (float)x0, ty = fy - (float)y0;
    auto px = [&](uint32_t x, uint32_t y) {
        const uint8_t* q = t.px + ((size_t)y * t.w + x) * 3;
        if (mode == 0) return mk(__ldg(S.srgb_lut + q[0]), __ldg(S.srgb_lut + q[1]), __ldg(S.srgb_lut + q[2]));
        if (mode == 1) return mk((float)q[0] / 255.0f, (float)q[1] / 255.0f, (float)q[2] / 255.0f);
        float r = (float)q[0] / 255.0f;
        return mk(r, r, r);
    };
    float3 c0 = px(x0, y0) * (1.0f - tx) + px(x1, y0) * tx;
    float3 c1 = px(x0, y1) * (1.0f - tx) + px(x1, y1) * tx;
    return c0 * (1.0f - ty) + c1 * ty;
}

// PbrMaterial::params (material.rs:758-786): the maps override the scalars;
// the albedo is multiplied by the ambient-occlusion map.  *sn receives the
// normal-mapped shading normal (tbn_normal: the face-forward normal `n` and
// the hit's tangent; a (0.5, 0.5, 0.5) texel keeps `n`).
RT_D PbrHit pbr_hit(const DevScene& S, const DevMaterial& m, const HitUV& uv, float3 n, float3* sn) {
    PbrHit h = pbr_scalars(m);
    *sn = n;
    if (m.normal_tex && len2(uv.tan) > 1e-6f) {
        float3 raw = tex_bilinear(S, m.normal_tex, uv.u, uv.v, 1);
        float3 ts = mk(raw.x * 2.0f - 1.0f, raw.y * 2.0f - 1.0f, raw.z * 2.0f - 1.0f);
        float3 b = cross3(n, uv.tan);
        float3 pert = uv.tan * ts.x + b * ts.y + n * ts.z;
        if (len2(pert) > 1e-12f) *sn = unit3(pert);
    }
    if (m.albedo_tex) h.albedo = tex_bilinear(S, m.albedo_tex, uv.u, uv.v, 0);
    if (m.ao_tex) h.albedo = h.albedo * tex_bilinear(S, m.ao_tex, uv.u, uv.v, 2).x;
    if (m.roughness_tex) h.roughness = tex_bilinear(S, m.roughness_tex, uv.u, uv.v, 2).x;
    if (m.metallic_tex) h.metallic = tex_bilinear(S, m.metallic_tex, uv.u, uv.v, 2).x;
    return h;
}
RT_D bool pbr_textured(const DevMaterial& m) {
    return m.albedo_tex | m.roughness_tex | m.metallic_tex | m.ao_tex | m.normal_tex;
}

}  // namespace rtd
