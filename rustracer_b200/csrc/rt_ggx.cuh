// rt_ggx.cuh — GGX microfacet helpers shared by the shading and photon kernels
// (material.rs:104-322) and the PbrMaterial lobes (material.rs:680-1050):
// Smith masking (isotropic and anisotropic), the GGX NDF, VNDF sampling
// (Heitz 2018), the E_ss energy-compensation lookup, Schlick Fresnel and the
// thin-film colour lookup.  The CPU oracle restates the same functions
// (oracle/rt_oracle.cpp).
#pragma once
#include "rt_device.cuh"

namespace rtd {

RT_D float smith_lambda(float c, float alpha) {                                     // material.rs:179-184
    float a2 = alpha * alpha, c2 = c * c;
    return (sqrtf(a2 + (1.0f - a2) * c2) - c) / (2.0f * c);
}
RT_D float smith_g1(float c, float alpha) {                                         // material.rs:163-167
    float a2 = alpha * alpha, c2 = c * c;
    return 2.0f * c / (c + sqrtf(a2 + (1.0f - a2) * c2));
}
RT_D float smith_lambda_aniso(float c, float tx, float ty, float ax, float ay) {    // material.rs:187-190
    return (sqrtf(c * c + ax * ax * tx * tx + ay * ay * ty * ty) - c) / (2.0f * c);
}
RT_D float smith_g1_aniso(float c, float tx, float ty, float ax, float ay) {        // material.rs:172-175
    float den = c + sqrtf(c * c + ax * ax * tx * tx + ay * ay * ty * ty);
    return clampf_(2.0f * c / fmaxf(den, 1e-6f), 0.0f, 1.0f);
}
RT_D float ggx_ndf(float cos_h, float alpha) {                                      // material.rs:308-312
    float a2 = alpha * alpha;
    float dd = 1.0f + cos_h * cos_h * (a2 - 1.0f);
    return a2 / fmaxf(PI_F * dd * dd, 1e-12f);
}
RT_D float ggx_ndf_aniso(float3 h, float ax, float ay) {                            // material.rs:316-321
    float hx = h.x / ax, hy = h.y / ay;
    float dd = hx * hx + hy * hy + h.z * h.z;
    return 1.0f / fmaxf(PI_F * ax * ay * dd * dd, 1e-12f);
}
// vndf_sample_aniso (material.rs:273-305): a microfacet normal in tangent space
RT_D float3 vndf_sample(float3 wo, float ax, float ay, float xi1, float xi2) {
    float3 wh = unit3(mk(ax * wo.x, ay * wo.y, wo.z));
    float len = sqrtf(wh.x * wh.x + wh.y * wh.y);
    float3 t1 = len > 1e-6f ? mk(-wh.y / len, wh.x / len, 0.0f) : mk(1.0f, 0.0f, 0.0f);
    float3 t2 = cross3(wh, t1);
    float a = 1.0f / (1.0f + wh.z);
    float r = sqrtf(xi1);
    float p1, p2, sphi, cphi;
    if (xi2 < a) {
        sincosf(xi2 / a * PI_F, &sphi, &cphi);
        p1 = r * cphi; p2 = r * sphi;
    } else {
        sincosf(PI_F + (xi2 - a) / (1.0f - a) * PI_F, &sphi, &cphi);
        p1 = r * cphi; p2 = r * sphi * wh.z;
    }
    float p3 = sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f));
    float3 nh = t1 * p1 + t2 * p2 + wh * p3;
    return unit3(mk(ax * nh.x, ay * nh.y, fmaxf(nh.z, 0.0f)));
}
// E_ss(mu, alpha) bilinear lookup (material.rs:200-262) and its compensation
RT_D float e_ss_lut(const DevScene& S, float mu, float alpha) {
    float x = clampf_(clampf_(mu, 0.0f, 1.0f) * 64.0f - 0.5f, 0.0f, 63.0f);
    float y = clampf_(clampf_(alpha, 0.0f, 1.0f) * 64.0f - 0.5f, 0.0f, 63.0f);
    int i0 = (int)x, j0 = (int)y, i1 = min(i0 + 1, 63), j1 = min(j0 + 1, 63);
    float fx = x - (float)i0, fy = y - (float)j0;
    float e00 = __ldg(S.elut + i0 * 64 + j0), e10 = __ldg(S.elut + i1 * 64 + j0);
    float e01 = __ldg(S.elut + i0 * 64 + j1), e11 = __ldg(S.elut + i1 * 64 + j1);
    return (e00 * (1.0f - fx) + e10 * fx) * (1.0f - fy) + (e01 * (1.0f - fx) + e11 * fx) * fy;
}
RT_D float energy_comp(const DevScene& S, float mu, float alpha) {                  // material.rs:265-267
    return fminf(1.0f / fmaxf(e_ss_lut(S, mu, alpha), 0.05f), 10.0f);
}

// ── PbrMaterial (material.rs:680-1050) ──────────────────────────────────────
RT_D float schlick(float cosine, float ref_idx) {                                   // material.rs:106-111
    float b = (1.0f - ref_idx) / (1.0f + ref_idx), r0 = b * b, u = 1.0f - cosine;
    return r0 + (1.0f - r0) * (u * u * u * u * u);
}
RT_D float3 schlick_rgb(float ct, float3 f0) {                                      // material.rs:155-160
    float u = fmaxf(1.0f - ct, 0.0f), t = u * u * u * u * u;
    return f0 + (mk(1.f, 1.f, 1.f) - f0) * t;
}
// Vec3::onb (vec3.rs:37-42)
RT_D void onb_y(float3 n, float3* u, float3* v) {
    float3 up = fabsf(n.y) < 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
    *u = unit3(cross3(n, up));
    *v = cross3(n, *u);
}
// nacre_color (material.rs:1130-1146): the thin-film LUT over the optical path
// difference, blended toward grey at grazing angles
RT_D float3 nacre_color(const DevScene& S, float ct, float film_ior, float thick) {
    float sin_sq = fmaxf(1.0f - ct * ct, 0.0f);
    float cos_t = sqrtf(fmaxf(1.0f - sin_sq / (film_ior * film_ior), 0.0f));
    float opd = 2.0f * film_ior * thick * cos_t;
    float t = clampf_(opd / 2500.0f, 0.0f, 1.0f) * 255.0f;
    int lo = (int)t, hi = min(lo + 1, 255);
    float f = t - (float)lo;
    float4 a = __ldg(S.nacre + lo), b = __ldg(S.nacre + hi);
    float3 raw = mk(a.x, a.y, a.z) * (1.0f - f) + mk(b.x, b.y, b.z) * f;
    float blend = powf(ct, 0.5f);
    return raw * blend + mk(0.5f, 0.5f, 0.5f) * (1.0f - blend);
}
// the per-hit PBR parameters (ShadingParams, material.rs:773-786): albedo,
// roughness and metallic from the scalars or the texture maps
struct PbrHit { float3 albedo; float roughness, metallic; };
RT_D PbrHit pbr_scalars(const DevMaterial& m) {
    PbrHit h;
    h.albedo = mk(m.albedo[0], m.albedo[1], m.albedo[2]);
    h.roughness = m.roughness;
    h.metallic = m.metallic;
    return h;
}
RT_D float3 pbr_f0(const PbrHit& h) {
    return mk(0.04f, 0.04f, 0.04f) * (1.0f - h.metallic) + h.albedo * h.metallic;
}
RT_D float pbr_p_coat(const DevMaterial& m, float cos_o) {
    return m.clearcoat > 1e-3f ? fmaxf(schlick(cos_o, 1.0f / 1.5f) * m.clearcoat, 0.12f * m.clearcoat) : 0.0f;
}
RT_D float pbr_p_spec(const PbrHit& h, float3 f0, float cos_o) {
    return h.metallic > 0.999f ? 1.0f : clampf_(lum3(schlick_rgb(cos_o, f0)), 0.04f, 0.9f);
}
// the anisotropic base-lobe frame: the onb rotated by anisotropy_angle
RT_D void pbr_frame(const DevMaterial& m, float3 n, float3* t, float3* b) {
    float3 t0, b0;
    onb_y(n, &t0, &b0);
    *t = t0 * m.aniso_c + b0 * m.aniso_s;
    *b = b0 * m.aniso_c - t0 * m.aniso_s;
}

enum { PBR_NONE = 0, PBR_SPECULAR = 1, PBR_DIFFUSE = 2 };
// PbrMaterial::scatter (material.rs:790-920): the coat, base-specular or
// diffuse(+sheen) lobe, chosen by xi_coat / xi_spec; xi1, xi2 sample the VNDF.
// Returns the lobe, its attenuation and (specular lobes) its direction.
RT_D int pbr_scatter(const DevScene& S, const DevMaterial& m, const PbrHit& ph, float3 wo, float3 n, float xi_coat,
                     float xi_spec, float xi1, float xi2, float3* att, float3* dir) {
    float cos_o = dot3(wo, n);
    if (cos_o <= 0.0f) return PBR_NONE;
    float alpha = fmaxf(ph.roughness * ph.roughness, 1e-4f);
    float3 albedo = ph.albedo;
    float3 f0 = pbr_f0(ph);
    float p_coat = pbr_p_coat(m, cos_o);
    float p_spec = pbr_p_spec(ph, f0, cos_o);
    if (xi_coat < p_coat) {
        float ac = fmaxf(m.clearcoat_roughness * m.clearcoat_roughness, 1e-4f);
        float3 t, b;
        onb_y(n, &t, &b);
        float3 ms = vndf_sample(mk(dot3(wo, t), dot3(wo, b), cos_o), ac, ac, xi1, xi2);
        float3 mm = unit3(t * ms.x + b * ms.y + n * ms.z);
        float vo_h = fmaxf(dot3(wo, mm), 0.0f);
        float3 wi = unit3(2.0f * vo_h * mm - wo);
        float cos_i = dot3(wi, n);
        if (cos_i <= 0.0f) return PBR_NONE;
        float f_coat = schlick(vo_h, 1.0f / 1.5f) * m.clearcoat;
        float lo = smith_lambda(cos_o, ac), li = smith_lambda(cos_i, ac);
        float w = ((1.0f + lo) / (1.0f + lo + li)) * energy_comp(S, cos_o, ac);
        float3 film = m.film_thickness > 0.0f ? nacre_color(S, vo_h, m.film_ior, m.film_thickness) : mk(1.f, 1.f, 1.f);
        *att = film * (f_coat * w / p_coat);
        *dir = wi;
        return PBR_SPECULAR;
    }
    if (xi_spec < p_spec) {
        float ax = alpha / m.aspect, ay = alpha * m.aspect;
        float3 t, b;
        pbr_frame(m, n, &t, &b);
        float3 wo_ts = mk(dot3(wo, t), dot3(wo, b), cos_o);
        float3 ms = vndf_sample(wo_ts, ax, ay, xi1, xi2);
        float3 mm = unit3(t * ms.x + b * ms.y + n * ms.z);
        float vo_h = fmaxf(dot3(wo, mm), 0.0f);
        float3 wi = unit3(2.0f * vo_h * mm - wo);
        float cos_i = dot3(wi, n);
        if (cos_i <= 0.0f) return PBR_NONE;
        float lo = smith_lambda_aniso(cos_o, wo_ts.x, wo_ts.y, ax, ay);
        float li = smith_lambda_aniso(cos_i, dot3(wi, t), dot3(wi, b), ax, ay);
        float w = ((1.0f + lo) / (1.0f + lo + li)) * energy_comp(S, cos_o, alpha);
        *att = schlick_rgb(vo_h, f0) * w / (p_spec * (1.0f - p_coat));
        *dir = wi;
        return PBR_SPECULAR;
    }
    float3 sheen = mk(0.f, 0.f, 0.f);
    if (m.sheen > 0.0f && ph.metallic < 0.999f) {
        float l = lum3(albedo);
        float3 c_tint = l > 1e-6f ? albedo / l : mk(1.f, 1.f, 1.f);
        float3 sc = mk(1.f, 1.f, 1.f) * (1.0f - m.sheen_tint) + c_tint * m.sheen_tint;
        float u = 1.0f - cos_o, f_h = u * u * u * u * u;
        sheen = sc * (m.sheen * (1.0f - ph.metallic) * f_h * PI_F);
    }
    *att = (albedo * (1.0f - ph.metallic) + sheen) / ((1.0f - p_spec) * (1.0f - p_coat));
    return PBR_DIFFUSE;
}
// PbrMaterial::specular_brdf_cos and specular_sampling_pdf (material.rs:935-1047)
RT_D float3 pbr_spec_brdf_cos(const DevScene& S, const DevMaterial& m, const PbrHit& ph, float3 wo, float3 n,
                              float3 wi, float* pdf) {
    *pdf = 0.0f;
    float cos_o = dot3(wo, n), cos_i = dot3(wi, n);
    if (cos_o <= 0.0f || cos_i <= 0.0f) return mk(0.f, 0.f, 0.f);
    float3 h = unit3(wo + wi);
    float wo_h = fmaxf(dot3(wo, h), 0.0f), h_n = fmaxf(dot3(h, n), 0.0f);
    float3 f0 = pbr_f0(ph);
    float p_coat = pbr_p_coat(m, cos_o), p_spec = pbr_p_spec(ph, f0, cos_o);
    float3 res = mk(0.f, 0.f, 0.f);
    float pd = 0.0f;
    if (m.clearcoat > 1e-3f) {
        float ac = fmaxf(m.clearcoat_roughness * m.clearcoat_roughness, 1e-4f);
        float d = ggx_ndf(h_n, ac);
        float g2 = 1.0f / (1.0f + smith_lambda(cos_o, ac) + smith_lambda(cos_i, ac));
        float fc = schlick(wo_h, 1.0f / 1.5f) * m.clearcoat;
        float3 film = m.film_thickness > 0.0f ? nacre_color(S, wo_h, m.film_ior, m.film_thickness) : mk(1.f, 1.f, 1.f);
        res = res + film * (d * fc * g2 / (4.0f * cos_o) * energy_comp(S, cos_o, ac));
        pd += p_coat * d * smith_g1(cos_o, ac) / (4.0f * cos_o);
    }
    float alpha = fmaxf(ph.roughness * ph.roughness, 1e-4f);
    float ax = alpha / m.aspect, ay = alpha * m.aspect;
    float3 t, b;
    pbr_frame(m, n, &t, &b);
    float3 h_ts = mk(dot3(h, t), dot3(h, b), h_n);
    float wox = dot3(wo, t), woy = dot3(wo, b);
    float d = ggx_ndf_aniso(h_ts, ax, ay);
    float g2 = 1.0f / (1.0f + smith_lambda_aniso(cos_o, wox, woy, ax, ay) +
                       smith_lambda_aniso(cos_i, dot3(wi, t), dot3(wi, b), ax, ay));
    res = res + schlick_rgb(wo_h, f0) * (d * g2 / (4.0f * cos_o) * energy_comp(S, cos_o, alpha));
    if ((1.0f - p_coat) * p_spec > 1e-6f)
        pd += (1.0f - p_coat) * p_spec * d * smith_g1_aniso(cos_o, wox, woy, ax, ay) / (4.0f * cos_o);
    *pdf = pd;
    return res;
}
// specular_sampling_pdf alone, for the MIS weight of a sampled specular bounce
RT_D float pbr_spec_pdf(const DevScene& S, const DevMaterial& m, const PbrHit& ph, float3 wo, float3 n, float3 wi) {
    float pdf;
    pbr_spec_brdf_cos(S, m, ph, wo, n, wi, &pdf);
    return pdf;
}

}  // namespace rtd
