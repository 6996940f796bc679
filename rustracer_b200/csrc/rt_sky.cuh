// rt_sky.cuh — the Physical background: Preetham sky with a sun disc
// (renderer.rs:18, 231-337), the sun cone pdf and its sampling (:340-362).
// Host and device: the host evaluates it for the sun's photon emitter.
#pragma once
#include "rt_device.cuh"

namespace rtd {

static constexpr float COS_SUN_MAX = 0.9999892f;
static constexpr float SUN_PDF = 1.0f / (2.0f * PI_F * (1.0f - COS_SUN_MAX));

RT_HD float sky_clamp(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
RT_HD float3 sky_unit(float3 a) { return a / sqrtf(len2(a)); }

RT_HD float perez(float a, float b, float c, float dp, float e, float ct, float g, float cg) {
    return (1.0f + a * expf(b / ct)) * (1.0f + c * expf(dp * g) + e * cg * cg);
}

RT_HD float3 preetham_sky_eval(float3 dir, float3 sun_dir, float turbidity) {
    float3 d = sky_unit(dir), sun = sky_unit(sun_dir);
    float cos_gamma = sky_clamp(dot3(d, sun), -1.0f, 1.0f);
    float gamma = acosf(cos_gamma);
    float t = sky_clamp(turbidity, 1.7f, 20.0f);
    float cos_theta_s = fmaxf(sun.y, 0.0175f);
    float theta_s = acosf(cos_theta_s);
    float ay = 0.1787f * t - 1.4630f, by = -0.3554f * t + 0.4275f, cy = 0.0227f * t + 5.3251f,
          dy = 0.1206f * t - 2.5771f, ey = -0.0670f * t + 0.3703f;
    float ax = -0.0193f * t - 0.2592f, bx = -0.0665f * t + 0.0008f, cx = -0.0004f * t + 0.2125f,
          dx = -0.0641f * t - 0.8989f, ex = -0.0033f * t + 0.0452f;
    float acy = -0.0167f * t - 0.2608f, bcy = -0.0950f * t + 0.0092f, ccy = -0.0079f * t + 0.2102f,
          dcy = -0.0441f * t - 1.6537f, ecy = -0.0109f * t + 0.0529f;
    float fn_y = perez(ay, by, cy, dy, ey, 1.0f, theta_s, cos_theta_s);
    float fn_x = perez(ax, bx, cx, dx, ex, 1.0f, theta_s, cos_theta_s);
    float fn_cy = perez(acy, bcy, ccy, dcy, ecy, 1.0f, theta_s, cos_theta_s);
    float yz = fmaxf((4.0453f * t - 4.9710f) * tanf((4.0f / 9.0f - t / 120.0f) * (PI_F - 2.0f * theta_s))
                     - 0.2155f * t + 2.4192f, 0.0f);
    if (cos_gamma > COS_SUN_MAX && sun.y > 0.0f && d.y > 0.0f) {
        float disc = yz * 111.0f;
        return mk(disc, disc * 0.95f, disc * 0.85f);
    }
    float ts = theta_s, ts2 = ts * ts, ts3 = ts2 * ts;
    float xz = t * t * (0.00166f * ts3 - 0.00375f * ts2 + 0.00209f * ts)
             + t * (-0.02903f * ts3 + 0.06377f * ts2 - 0.03202f * ts + 0.00394f)
             + (0.11693f * ts3 - 0.21196f * ts2 + 0.06052f * ts + 0.25886f);
    float yzc = t * t * (0.00275f * ts3 - 0.00610f * ts2 + 0.00317f * ts)
              + t * (-0.04214f * ts3 + 0.08970f * ts2 - 0.04153f * ts + 0.00516f)
              + (0.15346f * ts3 - 0.26756f * ts2 + 0.06670f * ts + 0.26688f);
    float ct = fmaxf(d.y, 0.001f);
    float fy = perez(ay, by, cy, dy, ey, ct, gamma, cos_gamma);
    float fx = perez(ax, bx, cx, dx, ex, ct, gamma, cos_gamma);
    float fcy = perez(acy, bcy, ccy, dcy, ecy, ct, gamma, cos_gamma);
    float cap_y = fmaxf(yz * fy / fn_y, 0.0f);
    float cap_x = sky_clamp(xz * fx / fn_x, 0.001f, 0.998f);
    float cap_yc = sky_clamp(yzc * fcy / fn_cy, 0.001f, 0.998f);
    float lum = cap_y * 0.05f;
    float big_x = cap_x / cap_yc * lum, big_y = lum;
    float big_z = fmaxf((1.0f - cap_x - cap_yc) / cap_yc * lum, 0.0f);
    float3 sky = mk(fmaxf(3.2406f * big_x - 1.5372f * big_y - 0.4986f * big_z, 0.0f),
                    fmaxf(-0.9689f * big_x + 1.8758f * big_y + 0.0415f * big_z, 0.0f),
                    fmaxf(0.0557f * big_x - 0.2040f * big_y + 1.0570f * big_z, 0.0f));
    if (d.y < 0.0f) {
        float tt = fminf(-d.y * 8.0f, 1.0f);
        return sky * (1.0f - tt) + mk(0.07f, 0.06f, 0.05f) * tt;
    }
    return sky;
}

RT_HD float3 preetham_sky(float3 dir, float3 sun_dir, float turbidity) {
    return preetham_sky_eval(dir, sun_dir, turbidity);
}

RT_HD float sun_pdf_value(const DevScene& S, float3 dir) {
    return (S.has_sun && dot3(sky_unit(dir), S.sun_dir) > COS_SUN_MAX) ? SUN_PDF : 0.0f;
}

RT_HD float3 sample_sun_cone(float3 axis, float r1, float r2) {
    float cos_t = 1.0f - r1 * (1.0f - COS_SUN_MAX);
    float sin_t = sqrtf(fmaxf(1.0f - cos_t * cos_t, 0.0f));
    float phi = 2.0f * PI_F * r2;
    float3 up = fabsf(axis.x) < 0.999f ? mk(1.f, 0.f, 0.f) : mk(0.f, 1.f, 0.f);
    float3 t = sky_unit(cross3(axis, up));
    float3 b = cross3(axis, t);
    return t * (sin_t * cosf(phi)) + b * (sin_t * sinf(phi)) + axis * cos_t;
}

}  // namespace rtd
