// rt_output.cu — develop linear radiance into 8-bit sRGB: the per-pixel mean
// of the accumulators (main.rs:571-583), lens optics in linear light
// (apply_optics, output.rs:159-190), exposure, the AgX or ACES tone curve and
// the sRGB encoding with the reference's quantisation (tone_map,
// output.rs:7-113).  Compiled without FMA contraction so the arithmetic
// rounds like the CPU restatement; only the library's log2f / powf differ in
// the last bits, which can move a byte by one.
#include "rt_internal.h"

using namespace rtd;

namespace {

RT_D float aces_curve(float x) {                                                   // output.rs:12-15
    x = fmaxf(x, 0.0f);
    return (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
}
RT_D float3 aces_tonemap(float3 c) {                                               // output.rs:17-31
    float r = c.x * 0.59719f + c.y * 0.35458f + c.z * 0.04823f;
    float g = c.x * 0.07600f + c.y * 0.90834f + c.z * 0.01566f;
    float b = c.x * 0.02840f + c.y * 0.13383f + c.z * 0.83777f;
    r = aces_curve(r); g = aces_curve(g); b = aces_curve(b);
    return mk(r * 1.60475f + g * -0.53108f + b * -0.07367f,
              r * -0.10208f + g * 1.10813f + b * -0.00605f,
              r * -0.00327f + g * -0.07276f + b * 1.07602f);
}
RT_D float agx_curve(float x) {                                                    // output.rs:39-43
    float x2 = x * x, x4 = x2 * x2;
    return 15.5f * x4 * x2 - 40.14f * x4 * x + 31.96f * x4 - 6.868f * x2 * x + 0.4298f * x2 + 0.1191f * x - 0.00232f;
}
RT_D float agx_log(float v) {
    const float MIN_EV = -12.47393f, RANGE = 16.5f;
    return clampf_((log2f(fmaxf(v, 1e-10f)) - MIN_EV) / RANGE, 0.0f, 1.0f);
}
RT_D float3 agx_tonemap(float3 c) {                                                // output.rs:45-80
    float r = c.x * 0.842479062253094f + c.y * 0.0784335999999992f + c.z * 0.0792237451477643f;
    float g = c.x * 0.0423282422610123f + c.y * 0.878468636469772f + c.z * 0.0791661274605434f;
    float b = c.x * 0.0423756549057051f + c.y * 0.0784336f + c.z * 0.879142973793104f;
    r = agx_curve(agx_log(r)); g = agx_curve(agx_log(g)); b = agx_curve(agx_log(b));
    // Punchy look: power 1.35 and 1.4× saturation about the luminance
    float luma = lum3(mk(r, g, b));
    r = luma + 1.4f * (powf(r, 1.35f) - luma);
    g = luma + 1.4f * (powf(g, 1.35f) - luma);
    b = luma + 1.4f * (powf(b, 1.35f) - luma);
    return mk(r * 1.19687900512017f + g * -0.0980208811401368f + b * -0.0990297440797205f,
              r * -0.0528968517574562f + g * 1.15190312990417f + b * -0.0989611768448433f,
              r * -0.0529716355144234f + g * -0.0980434501171241f + b * 1.15107567775604f);
}
RT_D uint8_t encode8(float x) {                                                    // output.rs:84-86, 104
    x = fmaxf(x, 0.0f);
    float e = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
    return (uint8_t)(clampf_(e, 0.0f, 0.999f) * 256.0f);
}

// one output pixel per thread; `lin` (per-sample means) or sum / max(count, 1)
__global__ void k_develop(const float* __restrict__ lin, const float* __restrict__ sum,
                          const uint32_t* __restrict__ cnt, uint32_t w, uint32_t h, float exposure, int tm,
                          float vignette, float distortion, uint8_t* __restrict__ out) {
    auto fetch = [&](uint32_t i) {
        if (lin) return mk(lin[i * 3], lin[i * 3 + 1], lin[i * 3 + 2]);
        float n = (float)max(cnt[i], 1u);
        return mk(sum[i * 3] / n, sum[i * 3 + 1] / n, sum[i * 3 + 2] / n);
    };
    uint32_t npix = w * h;
    float cx = ((float)w - 1.0f) * 0.5f, cy = ((float)h - 1.0f) * 0.5f;
    float rcorner = fmaxf(sqrtf(cx * cx + cy * cy), 1e-6f);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        uint32_t x = i % w, y = i / w;
        float3 c;
        if (vignette == 0.0f && distortion == 0.0f) {
            c = fetch(i);
        } else {                                                                    // output.rs:159-190
            float dx = ((float)x - cx) / rcorner, dy = ((float)y - cy) / rcorner;
            float r2 = dx * dx + dy * dy;
            float s = 1.0f - distortion * r2;
            float sx = clampf_(cx + dx * rcorner * s, 0.0f, (float)w - 1.0f);
            float sy = clampf_(cy + dy * rcorner * s, 0.0f, (float)h - 1.0f);
            uint32_t x0 = (uint32_t)sx, y0 = (uint32_t)sy;
            uint32_t x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
            float fx = sx - (float)x0, fy = sy - (float)y0;
            float3 c00 = fetch(y0 * w + x0), c10 = fetch(y0 * w + x1);
            float3 c01 = fetch(y1 * w + x0), c11 = fetch(y1 * w + x1);
            c = (c00 * (1.0f - fx) + c10 * fx) * (1.0f - fy) + (c01 * (1.0f - fx) + c11 * fx) * fy;
            c = c * fmaxf(1.0f - vignette * r2, 0.0f);
        }
        c = c * exposure;
        float3 m = tm == RT_TONEMAP_ACES ? aces_tonemap(c) : agx_tonemap(c);
        out[(size_t)i * 3] = encode8(m.x);
        out[(size_t)i * 3 + 1] = encode8(m.y);
        out[(size_t)i * 3 + 2] = encode8(m.z);
    }
}

}  // namespace

namespace rth {
void launch_develop(const float* lin, const float* sum, const uint32_t* cnt, uint32_t w, uint32_t h, float exposure,
                    int tm, float vignette, float distortion, uint8_t* out, int sms, cudaStream_t st) {
    uint32_t npix = w * h;
    uint32_t grid = std::max(1u, std::min((npix + 255u) / 256u, (uint32_t)sms * 8u));
    k_develop<<<grid, 256, 0, st>>>(lin, sum, cnt, w, h, exposure, tm, vignette, distortion, out);
}
}  // namespace rth
