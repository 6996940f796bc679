// rt_guide.cuh — the learned proposal of the path tracer (no counterpart in the
// reference, which samples every diffuse bounce from the cosine lobe,
// renderer.rs:545-571, pdf.rs:12-41).
//
// Network: position → 16-level hash grid (2 features per level, 2^19 entries
// per level, trilinear, the hashing of Müller et al. 2022 "Instant neural
// graphics primitives"), the outgoing direction ω_o (toward the previous vertex)
// → one-blob encoding (16 bins for each of θ/π and φ/2π, Müller et al. 2019
// "Neural importance sampling"); the shading normal enters only the cosine
// lobe of the mixture; the 64
// inputs pass three ReLU layers of width 64 and an output layer of 41 (padded
// to 48), no biases.  Weights and activations are BF16, products accumulate in
// FP32 on the tensor cores (mma.sync m16n8k16; one warp evaluates 16 rows).
//
// Outputs: 8 von Mises–Fisher lobes (unnormalised mean 3, log κ 1 clamped to
// [−5, lkmax], mixture logit 1) and the guide fraction α = amax·sigmoid(o40).  The bounce direction
// is drawn by one-sample MIS: with probability α from the vMF mixture, else
// from the cosine lobe; its density is α·p_vmf + (1 − α)·cos/π, which is > 0
// wherever the Lambertian integrand is, so the estimator stays unbiased.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace rtg {

constexpr int LEVELS = 16, FEAT = 2, LOG2_TSIZE = 19;
constexpr uint32_t TSIZE = 1u << LOG2_TSIZE;
constexpr int NIN = 64, NHID = 64, NOUT = 41, NOUTP = 48, NLOBE = 8, NBLOB = 16;
constexpr int OFF_W0 = 0, OFF_W1 = NHID * NIN, OFF_W2 = 2 * NHID * NIN, OFF_W3 = 3 * NHID * NIN;
constexpr int N_MLP = OFF_W3 + NOUTP * NHID;                      // 15360 weights
constexpr size_t N_TABLE = (size_t)LEVELS * TSIZE * FEAT;         // 16,777,216 table entries
constexpr size_t N_PARAMS = (size_t)N_MLP + N_TABLE;
constexpr int GP_F4 = 13;            // per-path mixture: 8 × (μ, κ), π0..3, π4..7, (α, -, -, -), β0..3, β4..7
                                     // with β_i = log(π_i · c(κ_i)) − κ_i, c the vMF normaliser
constexpr float LOGK_LO = -5.0f;     // log κ floor; the cap and α's cap are parameters
constexpr int LDW = NIN + 8;         // padded shared-memory row of a forward weight matrix (bf16)
constexpr int LDT3 = NOUTP + 8;      // padded row of the transposed output layer
constexpr int W_SMEM = (3 * NHID + NOUTP) * LDW;                  // forward weights, bf16 elements
constexpr int WT_SMEM = 3 * NIN * LDW + NHID * LDT3;              // transposed weights, bf16 elements
constexpr uint32_t REC_NONE = 0xFFFFFFFFu;

// What the render kernels see of the guide.  mode 0: off; 1: guided bounces;
// 2: guided bounces plus training records.
struct GuideDev {
    int mode;
    const float* table;               // [LEVELS][TSIZE][FEAT] fp32 master (Adam)
    const __nv_bfloat162* tbf;        // its bf16 copy, read by every encoding
    const __nv_bfloat16* wbf;         // the four layers, [out][in] row-major, bf16
    float lo[3], inv[3];              // hash-grid domain: pn = (p − lo) · inv, clamped to [0, 1]
    uint32_t res[LEVELS];             // grid resolution of each level
    float amax, lkmax;                // cap of α, cap of log κ
    float4* gpar;                     // GP_F4 float4 per path slot
    uint4* enc;                       // encoded inputs of the diffuse queue (8 uint4 per entry)
    float4 *rec_a, *rec_b, *rec_c;    // records: (p, Σ T·sf), (n, base Σ L), (ω_i, prev record)
    float2* rec_o;                    // records: one-blob angles (θ/π, φ/2π) of ω_o
    float* rec_w;                     // weight of each record, set when its path retires
    uint32_t* rec_count;
    uint32_t rec_cap;
};

#ifndef RTG_HD
#define RTG_HD __host__ __device__ __forceinline__
#endif
#define RTG_D __device__ __forceinline__

// ── encoding ─────────────────────────────────────────────────────────────────
RTG_HD uint32_t grid_index(uint32_t res, uint32_t x, uint32_t y, uint32_t z) {
    uint32_t n1 = res + 1u;
    if ((uint64_t)n1 * n1 * n1 <= TSIZE) return x + n1 * (y + n1 * z);     // dense coarse levels
    return (x ^ (y * 2654435761u) ^ (z * 805459861u)) & (TSIZE - 1u);
}

// Grid coordinates of one level: the cell's low corner and the fractions.
// Explicit _rn arithmetic, so every translation unit and the CPU restatement
// round alike.
RTG_D void level_cell(uint32_t res, float pn, uint32_t* i, float* f) {
    float x = __fmul_rn(pn, (float)res);
    uint32_t c = (uint32_t)floorf(x);
    if (c > res - 1u) c = res - 1u;
    *i = c;
    *f = __fsub_rn(x, (float)c);
}
RTG_D void normalise_pos(const GuideDev& G, float px, float py, float pz, float pn[3]) {
    float p[3] = {px, py, pz};
    for (int a = 0; a < 3; a++) pn[a] = fminf(fmaxf(__fmul_rn(__fsub_rn(p[a], G.lo[a]), G.inv[a]), 0.0f), 1.0f);
}
RTG_D float corner_weight(int c, const float f[3]) {
    float wx = (c & 1) ? f[0] : __fsub_rn(1.0f, f[0]);
    float wy = (c & 2) ? f[1] : __fsub_rn(1.0f, f[1]);
    float wz = (c & 4) ? f[2] : __fsub_rn(1.0f, f[2]);
    return __fmul_rn(__fmul_rn(wx, wy), wz);
}

RTG_D uint32_t pack_bf2(float lo, float hi);
RTG_D float bf_lo(uint32_t u);
RTG_D float bf_hi(uint32_t u);

// The one-blob coordinates of a unit direction: θ/π and φ/2π.
RTG_D void blob_angles(float3 d, float* th, float* ph) {
    *th = acosf(fminf(fmaxf(d.z, -1.0f), 1.0f)) * 0.318309886f;
    *ph = (atan2f(d.y, d.x) + 3.14159265f) * 0.159154943f;
}

// The 64 network inputs of one point, rounded to bf16, as 32 packed pairs:
// the hash grid at p, the one-blob of the direction with angles (th, ph).
RTG_D void encode_packed(const GuideDev& G, const __nv_bfloat162* __restrict__ table, float3 p, float th, float ph,
                         uint32_t (&out)[32]) {
    float pn[3];
    normalise_pos(G, p.x, p.y, p.z, pn);
#pragma unroll
    for (int l = 0; l < LEVELS; l++) {
        uint32_t res = G.res[l], ci[3];
        float f[3];
        for (int a = 0; a < 3; a++) level_cell(res, pn[a], &ci[a], &f[a]);
        const __nv_bfloat162* tl = table + (size_t)l * TSIZE;
        float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            uint32_t idx = grid_index(res, ci[0] + (c & 1), ci[1] + ((c >> 1) & 1), ci[2] + (c >> 2));
            uint32_t u = __ldg(reinterpret_cast<const unsigned int*>(tl + idx));
            float w = corner_weight(c, f);
            a0 = __fadd_rn(a0, __fmul_rn(w, bf_lo(u)));
            a1 = __fadd_rn(a1, __fmul_rn(w, bf_hi(u)));
        }
        out[l] = pack_bf2(a0, a1);
    }
#pragma unroll
    for (int k = 0; k < NBLOB; k += 2) {
        float d0 = __fsub_rn(__fmul_rn(16.0f, th), (float)k + 0.5f);
        float d1 = __fsub_rn(__fmul_rn(16.0f, th), (float)k + 1.5f);
        float e0 = __fsub_rn(__fmul_rn(16.0f, ph), (float)k + 0.5f);
        float e1 = __fsub_rn(__fmul_rn(16.0f, ph), (float)k + 1.5f);
        out[16 + k / 2] = pack_bf2(expf(-0.5f * d0 * d0), expf(-0.5f * d1 * d1));
        out[24 + k / 2] = pack_bf2(expf(-0.5f * e0 * e0), expf(-0.5f * e1 * e1));
    }
}

// The same inputs into a row of bf16 (shared or global memory, 4-byte aligned).
RTG_D void encode_row(const GuideDev& G, const __nv_bfloat162* __restrict__ table, float3 p, float th, float ph,
                      __nv_bfloat16* row) {
    uint32_t v[32];
    encode_packed(G, table, p, th, ph, v);
#pragma unroll
    for (int k = 0; k < 32; k++) reinterpret_cast<uint32_t*>(row)[k] = v[k];
}

// ── tensor-core tiles ────────────────────────────────────────────────────────
RTG_D uint32_t pack_bf2(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&h);
}
RTG_D float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
RTG_D float bf_hi(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }
RTG_D uint32_t ld_u32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

RTG_D void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A fragments (16 rows × 16·NK columns) of a row-major bf16 tile in shared memory.
template <int NK>
RTG_D void load_frags(const __nv_bfloat16* S, int ld, uint32_t (&x)[NK][4]) {
    int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kb = 0; kb < NK; kb++) {
        const __nv_bfloat16* r0 = S + g * ld + 16 * kb + 2 * t;
        const __nv_bfloat16* r1 = r0 + 8 * ld;
        x[kb][0] = ld_u32(r0); x[kb][1] = ld_u32(r1); x[kb][2] = ld_u32(r0 + 8); x[kb][3] = ld_u32(r1 + 8);
    }
}

// C (16 × 8·NT, fp32) = X (16 × 16·NK, A fragments) · Wᵀ with W in shared
// memory as NT·8 rows of `ld` bf16 (row = output column, contiguous along k).
template <int NK, int NT>
RTG_D void mm_tile(const uint32_t (&x)[NK][4], const __nv_bfloat16* W, int ld, float (&c)[NT][4]) {
    int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < NT; j++) {
        c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.0f;
        const __nv_bfloat16* row = W + (8 * j + g) * ld + 2 * t;
#pragma unroll
        for (int kb = 0; kb < NK; kb++) mma_bf16(c[j], x[kb], ld_u32(row + 16 * kb), ld_u32(row + 16 * kb + 8));
    }
}

// C tiles of one layer → A fragments of the next (the m16n8 accumulator layout
// of two adjacent tiles is the m16k16 operand layout), optionally through ReLU.
template <int NK, bool RELU>
RTG_D void to_frags(const float (&c)[2 * NK][4], uint32_t (&x)[NK][4]) {
#pragma unroll
    for (int kb = 0; kb < NK; kb++) {
        float v[8] = {c[2 * kb][0], c[2 * kb][1], c[2 * kb][2], c[2 * kb][3],
                      c[2 * kb + 1][0], c[2 * kb + 1][1], c[2 * kb + 1][2], c[2 * kb + 1][3]};
        if (RELU)
            for (int i = 0; i < 8; i++) v[i] = fmaxf(v[i], 0.0f);
        x[kb][0] = pack_bf2(v[0], v[1]); x[kb][1] = pack_bf2(v[2], v[3]);
        x[kb][2] = pack_bf2(v[4], v[5]); x[kb][3] = pack_bf2(v[6], v[7]);
    }
}

// Zero the gradient where the layer's activation is not positive (ReLU').
RTG_D void relu_mask(float (&c)[8][4], const uint32_t (&h)[4][4]) {
#pragma unroll
    for (int kb = 0; kb < 4; kb++)
#pragma unroll
        for (int r = 0; r < 4; r++) {
            int j = 2 * kb + (r >> 1), e = (r & 1) * 2;
            if (!(bf_lo(h[kb][r]) > 0.0f)) c[j][e] = 0.0f;
            if (!(bf_hi(h[kb][r]) > 0.0f)) c[j][e + 1] = 0.0f;
        }
}

// Forward pass of 16 rows: Ws holds W0, W1, W2 (64 rows each) and W3 (48 rows),
// rows of LDW bf16.
RTG_D void mlp_forward(const __nv_bfloat16* Ws, const uint32_t (&x0)[4][4], uint32_t (&h1)[4][4],
                       uint32_t (&h2)[4][4], uint32_t (&h3)[4][4], float (&o)[6][4]) {
    float c[8][4];
    mm_tile<4, 8>(x0, Ws, LDW, c);
    to_frags<4, true>(c, h1);
    mm_tile<4, 8>(h1, Ws + 64 * LDW, LDW, c);
    to_frags<4, true>(c, h2);
    mm_tile<4, 8>(h2, Ws + 128 * LDW, LDW, c);
    to_frags<4, true>(c, h3);
    mm_tile<4, 6>(h3, Ws + 192 * LDW, LDW, o);
}

// Output tiles → a row-major fp32 tile (16 × ld) in shared memory.
RTG_D void store_out(const float (&o)[6][4], float* So, int ld) {
    int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < 6; j++) {
        So[g * ld + 8 * j + 2 * t] = o[j][0];
        So[g * ld + 8 * j + 2 * t + 1] = o[j][1];
        So[(g + 8) * ld + 8 * j + 2 * t] = o[j][2];
        So[(g + 8) * ld + 8 * j + 2 * t + 1] = o[j][3];
    }
}

// Forward weights (global [out][in] bf16) into padded shared-memory rows.
RTG_D void load_weights(const __nv_bfloat16* __restrict__ wbf, __nv_bfloat16* Ws) {
    for (int i = threadIdx.x; i < (3 * NHID + NOUTP) * (NIN / 2); i += blockDim.x) {
        int r = i / (NIN / 2), c2 = i - r * (NIN / 2);
        *reinterpret_cast<uint32_t*>(Ws + r * LDW + 2 * c2) = ld_u32(wbf + r * NIN + 2 * c2);
    }
}

// ── the vMF mixture ──────────────────────────────────────────────────────────
RTG_HD float vmf_norm(float k) { return k / (6.2831853f * -expm1f(-2.0f * k)); }

// 41 outputs → mixture parameters (GP_F4 float4).
RTG_HD void mixture_from_outputs(const float* o, float4* gp, float amax, float lkmax) {
    float mx = o[4];
    for (int i = 1; i < NLOBE; i++) mx = fmaxf(mx, o[5 * i + 4]);
    float e[NLOBE], s = 0.0f;
    for (int i = 0; i < NLOBE; i++) { e[i] = expf(o[5 * i + 4] - mx); s += e[i]; }
    for (int i = 0; i < NLOBE; i++) {
        float vx = o[5 * i], vy = o[5 * i + 1], vz = o[5 * i + 2];
        float len = sqrtf(vx * vx + vy * vy + vz * vz);
        float k = expf(fminf(fmaxf(o[5 * i + 3], LOGK_LO), lkmax));
        gp[i] = len > 1e-12f ? make_float4(vx / len, vy / len, vz / len, k) : make_float4(0.f, 0.f, 1.f, k);
    }
    gp[8] = make_float4(e[0] / s, e[1] / s, e[2] / s, e[3] / s);
    gp[9] = make_float4(e[4] / s, e[5] / s, e[6] / s, e[7] / s);
    gp[10] = make_float4(amax / (1.0f + expf(-o[40])), 0.f, 0.f, 0.f);
    float beta[NLOBE], ls = logf(s);
    for (int i = 0; i < NLOBE; i++) {
        float k = gp[i].w;
        beta[i] = (o[5 * i + 4] - mx - ls) + logf(k) - 1.83787707f - logf(-expm1f(-2.0f * k)) - k;
    }
    gp[11] = make_float4(beta[0], beta[1], beta[2], beta[3]);
    gp[12] = make_float4(beta[4], beta[5], beta[6], beta[7]);
}

RTG_HD float lobe_weight(const float4* gp, int i) {
    float4 q = gp[8 + (i >> 2)];
    int r = i & 3;
    return r == 0 ? q.x : r == 1 ? q.y : r == 2 ? q.z : q.w;
}

// Density of the vMF mixture alone at unit direction w:
// Σ π_i c(κ_i) exp(κ_i (μ_i·w − 1)) = Σ exp(κ_i μ_i·w + β_i).
RTG_HD float vmf_mix_pdf(const float4* gp, float wx, float wy, float wz) {
    float4 b0 = gp[11], b1 = gp[12];
    float beta[NLOBE] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
    float p = 0.0f;
#pragma unroll
    for (int i = 0; i < NLOBE; i++) {
        float4 m = gp[i];
        p += expf(m.w * (m.x * wx + m.y * wy + m.z * wz) + beta[i]);
    }
    return p;
}

// Density of the one-sample mixture of the guide and the cosine lobe about n.
RTG_HD float guide_pdf(const float4* gp, float nx, float ny, float nz, float wx, float wy, float wz) {
    float a = gp[10].x;
    float pb = fmaxf(nx * wx + ny * wy + nz * wz, 0.0f) * 0.318309886f;
    return a * vmf_mix_pdf(gp, wx, wy, wz) + (1.0f - a) * pb;
}

// A direction from the vMF mixture: lobe by u0, then Jakob's stable inversion
// (2012, "Numerically stable sampling of the von Mises–Fisher distribution on
// S²") with u1, u2, about the lobe's mean in the orthonormal basis of Duff et
// al. (2017, "Building an orthonormal basis, revisited").
RTG_HD void vmf_mix_sample(const float4* gp, float u0, float u1, float u2, float* dx, float* dy, float* dz) {
    int lobe = NLOBE - 1;
    float cum = 0.0f;
    for (int i = 0; i < NLOBE - 1; i++) {
        cum += lobe_weight(gp, i);
        if (u0 < cum) { lobe = i; break; }
    }
    float4 m = gp[lobe];
    float k = m.w;
    float xi = 1.0f - u1;                                   // (0, 1]
    float w = 1.0f + logf(xi + (1.0f - xi) * expf(-2.0f * k)) / k;
    w = fminf(fmaxf(w, -1.0f), 1.0f);
    float sr = sqrtf(fmaxf(1.0f - w * w, 0.0f));
    float sp = sinf(6.2831853f * u2), cp = cosf(6.2831853f * u2);
    float sg = m.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sg + m.z), b = m.x * m.y * a;
    float tx = 1.0f + sg * m.x * m.x * a, ty = sg * b, tz = -sg * m.x;
    float bx = b, by = sg + m.y * m.y * a, bz = -m.y;
    float x = w * m.x + sr * (cp * tx + sp * bx);
    float y = w * m.y + sr * (cp * ty + sp * by);
    float z = w * m.z + sr * (cp * tz + sp * bz);
    float il = 1.0f / sqrtf(x * x + y * y + z * z);
    *dx = x * il; *dy = y * il; *dz = z * il;
}

// The training objective of one record, times `scale` (1/batch), with respect
// to the 41 outputs.  The lobes descend −w·log p_vmf(ω_i): the KL divergence
// from the density ∝ f·L_i·cos that the weights estimate to the vMF mixture
// alone, so they learn whatever α is.  α descends −w·log p_mix(ω_i) with the
// lobes held fixed (the selection probability learned on its own, as in
// Müller et al. 2019): minimising the mixture loss jointly collapses α to 0
// while the untrained lobes explain the records worse than the cosine lobe,
// and then every lobe gradient carries the factor α.  Densities are floored
// at 1e-8.  Returns −w·log p_mix.
RTG_HD float loss_grad(const float* o, float nx, float ny, float nz, float wx, float wy, float wz, float wt,
                       float scale, float amax, float lkmax, float* g) {
    float mx = o[4];
    for (int i = 1; i < NLOBE; i++) mx = fmaxf(mx, o[5 * i + 4]);
    float e[NLOBE], s = 0.0f;
    for (int i = 0; i < NLOBE; i++) { e[i] = expf(o[5 * i + 4] - mx); s += e[i]; }
    float pi[NLOBE], f[NLOBE], c[NLOBE], k[NLOBE], len[NLOBE], mu[NLOBE][3];
    float pg = 0.0f;
    for (int i = 0; i < NLOBE; i++) {
        pi[i] = e[i] / s;
        float vx = o[5 * i], vy = o[5 * i + 1], vz = o[5 * i + 2];
        len[i] = sqrtf(vx * vx + vy * vy + vz * vz);
        if (len[i] > 1e-12f) { mu[i][0] = vx / len[i]; mu[i][1] = vy / len[i]; mu[i][2] = vz / len[i]; }
        else { mu[i][0] = 0.0f; mu[i][1] = 0.0f; mu[i][2] = 1.0f; }
        k[i] = expf(fminf(fmaxf(o[5 * i + 3], LOGK_LO), lkmax));
        c[i] = mu[i][0] * wx + mu[i][1] * wy + mu[i][2] * wz;
        f[i] = vmf_norm(k[i]) * expf(k[i] * (c[i] - 1.0f));
        pg += pi[i] * f[i];
    }
    float sg = 1.0f / (1.0f + expf(-o[40]));
    float a = amax * sg;
    float pb = fmaxf(nx * wx + ny * wy + nz * wz, 0.0f) * 0.318309886f;
    float p = fmaxf(a * pg + (1.0f - a) * pb, 1e-8f);
    float loss = -wt * logf(p);
    float dp = -wt / p * scale;                              // mixture loss: α only
    g[40] = dp * (pg - pb) * amax * sg * (1.0f - sg);
    float dq = -wt / fmaxf(pg, 1e-8f) * scale;               // vMF loss: the lobes
    float gs = 0.0f;
    for (int i = 0; i < NLOBE; i++) gs += pi[i] * (dq * f[i]);
    for (int i = 0; i < NLOBE; i++) {
        g[5 * i + 4] = pi[i] * (dq * f[i] - gs);
        float df = dq * pi[i] * f[i];                        // ∂loss/∂f_i · f_i
        float lk = o[5 * i + 3];
        float dlk = 1.0f / k[i] - 2.0f / expm1f(2.0f * k[i]) + (c[i] - 1.0f);
        g[5 * i + 3] = (lk > LOGK_LO && lk < lkmax) ? df * dlk * k[i] : 0.0f;
        float cm = len[i] > 1e-12f ? df * k[i] / len[i] : 0.0f;
        g[5 * i] = cm * (wx - mu[i][0] * c[i]);
        g[5 * i + 1] = cm * (wy - mu[i][1] * c[i]);
        g[5 * i + 2] = cm * (wz - mu[i][2] * c[i]);
    }
    return loss;
}

}  // namespace rtg
