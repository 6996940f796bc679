// rt_guide.cu — training and evaluation of the path-guiding network
// (rt_guide.cuh): the records → training-sample compaction, the fused
// forward/backward pass (BF16 tensor-core tiles, FP32 accumulation, hash-grid
// gradients scattered with atomics), the weight-gradient contraction over the
// batch, Adam, and the evaluation kernel behind the rt_guide_* test entry
// points.  Compiled without FMA contraction, like the CPU restatement it is
// checked against.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "rt_internal.h"

using namespace rtg;

namespace {

constexpr int GW = 4;                  // warps per block of the network kernels
constexpr int LDO = 52;                // fp32 output tile row
constexpr int LDX = 33;                // fp32 input-gradient tile row
constexpr int ST = 18;                 // transposed staging row (bf16)
constexpr uint32_t WG_CHUNK = 1024;    // batch rows per block of the weight-gradient kernel

// transposed activation planes of one training batch (bf16, [feature][batch])
constexpr int ACT_H = 0;               // X0, H1, H2, H3 at 64·l
constexpr int ACT_D = 256;             // dZ1, dZ2, dZ3, dO at 256 + 64·l
constexpr int ACT_ROWS = 256 + 3 * 64 + NOUTP;

RTG_HD uint32_t mix32(uint32_t x) {    // lowbias32 (C. Wellons)
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}

// cosine-lobe direction about unit n (pdf.rs:12-41 restated with Duff et al.'s basis)
RTG_D void cosine_dir(float3 n, float r1, float r2, float3* d) {
    float sp = sinf(6.2831853f * r1), cp = cosf(6.2831853f * r1), sq = sqrtf(r2);
    float sg = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (sg + n.z), b = n.x * n.y * a;
    float3 t = make_float3(1.0f + sg * n.x * n.x * a, sg * b, -sg * n.x);
    float3 bb = make_float3(b, sg + n.y * n.y * a, -n.y);
    float z = sqrtf(fmaxf(1.0f - r2, 0.0f));
    float x = cp * sq, y = sp * sq;
    float3 v = make_float3(x * t.x + y * bb.x + z * n.x, x * t.y + y * bb.y + z * n.y, x * t.z + y * bb.z + z * n.z);
    float il = 1.0f / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    *d = make_float3(v.x * il, v.y * il, v.z * il);
}

// 16 rows of an A-fragment set → a row-major bf16 tile
RTG_D void frags_to_smem(const uint32_t (&x)[4][4], __nv_bfloat16* S, int ld) {
    int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kb = 0; kb < 4; kb++) {
        __nv_bfloat16* r0 = S + g * ld + 16 * kb + 2 * t;
        __nv_bfloat16* r1 = r0 + 8 * ld;
        *reinterpret_cast<uint32_t*>(r0) = x[kb][0];
        *reinterpret_cast<uint32_t*>(r1) = x[kb][1];
        *reinterpret_cast<uint32_t*>(r0 + 8) = x[kb][2];
        *reinterpret_cast<uint32_t*>(r1 + 8) = x[kb][3];
    }
}

// rows 0..15 × nf features of a row-major tile → plane[f][row0 + r], through a
// transposed staging tile (2-sample words per store)
RTG_D void store_planes(const __nv_bfloat16* S, int ld, int nf, __nv_bfloat16* St, __nv_bfloat16* plane,
                        size_t batch, uint32_t row0) {
    int lane = threadIdx.x & 31;
    __syncwarp();
    for (int i = lane; i < 16 * nf; i += 32) {
        int r = i / nf, f = i - r * nf;
        St[f * ST + r] = S[r * ld + f];
    }
    __syncwarp();
    for (int i = lane; i < nf * 8; i += 32) {
        int f = i >> 3, w = i & 7;
        *reinterpret_cast<uint32_t*>(plane + (size_t)f * batch + row0 + 2 * w) =
            *reinterpret_cast<const uint32_t*>(St + f * ST + 2 * w);
    }
    __syncwarp();
}

// transposed copies of the weights for the backward pass: WT_l[in][out]
RTG_D void load_weights_t(const __nv_bfloat16* __restrict__ wbf, __nv_bfloat16* WT) {
    for (int i = threadIdx.x; i < 3 * NHID * NIN; i += blockDim.x) {
        int l = i / (NHID * NIN), r = i - l * NHID * NIN, o = r / NIN, in = r - o * NIN;
        WT[l * NIN * LDW + in * LDW + o] = wbf[i];
    }
    for (int i = threadIdx.x; i < NOUTP * NHID; i += blockDim.x) {
        int o = i / NHID, in = i - o * NHID;
        WT[3 * NIN * LDW + in * LDT3 + o] = wbf[OFF_W3 + i];
    }
}

// Evaluate 32 points per warp; emit(mt, outputs) runs on lanes 0..15 for row 16·mt + lane.
template <class Emit>
RTG_D void warp_eval(const GuideDev& G, const __nv_bfloat16* Ws, __nv_bfloat16* S_in, float* S_o, bool valid,
                     float3 p, float3 wo, Emit emit) {
    int lane = threadIdx.x & 31;
    float th, ph;
    blob_angles(wo, &th, &ph);
    if (valid) encode_row(G, G.tbf, p, th, ph, S_in + lane * LDW);
    else
        for (int k = 0; k < NIN; k++) S_in[lane * LDW + k] = __float2bfloat16_rn(0.0f);
    __syncwarp();
    for (int mt = 0; mt < 2; mt++) {
        uint32_t x0[4][4], h1[4][4], h2[4][4], h3[4][4];
        float o[6][4];
        load_frags<4>(S_in + 16 * mt * LDW, LDW, x0);
        mlp_forward(Ws, x0, h1, h2, h3, o);
        store_out(o, S_o, LDO);
        __syncwarp();
        if (lane < 16) emit(mt, S_o + lane * LDO);
        __syncwarp();
    }
}

// rt_guide_eval / _pdf / _sample: q is n × 9 (position, unit normal, unit ω_o)
__global__ void __launch_bounds__(GW * 32) k_guide_api(GuideDev G, const float* __restrict__ q, uint32_t n,
                                                        const float* __restrict__ dirs, const float* __restrict__ u,
                                                        float* __restrict__ raw, float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char sm[];
    __nv_bfloat16* Ws = reinterpret_cast<__nv_bfloat16*>(sm);
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* S_in = Ws + W_SMEM + warp * 32 * LDW;
    float* S_o = reinterpret_cast<float*>(Ws + W_SMEM + GW * 32 * LDW) + warp * 16 * LDO;
    load_weights(G.wbf, Ws);
    __syncthreads();
    for (uint32_t base = (blockIdx.x * GW + warp) * 32; base < n; base += gridDim.x * GW * 32) {
        uint32_t i = base + lane;
        bool valid = i < n;
        float3 p = make_float3(0.f, 0.f, 0.f), wo = make_float3(0.f, 0.f, 1.f);
        if (valid) {
            p = make_float3(q[i * 9], q[i * 9 + 1], q[i * 9 + 2]);
            wo = make_float3(q[i * 9 + 6], q[i * 9 + 7], q[i * 9 + 8]);
        }
        warp_eval(G, Ws, S_in, S_o, valid, p, wo, [&](int mt, const float* o) {
            uint32_t r = base + 16 * mt + lane;
            if (r >= n) return;
            if (raw)
                for (int k = 0; k < NOUT; k++) raw[(size_t)r * NOUT + k] = o[k];
            if (!out) return;
            float4 gp[GP_F4];
            mixture_from_outputs(o, gp, G.amax, G.lkmax);
            float nx = q[r * 9 + 3], ny = q[r * 9 + 4], nz = q[r * 9 + 5];
            if (dirs) {
                out[r] = guide_pdf(gp, nx, ny, nz, dirs[r * 3], dirs[r * 3 + 1], dirs[r * 3 + 2]);
            } else if (u) {
                const float* uu = u + (size_t)r * 4;
                float dx, dy, dz;
                if (uu[0] < gp[10].x) {
                    vmf_mix_sample(gp, uu[1], uu[2], uu[3], &dx, &dy, &dz);
                } else {
                    float3 d;
                    cosine_dir(make_float3(nx, ny, nz), uu[2], uu[3], &d);
                    dx = d.x; dy = d.y; dz = d.z;
                }
                out[r * 4] = dx; out[r * 4 + 1] = dy; out[r * 4 + 2] = dz;
                out[r * 4 + 3] = guide_pdf(gp, nx, ny, nz, dx, dy, dz);
            }
        });
    }
}

// records of a render call → training samples (3 float4 each: (p, w), (n, θ_o/π),
// (ω_i, φ_o/2π), the angles being ω_o's one-blob coordinates)
__global__ void k_compact(const float4* __restrict__ ra, const float4* __restrict__ rb, const float4* __restrict__ rc,
                          const float2* __restrict__ ro, const float* __restrict__ rw, const uint32_t* counters,
                          uint32_t cap, float4* train, uint32_t* ntrain) {
    uint32_t n = min(counters[0], cap);
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        float w = rw[r];
        if (!(w > 0.0f) || !isfinite(w)) continue;
        uint32_t j = atomicAdd(ntrain, 1u);
        float4 a = ra[r], b = rb[r], c = rc[r];
        float2 ang = ro[r];
        train[(size_t)j * 3] = make_float4(a.x, a.y, a.z, w);
        train[(size_t)j * 3 + 1] = make_float4(b.x, b.y, b.z, ang.x);
        train[(size_t)j * 3 + 2] = make_float4(c.x, c.y, c.z, ang.y);
    }
}

struct TrainArgs {
    const float4* samples;   // 3 float4 per sample
    const uint32_t* n_dev;   // sample count on the device (select = 1), or null
    uint32_t n;              // sample count (select = 0)
    uint32_t batch;          // rows, a multiple of WG_CHUNK
    int select;              // 1: row b draws sample mix32(b ^ seed) % n; 0: row b is sample b
    uint32_t seed;
    __nv_bfloat16* act;      // ACT_ROWS × batch
    float* grad;             // N_PARAMS
    float* loss;             // Σ −w log p over the batch
};

RTG_D bool train_row(const TrainArgs& A, uint32_t row, uint32_t n, float4* s) {
    if (n == 0) return false;
    uint32_t j;
    if (A.select) j = mix32(row ^ A.seed) % n;
    else if (row < n) j = row;
    else return false;
    s[0] = A.samples[(size_t)j * 3]; s[1] = A.samples[(size_t)j * 3 + 1]; s[2] = A.samples[(size_t)j * 3 + 2];
    return true;
}

// fused forward + loss + backward of 32 rows per warp; writes the transposed
// activation planes for the weight gradients and scatters the hash-grid gradient
__global__ void __launch_bounds__(GW * 32) k_train(GuideDev G, TrainArgs A) {
    extern __shared__ __align__(16) unsigned char sm[];
    __nv_bfloat16* Ws = reinterpret_cast<__nv_bfloat16*>(sm);
    __nv_bfloat16* WT = Ws + W_SMEM;
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wsm = sm + (size_t)(W_SMEM + WT_SMEM) * 2;
    constexpr size_t PER_WARP = 32 * LDW * 2 + 16 * LDW * 2 + 16 * LDT3 * 2 + 64 * ST * 2 + 16 * LDO * 4 + 16 * LDX * 4;
    unsigned char* my = wsm + warp * PER_WARP;
    __nv_bfloat16* S_in = reinterpret_cast<__nv_bfloat16*>(my);
    __nv_bfloat16* S_t = S_in + 32 * LDW;
    __nv_bfloat16* S_do = S_t + 16 * LDW;
    __nv_bfloat16* S_st = S_do + 16 * LDT3;
    float* S_o = reinterpret_cast<float*>(S_st + 64 * ST);
    float* S_dx = S_o + 16 * LDO;
    load_weights(G.wbf, Ws);
    load_weights_t(G.wbf, WT);
    __syncthreads();
    uint32_t n = A.select ? *A.n_dev : A.n;
    float scale = 1.0f / (float)(A.select ? A.batch : max(A.n, 1u));
    size_t B = A.batch;
    float lsum = 0.0f;
    for (uint32_t base = (blockIdx.x * GW + warp) * 32; base < A.batch; base += gridDim.x * GW * 32) {
        float4 s[3];
        bool valid = train_row(A, base + lane, n, s);
        if (valid) encode_row(G, G.tbf, make_float3(s[0].x, s[0].y, s[0].z), s[1].w, s[2].w, S_in + lane * LDW);
        else
            for (int k = 0; k < NIN; k++) S_in[lane * LDW + k] = __float2bfloat16_rn(0.0f);
        __syncwarp();
        for (int mt = 0; mt < 2; mt++) {
            uint32_t row0 = base + 16 * mt;
            const __nv_bfloat16* Sx = S_in + 16 * mt * LDW;
            uint32_t x0[4][4], h1[4][4], h2[4][4], h3[4][4], d[4][4];
            float o[6][4];
            load_frags<4>(Sx, LDW, x0);
            store_planes(Sx, LDW, 64, S_st, A.act + (size_t)(ACT_H + 0) * B, B, row0);
            mlp_forward(Ws, x0, h1, h2, h3, o);
            frags_to_smem(h1, S_t, LDW);
            store_planes(S_t, LDW, 64, S_st, A.act + (size_t)(ACT_H + 64) * B, B, row0);
            frags_to_smem(h2, S_t, LDW);
            store_planes(S_t, LDW, 64, S_st, A.act + (size_t)(ACT_H + 128) * B, B, row0);
            frags_to_smem(h3, S_t, LDW);
            store_planes(S_t, LDW, 64, S_st, A.act + (size_t)(ACT_H + 192) * B, B, row0);
            store_out(o, S_o, LDO);
            __syncwarp();
            // loss gradient of row row0 + lane
            float4 r[3];
            bool rv = false;
            if (lane < 16) {
                rv = train_row(A, row0 + lane, n, r) && r[0].w > 0.0f;
                float g[NOUT];
                if (rv) {
                    lsum += loss_grad(S_o + lane * LDO, r[1].x, r[1].y, r[1].z, r[2].x, r[2].y, r[2].z, r[0].w, scale,
                                      G.amax, G.lkmax, g);
                } else {
                    for (int k = 0; k < NOUT; k++) g[k] = 0.0f;
                }
                for (int k = 0; k < NOUTP; k++) S_do[lane * LDT3 + k] = __float2bfloat16_rn(k < NOUT ? g[k] : 0.0f);
            }
            __syncwarp();
            uint32_t dO[3][4];
            load_frags<3>(S_do, LDT3, dO);
            store_planes(S_do, LDT3, NOUTP, S_st, A.act + (size_t)(ACT_D + 192) * B, B, row0);
            float c[8][4];
            mm_tile<3, 8>(dO, WT + 3 * NIN * LDW, LDT3, c);
            relu_mask(c, h3);
            to_frags<4, false>(c, d);
            frags_to_smem(d, S_t, LDW);
            store_planes(S_t, LDW, 64, S_st, A.act + (size_t)(ACT_D + 128) * B, B, row0);
            mm_tile<4, 8>(d, WT + 2 * NIN * LDW, LDW, c);
            relu_mask(c, h2);
            to_frags<4, false>(c, d);
            frags_to_smem(d, S_t, LDW);
            store_planes(S_t, LDW, 64, S_st, A.act + (size_t)(ACT_D + 64) * B, B, row0);
            mm_tile<4, 8>(d, WT + 1 * NIN * LDW, LDW, c);
            relu_mask(c, h1);
            to_frags<4, false>(c, d);
            frags_to_smem(d, S_t, LDW);
            store_planes(S_t, LDW, 64, S_st, A.act + (size_t)(ACT_D + 0) * B, B, row0);
            float cx[4][4];
            mm_tile<4, 4>(d, WT, LDW, cx);                   // ∂loss/∂(hash-grid features)
            {
                int g = lane >> 2, t = lane & 3;
                for (int j = 0; j < 4; j++) {
                    S_dx[g * LDX + 8 * j + 2 * t] = cx[j][0];
                    S_dx[g * LDX + 8 * j + 2 * t + 1] = cx[j][1];
                    S_dx[(g + 8) * LDX + 8 * j + 2 * t] = cx[j][2];
                    S_dx[(g + 8) * LDX + 8 * j + 2 * t + 1] = cx[j][3];
                }
            }
            __syncwarp();
            if (lane < 16 && rv) {
                float pn[3];
                normalise_pos(G, r[0].x, r[0].y, r[0].z, pn);
                float* gt = A.grad + N_MLP;
                for (int l = 0; l < LEVELS; l++) {
                    uint32_t res = G.res[l], ci[3];
                    float f[3];
                    for (int a = 0; a < 3; a++) level_cell(res, pn[a], &ci[a], &f[a]);
                    float d0 = S_dx[lane * LDX + 2 * l], d1 = S_dx[lane * LDX + 2 * l + 1];
                    for (int cc = 0; cc < 8; cc++) {
                        uint32_t idx = grid_index(res, ci[0] + (cc & 1), ci[1] + ((cc >> 1) & 1), ci[2] + (cc >> 2));
                        float w = corner_weight(cc, f);
                        size_t at = ((size_t)l * TSIZE + idx) * 2;
                        atomicAdd(gt + at, __fmul_rn(w, d0));
                        atomicAdd(gt + at + 1, __fmul_rn(w, d1));
                    }
                }
            }
            __syncwarp();
        }
    }
    if (lsum != 0.0f) atomicAdd(A.loss, lsum);
}

// ∂loss/∂W_l = Σ_b dZ_{l+1}[b]ᵀ · H_l[b]: block (chunk, l); warp w owns output rows 16w..16w+15
__global__ void __launch_bounds__(GW * 32) k_wgrad(const __nv_bfloat16* __restrict__ act, uint32_t batch,
                                                    float* __restrict__ grad) {
    int l = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    int M = l == 3 ? NOUTP : NHID;
    if (16 * warp >= M) return;
    size_t B = batch;
    const __nv_bfloat16* D = act + (size_t)(ACT_D + 64 * l) * B + (size_t)(16 * warp) * B;
    const __nv_bfloat16* H = act + (size_t)(ACT_H + 64 * l) * B;
    float c[8][4] = {};
    uint32_t k0 = blockIdx.x * WG_CHUNK;
    for (uint32_t kk = k0; kk < k0 + WG_CHUNK; kk += 16) {
        uint32_t a[4];
        a[0] = ld_u32(D + (size_t)g * B + kk + 2 * t);
        a[1] = ld_u32(D + (size_t)(g + 8) * B + kk + 2 * t);
        a[2] = ld_u32(D + (size_t)g * B + kk + 8 + 2 * t);
        a[3] = ld_u32(D + (size_t)(g + 8) * B + kk + 8 + 2 * t);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const __nv_bfloat16* hr = H + (size_t)(8 * j + g) * B + kk + 2 * t;
            mma_bf16(c[j], a, ld_u32(hr), ld_u32(hr + 8));
        }
    }
    int off = l == 0 ? OFF_W0 : l == 1 ? OFF_W1 : l == 2 ? OFF_W2 : OFF_W3;
    float* gw = grad + off;
    int o0 = 16 * warp + g;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        atomicAdd(gw + o0 * NIN + 8 * j + 2 * t, c[j][0]);
        atomicAdd(gw + o0 * NIN + 8 * j + 2 * t + 1, c[j][1]);
        atomicAdd(gw + (o0 + 8) * NIN + 8 * j + 2 * t, c[j][2]);
        atomicAdd(gw + (o0 + 8) * NIN + 8 * j + 2 * t + 1, c[j][3]);
    }
}

// Adam (Kingma & Ba 2015) with bias-corrected moments; refreshes the bf16 weights
__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, size_t n, float lr, float b1, float b2, float eps, float bc1,
                       float bc2, __nv_bfloat16* __restrict__ wbf, __nv_bfloat16* __restrict__ tbf) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = __fadd_rn(__fmul_rn(b1, m[i]), __fmul_rn(1.0f - b1, gi));
        float vi = __fadd_rn(__fmul_rn(b2, v[i]), __fmul_rn(1.0f - b2, __fmul_rn(gi, gi)));
        m[i] = mi;
        v[i] = vi;
        float step = __fdiv_rn(__fmul_rn(lr, __fdiv_rn(mi, bc1)), __fadd_rn(__fsqrt_rn(__fdiv_rn(vi, bc2)), eps));
        float pi = __fsub_rn(p[i], step);
        p[i] = pi;
        if (i < (size_t)N_MLP) wbf[i] = __float2bfloat16_rn(pi);
        else tbf[i - N_MLP] = __float2bfloat16_rn(pi);
    }
}

// bf16 copies of the weights and of the table from the fp32 parameters
__global__ void k_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ wbf,
                          __nv_bfloat16* __restrict__ tbf) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N_PARAMS; i += (size_t)gridDim.x * blockDim.x) {
        if (i < (size_t)N_MLP) wbf[i] = __float2bfloat16_rn(p[i]);
        else tbf[i - N_MLP] = __float2bfloat16_rn(p[i]);
    }
}

size_t api_smem() { return (size_t)W_SMEM * 2 + (size_t)GW * (32 * LDW * 2 + 16 * LDO * 4); }
size_t train_smem() {
    return (size_t)(W_SMEM + WT_SMEM) * 2 +
           (size_t)GW * (32 * LDW * 2 + 16 * LDW * 2 + 16 * LDT3 * 2 + 64 * ST * 2 + 16 * LDO * 4 + 16 * LDX * 4);
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

namespace rtgh {

struct Guide {
    RtGuideParams prm{};
    int mode = 0;
    float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16* wbf = nullptr;
    __nv_bfloat16* tbf = nullptr;     // bf16 copy of the table (the encodings read it)
    __nv_bfloat16* act = nullptr;
    uint32_t act_batch = 0;
    float4* gpar = nullptr;
    uint4* enc = nullptr;            // encoded inputs of the diffuse queue (128 B per path slot)
    uint32_t gpar_cap = 0;
    float4 *rec_a = nullptr, *rec_b = nullptr, *rec_c = nullptr;
    float2* rec_o = nullptr;
    float* rec_w = nullptr;
    uint32_t* counters = nullptr;   // records, training samples
    float4* train = nullptr;
    float* loss = nullptr;
    uint32_t rec_cap = 0;
    int64_t steps = 0, records = 0, samples = 0;
    double train_ms = 0.0;
    float lo[3], inv[3];
    uint32_t res[LEVELS];
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

void destroy(Guide* g) {
    if (!g) return;
    void* ptrs[] = {g->params, g->grad, g->m, g->v, g->wbf, g->tbf, g->act, g->gpar, g->enc, g->rec_a, g->rec_b, g->rec_c, g->rec_o,
                    g->rec_w, g->counters, g->train, g->loss};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (g->e0) cudaEventDestroy(g->e0);
    if (g->e1) cudaEventDestroy(g->e1);
    delete g;
}

static bool alloc_act(Guide* g, uint32_t batch) {
    if (g->act_batch >= batch) return true;
    if (g->act) cudaFree(g->act);
    g->act = nullptr;
    g->act_batch = 0;
    if (cudaMalloc(&g->act, (size_t)ACT_ROWS * batch * 2) != cudaSuccess) return false;
    g->act_batch = batch;
    return true;
}

Guide* create(const RtGuideParams& p, const float scene_lo[3], const float scene_hi[3], std::string* err) {
    Guide* g = new Guide();
    g->prm = p;
    bool use_scene = p.domain_min[0] == p.domain_max[0] && p.domain_min[1] == p.domain_max[1] &&
                     p.domain_min[2] == p.domain_max[2];
    for (int a = 0; a < 3; a++) {
        float lo = use_scene ? scene_lo[a] : p.domain_min[a];
        float hi = use_scene ? scene_hi[a] : p.domain_max[a];
        float ext = hi - lo;
        if (!(ext > 0.0f) || !std::isfinite(ext)) ext = 1.0f;
        g->lo[a] = lo;
        g->inv[a] = 1.0f / ext;
    }
    double r = p.min_resolution;
    for (int l = 0; l < LEVELS; l++) {
        g->res[l] = (uint32_t)std::max(2.0, std::floor(r));
        r *= p.level_scale;
    }
    g->rec_cap = p.record_capacity;
    bool ok = cudaMalloc(&g->params, N_PARAMS * 4) == cudaSuccess && cudaMalloc(&g->grad, N_PARAMS * 4) == cudaSuccess &&
              cudaMalloc(&g->m, N_PARAMS * 4) == cudaSuccess && cudaMalloc(&g->v, N_PARAMS * 4) == cudaSuccess &&
              cudaMalloc(&g->wbf, N_MLP * 2) == cudaSuccess && cudaMalloc(&g->tbf, N_TABLE * 2) == cudaSuccess &&
              cudaMalloc(&g->counters, 16) == cudaSuccess &&
              cudaMalloc(&g->loss, 4) == cudaSuccess &&
              cudaMalloc(&g->rec_a, (size_t)g->rec_cap * 16) == cudaSuccess &&
              cudaMalloc(&g->rec_b, (size_t)g->rec_cap * 16) == cudaSuccess &&
              cudaMalloc(&g->rec_c, (size_t)g->rec_cap * 16) == cudaSuccess &&
              cudaMalloc(&g->rec_o, (size_t)g->rec_cap * 8) == cudaSuccess &&
              cudaMalloc(&g->rec_w, (size_t)g->rec_cap * 4) == cudaSuccess &&
              cudaMalloc(&g->train, (size_t)g->rec_cap * 48) == cudaSuccess && alloc_act(g, p.batch) &&
              cudaEventCreate(&g->e0) == cudaSuccess && cudaEventCreate(&g->e1) == cudaSuccess;
    if (!ok) {
        *err = "cudaMalloc guide state";
        destroy(g);
        return nullptr;
    }
    // initial parameters: Glorot-uniform weights (output rows 41..47 zero), table U(−1e-4, 1e-4)
    std::vector<float> h(N_PARAMS);
    uint64_t s = p.seed;
    auto uni = [&]() { return (float)((splitmix(s) >> 40) * (1.0 / 16777216.0)) * 2.0f - 1.0f; };
    for (int l = 0; l < 4; l++) {
        int off = l * NHID * NIN, rows = l == 3 ? NOUTP : NHID, fan_out = l == 3 ? NOUT : NHID;
        float lim = std::sqrt(6.0f / (float)(NIN + fan_out));
        for (int o = 0; o < rows; o++)
            for (int i = 0; i < NIN; i++) h[off + o * NIN + i] = (l == 3 && o >= NOUT) ? 0.0f : lim * uni();
    }
    for (size_t i = N_MLP; i < N_PARAMS; i++) h[i] = 1e-4f * uni();
    if (cudaMemcpy(g->params, h.data(), N_PARAMS * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(g->m, 0, N_PARAMS * 4) != cudaSuccess || cudaMemset(g->v, 0, N_PARAMS * 4) != cudaSuccess ||
        cudaMemset(g->counters, 0, 16) != cudaSuccess) {
        *err = "guide parameter upload";
        destroy(g);
        return nullptr;
    }
    k_to_bf16<<<1024, 256>>>(g->params, g->wbf, g->tbf);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        *err = "guide initialisation";
        destroy(g);
        return nullptr;
    }
    if (cudaFuncSetAttribute(k_guide_api, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)api_smem()) ||
        cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem())) {
        *err = "guide kernels: shared-memory opt-in";
        destroy(g);
        return nullptr;
    }
    return g;
}

void set_mode(Guide* g, int mode) { g->mode = mode; }
int mode(const Guide* g) { return g ? g->mode : 0; }

GuideDev view(const Guide* g) {
    GuideDev d{};
    if (!g) return d;
    d.mode = g->mode;
    d.table = g->params + N_MLP;
    d.tbf = reinterpret_cast<const __nv_bfloat162*>(g->tbf);
    d.wbf = g->wbf;
    for (int a = 0; a < 3; a++) { d.lo[a] = g->lo[a]; d.inv[a] = g->inv[a]; }
    for (int l = 0; l < LEVELS; l++) d.res[l] = g->res[l];
    d.amax = g->prm.alpha_max;
    d.lkmax = g->prm.log_kappa_max;
    d.gpar = g->gpar;
    d.enc = g->enc;
    d.rec_a = g->rec_a; d.rec_b = g->rec_b; d.rec_c = g->rec_c; d.rec_o = g->rec_o; d.rec_w = g->rec_w;
    d.rec_count = g->counters;
    d.rec_cap = g->rec_cap;
    return d;
}

int ensure_paths(Guide* g, uint32_t cap) {
    if (g->gpar_cap >= cap) return 0;
    if (g->gpar) cudaFree(g->gpar);
    if (g->enc) cudaFree(g->enc);
    g->gpar = nullptr;
    g->enc = nullptr;
    g->gpar_cap = 0;
    if (cudaMalloc(&g->gpar, (size_t)cap * GP_F4 * sizeof(float4)) != cudaSuccess) return -1;
    if (cudaMalloc(&g->enc, (size_t)cap * 8 * sizeof(uint4)) != cudaSuccess) return -1;
    g->gpar_cap = cap;
    return 0;
}

cudaError_t params_io(Guide* g, float* host, int write, cudaStream_t st) {
    cudaError_t e;
    if (write) {
        if ((e = cudaMemcpyAsync(g->params, host, N_PARAMS * 4, cudaMemcpyHostToDevice, st))) return e;
        if ((e = cudaMemsetAsync(g->m, 0, N_PARAMS * 4, st))) return e;
        if ((e = cudaMemsetAsync(g->v, 0, N_PARAMS * 4, st))) return e;
        g->steps = 0;
        k_to_bf16<<<1024, 256, 0, st>>>(g->params, g->wbf, g->tbf);
        return cudaGetLastError();
    }
    if ((e = cudaMemcpyAsync(host, g->params, N_PARAMS * 4, cudaMemcpyDeviceToHost, st))) return e;
    return cudaStreamSynchronize(st);
}

void eval(Guide* g, const float* q, uint32_t n, const float* dirs, const float* u, float* raw, float* out, int sms,
          cudaStream_t st) {
    if (n == 0) return;
    uint32_t blocks = std::min<uint32_t>((n + GW * 32 - 1) / (GW * 32), (uint32_t)sms * 4);
    k_guide_api<<<blocks, GW * 32, api_smem(), st>>>(view(g), q, n, dirs, u, raw, out);
}

// one forward/backward pass and, if `adam`, one Adam step
static cudaError_t step(Guide* g, const TrainArgs& a0, bool adam, int sms, cudaStream_t st) {
    cudaError_t e;
    TrainArgs a = a0;
    a.act = g->act;
    a.grad = g->grad;
    a.loss = g->loss;
    if ((e = cudaMemsetAsync(g->grad, 0, N_PARAMS * 4, st))) return e;
    uint32_t blocks = std::min<uint32_t>(a.batch / (GW * 32), (uint32_t)sms * 2);
    k_train<<<blocks, GW * 32, train_smem(), st>>>(view(g), a);
    k_wgrad<<<dim3(a.batch / WG_CHUNK, 4), GW * 32, 0, st>>>(g->act, a.batch, g->grad);
    if (adam) {
        g->steps++;
        float b1 = g->prm.beta1, b2 = g->prm.beta2;
        float bc1 = (float)(1.0 - std::pow((double)b1, (double)g->steps));
        float bc2 = (float)(1.0 - std::pow((double)b2, (double)g->steps));
        k_adam<<<sms * 8, 256, 0, st>>>(g->params, g->m, g->v, g->grad, N_PARAMS, g->prm.learning_rate, b1, b2,
                                        g->prm.epsilon, bc1, bc2, g->wbf, g->tbf);
    }
    return cudaGetLastError();
}

// explicit samples (device, 3 float4 each): `steps` Adam steps over the whole
// set (steps = 0: gradient only, left in the gradient buffer)
cudaError_t train_explicit(Guide* g, const float4* samples, uint32_t n, int steps, float* loss_host, int sms,
                           cudaStream_t st) {
    uint32_t batch = std::max<uint32_t>(WG_CHUNK, (n + WG_CHUNK - 1) / WG_CHUNK * WG_CHUNK);
    if (!alloc_act(g, batch)) return cudaErrorMemoryAllocation;
    TrainArgs a{};
    a.samples = samples;
    a.n = n;
    a.batch = batch;
    a.select = 0;
    cudaError_t e;
    int runs = std::max(steps, 1);
    for (int i = 0; i < runs; i++) {
        if ((e = cudaMemsetAsync(g->loss, 0, 4, st))) return e;
        if ((e = step(g, a, steps > 0, sms, st))) return e;
    }
    if (loss_host) {
        if ((e = cudaMemcpyAsync(loss_host, g->loss, 4, cudaMemcpyDeviceToHost, st))) return e;
    }
    return cudaStreamSynchronize(st);
}

cudaError_t grad_out(Guide* g, float* host, cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(host, g->grad, N_PARAMS * 4, cudaMemcpyDeviceToHost, st);
    if (e) return e;
    return cudaStreamSynchronize(st);
}

cudaError_t begin_pass(Guide* g, cudaStream_t st) {
    if (g->mode != 2) return cudaSuccess;
    return cudaMemsetAsync(g->counters, 0, 8, st);
}

// after a training render call: compact the weighted records, then Adam steps
// on minibatches drawn from them
cudaError_t train_pass(Guide* g, int sms, cudaStream_t st, int64_t* launches) {
    if (g->mode != 2) return cudaSuccess;
    cudaError_t e;
    cudaEventRecord(g->e0, st);
    k_compact<<<sms * 8, 256, 0, st>>>(g->rec_a, g->rec_b, g->rec_c, g->rec_o, g->rec_w, g->counters, g->rec_cap, g->train,
                                       g->counters + 1);
    uint32_t cnt[2];
    if ((e = cudaMemcpyAsync(cnt, g->counters, 8, cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaStreamSynchronize(st))) return e;
    g->records += std::min(cnt[0], g->rec_cap);
    g->samples += cnt[1];
    if (launches) *launches += 1 + (cnt[1] > 0 ? 3 * (int64_t)g->prm.steps_per_pass : 0);
    if (cnt[1] > 0) {
        uint32_t batch = std::max<uint32_t>(WG_CHUNK, g->prm.batch / WG_CHUNK * WG_CHUNK);
        if (!alloc_act(g, batch)) return cudaErrorMemoryAllocation;
        for (uint32_t i = 0; i < g->prm.steps_per_pass; i++) {
            TrainArgs a{};
            a.samples = g->train;
            a.n_dev = g->counters + 1;
            a.batch = batch;
            a.select = 1;
            a.seed = mix32((uint32_t)g->prm.seed ^ mix32((uint32_t)g->steps + 1u));
            if ((e = cudaMemsetAsync(g->loss, 0, 4, st))) return e;
            if ((e = step(g, a, true, sms, st))) return e;
        }
    }
    cudaEventRecord(g->e1, st);
    if ((e = cudaEventSynchronize(g->e1))) return e;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, g->e0, g->e1);
    g->train_ms += ms;
    return cudaGetLastError();
}

void stats(const Guide* g, int64_t* records, int64_t* samples, int64_t* steps, double* ms) {
    if (records) *records = g->records;
    if (samples) *samples = g->samples;
    if (steps) *steps = g->steps;
    if (ms) *ms = g->train_ms;
}

}  // namespace rtgh
