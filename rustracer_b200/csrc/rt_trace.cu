// rt_trace.cu — 8-wide BVH traversal kernels (closest hit, any hit).
//
// Compiled with --fmad=false: the reference (Rust) never fuses a*b+c, and the
// hit ids / t values must be bit-identical to that arithmetic, so no FFMA may
// appear in the primitive tests.  The slab test is FSUB+FMUL+FMNMX only.
//
// Traversal (replaces BvhTree::hit_index, src/bvh.rs:229-288, and the AVX2
// slab test :326-364): one ray per lane in persistent warps; lanes that finish
// pull new rays as soon as enough of the warp is idle (lane refill), which keeps
// SIMD lanes busy across very uneven ray costs.
// Per node the thread issues 14 128-bit loads (224 B, the reference node),
// tests all 8 child boxes, intersects hit leaves immediately (closest-t
// first-wins, ties → smaller canonical id), then sorts the hit inner children
// by entry distance with a 19-comparator network on packed (t | slot) keys and
// continues with the nearest while the others go on a per-thread stack.
#include <algorithm>

#include <cub/block/block_scan.cuh>

#include "rt_internal.h"
#include "rt_media.cuh"

using namespace rtd;

namespace {

struct Best { float t, b1, b2; uint32_t ref, gid, mat; };

RT_D uint32_t f2u(float f) { return __float_as_uint(f); }

// Leaf test for one reference; updates `best` and returns nothing.
// ANA: the scene has convex solids or shapes; without them the type-3 branch
// is compiled out, so triangle scenes keep a lean traversal kernel.
template <bool ANA>
RT_D void leaf_closest(const DevScene& S, uint32_t ref, float3 o, float3 d, float tmin, Best& best) {
    uint32_t type = (ref >> 28) & 7u, idx = ref & 0x0FFFFFFFu;
    float t, b1, b2;
    uint32_t gid, mat;
    bool h;
    if (type == RT_PRIM_TRI) {
        const float4* g = S.tri + (size_t)idx * 3;
        float4 a = __ldg(g), b = __ldg(g + 1), c = __ldg(g + 2);
        h = tri_test(a, b, c, o, d, tmin, best.t, &t, &b1, &b2);
        gid = f2u(c.y);
        mat = f2u(c.z);
    } else if (type == RT_PRIM_QUAD) {
        const float4* g = S.quad + (size_t)idx * 5;
        float4 gg[4] = {__ldg(g), __ldg(g + 1), __ldg(g + 2), __ldg(g + 3)};
        h = quad_test(gg, o, d, tmin, best.t, &t, &b1, &b2);
        float4 gm = h ? __ldg(g + 4) : make_float4(0.f, 0.f, 0.f, 0.f);
        gid = f2u(gm.x);
        mat = f2u(gm.y);
    } else if (type == RT_PRIM_SPHERE) {
        const float4* g = S.sphere + (size_t)idx * 2;
        h = sphere_test(__ldg(g), o, d, tmin, best.t, &t);
        b1 = b2 = 0.0f;
        float4 gm = h ? __ldg(g + 1) : make_float4(0.f, 0.f, 0.f, 0.f);
        gid = f2u(gm.x);
        mat = f2u(gm.y);
    } else if (!ANA) {
        return;
    } else {                                        // convex solid or shape; b1 carries the plane / surface
        float4 c0 = __ldg(S.cvx + (size_t)idx * 2);
        int pi = -1, cnt = __float_as_int(c0.y);
        if (cnt > 0) {
            h = convex_test(S.cvx_planes + __float_as_int(c0.x), cnt, o, d, tmin, best.t, &t, &pi);
        } else {
            const float4* P = S.shape_par + __float_as_int(c0.x);
            float3 lo, ld;
            shape_local(P, o, d, &lo, &ld);
            h = shape_test(-1 - cnt, P, lo, ld, tmin, best.t, &t, &pi);
        }
        b1 = __int_as_float(pi);
        b2 = 0.0f;
        gid = h ? f2u(__ldg(S.cvx + (size_t)idx * 2 + 1).x) : 0u;
        mat = f2u(c0.z);
    }
    if (h && (t < best.t || best.ref == RT_MISS_REF || gid < best.gid)) {
        best.t = t; best.b1 = b1; best.b2 = b2; best.ref = ref; best.gid = gid; best.mat = mat;
    }
}

template <bool ANA>
RT_D bool leaf_any(const DevScene& S, uint32_t ref, float3 o, float3 d, float tmin, float tmax) {
    uint32_t type = (ref >> 28) & 7u, idx = ref & 0x0FFFFFFFu;
    float t, b1, b2;
    if (type == RT_PRIM_TRI) {
        const float4* g = S.tri + (size_t)idx * 3;
        return tri_test(__ldg(g), __ldg(g + 1), __ldg(g + 2), o, d, tmin, tmax, &t, &b1, &b2);
    } else if (type == RT_PRIM_QUAD) {
        const float4* g = S.quad + (size_t)idx * 5;
        float4 gg[4] = {__ldg(g), __ldg(g + 1), __ldg(g + 2), __ldg(g + 3)};
        return quad_test(gg, o, d, tmin, tmax, &t, &b1, &b2);
    }
    if (type == RT_PRIM_SPHERE) return sphere_test(__ldg(S.sphere + (size_t)idx * 2), o, d, tmin, tmax, &t);
    if (!ANA) return false;
    float4 c0 = __ldg(S.cvx + (size_t)idx * 2);
    int pi, cnt = __float_as_int(c0.y);
    if (cnt > 0) return convex_test(S.cvx_planes + __float_as_int(c0.x), cnt, o, d, tmin, tmax, &t, &pi);
    const float4* P = S.shape_par + __float_as_int(c0.x);
    float3 lo, ld;
    shape_local(P, o, d, &lo, &ld);
    return shape_test(-1 - cnt, P, lo, ld, tmin, tmax, &t, &pi);
}

#ifndef RT_MNMX3
#define RT_MNMX3 1
#endif
#ifndef RT_EMPTY_INVERTED
#define RT_EMPTY_INVERTED 1
#endif
// three-input min / max (sm_100)
RT_D float fmax3f(float a, float b, float c) {
#if RT_MNMX3
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
#else
    return fmaxf(fmaxf(a, b), c);
#endif
}
RT_D float fmin3f(float a, float b, float c) {
#if RT_MNMX3
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
#else
    return fminf(fminf(a, b), c);
#endif
}

#define CAS(a, b) { uint32_t lo_ = min(k[a], k[b]); uint32_t hi_ = max(k[a], k[b]); k[a] = lo_; k[b] = hi_; }

// Per-ray slab constants.  Fast path (every direction component non-zero and
// t_min ≥ 0): the near and far planes of each axis are chosen once per ray from
// the sign of the direction, so a child costs 6 FSUB + 6 FMUL + 6 FMNMX.  The
// far-plane reciprocal is widened by 2^-15, which after the two roundings of
// (b − o)·inv still exceeds the exact exit distance by ≥ 2^-16 relative — the
// culling stays conservative, so any layout returns the brute-force answer.
// General path (a zero or denormal component, or t_min < 0): both planes with
// min/max, a NaN slab (ray lying in a face plane) spanning the whole line, and
// the exit widened explicitly.
struct RayC {
    float3 o, inv, invf;
    int nx, ny, nz;          // float4 offsets of the near-plane arrays in a node
    bool general;
    bool qgeneral;           // quantised nodes: also any |1/d| outside [2^-60, 2^60]
};

RT_D bool inv_in_range(float x) {
    float a = fabsf(x);
    return a >= 8.673617379884035e-19f && a <= 1.152921504606846976e18f;   // 2^-60 .. 2^60
}

RT_D RayC make_rayc(float3 o, float3 d, float tmin) {
    RayC r;
    r.o = o;
    r.inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    const float W = 1.000030517578125f;   // 1 + 2^-15
    r.invf = mk(r.inv.x * W, r.inv.y * W, r.inv.z * W);
    r.general = isinf(r.inv.x) || isinf(r.inv.y) || isinf(r.inv.z) || !(tmin >= 0.0f);
    r.qgeneral = r.general || !inv_in_range(r.inv.x) || !inv_in_range(r.inv.y) || !inv_in_range(r.inv.z);
    r.nx = signbit(r.inv.x) ? 6 : 0;
    r.ny = signbit(r.inv.y) ? 8 : 2;
    r.nz = signbit(r.inv.z) ? 10 : 4;
    return r;
}

__device__ __noinline__ uint32_t node_test_general(const DevScene& S, uint32_t ni, const RayC& R, float tmin,
                                                   float tmax, float* tn);

// Slab test of the 8 children of node `ni` against [tmin, tmax]; returns the
// hit mask and the entry distances.
RT_D uint32_t node_test(const DevScene& S, uint32_t ni, const RayC& R, float tmin, float tmax, float tn[8],
                        uint32_t ch[8]) {
    const float4* N = S.nodes + (size_t)ni * 14;
    uint32_t mask = 0;
    float4 c0 = __ldg(N + 12), c1 = __ldg(N + 13);
    const uint32_t cc[8] = {__float_as_uint(c0.x), __float_as_uint(c0.y), __float_as_uint(c0.z), __float_as_uint(c0.w),
                            __float_as_uint(c1.x), __float_as_uint(c1.y), __float_as_uint(c1.z), __float_as_uint(c1.w)};
#pragma unroll
    for (int c = 0; c < 8; c++) ch[c] = cc[c];
    if (!R.general) {
        float4 q[12];
        q[0] = __ldg(N + R.nx); q[1] = __ldg(N + R.nx + 1);
        q[2] = __ldg(N + R.ny); q[3] = __ldg(N + R.ny + 1);
        q[4] = __ldg(N + R.nz); q[5] = __ldg(N + R.nz + 1);
        q[6] = __ldg(N + 6 - R.nx); q[7] = __ldg(N + 7 - R.nx);
        q[8] = __ldg(N + 10 - R.ny); q[9] = __ldg(N + 11 - R.ny);
        q[10] = __ldg(N + 14 - R.nz); q[11] = __ldg(N + 15 - R.nz);
        const float* f = reinterpret_cast<const float*>(q);
#pragma unroll
        for (int c = 0; c < 8; c++) {
            float nx = (f[0 + c] - R.o.x) * R.inv.x, fx = (f[24 + c] - R.o.x) * R.invf.x;
            float ny = (f[8 + c] - R.o.y) * R.inv.y, fy = (f[32 + c] - R.o.y) * R.invf.y;
            float nz = (f[16 + c] - R.o.z) * R.inv.z, fz = (f[40 + c] - R.o.z) * R.invf.z;
            float t0 = fmax3f(fmaxf(tmin, nx), ny, nz);
            float t1 = fmin3f(fminf(tmax, fx), fy, fz);
            tn[c] = t0;
#if RT_EMPTY_INVERTED
            if (t0 <= t1) mask |= 1u << c;     // empty slots hold inverted boxes
#else
            if (t0 <= t1 && ch[c] != RT_EMPTY_REF) mask |= 1u << c;
#endif
        }
        return mask;
    }
    float tg[8];
    mask = node_test_general(S, ni, R, tmin, tmax, tg);
#pragma unroll
    for (int c = 0; c < 8; c++) tn[c] = tg[c];
    return mask;
}

__device__ __noinline__ uint32_t node_test_general(const DevScene& S, uint32_t ni, const RayC& R, float tmin,
                                                   float tmax, float* tn) {
    const float4* N = S.nodes + (size_t)ni * 14;
    uint32_t mask = 0;
    float4 q[14];
#pragma unroll
    for (int i = 0; i < 14; i++) q[i] = __ldg(N + i);
    const float* f = reinterpret_cast<const float*>(q);
    const uint32_t* ch = reinterpret_cast<const uint32_t*>(f + 48);
#pragma unroll
    for (int c = 0; c < 8; c++) {
        float dax = (f[0 + c] - R.o.x) * R.inv.x, dbx = (f[24 + c] - R.o.x) * R.inv.x;
        float day = (f[8 + c] - R.o.y) * R.inv.y, dby = (f[32 + c] - R.o.y) * R.inv.y;
        float daz = (f[16 + c] - R.o.z) * R.inv.z, dbz = (f[40 + c] - R.o.z) * R.inv.z;
        float lx = fminf(dax, dbx), hx = fmaxf(dax, dbx);
        float ly = fminf(day, dby), hy = fmaxf(day, dby);
        float lz = fminf(daz, dbz), hz = fmaxf(daz, dbz);
        if (isnan(dax) || isnan(dbx)) { lx = -INFINITY; hx = INFINITY; }
        if (isnan(day) || isnan(dby)) { ly = -INFINITY; hy = INFINITY; }
        if (isnan(daz) || isnan(dbz)) { lz = -INFINITY; hz = INFINITY; }
        float t0 = fmaxf(fmaxf(fmaxf(tmin, lx), ly), lz);
        float t1 = fminf(fminf(fminf(tmax, hx), hy), hz);
        float t1w = t1 + fabsf(t1) * SLAB_WIDEN;
        tn[c] = t0;
        if (t0 <= t1w && ch[c] != RT_EMPTY_REF) mask |= 1u << c;
    }
    return mask;
}

// ── quantised nodes (8 float4: see encode_qnode in rt_host.cu) ───────────────
// Child planes are the real numbers p + q·s (s = 2^e per axis), which contain
// the exact child boxes.  Per ray and node, S = s/d is exact and
// A = (p − o)/d is computed with two roundings; q·S + A then differs from the
// exact plane distance by at most u·(255|S| + 3.02|A|) (u = 2^-24), so with
// err = 2^-20·(|A| + 256|S|) the near distance fma(2^23 + q, S, A − err − 2^23·S)
// rounded down is below it and the far one rounded up is above it: the
// culling stays conservative and the hits are the brute-force ones.  The
// byte q enters as the float 2^23 + q (one byte permute), its 2^23 folded
// into the per-node constant.
RT_D float qbyte(uint32_t w, uint32_t sel) { return __uint_as_float(__byte_perm(w, 0x4B000000u, sel)); }

__device__ __noinline__ uint32_t qnode_test_general(const DevScene& S, uint32_t ni, const RayC& R, float tmin,
                                                    float tmax, float* tn);

RT_D uint32_t qnode_test(const DevScene& S, uint32_t ni, const RayC& R, float tmin, float tmax, float tn[8],
                         uint32_t ch[8]) {
    const float4* N = S.qnodes + (size_t)ni * 8;
    float4 h = __ldg(N);
    uint4 bq[3] = {__ldg(reinterpret_cast<const uint4*>(N + 1)), __ldg(reinterpret_cast<const uint4*>(N + 2)),
                   __ldg(reinterpret_cast<const uint4*>(N + 3))};
    float4 c0 = __ldg(N + 4), c1 = __ldg(N + 5);
    const uint32_t cc[8] = {__float_as_uint(c0.x), __float_as_uint(c0.y), __float_as_uint(c0.z), __float_as_uint(c0.w),
                            __float_as_uint(c1.x), __float_as_uint(c1.y), __float_as_uint(c1.z), __float_as_uint(c1.w)};
#pragma unroll
    for (int c = 0; c < 8; c++) ch[c] = cc[c];
    const uint32_t meta = __float_as_uint(h.w);
    if (R.qgeneral) {
        float tg[8];
        uint32_t m = qnode_test_general(S, ni, R, tmin, tmax, tg);
#pragma unroll
        for (int c = 0; c < 8; c++) tn[c] = tg[c];
        return m;
    }
    const float M = 8388608.0f;                        // 2^23
    const float P[3] = {h.x, h.y, h.z}, O[3] = {R.o.x, R.o.y, R.o.z}, I[3] = {R.inv.x, R.inv.y, R.inv.z};
    float Sa[3], An[3], Af[3];
    uint32_t wn[3][2], wf[3][2];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float sa = __uint_as_float(((meta >> (8 * a)) & 0xFFu) << 23);   // 2^e
        float Sx = sa * I[a];
        float Ax = (P[a] - O[a]) * I[a];
        float err = __fmul_ru(__fmaf_ru(fabsf(Sx), 256.0f, fabsf(Ax)), 9.5367431640625e-07f);   // × 2^-20
        An[a] = __fmaf_rd(-M, Sx, __fsub_rd(Ax, err));
        Af[a] = __fmaf_ru(-M, Sx, __fadd_ru(Ax, err));
        Sa[a] = Sx;
        // the near planes are the lower ones for a positive direction
        bool neg = I[a] < 0.0f;
        wn[a][0] = neg ? bq[a].z : bq[a].x; wn[a][1] = neg ? bq[a].w : bq[a].y;
        wf[a][0] = neg ? bq[a].x : bq[a].z; wf[a][1] = neg ? bq[a].y : bq[a].w;
    }
    uint32_t mask = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const uint32_t sel = 0x7540u + (uint32_t)(c & 3);
        float nx = __fmaf_rd(qbyte(wn[0][c >> 2], sel), Sa[0], An[0]);
        float ny = __fmaf_rd(qbyte(wn[1][c >> 2], sel), Sa[1], An[1]);
        float nz = __fmaf_rd(qbyte(wn[2][c >> 2], sel), Sa[2], An[2]);
        float fx = __fmaf_ru(qbyte(wf[0][c >> 2], sel), Sa[0], Af[0]);
        float fy = __fmaf_ru(qbyte(wf[1][c >> 2], sel), Sa[1], Af[1]);
        float fz = __fmaf_ru(qbyte(wf[2][c >> 2], sel), Sa[2], Af[2]);
        float t0 = fmax3f(fmaxf(tmin, nx), ny, nz);
        float t1 = fmin3f(fminf(tmax, fx), fy, fz);
        tn[c] = t0;
        if (t0 <= t1) mask |= 1u << c;
    }
    return mask & (meta >> 24);
}

// General rays (a zero, denormal or extreme direction component, or t_min < 0):
// the planes decoded with outward rounding, then the general slab test.
__device__ __noinline__ uint32_t qnode_test_general(const DevScene& S, uint32_t ni, const RayC& R, float tmin,
                                                    float tmax, float* tn) {
    const float4* N = S.qnodes + (size_t)ni * 8;
    float4 h = __ldg(N);
    const uint32_t meta = __float_as_uint(h.w);
    const float P[3] = {h.x, h.y, h.z};
    float lo[3][8], hi[3][8];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        uint4 b = __ldg(reinterpret_cast<const uint4*>(N + 1 + a));
        float sa = __uint_as_float(((meta >> (8 * a)) & 0xFFu) << 23);
#pragma unroll
        for (int c = 0; c < 8; c++) {
            uint32_t wl = c < 4 ? b.x : b.y, wh = c < 4 ? b.z : b.w;
            float ql = (float)((wl >> (8 * (c & 3))) & 0xFFu), qh = (float)((wh >> (8 * (c & 3))) & 0xFFu);
            lo[a][c] = __fmaf_rd(ql, sa, P[a]);
            hi[a][c] = __fmaf_ru(qh, sa, P[a]);
        }
    }
    uint32_t mask = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        float dax = (lo[0][c] - R.o.x) * R.inv.x, dbx = (hi[0][c] - R.o.x) * R.inv.x;
        float day = (lo[1][c] - R.o.y) * R.inv.y, dby = (hi[1][c] - R.o.y) * R.inv.y;
        float daz = (lo[2][c] - R.o.z) * R.inv.z, dbz = (hi[2][c] - R.o.z) * R.inv.z;
        float lx = fminf(dax, dbx), hx = fmaxf(dax, dbx);
        float ly = fminf(day, dby), hy = fmaxf(day, dby);
        float lz = fminf(daz, dbz), hz = fmaxf(daz, dbz);
        if (isnan(dax) || isnan(dbx)) { lx = -INFINITY; hx = INFINITY; }
        if (isnan(day) || isnan(dby)) { ly = -INFINITY; hy = INFINITY; }
        if (isnan(daz) || isnan(dbz)) { lz = -INFINITY; hz = INFINITY; }
        float t0 = fmaxf(fmaxf(fmaxf(tmin, lx), ly), lz);
        float t1 = fminf(fminf(fminf(tmax, hx), hy), hz);
        float t1w = t1 + fabsf(t1) * SLAB_WIDEN;
        tn[c] = t0;
        if (t0 <= t1w) mask |= 1u << c;
    }
    return mask & (meta >> 24);
}

// ── 4-wide nodes (7 float4: lower x, y, z, upper x, y, z, references) ──────
__device__ __noinline__ uint32_t node4_test_general(const DevScene& S, uint32_t ni, const RayC& R, float tmin,
                                                    float tmax, float* tn);

RT_D uint32_t node4_test(const DevScene& S, uint32_t ni, const RayC& R, float tmin, float tmax, float tn[8],
                         uint32_t ch[8]) {
    const float4* N = S.nodes4 + (size_t)ni * 7;
    float4 c0 = __ldg(N + 6);
    ch[0] = __float_as_uint(c0.x); ch[1] = __float_as_uint(c0.y);
    ch[2] = __float_as_uint(c0.z); ch[3] = __float_as_uint(c0.w);
    if (!R.general) {
        // the near planes of an axis are the lower ones for a positive direction
        // (R.nx / 2 is 0 or 3, R.ny / 2 is 1 or 4, R.nz / 2 is 2 or 5)
        float4 q[6];
        q[0] = __ldg(N + R.nx / 2); q[1] = __ldg(N + R.ny / 2); q[2] = __ldg(N + R.nz / 2);
        q[3] = __ldg(N + 3 - R.nx / 2); q[4] = __ldg(N + 5 - R.ny / 2); q[5] = __ldg(N + 7 - R.nz / 2);
        const float* f = reinterpret_cast<const float*>(q);
        uint32_t mask = 0;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            float nx = (f[0 + c] - R.o.x) * R.inv.x, fx = (f[12 + c] - R.o.x) * R.invf.x;
            float ny = (f[4 + c] - R.o.y) * R.inv.y, fy = (f[16 + c] - R.o.y) * R.invf.y;
            float nz = (f[8 + c] - R.o.z) * R.inv.z, fz = (f[20 + c] - R.o.z) * R.invf.z;
            float t0 = fmax3f(fmaxf(tmin, nx), ny, nz);
            float t1 = fmin3f(fminf(tmax, fx), fy, fz);
            tn[c] = t0;
            if (t0 <= t1) mask |= 1u << c;     // empty slots hold inverted boxes
        }
        return mask;
    }
    float tg[4];
    uint32_t mask = node4_test_general(S, ni, R, tmin, tmax, tg);
#pragma unroll
    for (int c = 0; c < 4; c++) tn[c] = tg[c];
    return mask;
}

__device__ __noinline__ uint32_t node4_test_general(const DevScene& S, uint32_t ni, const RayC& R, float tmin,
                                                    float tmax, float* tn) {
    const float4* N = S.nodes4 + (size_t)ni * 7;
    float4 q[7];
#pragma unroll
    for (int i = 0; i < 7; i++) q[i] = __ldg(N + i);
    const float* f = reinterpret_cast<const float*>(q);
    const uint32_t* ch = reinterpret_cast<const uint32_t*>(f + 24);
    uint32_t mask = 0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        float dax = (f[0 + c] - R.o.x) * R.inv.x, dbx = (f[12 + c] - R.o.x) * R.inv.x;
        float day = (f[4 + c] - R.o.y) * R.inv.y, dby = (f[16 + c] - R.o.y) * R.inv.y;
        float daz = (f[8 + c] - R.o.z) * R.inv.z, dbz = (f[20 + c] - R.o.z) * R.inv.z;
        float lx = fminf(dax, dbx), hx = fmaxf(dax, dbx);
        float ly = fminf(day, dby), hy = fmaxf(day, dby);
        float lz = fminf(daz, dbz), hz = fmaxf(daz, dbz);
        if (isnan(dax) || isnan(dbx)) { lx = -INFINITY; hx = INFINITY; }
        if (isnan(day) || isnan(dby)) { ly = -INFINITY; hy = INFINITY; }
        if (isnan(daz) || isnan(dbz)) { lz = -INFINITY; hz = INFINITY; }
        float t0 = fmaxf(fmaxf(fmaxf(tmin, lx), ly), lz);
        float t1 = fminf(fminf(fminf(tmax, hx), hy), hz);
        float t1w = t1 + fabsf(t1) * SLAB_WIDEN;
        tn[c] = t0;
        if (t0 <= t1w && ch[c] != RT_EMPTY_REF) mask |= 1u << c;
    }
    return mask;
}

// the node test and the child-reference words of node `ni` in the layout NF
// (RT_NODES_FULL, RT_NODES_QUANTISED, RT_NODES_WIDE4), and its width
template <int NF>
RT_D uint32_t node_test_any(const DevScene& S, uint32_t ni, const RayC& R, float tmin, float tmax, float tn[8],
                            uint32_t ch[8]) {
    if constexpr (NF == RT_NODES_QUANTISED) return qnode_test(S, ni, R, tmin, tmax, tn, ch);
    else if constexpr (NF == RT_NODES_WIDE4) return node4_test(S, ni, R, tmin, tmax, tn, ch);
    else return node_test(S, ni, R, tmin, tmax, tn, ch);
}
template <int NF>
RT_D const uint32_t* node_refs(const DevScene& S, uint32_t ni) {
    if constexpr (NF == RT_NODES_QUANTISED) return reinterpret_cast<const uint32_t*>(S.qnodes + (size_t)ni * 8 + 4);
    else if constexpr (NF == RT_NODES_WIDE4) return reinterpret_cast<const uint32_t*>(S.nodes4 + (size_t)ni * 7 + 6);
    else return reinterpret_cast<const uint32_t*>(S.nodes + (size_t)ni * 14 + 12);
}
template <int NF> constexpr int node_width() { return NF == RT_NODES_WIDE4 ? 4 : 8; }

}  // namespace

namespace rtk {

// Per-thread traversal stack (the reference keeps 128 entries inline and
// spills to a heap Vec, bvh.rs:229-239).  The newest RT_SHORT_STACK entries
// live in a ring: the thread's local memory (RT_STACK_LOCAL, the default) or
// shared memory laid out [entry][thread], so the lanes of a warp hit 32
// different banks whatever their depths.  Entry e ≥ RT_SHORT_STACK of a
// deeper stack waits in the thread's global column spill[(e − RT_SHORT_STACK)
// · stride] (rt_set_tuning can shrink the ring to fewer slots, so the tests
// run every traversal through the spill path).  A push beyond the ring first
// moves the ring slot's old entry to its column, a pop that uncovers a
// spilled entry brings it back.  `cap` (7 per tree level, sized at scene
// creation) is never reached by a traversal of the scene's own tree; a lower
// cap from rt_set_tuning makes the traversal stop with RT_ERR_CAPACITY.
constexpr int RING_STRIDE = RT_STACK_LOCAL ? 1 : RT_TRACE_BLOCK;
struct TStack {
    uint32_t* ring;          // ring slot k at ring[k · RING_STRIDE] (shared: &ring[threadIdx.x])
    uint32_t* spill;         // &S.stack_spill[global thread]; entry e at spill[(e − ring_n) · stride]
    uint32_t stride;
    int sp, cap;
    int ring_n;              // ring slots in use: RT_SHORT_STACK, or fewer (a power of two) when tuned

    RT_D bool room(int k) const { return sp + k <= cap; }
    RT_D void push(uint32_t v) {
        int slot = sp & (ring_n - 1);
        if (sp >= ring_n) spill[(size_t)(sp - ring_n) * stride] = ring[slot * RING_STRIDE];
        ring[slot * RING_STRIDE] = v;
        sp++;
    }
    RT_D uint32_t pop() {
        sp--;
        int slot = sp & (ring_n - 1);
        uint32_t v = ring[slot * RING_STRIDE];
        if (sp >= ring_n) ring[slot * RING_STRIDE] = spill[(size_t)(sp - ring_n) * stride];
        return v;
    }
};

RT_D TStack make_stack(const DevScene& S, uint32_t* ring_base) {
    TStack st;
    st.ring = RT_STACK_LOCAL ? ring_base : ring_base + threadIdx.x;
    st.stride = gridDim.x * blockDim.x;
    st.spill = S.stack_spill + blockIdx.x * blockDim.x + threadIdx.x;
    st.sp = 0;
    st.cap = S.stack_cap;
    st.ring_n = S.stack_ring;
    return st;
}

// One node visit of the closest-hit traversal: tests the 8 children of `node`,
// intersects hit leaves in slot order, then continues with the nearest hit inner
// child (sorted by a 19-comparator network on packed (t | slot) keys) and pushes
// the others far → near.  Returns false when the traversal is finished.
template <bool ANA, int NF>
RT_D bool closest_step(const DevScene& S, const RayC& R, float3 d, float tmin, Best& best,
                       uint32_t& node, TStack& stk, bool& ok) {
    constexpr int WN = node_width<NF>();
    float tn[8];
    uint32_t ch[8];
    // the closest hit so far bounds the boxes; widened like every exit distance
    float cwin = best.t + fabsf(best.t) * SLAB_WIDEN;
    uint32_t mask = node_test_any<NF>(S, node, R, tmin, R.general ? best.t : cwin, tn, ch);
    uint32_t leaves = 0;
#pragma unroll
    for (int c = 0; c < WN; c++) leaves |= ((ch[c] & RT_LEAF_BIT) ? 1u : 0u) << c;
    leaves &= mask;
    if (leaves) {
        const uint32_t* refs = node_refs<NF>(S, node);
#pragma unroll 1
        while (leaves) {
            int c = __ffs(leaves) - 1;
            leaves &= leaves - 1;
            leaf_closest<ANA>(S, __ldg(refs + c), R.o, d, tmin, best);
        }
    }
    float cw = best.t + fabsf(best.t) * SLAB_WIDEN;
    uint32_t k[8];
    int n = 0;
#pragma unroll
    for (int c = 0; c < WN; c++) {
        bool inner = ((mask >> c) & 1u) && !(ch[c] & RT_LEAF_BIT) && tn[c] <= cw;
        k[c] = inner ? ((__float_as_uint(fmaxf(tn[c], 0.0f)) & ~7u) | (uint32_t)c) : 0xFFFFFFFFu;
        n += inner ? 1 : 0;
    }
    if (n == 0) {
        if (stk.sp == 0) return false;
        node = stk.pop();
        return true;
    }
    if (n == 2) {
        // two inner children: continue with the nearer, push the farther
        uint32_t a = 0xFFFFFFFFu, b = 0xFFFFFFFFu;
#pragma unroll
        for (int c = 0; c < WN; c++) {
            if (k[c] == 0xFFFFFFFFu) continue;
            if (a == 0xFFFFFFFFu) a = k[c]; else b = k[c];
        }
        uint32_t lo = min(a, b), hi = max(a, b);
        if (!stk.room(1)) { ok = false; return false; }
        const uint32_t* refs = node_refs<NF>(S, node);
        stk.push(__ldg(refs + (hi & 7u)));
        node = __ldg(refs + (lo & 7u));
    } else if (n > 2) {
        if constexpr (WN == 4) {
            CAS(0, 1) CAS(2, 3)
            CAS(0, 2) CAS(1, 3)
            CAS(1, 2)
        } else {
            CAS(0, 1) CAS(2, 3) CAS(4, 5) CAS(6, 7)
            CAS(0, 2) CAS(1, 3) CAS(4, 6) CAS(5, 7)
            CAS(1, 2) CAS(5, 6) CAS(0, 4) CAS(3, 7)
            CAS(1, 5) CAS(2, 6)
            CAS(1, 4) CAS(3, 6)
            CAS(2, 4) CAS(3, 5)
            CAS(3, 4)
        }
        if (!stk.room(n - 1)) { ok = false; return false; }
        const uint32_t* refs = node_refs<NF>(S, node);
#pragma unroll
        for (int j = WN - 1; j >= 1; j--)
            if (j < n) stk.push(__ldg(refs + (k[j] & 7u)));
        node = __ldg(refs + (k[0] & 7u));
    } else {
        uint32_t c = 0;
#pragma unroll
        for (int j = 0; j < WN; j++) if (k[j] != 0xFFFFFFFFu) c = j;
        node = ch[c];
    }
    return true;
}

// One node visit of the any-hit traversal (bvh.rs:487-530).  Returns false when
// finished; *hit is set when a primitive was hit.
template <bool ANA, int NF>
RT_D bool any_step(const DevScene& S, const RayC& R, float3 d, float tmin, float tmax,
                   uint32_t& node, TStack& stk, bool& hit, bool& ok) {
    constexpr int WN = node_width<NF>();
    float tn[8];
    uint32_t ch[8];
    float tw = tmax + fabsf(tmax) * SLAB_WIDEN;
    uint32_t mask = node_test_any<NF>(S, node, R, tmin, R.general ? tmax : tw, tn, ch);
    uint32_t inner = 0, leaves = 0;
#pragma unroll
    for (int c = 0; c < WN; c++) {
        bool lf = ch[c] & RT_LEAF_BIT;
        leaves |= (lf ? 1u : 0u) << c;
        inner |= (lf ? 0u : 1u) << c;
    }
    leaves &= mask;
    inner &= mask;
    if (leaves) {
        const uint32_t* refs = node_refs<NF>(S, node);
#pragma unroll 1
        while (leaves) {
            int c = __ffs(leaves) - 1;
            leaves &= leaves - 1;
            if (leaf_any<ANA>(S, __ldg(refs + c), R.o, d, tmin, tmax)) { hit = true; return false; }
        }
    }
    if (inner == 0) {
        if (stk.sp == 0) return false;
        node = stk.pop();
        return true;
    }
    int first = __ffs(inner) - 1;
    uint32_t rest = inner & (inner - 1);
    if (!stk.room(__popc(rest))) { ok = false; return false; }
#pragma unroll
    for (int c = 0; c < WN; c++)
        if ((rest >> c) & 1u) stk.push(ch[c]);
    node = ch[first];
    return true;
}

RT_D bool nan_ray(float3 o, float3 d, float tmin, float tmax) {
    return isnan(o.x) || isnan(o.y) || isnan(o.z) || isnan(d.x) || isnan(d.y) || isnan(d.z) || isnan(tmin) ||
           isnan(tmax);
}

}  // namespace rtk

// ── persistent traversal with lane refill ───────────────────────────────────
// Each lane owns one ray; every loop iteration performs one node visit per
// active lane.  When at least RT_REFILL lanes of a warp are idle, they pull
// new rays from the queue together (one atomic per warp), so a warp is not held
// by its slowest ray (persistent threads with dynamic fetch, Aila & Laine 2009).
#ifndef RT_REFILL
#define RT_REFILL 12
#endif
// the closest-hit kernel refills later: its rays are longer, and fewer,
// larger refills measured faster (icosphere workload, extend 62.8 → 60.6 ms
// at 24; any-hit stays best at 12)
#ifndef RT_REFILL_CLOSEST
#define RT_REFILL_CLOSEST 24
#endif
#define FULLMASK 0xFFFFFFFFu

// MODE 0: wavefront extend (queue of path ids, rays in PathState, hits to PathState)
// MODE 1: API (rays n×8 in memory, hits as int4)

template <int MODE, bool ANA, int NF>
__global__ void __launch_bounds__(RT_TRACE_BLOCK, RT_TRACE_MINB) k_closest(DevScene S, PathState P, const uint32_t* __restrict__ queue,
                                                            const float* __restrict__ rays, uint32_t n_api,
                                                            const uint32_t* count, uint32_t* next,
                                                            int4* __restrict__ out, int* err) {
    const uint32_t n = MODE == 0 ? *count : n_api;
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
#if RT_STACK_LOCAL
    uint32_t ring[RT_SHORT_STACK];
#else
    __shared__ uint32_t ring[RT_SHORT_STACK * RT_TRACE_BLOCK];
#endif
    rtk::TStack stk = rtk::make_stack(S, ring);
    bool active = false, exhausted = false, ok = true;
    uint32_t item = 0, node = 0, pid = 0;
    float3 o = mk(0.f, 0.f, 0.f), d = o;
    RayC R = make_rayc(o, mk(1.f, 1.f, 1.f), 0.0f);
    float tmin = 0.0f;
    Best best{0.0f, 0.0f, 0.0f, RT_MISS_REF, 0xFFFFFFFFu, 0u};
    while (true) {
        uint32_t idle = __ballot_sync(FULLMASK, !active);
        if (!exhausted && __popc(idle) >= RT_REFILL_CLOSEST) {
            uint32_t k = __popc(idle), base = 0;
            if (lane == 0) base = atomicAdd(next, k);
            base = __shfl_sync(FULLMASK, base, 0);
            if (base + k >= n) exhausted = true;
            if (!active) {
                uint32_t i = base + __popc(idle & lt);
                if (i < n) {
                    item = i;
                    float tmax;
                    if (MODE == 0) {
                        pid = queue ? queue[i] : i;
                        float4 ro = P.ray_o[pid], rd = P.ray_d[pid];
                        o = mk(ro.x, ro.y, ro.z); d = mk(rd.x, rd.y, rd.z);
                        tmin = 0.001f; tmax = INFINITY;
                    } else {
                        const float* r = rays + (size_t)i * 8;
                        o = mk(r[0], r[1], r[2]); d = mk(r[3], r[4], r[5]);
                        tmin = r[6]; tmax = r[7];
                    }
                    R = make_rayc(o, d, tmin);
                    best = Best{tmax, 0.0f, 0.0f, RT_MISS_REF, 0xFFFFFFFFu, 0u};
                    node = 0; stk.sp = 0;
                    active = !rtk::nan_ray(o, d, tmin, tmax);
                    if (!active) {
                        if (MODE == 0) P.hit[pid] = make_float4(__uint_as_float(RT_MISS_REF), 0.f, 0.f, 0.f);
                        else out[i] = make_int4(-1, 0, 0, 0);
                    }
                }
            }
        }
        if (exhausted && __ballot_sync(FULLMASK, active) == 0) break;
        if (active) {
            bool lok = true;
            bool more = rtk::closest_step<ANA, NF>(S, R, d, tmin, best, node, stk, lok);
            if (!lok) ok = false;
            if (!more) {
                active = false;
                bool hit = best.ref != RT_MISS_REF;
                if (MODE == 0) {
                    uint32_t href = hit ? RT_HIT_MAKE(best.ref, __ldg(S.mat_code + best.mat)) : RT_MISS_REF;
                    P.hit[pid] = make_float4(__uint_as_float(href), best.t, best.b1, best.b2);
                } else {
                    out[item] = make_int4(hit ? (int)best.gid : -1, __float_as_int(hit ? best.t : 0.0f),
                                          __float_as_int(hit ? best.b1 : 0.0f), __float_as_int(hit ? best.b2 : 0.0f));
                }
            }
        }
    }
    if (!ok) atomicExch(err, RT_ERR_CAPACITY);
}

// MODE 0: wavefront shadow rays (an occluded ray cancels its parked contribution)
// MODE 1: API any-hit (occluded flags)
// MODE 2: wavefront shadow rays in a scene with media (an unoccluded ray scales
//         its parked contribution by the media's transmittance)
template <int MODE, bool ANA, int NF>
__global__ void __launch_bounds__(RT_TRACE_BLOCK, RT_TRACE_MINB) k_any(DevScene S, PendTargets T, const float4* __restrict__ sq,
                                                        const float* __restrict__ rays, uint32_t n_api,
                                                        const uint32_t* count, uint32_t* next,
                                                        uint8_t* __restrict__ out, int* err) {
    const uint32_t n = MODE != 1 ? *count : n_api;
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
#if RT_STACK_LOCAL
    uint32_t ring[RT_SHORT_STACK];
#else
    __shared__ uint32_t ring[RT_SHORT_STACK * RT_TRACE_BLOCK];
#endif
    rtk::TStack stk = rtk::make_stack(S, ring);
    bool active = false, exhausted = false, ok = true;
    uint32_t item = 0, node = 0, tag = 0;
    float3 o = mk(0.f, 0.f, 0.f), d = o;
    RayC R = make_rayc(o, mk(1.f, 1.f, 1.f), 0.0f);
    float tmin = 0.0f, tmax = 0.0f;
    bool hit = false;
    while (true) {
        uint32_t idle = __ballot_sync(FULLMASK, !active);
        if (!exhausted && __popc(idle) >= RT_REFILL) {
            uint32_t k = __popc(idle), base = 0;
            if (lane == 0) base = atomicAdd(next, k);
            base = __shfl_sync(FULLMASK, base, 0);
            if (base + k >= n) exhausted = true;
            if (!active) {
                uint32_t i = base + __popc(idle & lt);
                if (i < n) {
                    item = i;
                    if (MODE != 1) {
                        float4 a = sq[(size_t)i * 2], b = sq[(size_t)i * 2 + 1];
                        o = mk(a.x, a.y, a.z); d = mk(b.x, b.y, b.z);
                        tmin = 0.001f; tmax = a.w;
                        tag = __float_as_uint(b.w);
                    } else {
                        const float* r = rays + (size_t)i * 8;
                        o = mk(r[0], r[1], r[2]); d = mk(r[3], r[4], r[5]);
                        tmin = r[6]; tmax = r[7];
                    }
                    R = make_rayc(o, d, tmin);
                    node = 0; stk.sp = 0; hit = false;
                    active = !rtk::nan_ray(o, d, tmin, tmax);
                    if (!active && MODE == 1) out[i] = 0;
                }
            }
        }
        if (exhausted && __ballot_sync(FULLMASK, active) == 0) break;
        if (active) {
            bool lok = true;
            bool more = rtk::any_step<ANA, NF>(S, R, d, tmin, tmax, node, stk, hit, lok);
            if (!lok) ok = false;
            if (!more) {
                active = false;
                if (MODE != 1) {
                    if (hit) {
                        T.pend[tag & 3u][tag >> 2] = make_float4(0.f, 0.f, 0.f, 0.f);
                    } else if (MODE == 2) {
                        // world.transmittance (bvh.rs:532-575): the media scale what got through
                        float tr = media_transmittance(S, o, d, tmin, tmax);
                        if (tr < 1.0f) {
                            float4* pp = T.pend[tag & 3u] + (tag >> 2);
                            float4 v = *pp;
                            *pp = make_float4(v.x * tr, v.y * tr, v.z * tr, v.w);
                        }
                    }
                } else {
                    out[item] = hit ? 1 : 0;
                }
            }
        }
    }
    if (!ok) atomicExch(err, RT_ERR_CAPACITY);
}

// ── participating media next to the traversal ───────────────────────────────
// A medium's scatter distance depends on the ray alone, so after the closest
// hit each ray takes the nearest medium event before its surface hit (media
// ids follow the primitives: a tie goes to the surface).
// MODE 0: wavefront paths (dense set, wavelength in meta.w)
// MODE 1: photons (queued, wavelength in ray_d.w)
template <int MODE>
__global__ void k_media(DevScene S, PathState P, const uint32_t* __restrict__ queue, const uint32_t* count) {
    uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t pid = MODE == 1 ? queue[i] : i;
        float4 ro = P.ray_o[pid], rd = P.ray_d[pid], hv = P.hit[pid];
        float lam = MODE == 1 ? rd.w : __uint_as_float(P.meta[pid].w);
        float3 o = mk(ro.x, ro.y, ro.z), d = mk(rd.x, rd.y, rd.z);
        if (rtk::nan_ray(o, d, 0.001f, INFINITY)) continue;
        float tsurf = __float_as_uint(hv.x) == RT_MISS_REF ? INFINITY : hv.y;
        float tm;
        int med = media_event(S, o, d, lam, 0.001f, tsurf, &tm);
        if (med >= 0) P.hit[pid] = make_float4(__uint_as_float(RT_HIT_MEDIUM_BASE | (uint32_t)med), tm, 0.f, 0.f);
    }
}

// API: rays n × 8 (o, d, t_min, t_max) with closest hits already in `out`
// (fill_miss: there is no BVH, every ray starts as a miss)
__global__ void k_media_api(DevScene S, const float* __restrict__ rays, uint32_t n, int4* out, int32_t n_prims,
                            int fill_miss) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* r = rays + (size_t)i * 8;
        float3 o = mk(r[0], r[1], r[2]), d = mk(r[3], r[4], r[5]);
        if (fill_miss) out[i] = make_int4(-1, 0, 0, 0);
        if (rtk::nan_ray(o, d, r[6], r[7])) continue;
        int4 h = out[i];
        float tsurf = h.x < 0 ? r[7] : __int_as_float(h.y);
        float tm;
        int med = media_event(S, o, d, 550.0f, r[6], tsurf, &tm);
        if (med >= 0) out[i] = make_int4(n_prims + med, __float_as_int(tm), 0, 0);
    }
}

// API: world.transmittance per ray, from the any-hit flags (NULL: no primitives)
__global__ void k_transmittance_api(DevScene S, const float* __restrict__ rays, uint32_t n,
                                    const uint8_t* __restrict__ occ, float* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* r = rays + (size_t)i * 8;
        float3 o = mk(r[0], r[1], r[2]), d = mk(r[3], r[4], r[5]);
        float tr = (occ && occ[i]) ? 0.0f : 1.0f;
        if (tr > 0.0f && S.n_media > 0 && !rtk::nan_ray(o, d, r[6], r[7])) tr = media_transmittance(S, o, d, r[6], r[7]);
        out[i] = tr;
    }
}

// ── host launchers ──────────────────────────────────────────────────────────
// ── ray binning before extend (RT_RAY_BINS) ────────────────────────────────
// A counting sort of the set's rays by direction octant and a coarse cell of
// the origin: the extend kernel then takes its rays in bin order, so the lanes
// of a warp start rays that visit similar nodes in a similar order.  Each
// block sorts a contiguous chunk, so neighbours in the set stay neighbours
// within a bin.  The hits do not depend on the order.
#define BIN_BLOCK 256
#define BIN_ITEMS 8
#define BIN_CHUNK (BIN_BLOCK * BIN_ITEMS)
__device__ __forceinline__ uint32_t ray_bin(float4 ro, float4 rd, float3 lo, float3 sc) {
    uint32_t oct = (rd.x < 0.f ? 1u : 0u) | (rd.y < 0.f ? 2u : 0u) | (rd.z < 0.f ? 4u : 0u);
    int cx = min(max(__float2int_rz((ro.x - lo.x) * sc.x), 0), RT_BIN_CELLS - 1);
    int cy = min(max(__float2int_rz((ro.y - lo.y) * sc.y), 0), RT_BIN_CELLS - 1);
    int cz = min(max(__float2int_rz((ro.z - lo.z) * sc.z), 0), RT_BIN_CELLS - 1);
    return ((oct * RT_BIN_CELLS + (uint32_t)cx) * RT_BIN_CELLS + (uint32_t)cy) * RT_BIN_CELLS + (uint32_t)cz;
}
__global__ void __launch_bounds__(BIN_BLOCK) k_bin_count(PathState A, const uint32_t* __restrict__ count, float3 lo,
                                                         float3 sc, uint32_t* hist) {
    __shared__ uint32_t h[RT_NBINS];
    const uint32_t n = *count, base = blockIdx.x * BIN_CHUNK;
    if (base >= n) return;                       // uniform in the block
    for (int b = threadIdx.x; b < RT_NBINS; b += BIN_BLOCK) h[b] = 0;
    __syncthreads();
    for (int k = 0; k < BIN_ITEMS; k++) {
        uint32_t i = base + k * BIN_BLOCK + threadIdx.x;
        if (i < n) atomicAdd(&h[ray_bin(A.ray_o[i], A.ray_d[i], lo, sc)], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < RT_NBINS; b += BIN_BLOCK)
        if (h[b]) atomicAdd(hist + b, h[b]);
}
__global__ void __launch_bounds__(BIN_BLOCK) k_bin_scatter(PathState A, const uint32_t* __restrict__ count, float3 lo,
                                                           float3 sc, const uint32_t* __restrict__ hist,
                                                           uint32_t* cursor, uint32_t* out) {
    static_assert(RT_NBINS == 2 * BIN_BLOCK, "two bins per thread in the scan");
    typedef cub::BlockScan<uint32_t, BIN_BLOCK> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint32_t h[RT_NBINS], start[RT_NBINS];
    const uint32_t n = *count, base = blockIdx.x * BIN_CHUNK;
    if (base >= n) return;                       // uniform in the block
    // the bins' starts: exclusive prefix of the histogram
    uint32_t v[2] = {hist[2 * threadIdx.x], hist[2 * threadIdx.x + 1]};
    Scan(tmp).ExclusiveSum(v, v);
    start[2 * threadIdx.x] = v[0];
    start[2 * threadIdx.x + 1] = v[1];
    h[2 * threadIdx.x] = 0;
    h[2 * threadIdx.x + 1] = 0;
    __syncthreads();
    uint32_t key[BIN_ITEMS], rank[BIN_ITEMS];
    for (int k = 0; k < BIN_ITEMS; k++) {
        uint32_t i = base + k * BIN_BLOCK + threadIdx.x;
        key[k] = i < n ? ray_bin(A.ray_o[i], A.ray_d[i], lo, sc) : RT_NBINS;
        rank[k] = key[k] < RT_NBINS ? atomicAdd(&h[key[k]], 1u) : 0u;
    }
    __syncthreads();
    // this block's run in each bin
    for (int b = threadIdx.x; b < RT_NBINS; b += BIN_BLOCK)
        if (h[b]) h[b] = start[b] + atomicAdd(cursor + b, h[b]);
    __syncthreads();
    for (int k = 0; k < BIN_ITEMS; k++)
        if (key[k] < RT_NBINS) out[h[key[k]] + rank[k]] = base + k * BIN_BLOCK + threadIdx.x;
}

namespace rth {
#ifndef RT_TRACE_GRID_PER_SM
#define RT_TRACE_GRID_PER_SM RT_TRACE_MINB
#endif
// persistent kernels: one wave of resident blocks, or fewer when tuned
int trace_grid(const DevScene& S, int dev_sms) {
    int per = S.trace_per_sm > 0 ? std::min(S.trace_per_sm, RT_TRACE_MINB) : RT_TRACE_GRID_PER_SM;
    return dev_sms * per;
}

// the traversal kernels with (ANA) or without analytic solids
#define RT_TRACE_LAUNCH(K, MODE, ...)                                                                         \
    do {                                                                                                      \
        const int g_ = trace_grid(S, sms);                                                                    \
        const int f_ = S.node_format;                                                                        \
        if (S.n_analytic > 0) {                                                                               \
            if (f_ == RT_NODES_QUANTISED)  K<MODE, true, RT_NODES_QUANTISED><<<g_, RT_TRACE_BLOCK, 0, st>>>(__VA_ARGS__); \
            else if (f_ == RT_NODES_WIDE4) K<MODE, true, RT_NODES_WIDE4><<<g_, RT_TRACE_BLOCK, 0, st>>>(__VA_ARGS__);     \
            else                           K<MODE, true, RT_NODES_FULL><<<g_, RT_TRACE_BLOCK, 0, st>>>(__VA_ARGS__);      \
        } else {                                                                                              \
            if (f_ == RT_NODES_QUANTISED)  K<MODE, false, RT_NODES_QUANTISED><<<g_, RT_TRACE_BLOCK, 0, st>>>(__VA_ARGS__); \
            else if (f_ == RT_NODES_WIDE4) K<MODE, false, RT_NODES_WIDE4><<<g_, RT_TRACE_BLOCK, 0, st>>>(__VA_ARGS__);     \
            else                           K<MODE, false, RT_NODES_FULL><<<g_, RT_TRACE_BLOCK, 0, st>>>(__VA_ARGS__);      \
        }                                                                                                     \
    } while (0)
void launch_trace_closest_api(const DevScene& S, const float* rays, uint32_t n, int4* out, uint32_t* next, int* err,
                              int sms, cudaStream_t st) {
    RT_TRACE_LAUNCH(k_closest, 1, S, PathState{}, nullptr, rays, n, nullptr, next, out, err);
}
void launch_trace_any_api(const DevScene& S, const float* rays, uint32_t n, uint8_t* out, uint32_t* next, int* err,
                          int sms, cudaStream_t st) {
    RT_TRACE_LAUNCH(k_any, 1, S, PendTargets{}, nullptr, rays, n, nullptr, next, out, err);
}
void launch_bin_rays(const PathState& A, const uint32_t* count, uint32_t capacity, float3 lo, float3 scale,
                     uint32_t* bins, uint32_t* out, cudaStream_t st) {
    uint32_t grid = std::max<uint32_t>(1u, (capacity + BIN_CHUNK - 1) / BIN_CHUNK);
    cudaMemsetAsync(bins, 0, 2 * RT_NBINS * sizeof(uint32_t), st);
    k_bin_count<<<grid, BIN_BLOCK, 0, st>>>(A, count, lo, scale, bins);
    k_bin_scatter<<<grid, BIN_BLOCK, 0, st>>>(A, count, lo, scale, bins, bins + RT_NBINS, out);
}
void launch_extend(const DevScene& S, const PathState& P, const uint32_t* queue, const uint32_t* count,
                   uint32_t* next, int* err, int sms, cudaStream_t st) {
    RT_TRACE_LAUNCH(k_closest, 0, S, P, queue, nullptr, 0, count, next, nullptr, err);
}
void launch_shadow(const DevScene& S, const PendTargets& T, const float4* sq, const uint32_t* count,
                   uint32_t* next, int* err, int sms, cudaStream_t st) {
    if (S.n_media > 0) RT_TRACE_LAUNCH(k_any, 2, S, T, sq, nullptr, 0, count, next, nullptr, err);
    else               RT_TRACE_LAUNCH(k_any, 0, S, T, sq, nullptr, 0, count, next, nullptr, err);
}
#undef RT_TRACE_LAUNCH
void launch_media(const DevScene& S, const PathState& P, const uint32_t* queue, const uint32_t* count, int sms,
                  cudaStream_t st) {
    if (queue) k_media<1><<<sms * 8, 128, 0, st>>>(S, P, queue, count);
    else       k_media<0><<<sms * 8, 128, 0, st>>>(S, P, nullptr, count);
}
void launch_media_api(const DevScene& S, const float* rays, uint32_t n, int4* out, int32_t n_prims, int fill_miss,
                      int sms, cudaStream_t st) {
    k_media_api<<<sms * 8, 128, 0, st>>>(S, rays, n, out, n_prims, fill_miss);
}
void launch_transmittance_api(const DevScene& S, const float* rays, uint32_t n, const uint8_t* occ, float* out,
                              int sms, cudaStream_t st) {
    k_transmittance_api<<<sms * 8, 128, 0, st>>>(S, rays, n, occ, out);
}
}  // namespace rth
