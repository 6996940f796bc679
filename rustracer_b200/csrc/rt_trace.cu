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
#include "rt_internal.h"

using namespace rtd;

namespace {

struct Best { float t, b1, b2; uint32_t ref, gid; };

RT_D uint32_t f2u(float f) { return __float_as_uint(f); }

// Leaf test for one reference; updates `best` and returns nothing.
RT_D void leaf_closest(const DevScene& S, uint32_t ref, float3 o, float3 d, float tmin, Best& best) {
    uint32_t type = (ref >> 28) & 7u, idx = ref & 0x0FFFFFFFu;
    float t, b1, b2;
    uint32_t gid;
    bool h;
    if (type == RT_PRIM_TRI) {
        const float4* g = S.tri + (size_t)idx * 3;
        float4 a = __ldg(g), b = __ldg(g + 1), c = __ldg(g + 2);
        h = tri_test(a, b, c, o, d, tmin, best.t, &t, &b1, &b2);
        gid = f2u(c.y);
    } else if (type == RT_PRIM_QUAD) {
        const float4* g = S.quad + (size_t)idx * 5;
        float4 gg[4] = {__ldg(g), __ldg(g + 1), __ldg(g + 2), __ldg(g + 3)};
        h = quad_test(gg, o, d, tmin, best.t, &t, &b1, &b2);
        gid = h ? f2u(__ldg(g + 4).x) : 0u;
    } else {
        const float4* g = S.sphere + (size_t)idx * 2;
        h = sphere_test(__ldg(g), o, d, tmin, best.t, &t);
        b1 = b2 = 0.0f;
        gid = h ? f2u(__ldg(g + 1).x) : 0u;
    }
    if (h && (t < best.t || best.ref == RT_MISS_REF || gid < best.gid)) {
        best.t = t; best.b1 = b1; best.b2 = b2; best.ref = ref; best.gid = gid;
    }
}

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
    return sphere_test(__ldg(S.sphere + (size_t)idx * 2), o, d, tmin, tmax, &t);
}

#define CAS(a, b) { uint32_t lo_ = min(k[a], k[b]); uint32_t hi_ = max(k[a], k[b]); k[a] = lo_; k[b] = hi_; }

// Slab test of the 8 children of node `ni`; returns the hit mask and the entry
// distances.  Bit-identical to the CPU checker's AVX2 slab test.
template <bool NANSAFE>
RT_D uint32_t node_test(const DevScene& S, uint32_t ni, float3 o, float3 inv, float tmin, float tmax,
                        float tn[8], uint32_t ch[8]) {
    const float4* N = S.nodes + (size_t)ni * 14;
    float4 q[14];
#pragma unroll
    for (int i = 0; i < 14; i++) q[i] = __ldg(N + i);
    const float* f = reinterpret_cast<const float*>(q);
    uint32_t mask = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        ch[c] = __float_as_uint(f[48 + c]);
        float dax = (f[0 + c] - o.x) * inv.x, dbx = (f[24 + c] - o.x) * inv.x;
        float day = (f[8 + c] - o.y) * inv.y, dby = (f[32 + c] - o.y) * inv.y;
        float daz = (f[16 + c] - o.z) * inv.z, dbz = (f[40 + c] - o.z) * inv.z;
        float lx = fminf(dax, dbx), hx = fmaxf(dax, dbx);
        float ly = fminf(day, dby), hy = fmaxf(day, dby);
        float lz = fminf(daz, dbz), hz = fmaxf(daz, dbz);
        if (NANSAFE) {
            if (isnan(dax) || isnan(dbx)) { lx = -INFINITY; hx = INFINITY; }
            if (isnan(day) || isnan(dby)) { ly = -INFINITY; hy = INFINITY; }
            if (isnan(daz) || isnan(dbz)) { lz = -INFINITY; hz = INFINITY; }
        }
        float t0 = fmaxf(fmaxf(fmaxf(tmin, lx), ly), lz);
        float t1 = fminf(fminf(fminf(tmax, hx), hy), hz);
        float t1w = t1 + fabsf(t1) * SLAB_WIDEN;
        tn[c] = t0;
        if (t0 <= t1w && ch[c] != RT_EMPTY_REF) mask |= 1u << c;
    }
    return mask;
}

}  // namespace

namespace rtk {

// One node visit of the closest-hit traversal: tests the 8 children of `node`,
// intersects hit leaves in slot order, then continues with the nearest hit inner
// child (sorted by a 19-comparator network on packed (t | slot) keys) and pushes
// the others far → near.  Returns false when the traversal is finished.
RT_D bool closest_step(const DevScene& S, float3 o, float3 d, float3 inv, bool nansafe, float tmin, Best& best,
                       uint32_t& node, int& sp, uint32_t* stack, bool& ok) {
    float tn[8];
    uint32_t ch[8];
    uint32_t mask = nansafe ? node_test<true>(S, node, o, inv, tmin, best.t, tn, ch)
                            : node_test<false>(S, node, o, inv, tmin, best.t, tn, ch);
#pragma unroll
    for (int c = 0; c < 8; c++)
        if ((mask >> c) & 1u && (ch[c] & RT_LEAF_BIT)) leaf_closest(S, ch[c], o, d, tmin, best);
    float cw = best.t + fabsf(best.t) * SLAB_WIDEN;
    uint32_t k[8];
    int n = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        bool inner = ((mask >> c) & 1u) && !(ch[c] & RT_LEAF_BIT) && tn[c] <= cw;
        k[c] = inner ? ((__float_as_uint(fmaxf(tn[c], 0.0f)) & ~7u) | (uint32_t)c) : 0xFFFFFFFFu;
        n += inner ? 1 : 0;
    }
    if (n == 0) {
        if (sp == 0) return false;
        node = stack[--sp];
        return true;
    }
    if (n > 1) {
        CAS(0, 1) CAS(2, 3) CAS(4, 5) CAS(6, 7)
        CAS(0, 2) CAS(1, 3) CAS(4, 6) CAS(5, 7)
        CAS(1, 2) CAS(5, 6) CAS(0, 4) CAS(3, 7)
        CAS(1, 5) CAS(2, 6)
        CAS(1, 4) CAS(3, 6)
        CAS(2, 4) CAS(3, 5)
        CAS(3, 4)
        if (sp + n - 1 > RT_STACK) { ok = false; return false; }
        const uint32_t* refs = reinterpret_cast<const uint32_t*>(S.nodes + (size_t)node * 14 + 12);
#pragma unroll
        for (int j = 7; j >= 1; j--)
            if (j < n) stack[sp++] = __ldg(refs + (k[j] & 7u));
        node = __ldg(refs + (k[0] & 7u));
    } else {
        uint32_t c = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) if (k[j] != 0xFFFFFFFFu) c = j;
        node = ch[c];
    }
    return true;
}

// One node visit of the any-hit traversal (bvh.rs:487-530).  Returns false when
// finished; *hit is set when a primitive was hit.
RT_D bool any_step(const DevScene& S, float3 o, float3 d, float3 inv, bool nansafe, float tmin, float tmax,
                   uint32_t& node, int& sp, uint32_t* stack, bool& hit, bool& ok) {
    float tn[8];
    uint32_t ch[8];
    uint32_t mask = nansafe ? node_test<true>(S, node, o, inv, tmin, tmax, tn, ch)
                            : node_test<false>(S, node, o, inv, tmin, tmax, tn, ch);
    uint32_t inner = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        if (!((mask >> c) & 1u)) continue;
        if (ch[c] & RT_LEAF_BIT) {
            if (!hit && leaf_any(S, ch[c], o, d, tmin, tmax)) hit = true;
        } else {
            inner |= 1u << c;
        }
    }
    if (hit) return false;
    if (inner == 0) {
        if (sp == 0) return false;
        node = stack[--sp];
        return true;
    }
    int first = __ffs(inner) - 1;
    uint32_t rest = inner & (inner - 1);
    if (sp + __popc(rest) > RT_STACK) { ok = false; return false; }
#pragma unroll
    for (int c = 0; c < 8; c++)
        if ((rest >> c) & 1u) stack[sp++] = ch[c];
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
#define RT_REFILL 12
#define FULLMASK 0xFFFFFFFFu

// MODE 0: wavefront extend (queue of path ids, rays in PathState, hits to PathState)
// MODE 1: API (rays n×8 in memory, hits as int4)
template <int MODE>
__global__ void __launch_bounds__(RT_TRACE_BLOCK) k_closest(DevScene S, PathState P, const uint32_t* __restrict__ queue,
                                                            const float* __restrict__ rays, uint32_t n_api,
                                                            const uint32_t* count, uint32_t* next,
                                                            int4* __restrict__ out, int* err) {
    const uint32_t n = MODE == 0 ? *count : n_api;
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
    uint32_t stack[RT_STACK];
    bool active = false, exhausted = false, ok = true;
    uint32_t item = 0, node = 0, pid = 0;
    int sp = 0;
    float3 o = mk(0.f, 0.f, 0.f), d = o, inv = o;
    bool nansafe = false;
    float tmin = 0.0f;
    Best best{0.0f, 0.0f, 0.0f, RT_MISS_REF, 0xFFFFFFFFu};
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
                    float tmax;
                    if (MODE == 0) {
                        pid = queue[i];
                        float4 ro = P.ray_o[pid], rd = P.ray_d[pid];
                        o = mk(ro.x, ro.y, ro.z); d = mk(rd.x, rd.y, rd.z);
                        tmin = 0.001f; tmax = INFINITY;
                    } else {
                        const float* r = rays + (size_t)i * 8;
                        o = mk(r[0], r[1], r[2]); d = mk(r[3], r[4], r[5]);
                        tmin = r[6]; tmax = r[7];
                    }
                    inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
                    nansafe = isinf(inv.x) || isinf(inv.y) || isinf(inv.z);
                    best = Best{tmax, 0.0f, 0.0f, RT_MISS_REF, 0xFFFFFFFFu};
                    node = 0; sp = 0;
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
            bool more = rtk::closest_step(S, o, d, inv, nansafe, tmin, best, node, sp, stack, lok);
            if (!lok) ok = false;
            if (!more) {
                active = false;
                bool hit = best.ref != RT_MISS_REF;
                if (MODE == 0) {
                    P.hit[pid] = make_float4(__uint_as_float(best.ref), best.t, best.b1, best.b2);
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
template <int MODE>
__global__ void __launch_bounds__(RT_TRACE_BLOCK) k_any(DevScene S, PathState P, const float4* __restrict__ sq,
                                                        const float* __restrict__ rays, uint32_t n_api,
                                                        const uint32_t* count, uint32_t* next,
                                                        uint8_t* __restrict__ out, int* err) {
    const uint32_t n = MODE == 0 ? *count : n_api;
    const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
    uint32_t stack[RT_STACK];
    bool active = false, exhausted = false, ok = true;
    uint32_t item = 0, node = 0, tag = 0;
    int sp = 0;
    float3 o = mk(0.f, 0.f, 0.f), d = o, inv = o;
    bool nansafe = false;
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
                    if (MODE == 0) {
                        float4 a = sq[(size_t)i * 2], b = sq[(size_t)i * 2 + 1];
                        o = mk(a.x, a.y, a.z); d = mk(b.x, b.y, b.z);
                        tmin = 0.001f; tmax = a.w;
                        tag = __float_as_uint(b.w);
                    } else {
                        const float* r = rays + (size_t)i * 8;
                        o = mk(r[0], r[1], r[2]); d = mk(r[3], r[4], r[5]);
                        tmin = r[6]; tmax = r[7];
                    }
                    inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
                    nansafe = isinf(inv.x) || isinf(inv.y) || isinf(inv.z);
                    node = 0; sp = 0; hit = false;
                    active = !rtk::nan_ray(o, d, tmin, tmax);
                    if (!active && MODE == 1) out[i] = 0;
                }
            }
        }
        if (exhausted && __ballot_sync(FULLMASK, active) == 0) break;
        if (active) {
            bool lok = true;
            bool more = rtk::any_step(S, o, d, inv, nansafe, tmin, tmax, node, sp, stack, hit, lok);
            if (!lok) ok = false;
            if (!more) {
                active = false;
                if (MODE == 0) {
                    if (hit) {
                        uint32_t p = tag >> 1;
                        if (tag & 1u) P.pend1[p] = make_float4(0.f, 0.f, 0.f, 0.f);
                        else          P.pend0[p] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                } else {
                    out[item] = hit ? 1 : 0;
                }
            }
        }
    }
    if (!ok) atomicExch(err, RT_ERR_CAPACITY);
}

// ── host launchers ──────────────────────────────────────────────────────────
namespace rth {
int trace_grid(int dev_sms) { return dev_sms * RT_TRACE_BLOCKS_PER_SM; }

void launch_trace_closest_api(const DevScene& S, const float* rays, uint32_t n, int4* out, uint32_t* next, int* err,
                              int sms, cudaStream_t st) {
    k_closest<1><<<trace_grid(sms), RT_TRACE_BLOCK, 0, st>>>(S, PathState{}, nullptr, rays, n, nullptr, next, out, err);
}
void launch_trace_any_api(const DevScene& S, const float* rays, uint32_t n, uint8_t* out, uint32_t* next, int* err,
                          int sms, cudaStream_t st) {
    k_any<1><<<trace_grid(sms), RT_TRACE_BLOCK, 0, st>>>(S, PathState{}, nullptr, rays, n, nullptr, next, out, err);
}
void launch_extend(const DevScene& S, const PathState& P, const uint32_t* queue, const uint32_t* count,
                   uint32_t* next, int* err, int sms, cudaStream_t st) {
    k_closest<0><<<trace_grid(sms), RT_TRACE_BLOCK, 0, st>>>(S, P, queue, nullptr, 0, count, next, nullptr, err);
}
void launch_shadow(const DevScene& S, const PathState& P, const float4* sq, const uint32_t* count,
                   uint32_t* next, int* err, int sms, cudaStream_t st) {
    k_any<0><<<trace_grid(sms), RT_TRACE_BLOCK, 0, st>>>(S, P, sq, nullptr, 0, count, next, nullptr, err);
}
}  // namespace rth
