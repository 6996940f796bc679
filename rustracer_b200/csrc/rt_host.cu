// rt_host.cu — C ABI of librtb200.so (include/rt_api.h): scene upload, BVH
// build, environment alias tables, spectral tables, and the wavefront render
// loop that drives the kernels of rt_trace.cu / rt_shade.cu on one stream.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <chrono>
#include <thread>
#include <vector>

#include "../../include/rt_spectral_tables.h"
#include "rt_internal.h"
#include "rt_sky.cuh"

using namespace rtd;

namespace {

// ── small host math (f32, no contraction: built with -ffp-contract=off) ─────
struct H3 { float x, y, z; };
static inline H3 h3(float x, float y, float z) { return H3{x, y, z}; }
static inline H3 operator+(H3 a, H3 b) { return h3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline H3 operator-(H3 a, H3 b) { return h3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline H3 operator*(H3 a, float t) { return h3(a.x * t, a.y * t, a.z * t); }
static inline H3 operator/(H3 a, float t) { return h3(a.x / t, a.y / t, a.z / t); }
static inline float hdot(H3 a, H3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline H3 hcross(H3 a, H3 b) { return h3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float hlen(H3 a) { return std::sqrt(hdot(a, a)); }
static inline float hc(H3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

struct Box { H3 mn, mx; };
static inline Box unite(const Box& a, const Box& b) {
    return Box{h3(std::fmin(a.mn.x, b.mn.x), std::fmin(a.mn.y, b.mn.y), std::fmin(a.mn.z, b.mn.z)),
               h3(std::fmax(a.mx.x, b.mx.x), std::fmax(a.mx.y, b.mx.y), std::fmax(a.mx.z, b.mx.z))};
}
static inline Box pad(Box b) {                                                      // aabb.rs:18-29
    const float D = 0.0001f;
    float px = b.mx.x - b.mn.x < D ? D : 0.0f, py = b.mx.y - b.mn.y < D ? D : 0.0f, pz = b.mx.z - b.mn.z < D ? D : 0.0f;
    return Box{h3(b.mn.x - px, b.mn.y - py, b.mn.z - pz), h3(b.mx.x + px, b.mx.y + py, b.mx.z + pz)};
}
// ── convex placement (transform.rs:15-27, 140-224; scene_file.rs:924-930) ──
// x_world = R·(s·x − pivot) + pivot + t.  A plane n·x ≤ d maps to n'·x ≤ d'
// with n' = R·n and d' = n'·(pivot + t) + (s·d − n·pivot).
static bool rotation_ok(const float* R) {
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double dot = 0.0;
            for (int k = 0; k < 3; k++) dot += (double)R[a * 3 + k] * R[b * 3 + k];
            if (!(std::fabs(dot - (a == b ? 1.0 : 0.0)) < 1e-3)) return false;
        }
    return true;
}
static inline H3 rot_apply(const float* R, H3 v) {                                  // transform.rs:150-156
    return h3(R[0] * v.x + R[1] * v.y + R[2] * v.z, R[3] * v.x + R[4] * v.y + R[5] * v.z,
              R[6] * v.x + R[7] * v.y + R[8] * v.z);
}
// micro_tilt (hittable.rs:261-270) on the host
static H3 micro_tilt_h(uint64_t idx, float amp, H3 n) {
    if (!(amp > 0.0f)) return n;
    uint64_t h = idx * 0x9E3779B97F4A7C15ull ^ 0xD1B54A32D192ED03ull;
    float a = (float)(uint32_t)(h >> 32) / 4294967295.0f * 2.0f - 1.0f;
    float b = (float)(uint32_t)h / 4294967295.0f * 2.0f - 1.0f;
    H3 up = std::fabs(n.x) < 0.9f ? h3(1.f, 0.f, 0.f) : h3(0.f, 1.f, 0.f);
    H3 t = hcross(n, up);
    t = t / hlen(t);
    H3 b2 = hcross(n, t);
    H3 m = n + t * (a * amp) + b2 * (b * amp);
    return m / hlen(m);
}
static void place_convex(const RtConvex& c, const float* pl, float4* out, float4* shade) {
    H3 pv = h3(c.pivot[0], c.pivot[1], c.pivot[2]);
    H3 pt = h3(c.pivot[0] + c.translate[0], c.pivot[1] + c.translate[1], c.pivot[2] + c.translate[2]);
    for (int j = 0; j < c.n_planes; j++) {
        H3 n = h3(pl[j * 4], pl[j * 4 + 1], pl[j * 4 + 2]);
        H3 nw = rot_apply(c.rot, n);
        float dw = hdot(nw, pt) + (c.scale * pl[j * 4 + 3] - hdot(n, pv));
        out[j] = make_float4(nw.x, nw.y, nw.z, dw);
        // the facet a polished normal is keyed on: the first plane with this normal (diamond.rs:267-269)
        int f = 0;
        while (f < j && !(std::fabs(pl[f * 4] - n.x) < 1e-6f && std::fabs(pl[f * 4 + 1] - n.y) < 1e-6f &&
                          std::fabs(pl[f * 4 + 2] - n.z) < 1e-6f)) f++;
        H3 sf = rot_apply(c.rot, micro_tilt_h((uint64_t)f, c.polish, n));
        H3 sb = rot_apply(c.rot, micro_tilt_h((uint64_t)f, c.polish, h3(-n.x, -n.y, -n.z)));
        shade[j * 2] = make_float4(sf.x, sf.y, sf.z, 0.f);
        shade[j * 2 + 1] = make_float4(sb.x, sb.y, sb.z, 0.f);
    }
}
static Box placed_box(const RtConvex& c) {                                          // transform.rs:180-200
    Box b{h3(INFINITY, INFINITY, INFINITY), h3(-INFINITY, -INFINITY, -INFINITY)};
    H3 pv = h3(c.pivot[0], c.pivot[1], c.pivot[2]), t = h3(c.translate[0], c.translate[1], c.translate[2]);
    for (int k = 0; k < 8; k++) {
        H3 x = h3(k & 1 ? c.box_hi[0] : c.box_lo[0], k & 2 ? c.box_hi[1] : c.box_lo[1], k & 4 ? c.box_hi[2] : c.box_lo[2]);
        H3 w = rot_apply(c.rot, x * c.scale - pv) + pv + t;
        b = unite(b, Box{w, w});
    }
    // the corners' rounding must not cut into the solid
    float e = 1e-5f * std::max(std::max(std::fabs(b.mn.x), std::fabs(b.mx.x)),
                               std::max(std::max(std::fabs(b.mn.y), std::fabs(b.mx.y)),
                                        std::max(std::fabs(b.mn.z), std::fabs(b.mx.z)))) + 1e-6f;
    return Box{b.mn - h3(e, e, e), b.mx + h3(e, e, e)};
}

// Cylinder / cone / disk / plane records (8 float4): (centre, radius),
// (unit normal, height), (u axis, wave amplitude), (v axis, wave scale), the
// rotation rows with (scale, 1/scale, placed), (translation, 0); returns the
// placed box (cylinder.rs:226-232, cone.rs:126-132, disk.rs:166-175,
// plane.rs:80-95, transform.rs:180-200).
static Box shape_params(const RtShape& q, float4* P) {
    H3 c = h3(q.center[0], q.center[1], q.center[2]);
    bool planar = q.type == RT_SHAPE_DISK || q.type == RT_SHAPE_PLANE;
    H3 n = h3(0.f, 1.f, 0.f);
    if (planar) {
        H3 nr = h3(q.normal[0], q.normal[1], q.normal[2]);
        n = nr / hlen(nr);
    }
    H3 up = std::fabs(n.y) < 0.9f ? h3(0.f, 1.f, 0.f) : h3(1.f, 0.f, 0.f);              // vec3.rs:37-42
    H3 u = hcross(n, up);
    u = u / hlen(u);
    H3 v = hcross(n, u);
    const float* R = q.rot;
    bool ident = R[0] == 1.f && R[4] == 1.f && R[8] == 1.f && R[1] == 0.f && R[2] == 0.f && R[3] == 0.f &&
                 R[5] == 0.f && R[6] == 0.f && R[7] == 0.f && q.scale == 1.f && q.translate[0] == 0.f &&
                 q.translate[1] == 0.f && q.translate[2] == 0.f;
    P[0] = make_float4(c.x, c.y, c.z, q.radius);
    P[1] = make_float4(n.x, n.y, n.z, q.height);
    P[2] = make_float4(u.x, u.y, u.z, q.wave_amplitude);
    P[3] = make_float4(v.x, v.y, v.z, q.wave_scale);
    P[4] = make_float4(R[0], R[1], R[2], q.scale);
    P[5] = make_float4(R[3], R[4], R[5], 1.0f / q.scale);
    P[6] = make_float4(R[6], R[7], R[8], ident ? 0.f : 1.f);
    P[7] = make_float4(q.translate[0], q.translate[1], q.translate[2], 0.f);
    Box ob;
    if (!planar) {
        H3 rr = h3(q.radius, 0.f, q.radius);
        ob = Box{c - rr, c + rr + h3(0.f, q.height, 0.f)};
    } else if (q.type == RT_SHAPE_DISK) {
        H3 ext = h3(q.radius * std::sqrt(std::fmax(1.f - n.x * n.x, 0.f)), q.radius * std::sqrt(std::fmax(1.f - n.y * n.y, 0.f)),
                    q.radius * std::sqrt(std::fmax(1.f - n.z * n.z, 0.f)));
        ob = pad(Box{c - ext, c + ext});
    } else {
        const float B = 1e5f, E = 1e-3f;
        float lo[3], hi[3], nn[3] = {n.x, n.y, n.z}, pp[3] = {c.x, c.y, c.z};
        for (int a = 0; a < 3; a++) {
            if (std::fabs(nn[a]) > 0.999f) { lo[a] = pp[a] - E; hi[a] = pp[a] + E; }
            else { lo[a] = -B; hi[a] = B; }
        }
        ob = Box{h3(lo[0], lo[1], lo[2]), h3(hi[0], hi[1], hi[2])};
    }
    if (ident) return ob;
    Box b{h3(INFINITY, INFINITY, INFINITY), h3(-INFINITY, -INFINITY, -INFINITY)};
    H3 t = h3(q.translate[0], q.translate[1], q.translate[2]);
    for (int k = 0; k < 8; k++) {
        H3 x = h3(k & 1 ? ob.mx.x : ob.mn.x, k & 2 ? ob.mx.y : ob.mn.y, k & 4 ? ob.mx.z : ob.mn.z) * q.scale;
        H3 w = rot_apply(R, x) + t;
        b = unite(b, Box{w, w});
    }
    float e = 1e-5f * std::max(std::max(std::fabs(b.mn.x), std::fabs(b.mx.x)),
                               std::max(std::max(std::fabs(b.mn.y), std::fabs(b.mx.y)),
                                        std::max(std::fabs(b.mn.z), std::fabs(b.mx.z)))) + 1e-6f;
    return Box{b.mn - h3(e, e, e), b.mx + h3(e, e, e)};
}

static inline float area(const Box& b) {
    H3 d = b.mx - b.mn;
    return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
}

// Reference-layout node (bvh.rs:25-32).
struct RefNode { float mn[3][8], mx[3][8]; int32_t ch[8]; };

// ── quantised node (128 B): the child boxes as 8-bit offsets from the node's
// lower corner p in steps of s = 2^e per axis, rounded outward so that the
// real planes p + q·s contain the exact child box (Ylitie et al. 2017 store
// child boxes this way; the rounding here is made conservative so the hits
// stay the brute-force ones).  Layout (float4 words):
//   0: p.x, p.y, p.z, (e_x + 127) | (e_y + 127) << 8 | (e_z + 127) << 16 | valid-slot mask << 24
//   1-3: per axis x, y, z: q_lo of slots 0-3, 4-7, then q_hi of slots 0-3, 4-7 (a byte each)
//   4-5: the 8 child references (as in the full node); 6-7: unused
// x − y rounded down / up, exactly (TwoSum gives the rounding error of x − y)
static inline float sub_dir(float x, float y, bool up) {
    float a = x, b = -y;
    float sm = a + b, bb = sm - a;
    float err = (a - (sm - bb)) + (b - bb);
    if (up) return err > 0.0f ? std::nextafter(sm, INFINITY) : sm;
    return err < 0.0f ? std::nextafter(sm, -INFINITY) : sm;
}
// quantise one node; false when an extent needs a step beyond 2^60 (steps are
// kept in [2^-60, 2^60], so with |1/d| in [2^-60, 2^60] every s/d is a normal float)
static bool encode_qnode(const RefNode& r, const float4* full, float4* out) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    uint32_t valid = 0;
    for (int c = 0; c < 8; c++) {
        if (r.ch[c] == INT32_MIN) continue;
        valid |= 1u << c;
        for (int a = 0; a < 3; a++) { lo[a] = std::fmin(lo[a], r.mn[a][c]); hi[a] = std::fmax(hi[a], r.mx[a][c]); }
    }
    if (!valid) for (int a = 0; a < 3; a++) lo[a] = hi[a] = 0.0f;
    int e[3];
    bool flat[3];
    int e_any = -60;
    for (int a = 0; a < 3; a++) {
        float ext = sub_dir(hi[a], lo[a], true);
        flat[a] = !(ext > 0.0f);
        if (flat[a]) continue;
        int ex;
        std::frexp(ext / 255.0f, &ex);              // ext/255 < 2^ex
        while (ex > -60 && std::ldexp(255.0f, ex - 1) >= ext) ex--;
        while (std::ldexp(255.0f, ex) < ext) ex++;
        e[a] = std::max(ex, -60);                    // steps of at least 2^-60
        e_any = std::max(e_any, e[a]);
    }
    for (int a = 0; a < 3; a++) {
        if (flat[a]) e[a] = e_any;
        if (e[a] > 60) return false;
    }
    uint8_t qlo[3][8], qhi[3][8];
    for (int a = 0; a < 3; a++) {
        float sa = std::ldexp(1.0f, e[a]);
        for (int c = 0; c < 8; c++) {
            if (!((valid >> c) & 1u)) { qlo[a][c] = 255; qhi[a][c] = 0; continue; }
            float dl = sub_dir(r.mn[a][c], lo[a], false), dh = sub_dir(r.mx[a][c], lo[a], true);
            float ql = std::floor(dl / sa), qh = std::ceil(dh / sa);
            qlo[a][c] = (uint8_t)std::min(std::max(ql, 0.0f), 255.0f);
            qhi[a][c] = (uint8_t)std::min(std::max(qh, 0.0f), 255.0f);
        }
    }
    uint32_t meta = (uint32_t)(e[0] + 127) | (uint32_t)(e[1] + 127) << 8 | (uint32_t)(e[2] + 127) << 16 | valid << 24;
    float fm;
    memcpy(&fm, &meta, 4);
    out[0] = make_float4(lo[0], lo[1], lo[2], fm);
    for (int a = 0; a < 3; a++) {
        uint32_t w[4] = {0, 0, 0, 0};
        for (int c = 0; c < 8; c++) {
            w[c >> 2] |= (uint32_t)qlo[a][c] << (8 * (c & 3));
            w[2 + (c >> 2)] |= (uint32_t)qhi[a][c] << (8 * (c & 3));
        }
        float f[4];
        memcpy(f, w, 16);
        out[1 + a] = make_float4(f[0], f[1], f[2], f[3]);
    }
    out[4] = full[12];
    out[5] = full[13];
    out[6] = out[7] = make_float4(0.f, 0.f, 0.f, 0.f);
    return true;
}

// ── binned-SAH 8-wide builder (cost model of bvh.rs:52-174) ─────────────────
// In place on an index array: each partition reorders idx[lo, hi) by a stable
// counting sort on bucket id, which is what the reference's stable
// `sort_by_key` + `partition_point` does (bvh.rs:132-137).
struct SahBuilder {
    const std::vector<Box>& boxes;
    std::vector<float> cen[3];
    std::vector<int32_t> idx, tmp;
    std::vector<RefNode> nodes;
    std::vector<int32_t> leaves;
    int max_depth = 0;

    explicit SahBuilder(const std::vector<Box>& b) : boxes(b) {
        size_t n = b.size();
        for (int a = 0; a < 3; a++) {
            cen[a].resize(n);
            for (size_t i = 0; i < n; i++) cen[a][i] = (hc(b[i].mn, a) + hc(b[i].mx, a)) * 0.5f;
        }
        idx.resize(n);
        tmp.resize(n);
        for (size_t i = 0; i < n; i++) idx[i] = (int32_t)i;
    }

    size_t partition(size_t lo, size_t hi) {
        const int NB = 12;
        size_t span = hi - lo;
        float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
        Box nb = boxes[idx[lo]];
        for (size_t k = lo; k < hi; k++) {
            int32_t o = idx[k];
            for (int a = 0; a < 3; a++) { cmn[a] = std::fmin(cmn[a], cen[a][o]); cmx[a] = std::fmax(cmx[a], cen[a][o]); }
            if (k > lo) nb = unite(nb, boxes[o]);
        }
        float nsa = area(nb);
        float best = INFINITY;
        int bax = 0, bsp = 0;
        for (int ax = 0; ax < 3; ax++) {
            float ext = cmx[ax] - cmn[ax];
            if (ext < 1e-6f) continue;
            bool has[NB] = {};
            Box bb[NB];
            uint32_t cnt[NB] = {};
            for (size_t k = lo; k < hi; k++) {
                int32_t o = idx[k];
                float t = (cen[ax][o] - cmn[ax]) / ext;
                int bi = std::min((int)((float)NB * t), NB - 1);
                cnt[bi]++;
                bb[bi] = has[bi] ? unite(bb[bi], boxes[o]) : boxes[o];
                has[bi] = true;
            }
            float lsa[NB];
            uint32_t ln[NB];
            bool ah = false;
            Box acc;
            uint32_t an = 0;
            for (int i = 0; i < NB; i++) {
                an += cnt[i];
                if (has[i]) { acc = ah ? unite(acc, bb[i]) : bb[i]; ah = true; }
                ln[i] = an;
                lsa[i] = ah ? area(acc) : 0.0f;
            }
            ah = false; an = 0;
            for (int s = NB - 2; s >= 0; s--) {
                an += cnt[s + 1];
                if (has[s + 1]) { acc = ah ? unite(acc, bb[s + 1]) : bb[s + 1]; ah = true; }
                uint32_t nl = ln[s], nr = an;
                if (nl == 0 || nr == 0) continue;
                float rsa = ah ? area(acc) : 0.0f;
                float cost = 1.0f + (lsa[s] * (float)nl + rsa * (float)nr) / nsa;
                if (cost < best) { best = cost; bax = ax; bsp = s; }
            }
        }
        float ext = cmx[bax] - cmn[bax];
        uint32_t cnt[NB] = {};
        std::vector<uint8_t> bid(span);
        for (size_t k = lo; k < hi; k++) {
            int bi = 0;
            if (!(ext < 1e-6f)) {
                float t = (cen[bax][idx[k]] - cmn[bax]) / ext;
                bi = std::min((int)((float)NB * t), NB - 1);
            }
            bid[k - lo] = (uint8_t)bi;
            cnt[bi]++;
        }
        uint32_t off[NB];
        uint32_t run = 0;
        size_t mid_off = 0;
        for (int b = 0; b < NB; b++) { off[b] = run; run += cnt[b]; if (b == bsp) mid_off = run; }
        for (size_t k = lo; k < hi; k++) tmp[lo + off[bid[k - lo]]++] = idx[k];
        std::copy(tmp.begin() + lo, tmp.begin() + hi, idx.begin() + lo);
        size_t mid = (mid_off == 0 || mid_off == span) ? span / 2 : mid_off;
        return lo + mid;
    }

    // ── binary SAH tree + greedy collapse to 8-wide nodes ───────────────────
    // The binary tree applies the reference's sah_partition recursively (the
    // same tree its fixed 3-level split walks), down to one primitive per
    // leaf.  The internal node that splits [lo, hi) at `mid` gets id mid − 1, a
    // bijection onto [0, n−1), so subtrees can be built by threads and the
    // result is still deterministic.  Children: ≥ 0 internal id, < 0 leaf
    // −(position in idx + 1).
    struct BinNode { int32_t l, r; Box box; };
    std::vector<BinNode> bin;

    void build_binary(size_t lo, size_t hi, int32_t* ref, Box* box, int depth) {
        if (hi - lo == 1) { *ref = -(int32_t)lo - 1; *box = boxes[idx[lo]]; return; }
        size_t mid = partition(lo, hi);
        int32_t id = (int32_t)mid - 1;
        BinNode& b = bin[id];
        Box lb, rb;
        if (depth < 4 && hi - lo > 65536) {
            std::thread t([&]() { build_binary(lo, mid, &b.l, &lb, depth + 1); });
            build_binary(mid, hi, &b.r, &rb, depth + 1);
            t.join();
        } else {
            build_binary(lo, mid, &b.l, &lb, depth + 1);
            build_binary(mid, hi, &b.r, &rb, depth + 1);
        }
        b.box = unite(lb, rb);
        *ref = id;
        *box = b.box;
    }

    const Box& bbox_of(int32_t ref) const { return ref >= 0 ? bin[ref].box : boxes[idx[-ref - 1]]; }

    // Wide node from binary node `b`: open the inner child of largest surface
    // area until 8 children (or only leaves) remain; preorder node numbering.
    int32_t collapse(int32_t b, int depth) {
        max_depth = std::max(max_depth, depth);
        int32_t kids[8];
        int nk = 2;
        kids[0] = bin[b].l; kids[1] = bin[b].r;
        while (nk < 8) {
            int best = -1;
            float ba = -1.0f;
            for (int i = 0; i < nk; i++)
                if (kids[i] >= 0) { float a = area(bin[kids[i]].box); if (a > ba) { ba = a; best = i; } }
            if (best < 0) break;
            int32_t o = kids[best];
            kids[best] = bin[o].l;
            kids[nk++] = bin[o].r;
        }
        size_t my = nodes.size();
        RefNode nd;
        memset(&nd, 0, sizeof(nd));
        for (int c = 0; c < 8; c++) nd.ch[c] = INT32_MIN;
        nodes.push_back(nd);
        for (int c = 0; c < nk; c++) {
            const Box cb = bbox_of(kids[c]);
            for (int a = 0; a < 3; a++) { nd.mn[a][c] = hc(cb.mn, a); nd.mx[a][c] = hc(cb.mx, a); }
            if (kids[c] < 0) {
                int32_t slot = (int32_t)leaves.size();
                leaves.push_back(idx[-kids[c] - 1]);
                nd.ch[c] = -(slot + 1);
            } else {
                nd.ch[c] = collapse(kids[c], depth + 1);
            }
        }
        nodes[my] = nd;
        return (int32_t)my;
    }

    // the binary tree from the device builder (rth::gpu_build_binary): the same
    // partition, so the same tree; 0 or a CUDA error
    int build_binary_device(int32_t* root, int sms, cudaStream_t st) {
        size_t n = boxes.size();
        std::vector<float> bx(n * 6), nb(n > 1 ? (n - 1) * 6 : 6);
        for (size_t i = 0; i < n; i++)
            for (int a = 0; a < 3; a++) { bx[i * 6 + a] = hc(boxes[i].mn, a); bx[i * 6 + 3 + a] = hc(boxes[i].mx, a); }
        std::vector<int32_t> l(n > 1 ? n - 1 : 1), r(n > 1 ? n - 1 : 1);
        int rc = rth::gpu_build_binary(bx.data(), (int32_t)n, idx.data(), l.data(), r.data(), nb.data(), root, sms, st);
        if (rc) return rc;
        for (size_t i = 0; i + 1 < n; i++) {
            bin[i].l = l[i]; bin[i].r = r[i];
            bin[i].box = Box{h3(nb[i * 6], nb[i * 6 + 1], nb[i * 6 + 2]), h3(nb[i * 6 + 3], nb[i * 6 + 4], nb[i * 6 + 5])};
        }
        return 0;
    }

    // device: build the binary tree on the GPU (sms > 0), else on the host threads
    int build_wide(int sms = 0, cudaStream_t st = 0) {
        size_t n = boxes.size();
        bin.assign(n > 1 ? n - 1 : 1, BinNode{});
        int32_t root;
        Box rb;
        if (sms > 0) {
            int rc = build_binary_device(&root, sms, st);
            if (rc) return rc;
            rb = root < 0 ? boxes[idx[-root - 1]] : bin[root].box;
        } else {
            build_binary(0, n, &root, &rb, 0);
        }
        if (root < 0) {                       // single primitive: one node with one leaf
            RefNode nd;
            memset(&nd, 0, sizeof(nd));
            for (int c = 0; c < 8; c++) nd.ch[c] = INT32_MIN;
            nd.ch[0] = -1;
            leaves.push_back(idx[0]);
            for (int a = 0; a < 3; a++) { nd.mn[a][0] = hc(rb.mn, a); nd.mx[a][0] = hc(rb.mx, a); }
            nodes.push_back(nd);
            return 0;
        }
        collapse(root, 0);
        return 0;
    }

};

// ── E_ss LUT on the host (material.rs:206-241), once per process ─────────────
static float g_elut[64 * 64];
static std::once_flag g_elut_once;
static void host_vndf(float wx, float wy, float wz, float alpha, float xi1, float xi2, float* m) {
    const float PI = 3.14159265358979323846f;
    H3 wh = h3(alpha * wx, alpha * wy, wz);
    wh = wh / hlen(wh);
    float len = std::sqrt(wh.x * wh.x + wh.y * wh.y);
    H3 t1 = len > 1e-6f ? h3(-wh.y / len, wh.x / len, 0.0f) : h3(1, 0, 0);
    H3 t2 = hcross(wh, t1);
    float a = 1.0f / (1.0f + wh.z);
    float r = std::sqrt(xi1);
    float p1, p2;
    if (xi2 < a) { float phi = xi2 / a * PI; p1 = r * std::cos(phi); p2 = r * std::sin(phi); }
    else { float phi = PI + (xi2 - a) / (1.0f - a) * PI; p1 = r * std::cos(phi); p2 = r * std::sin(phi) * wh.z; }
    float p3 = std::sqrt(std::fmax(1.0f - p1 * p1 - p2 * p2, 0.0f));
    H3 nh = t1 * p1 + t2 * p2 + wh * p3;
    H3 mm = h3(alpha * nh.x, alpha * nh.y, std::fmax(nh.z, 0.0f));
    mm = mm / hlen(mm);
    m[0] = mm.x; m[1] = mm.y; m[2] = mm.z;
}
static float host_lambda(float c, float alpha) {
    float a2 = alpha * alpha, c2 = c * c;
    return (std::sqrt(a2 + (1.0f - a2) * c2) - c) / (2.0f * c);
}
static void build_elut() {
    const int N = 64, G = 64;
    for (int i = 0; i < N; i++) {
        float mu = ((float)i + 0.5f) / (float)N;
        for (int j = 0; j < N; j++) {
            float alpha = std::fmax(((float)j + 0.5f) / (float)N, 1e-3f);
            float lo = host_lambda(mu, alpha);
            double sum = 0.0;
            uint32_t texel = (uint32_t)(i * N + j);
            for (int k = 0; k < G; k++)
                for (int l = 0; l < G; l++) {
                    uint32_t smp = (uint32_t)(k * G + l);
                    float r1 = (float)(pcg3d_x(texel, smp, 0xE55E0001u) >> 8) * (1.0f / 16777216.0f);
                    float r2 = (float)(pcg3d_x(texel, smp, 0xE55E0002u) >> 8) * (1.0f / 16777216.0f);
                    float m[3];
                    host_vndf(0.0f, 0.0f, mu, alpha, ((float)k + r1) / (float)G, ((float)l + r2) / (float)G, m);
                    float voh = std::fmax(mu * m[2], 0.0f);
                    // wi = 2·(wo·m)·m − wo, wo = (0, 0, mu)
                    float wiz = 2.0f * voh * m[2] - mu;
                    if (wiz <= 0.0f) continue;
                    float li = host_lambda(wiz, alpha);
                    sum += (double)((1.0f + lo) / (1.0f + lo + li));
                }
            g_elut[i * N + j] = (float)(sum / (double)(G * G));
        }
    }
}

static void xyz_srgb_h(float x, float y, float z, float o[3]) {
    o[0] = std::fmax(3.2406f * x - 1.5372f * y - 0.4986f * z, 0.0f);
    o[1] = std::fmax(-0.9689f * x + 1.8758f * y + 0.0415f * z, 0.0f);
    o[2] = std::fmax(0.0557f * x - 0.2040f * y + 1.0570f * z, 0.0f);
}
// NACRE_LUT (material.rs:1096-1118): the thin-film colour over OPD 0..2500 nm
// in 256 steps, the mean over 380..700 nm of spectral_to_rgb(λ)·½(1 + cos 2π·OPD/λ);
// spectral_to_rgb uses the 380..700 nm table and its per-channel normalisation
static float4 g_nacre[256];
static std::once_flag g_nacre_once;
static void build_nacre() {
    float sum[3] = {0, 0, 0};
    for (int i = 0; i < RT_CIE_N; i++) {
        float rgb[3];
        xyz_srgb_h(RT_CIE_XYZ[i][0], RT_CIE_XYZ[i][1], RT_CIE_XYZ[i][2], rgb);
        for (int k = 0; k < 3; k++) sum[k] += rgb[k];
    }
    float norm[3];
    for (int k = 0; k < 3; k++) norm[k] = (float)RT_CIE_N / std::fmax(sum[k], 1e-6f);
    for (int i = 0; i < 256; i++) {
        float opd = (float)i / 255.0f * 2500.0f;
        float c[3] = {0, 0, 0};
        for (float lambda = 380.0f; lambda <= 700.01f; lambda += 5.0f) {
            float t = std::fmin(std::fmax((lambda - 380.0f) / 5.0f, 0.0f), (float)(RT_CIE_N - 1));
            int k = std::min((int)t, RT_CIE_N - 2);
            float f = t - (float)k, xyz[3];
            for (int q = 0; q < 3; q++) xyz[q] = RT_CIE_XYZ[k][q] + f * (RT_CIE_XYZ[k + 1][q] - RT_CIE_XYZ[k][q]);
            float rgb[3];
            xyz_srgb_h(xyz[0], xyz[1], xyz[2], rgb);
            float irid = 0.5f * (1.0f + std::cos(2.0f * 3.14159265358979f * opd / lambda));
            for (int q = 0; q < 3; q++) c[q] = c[q] + rgb[q] * norm[q] * irid;
        }
        g_nacre[i] = make_float4(c[0] / 65.0f, c[1] / 65.0f, c[2] / 65.0f, 0.0f);
    }
}
static void fire_h(float x, float y, float z, float c[3]) {
    float w = std::fmax(std::pow(y, 0.5f), 0.08f);
    float rgb[3];
    xyz_srgb_h(x, y, z, rgb);
    for (int k = 0; k < 3; k++) c[k] = rgb[k] * w;
    float lum = 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
    for (int k = 0; k < 3; k++) c[k] = c[k] * (1.0f - 0.5f) + lum * 0.5f;
}
static float planck_h(float l, float tk) {
    float x = 14388000.0f / (l * tk);
    float l2 = l * l, l4 = l2 * l2;
    return 1.0f / (l * l4 * std::fmax(std::exp(x) - 1.0f, 1e-30f));
}

}  // namespace

// ── the scene handle ────────────────────────────────────────────────────────
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct RtScene {
    int device = 0, sms = 148;
    cudaStream_t stream = nullptr;
    // the caller's stream (rt_set_caller_stream; default: the legacy default
    // stream): every call first makes `stream` wait for the work already queued
    // there, so device buffers the caller is still writing are complete
    cudaStream_t caller = 0;
    cudaEvent_t caller_ev = nullptr;
    std::string err;
    DevScene S{};
    std::vector<DevBuf> owned;
    int64_t n_nodes = 0, n_leaves = 0, n_prims = 0;
    int32_t max_depth = 0;
    int stack_cap_built = 0;          // traversal stack entries the spill columns hold
    bool qnodes_ok = false;           // the quantised node copy exists (extents within 255·2^60)
    bool wide4_ok = false;            // the 4-wide node copy exists (trees built on the device)
    std::vector<DevLight> h_lights;   // host copy of the NEE light list (photon emitters from lights)
    std::vector<float> h_emission;    // per material: RGB emission of a light material (3 floats)
    float photon_stage_ms[3] = {0, 0, 0};   // last photon build: trace, compaction, tree
    uint64_t max_iterations = 0;      // wavefront iteration bound (rt_set_tuning; 0 = derived)
    mutable double sah_cost = 0.0;
    double build_ms = 0.0;
    // reference-layout copy for rt_scene_bvh_export and the SAH statistic; with
    // the device collapse it is made from the device nodes on first use
    mutable std::vector<RefNode> ref_nodes;
    mutable bool ref_ready = false;
    const int32_t* d_export_ch = nullptr;   // device collapse: children in export form, 8 per node
    std::vector<int32_t> leaf_gids;
    bool empty = true;
    // wavefront buffers (grown on demand)
    uint32_t cap = 0;
    PathState P{};                    // set 0 (also the photon tracer's state)
    PathState P2{};                   // set 1 (shares hit and gq with set 0)
    PathState Rt{};                   // retire records: L, pend0, pend1, pendC, meta
    rtgh::Guide* guide = nullptr;     // path-guiding network (rt_guide_init)
    uint32_t max_paths = 1u << 23;    // path-pool capacity (rt_set_tuning)
    uint32_t* queue[2] = {nullptr, nullptr};   // photon tracer queues
    ClassQueues cq{};
    float4* sq = nullptr;
    uint32_t* counters = nullptr;     // RT_CTR_WORDS (header + ring of iteration blocks)
    int* d_err = nullptr;
    uint32_t* d_bins = nullptr;       // ray binning histogram and cursors
    RenderLaunch* d_R = nullptr;      // device copy of the current call's RenderLaunch
    // the wavefront as one captured graph (rt_set_tuning graph = 1, and the
    // asynchronous entry point): kept while its key (buffers, scene state,
    // pool, flags) matches and its iteration capacity K covers the call's bound
    struct WaveGraph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        std::vector<uint8_t> key;
        uint64_t K = 0;
    } wg;
    bool graph_mode = false;
    uint32_t* d_gstat = nullptr;      // next-iteration ray count and iterations run, left by the graph
    uint64_t* h_tot = nullptr;        // pinned: ray totals of an asynchronous call
    bool async_pending = false;       // an asynchronous call's statistics wait for rt_sync
    int64_t async_per_it = 0;
    uint32_t* d_active = nullptr;     // active-pixel list of a converged mask
    uint32_t active_cap = 0;
    // lagged end-of-work check: next-iteration ray counts copied to pinned memory
    uint32_t* h_status = nullptr;
    cudaEvent_t st_ev[8] = {};
    // side streams of the per-class shading kernels (rth::launch_shade)
    ShadeFork fk{};
    float* scratch = nullptr;
    size_t scratch_bytes = 0;
    uint8_t* d_conv = nullptr;
    size_t conv_bytes = 0;
    // accumulators
    float *acc = nullptr, *m2 = nullptr;
    uint32_t* cnt = nullptr;
    uint32_t acc_npix = 0;
    // packed batches: accumulators of all requests and the device request table
    float *b_acc = nullptr, *b_m2 = nullptr;
    uint32_t* b_cnt = nullptr;
    uint64_t batch_pix = 0;
    JobDev* d_jobs = nullptr;
    uint32_t jobs_cap = 0;
    // api staging
    void* stage = nullptr;
    size_t stage_bytes = 0;
    // caustic photon map and the union of the primitive boxes (photon_bounds)
    PhotonMapDev photons;
    float world_lo[3] = {0, 0, 0}, world_hi[3] = {0, 0, 0};
    // per-stage profiling
    bool profiling = false;
    std::vector<cudaEvent_t> pev;
    std::vector<int> pkind;
    double kms[4] = {0, 0, 0, 0};
    int64_t kcount[4] = {0, 0, 0, 0};
    // ray capture (diagnostics)
    int32_t cap_depth = -1;
    float* cap_out = nullptr;
    int64_t cap_max = 0, cap_n = 0;
    // stats
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    int64_t last_ext = 0, last_shadow = 0, last_launches = 0;
};

static void free_paths(RtScene* s);
static inline float __int_as_float_h(int32_t v) { float f; memcpy(&f, &v, 4); return f; }

static int fail(RtScene* s, int code, const std::string& msg) {
    if (s) s->err = msg;
    return code;
}
#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(s, RT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static int dalloc(RtScene* s, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) return fail(s, RT_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    s->owned.push_back(DevBuf{*p, bytes});
    return RT_OK;
}
template <class T>
static int upload(RtScene* s, const T* src, size_t count, const T** dst) {
    void* p = nullptr;
    int rc = dalloc(s, &p, count * sizeof(T));
    if (rc) return rc;
    if (count) CK(cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice));
    *dst = (const T*)p;
    return RT_OK;
}

static void free_dev(void*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// Start of every call that launches work: make the scene's device current and
// order its stream after the work already queued on the caller's stream (the
// stream is non-blocking, so without this a caller kernel still writing an
// input buffer, or a caching allocator's freed block still in use, would race
// with the library's kernels).  Every call synchronises its own stream before
// it returns, so work the caller queues afterwards needs no ordering.
static int fold_async(RtScene* s);
static int enter(RtScene* s) {
    CK(cudaSetDevice(s->device));
    if (s->async_pending) {
        // a queued asynchronous call's statistics are folded before its
        // pinned status words are reused (its device status stays in the
        // error word for the next check)
        if (int rc = fold_async(s)) return rc;
    }
    CK(cudaEventRecord(s->caller_ev, s->caller));
    CK(cudaStreamWaitEvent(s->stream, s->caller_ev, 0));
    return RT_OK;
}
// SAH cost of a wide tree (statistics): Σ_inner area(node)/area(root) +
// Σ_leaf area(leaf)/area(root), inner nodes costing 1 per traversal
static double sah_cost_of(const std::vector<RefNode>& nodes) {
    if (nodes.empty()) return 0.0;
    Box rb{h3(INFINITY, INFINITY, INFINITY), h3(-INFINITY, -INFINITY, -INFINITY)};
    const RefNode& r0 = nodes[0];
    for (int c = 0; c < 8; c++) if (r0.ch[c] != INT32_MIN)
        rb = unite(rb, Box{h3(r0.mn[0][c], r0.mn[1][c], r0.mn[2][c]), h3(r0.mx[0][c], r0.mx[1][c], r0.mx[2][c])});
    double root_sa = area(rb), cost = 0.0;
    for (const RefNode& r : nodes) {
        Box nb{h3(INFINITY, INFINITY, INFINITY), h3(-INFINITY, -INFINITY, -INFINITY)};
        for (int c = 0; c < 8; c++) if (r.ch[c] != INT32_MIN) {
            Box cb{h3(r.mn[0][c], r.mn[1][c], r.mn[2][c]), h3(r.mx[0][c], r.mx[1][c], r.mx[2][c])};
            nb = unite(nb, cb);
            if (r.ch[c] < 0) cost += (double)area(cb) / root_sa;
        }
        cost += (double)area(nb) / root_sa;
    }
    return cost;
}

// the reference-layout nodes of a device-collapsed tree, downloaded on first use
static int ensure_ref_nodes(const RtScene* s) {
    if (s->ref_ready) return RT_OK;
    if (s->d_export_ch && s->n_nodes > 0) {
        std::vector<float4> nodes((size_t)s->n_nodes * 14);
        std::vector<int32_t> ch((size_t)s->n_nodes * 8);
        if (cudaSetDevice(s->device) != cudaSuccess ||
            cudaMemcpy(nodes.data(), s->S.nodes, nodes.size() * 16, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(ch.data(), s->d_export_ch, ch.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            return RT_ERR_CUDA;
        s->ref_nodes.assign((size_t)s->n_nodes, RefNode{});
        for (int64_t k = 0; k < s->n_nodes; k++) {
            RefNode& r = s->ref_nodes[k];
            const float* f = reinterpret_cast<const float*>(&nodes[(size_t)k * 14]);
            for (int c = 0; c < 8; c++) {
                r.ch[c] = ch[(size_t)k * 8 + c];
                bool empty = r.ch[c] == INT32_MIN;     // empty slots keep the reference's zero box
                for (int a = 0; a < 3; a++) {
                    r.mn[a][c] = empty ? 0.0f : f[a * 8 + c];
                    r.mx[a][c] = empty ? 0.0f : f[24 + a * 8 + c];
                }
            }
        }
    }
    s->sah_cost = sah_cost_of(s->ref_nodes);
    s->ref_ready = true;
    return RT_OK;
}

#define ENTER(s)                          \
    do {                                  \
        int rc_e_ = enter(s);             \
        if (rc_e_) return rc_e_;          \
    } while (0)

extern "C" {

int32_t rt_version(void) { return RT_API_VERSION; }

int32_t rt_device_count(int32_t* count) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
    if (count) *count = n;
    return RT_OK;
}

int32_t rt_last_error(const RtScene* s, char* buf, size_t len) {
    if (!buf || len == 0) return RT_ERR_INVALID;
    std::string m = s ? s->err : std::string("null scene");
    size_t n = std::min(len - 1, m.size());
    memcpy(buf, m.data(), n);
    buf[n] = 0;
    return RT_OK;
}

int32_t rt_scene_destroy(RtScene* s) {
    if (!s) return RT_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& b : s->owned) cudaFree(b.p);
    void* ps[] = {s->counters, s->d_err, s->scratch, s->d_conv, s->acc, s->m2, s->cnt, s->stage, s->d_active,
                  s->b_acc, s->b_m2, s->b_cnt, s->d_jobs, s->d_R, s->d_gstat, s->d_bins};
    if (s->wg.exec) cudaGraphExecDestroy(s->wg.exec);
    if (s->wg.graph) cudaGraphDestroy(s->wg.graph);
    if (s->h_tot) cudaFreeHost(s->h_tot);
    free_paths(s);
    rtgh::destroy(s->guide);
    s->photons.release();
    for (void* p : ps) if (p) cudaFree(p);
    for (auto e : s->pev) cudaEventDestroy(e);
    for (auto e : s->st_ev) if (e) cudaEventDestroy(e);
    if (s->h_status) cudaFreeHost(s->h_status);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->caller_ev) cudaEventDestroy(s->caller_ev);
    for (auto e : s->fk.join) if (e) cudaEventDestroy(e);
    if (s->fk.fork) cudaEventDestroy(s->fk.fork);
    for (auto q : s->fk.side) if (q) cudaStreamDestroy(q);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return RT_OK;
}

int32_t rt_scene_create(const RtSceneDesc* d, int32_t device, RtScene** out) {
    if (!d || !out) return RT_ERR_INVALID;
    *out = nullptr;
    RtScene* s = new RtScene();
    auto bail = [&](int rc) { RtScene* keep = s; *out = keep; return rc; };   // handle kept for rt_last_error
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bail(fail(s, RT_ERR_CUDA, "no CUDA device"));
    if (device < 0 || device >= ndev) return bail(fail(s, RT_ERR_INVALID, "device index out of range"));
    s->device = device;
    if (cudaSetDevice(device) != cudaSuccess) return bail(fail(s, RT_ERR_CUDA, "cudaSetDevice failed"));
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    s->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(s, RT_ERR_CUDA, "cudaStreamCreate failed"));
    cudaEventCreate(&s->ev0);
    cudaEventCreate(&s->ev1);
    if (cudaEventCreateWithFlags(&s->caller_ev, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(s, RT_ERR_CUDA, "cudaEventCreate failed"));
    for (auto& e : s->st_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(s, RT_ERR_CUDA, "cudaEventCreate failed"));
    for (auto& q : s->fk.side)
        if (cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(s, RT_ERR_CUDA, "cudaStreamCreate failed"));
    if (cudaEventCreateWithFlags(&s->fk.fork, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(s, RT_ERR_CUDA, "cudaEventCreate failed"));
    for (auto& e : s->fk.join)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(s, RT_ERR_CUDA, "cudaEventCreate failed"));
    if (cudaHostAlloc((void**)&s->h_status, 8 * sizeof(uint32_t), cudaHostAllocDefault) != cudaSuccess)
        return bail(fail(s, RT_ERR_NOMEM, "cudaHostAlloc status words"));

    // ── validate ────────────────────────────────────────────────────────────
    if (d->n_tris < 0 || d->n_quads < 0 || d->n_spheres < 0 || d->n_mats < 0 || d->n_lights < 0)
        return bail(fail(s, RT_ERR_INVALID, "negative count"));
    if (d->n_convex < 0 || (d->n_convex > 0 && (!d->convex || !d->convex_planes)))
        return bail(fail(s, RT_ERR_INVALID, "convex solids without their arrays"));
    // hit records carry a 27-bit index per primitive type
    if (d->n_tris > (int64_t)RT_HIT_MAX_INDEX + 1 || d->n_quads > (int64_t)RT_HIT_MAX_INDEX + 1 ||
        d->n_spheres > (int64_t)RT_HIT_MAX_INDEX + 1 || d->n_convex > (int64_t)RT_HIT_MAX_INDEX + 1 ||
        d->n_media > (int64_t)RT_HIT_MAX_INDEX + 1)
        return bail(fail(s, RT_ERR_CAPACITY, "more than 2^27 primitives of one type"));
    if (d->n_shapes < 0 || (d->n_shapes > 0 && !d->shapes)) return bail(fail(s, RT_ERR_INVALID, "shapes without their array"));
    const int64_t n_sph_end = d->n_tris + d->n_quads + d->n_spheres;   // canonical ids of the convex solids start here
    const int64_t n_cvx_end = n_sph_end + d->n_convex;                   // ... and of the other shapes here
    if (d->n_convex + d->n_shapes > (int64_t)RT_HIT_MAX_INDEX + 1)
        return bail(fail(s, RT_ERR_CAPACITY, "more than 2^27 convex solids and shapes"));
    int64_t n = n_cvx_end + d->n_shapes;
    if (n >= (1ll << 28) - 1) return bail(fail(s, RT_ERR_CAPACITY, "more than 2^28 - 2 primitives"));
    s->n_prims = n;
    if ((d->n_tris && (!d->tri_v || !d->tri_mat)) || (d->n_quads && (!d->quad_quv || !d->quad_mat)) ||
        (d->n_spheres && (!d->sphere || !d->sphere_mat)) || (d->n_mats && !d->mats) || (d->n_lights && !d->light_prims))
        return bail(fail(s, RT_ERR_INVALID, "null array with non-zero count"));
    auto bad_mat = [&](int32_t m) { return m < 0 || m >= d->n_mats; };
    for (int64_t i = 0; i < d->n_tris; i++) if (bad_mat(d->tri_mat[i])) return bail(fail(s, RT_ERR_INVALID, "triangle material index out of range"));
    for (int64_t i = 0; i < d->n_quads; i++) if (bad_mat(d->quad_mat[i])) return bail(fail(s, RT_ERR_INVALID, "quad material index out of range"));
    for (int64_t i = 0; i < d->n_spheres; i++) if (bad_mat(d->sphere_mat[i])) return bail(fail(s, RT_ERR_INVALID, "sphere material index out of range"));
    for (int32_t i = 0; i < d->n_mats; i++) {
        const RtMaterial& m = d->mats[i];
        if (m.type < RT_MAT_LAMBERTIAN || m.type > RT_MAT_PBR) return bail(fail(s, RT_ERR_INVALID, "unknown material type"));
        if (m.type == RT_MAT_PBR) {
            const float v[] = {m.albedo[0], m.albedo[1], m.albedo[2], m.roughness, m.metallic, m.anisotropy,
                               m.anisotropy_angle, m.clearcoat, m.clearcoat_roughness, m.film_thickness, m.film_ior,
                               m.sheen, m.sheen_tint, m.emission[0], m.emission[1], m.emission[2], m.emission_strength};
            for (float x : v)
                if (!std::isfinite(x)) return bail(fail(s, RT_ERR_INVALID, "non-finite PBR parameter"));
            if (m.film_thickness > 0.0f && !(m.film_ior > 0.0f))
                return bail(fail(s, RT_ERR_INVALID, "a PBR thin film needs a positive film_ior"));
        }
        if (m.type == RT_MAT_SPECTRAL_METAL && m.metal == RT_METAL_CUSTOM && (m.nk_count < 2 || m.nk_count > RT_MAX_NK || !(m.nk_step > 0.0f)))
            return bail(fail(s, RT_ERR_INVALID, "custom conductor table needs 2..16 samples and a positive step"));
        if (m.type == RT_MAT_SPECTRAL_METAL && (m.metal < RT_METAL_GOLD || m.metal > RT_METAL_CUSTOM))
            return bail(fail(s, RT_ERR_INVALID, "unknown conductor"));
    }
    if (d->n_lights > 4096) return bail(fail(s, RT_ERR_CAPACITY, "more than 4096 NEE lights"));
    for (int32_t i = 0; i < d->n_lights; i++) {
        int64_t g = d->light_prims[i];
        if (g < d->n_tris || g >= n_sph_end) return bail(fail(s, RT_ERR_INVALID, "light list entries must be quads or spheres"));
    }
    int64_t n_planes_total = 0, n_world_planes = 0;
    for (int64_t i = 0; i < d->n_convex; i++) {
        const RtConvex& c = d->convex[i];
        if (c.n_planes < 4 || c.n_planes > 1024 || c.plane_offset < 0 || bad_mat(c.mat))
            return bail(fail(s, RT_ERR_INVALID, "convex solid " + std::to_string(i) + ": 4..1024 planes and a valid material"));
        int mt = d->mats[c.mat].type;
        if (mt == RT_MAT_DIFFUSE_LIGHT || mt == RT_MAT_BLACKBODY_LIGHT)
            return bail(fail(s, RT_ERR_INVALID, "convex solid " + std::to_string(i) + ": emissive materials are not supported"));
        for (int a = 0; a < 3; a++)
            if (!(c.box_lo[a] <= c.box_hi[a]) || !std::isfinite(c.box_lo[a]) || !std::isfinite(c.box_hi[a]))
                return bail(fail(s, RT_ERR_INVALID, "convex solid " + std::to_string(i) + ": invalid box"));
        if (!(c.polish >= 0.0f && c.polish <= 0.25f) || !(c.scale > 0.0f) || !std::isfinite(c.scale) ||
            !rotation_ok(c.rot) || !std::isfinite(c.pivot[0] + c.pivot[1] + c.pivot[2]) ||
            !std::isfinite(c.translate[0] + c.translate[1] + c.translate[2]))
            return bail(fail(s, RT_ERR_INVALID, "convex solid " + std::to_string(i) +
                                                    ": polish in [0, 0.25], a positive scale, a rotation matrix"));
        n_planes_total = std::max<int64_t>(n_planes_total, (int64_t)c.plane_offset + c.n_planes);
        n_world_planes += c.n_planes;
    }
    for (int64_t k = 0; k < n_planes_total * 4; k++)
        if (!std::isfinite(d->convex_planes[k])) return bail(fail(s, RT_ERR_INVALID, "non-finite convex plane"));
    for (int64_t i = 0; i < d->n_shapes; i++) {
        const RtShape& q = d->shapes[i];
        std::string what = "shape " + std::to_string(i);
        if (q.type < RT_SHAPE_CYLINDER || q.type > RT_SHAPE_PLANE || bad_mat(q.mat))
            return bail(fail(s, RT_ERR_INVALID, what + ": unknown type or material"));
        int mt = d->mats[q.mat].type;
        if (mt == RT_MAT_DIFFUSE_LIGHT || mt == RT_MAT_BLACKBODY_LIGHT)
            return bail(fail(s, RT_ERR_INVALID, what + ": emissive materials are not supported (shapes are not NEE lights)"));
        float v[] = {q.center[0], q.center[1], q.center[2], q.normal[0], q.normal[1], q.normal[2], q.radius, q.height,
                     q.wave_amplitude, q.wave_scale, q.scale, q.translate[0], q.translate[1], q.translate[2]};
        for (float x : v)
            if (!std::isfinite(x)) return bail(fail(s, RT_ERR_INVALID, what + ": non-finite parameter"));
        bool planar = q.type == RT_SHAPE_DISK || q.type == RT_SHAPE_PLANE;
        float nl2 = q.normal[0] * q.normal[0] + q.normal[1] * q.normal[1] + q.normal[2] * q.normal[2];
        if (!(q.scale > 0.0f) || !rotation_ok(q.rot) || (planar && !(nl2 > 1e-12f)) ||
            (q.type != RT_SHAPE_PLANE && !(q.radius > 0.0f)) || (!planar && !(q.height > 0.0f)))
            return bail(fail(s, RT_ERR_INVALID, what + ": positive scale, radius and height, a non-zero normal, a rotation"));
    }
    if (d->tri_uv && !d->tri_tangent) return bail(fail(s, RT_ERR_INVALID, "tri_uv needs tri_tangent"));
    if (d->n_textures < 0 || (d->n_textures > 0 && !d->textures)) return bail(fail(s, RT_ERR_INVALID, "bad texture list"));
    for (int32_t i = 0; i < d->n_textures; i++) {
        const RtTexture& t = d->textures[i];
        bool ok = t.type == RT_TEX_IMAGE ? (t.width > 0 && t.height > 0 && t.rgb8 && (int64_t)t.width * t.height < (1ll << 31))
                : t.type == RT_TEX_MOTTLE ? std::isfinite(t.scale) : false;
        for (int k = 0; ok && t.type == RT_TEX_MOTTLE && k < 768; k++)
            ok = t.perlin_perm[k] >= 0 && t.perlin_perm[k] < 256 && std::isfinite(t.perlin_vec[k]);
        if (!ok) return bail(fail(s, RT_ERR_INVALID, "texture " + std::to_string(i) + ": bad image or mottle tables"));
    }
    for (int32_t i = 0; i < d->n_mats; i++) {
        const RtMaterial& m = d->mats[i];
        const int32_t ids[] = {m.albedo_tex, m.roughness_tex, m.metallic_tex, m.ao_tex, m.normal_tex};
        for (int32_t id : ids)
            if (id < 0 || id > d->n_textures) return bail(fail(s, RT_ERR_INVALID, "material texture id out of range"));
        if ((m.roughness_tex || m.metallic_tex || m.ao_tex || m.normal_tex) && m.type != RT_MAT_PBR)
            return bail(fail(s, RT_ERR_INVALID, "only PBR materials take roughness / metallic / ao / normal maps"));
        if (m.albedo_tex && m.type != RT_MAT_PBR && m.type != RT_MAT_LAMBERTIAN)
            return bail(fail(s, RT_ERR_INVALID, "albedo maps belong to Lambertian or PBR materials"));
        if (m.type == RT_MAT_PBR && (m.roughness_tex || m.metallic_tex || m.ao_tex || m.normal_tex || m.albedo_tex)) {
            const int32_t maps[] = {m.albedo_tex, m.roughness_tex, m.metallic_tex, m.ao_tex, m.normal_tex};
            for (int32_t id : maps)
                if (id && d->textures[id - 1].type != RT_TEX_IMAGE)
                    return bail(fail(s, RT_ERR_INVALID, "PBR maps must be image textures"));
        }
    }
    if (d->bg.type == RT_BG_ENVMAP && (!d->bg.env_rgb || d->bg.env_w <= 0 || d->bg.env_h <= 0))
        return bail(fail(s, RT_ERR_INVALID, "env map background without an image"));

    // ── primitive boxes, quad constants (quad.rs:21-33) ─────────────────────
    std::vector<Box> boxes(n);
    std::vector<float> qn(d->n_quads * 3), qd(d->n_quads), qw(d->n_quads * 3), qarea(d->n_quads);
    for (int64_t i = 0; i < d->n_tris; i++) {                                       // triangle.rs:128-140
        const float* v = d->tri_v + i * 9;
        H3 a = h3(v[0], v[1], v[2]);
        H3 e1 = h3(v[3], v[4], v[5]) - a, e2 = h3(v[6], v[7], v[8]) - a;
        H3 b = a + e1, c = a + e2;
        Box bb{h3(std::fmin(std::fmin(a.x, b.x), c.x), std::fmin(std::fmin(a.y, b.y), c.y), std::fmin(std::fmin(a.z, b.z), c.z)),
               h3(std::fmax(std::fmax(a.x, b.x), c.x), std::fmax(std::fmax(a.y, b.y), c.y), std::fmax(std::fmax(a.z, b.z), c.z))};
        boxes[i] = pad(bb);
    }
    for (int64_t i = 0; i < d->n_quads; i++) {
        const float* q = d->quad_quv + i * 9;
        H3 Q = h3(q[0], q[1], q[2]), u = h3(q[3], q[4], q[5]), v = h3(q[6], q[7], q[8]);
        H3 nn = hcross(u, v);
        float ar = hlen(nn);
        if (!(ar > 1e-6f * hlen(u) * hlen(v)))
            return bail(fail(s, RT_ERR_INVALID, "degenerate quad " + std::to_string(i) + ": u and v are parallel or zero"));
        H3 nrm = nn / ar, w = nn / hdot(nn, nn);
        qn[i * 3] = nrm.x; qn[i * 3 + 1] = nrm.y; qn[i * 3 + 2] = nrm.z;
        qd[i] = hdot(nrm, Q);
        qw[i * 3] = w.x; qw[i * 3 + 1] = w.y; qw[i * 3 + 2] = w.z;
        qarea[i] = ar;
        H3 cs[4] = {Q, Q + u, Q + v, Q + u + v};
        Box bb{cs[0], cs[0]};
        for (int k = 1; k < 4; k++) bb = unite(bb, Box{cs[k], cs[k]});
        boxes[d->n_tris + i] = pad(bb);
    }
    for (int64_t i = 0; i < d->n_spheres; i++) {
        const float* p = d->sphere + i * 4;
        H3 c = h3(p[0], p[1], p[2]), r = h3(p[3], p[3], p[3]);
        boxes[d->n_tris + d->n_quads + i] = Box{c - r, c + r};
    }
    // convex solids: planes, shading normals and boxes in world space
    std::vector<float4> wpl(std::max<int64_t>(n_world_planes, 1)), wsh(std::max<int64_t>(n_world_planes * 2, 2));
    std::vector<int32_t> wofs(d->n_convex);
    for (int64_t i = 0, o = 0; i < d->n_convex; i++) {
        const RtConvex& c = d->convex[i];
        wofs[i] = (int32_t)o;
        place_convex(c, d->convex_planes + (size_t)c.plane_offset * 4, wpl.data() + o, wsh.data() + o * 2);
        boxes[n_sph_end + i] = placed_box(c);
        o += c.n_planes;
    }

    // other shapes: 8 float4 each (shape_params) and their boxes
    std::vector<float4> gshape(std::max<int64_t>(d->n_shapes * 8, 8));
    for (int64_t i = 0; i < d->n_shapes; i++) boxes[n_cvx_end + i] = shape_params(d->shapes[i], gshape.data() + i * 8);

    // the photon-emitter bounds leave infinite planes out (plane.rs:97-102)
    bool any = false;
    Box wb{};
    for (int64_t i = 0; i < n; i++) {
        if (i >= n_cvx_end && d->shapes[i - n_cvx_end].type == RT_SHAPE_PLANE) continue;
        wb = any ? unite(wb, boxes[i]) : boxes[i];
        any = true;
    }
    if (any)
        for (int a = 0; a < 3; a++) { s->world_lo[a] = hc(wb.mn, a); s->world_hi[a] = hc(wb.mx, a); }

    // ── BVH ─────────────────────────────────────────────────────────────────
    std::vector<float4> gnodes;
    std::vector<float4> gtri, gtri_n, gquad, gsph, gtri_uv, gtri_tan;
    if (n > 0) {
        SahBuilder B(boxes);
        // the tree is built on the device (the binary SAH tree and its collapse to
        // 8-wide nodes) unless the description asks for the host builder
        const bool dev_wide = d->bvh_builder != RT_BVH_HOST && n >= 2;
        rth::WideOut W;
        auto tb = std::chrono::steady_clock::now();
        if (dev_wide) {
            std::vector<float> bx((size_t)n * 6);
            for (int64_t i = 0; i < n; i++)
                for (int a = 0; a < 3; a++) { bx[i * 6 + a] = hc(boxes[i].mn, a); bx[i * 6 + 3 + a] = hc(boxes[i].mx, a); }
            B.leaves.resize((size_t)n);
            W.type_end[0] = d->n_tris; W.type_end[1] = d->n_tris + d->n_quads; W.type_end[2] = n_sph_end;
            W.leaf_gids_h = B.leaves.data();
            int32_t root = 0;
            int brc = rth::gpu_build_binary(bx.data(), (int32_t)n, nullptr, nullptr, nullptr, nullptr, &root, s->sms,
                                            s->stream, &W);
            if (brc) return bail(fail(s, RT_ERR_CUDA, std::string("device BVH build: ") + cudaGetErrorString((cudaError_t)brc)));
            void* owned_ptrs[] = {W.nodes, W.qnodes, W.export_ch, W.nodes4};
            for (void* p : owned_ptrs) if (p) s->owned.push_back(DevBuf{p, 0});
            B.max_depth = W.max_depth;
        } else {
            int brc = B.build_wide(d->bvh_builder == RT_BVH_HOST ? 0 : s->sms, s->stream);
            if (brc) return bail(fail(s, RT_ERR_CUDA, std::string("device BVH build: ") + cudaGetErrorString((cudaError_t)brc)));
        }
        s->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
        s->max_depth = B.max_depth;
        // traversal stack: a visit of a node at depth k leaves at most 7 entries
        // per level above it, so 7 · (depth + 1) entries always suffice; the
        // ones beyond the shared-memory ring spill to a column per persistent
        // traversal thread (grid ≤ SMs × RT_TRACE_MINB blocks)
        if (B.max_depth > 4096) return bail(fail(s, RT_ERR_CAPACITY, "BVH deeper than 4096 levels"));
        s->stack_cap_built = 7 * (B.max_depth + 1) + 8;
        // the 4-wide tree is deeper; a visit there pushes at most 3 entries
        if (dev_wide) s->stack_cap_built = std::max(s->stack_cap_built, 3 * (W.max_depth4 + 1) + 8);
        s->S.stack_cap = s->stack_cap_built;
        s->S.stack_ring = RT_SHORT_STACK;
        size_t spill_entries = (size_t)s->stack_cap_built;   // also room for a ring shrunk by rt_set_tuning
        size_t spill_threads = (size_t)s->sms * RT_TRACE_MINB * RT_TRACE_BLOCK;
        void* sp_buf = nullptr;
        if (int rc = dalloc(s, &sp_buf, std::max<size_t>(spill_entries, 1) * spill_threads * sizeof(uint32_t)))
            return bail(rc);
        s->S.stack_spill = (uint32_t*)sp_buf;
        s->ref_nodes = std::move(B.nodes);
        s->leaf_gids = std::move(B.leaves);
        s->n_nodes = dev_wide ? W.n_nodes : (int64_t)s->ref_nodes.size();
        s->n_leaves = (int64_t)s->leaf_gids.size();
        s->d_export_ch = W.export_ch;
        s->ref_ready = !dev_wide;
        // leaf order per type
        std::vector<int32_t> typed_slot(s->n_leaves);
        std::vector<int64_t> order_tri, order_quad, order_sph, order_cvx;
        if (dev_wide) {   // the device's leaf order must be a permutation of the primitives
            std::vector<uint8_t> seen((size_t)n, 0);
            for (int64_t k = 0; k < s->n_leaves; k++) {
                int64_t g = s->leaf_gids[k];
                if (g < 0 || g >= n || seen[g]) return bail(fail(s, RT_ERR_CUDA, "device BVH collapse: invalid leaf order"));
                seen[g] = 1;
            }
        }
        for (int64_t k = 0; k < s->n_leaves; k++) {
            int64_t g = s->leaf_gids[k];
            if (g < d->n_tris) { typed_slot[k] = (int32_t)order_tri.size(); order_tri.push_back(g); }
            else if (g < d->n_tris + d->n_quads) { typed_slot[k] = (int32_t)order_quad.size(); order_quad.push_back(g - d->n_tris); }
            else if (g < n_sph_end) { typed_slot[k] = (int32_t)order_sph.size(); order_sph.push_back(g - d->n_tris - d->n_quads); }
            else { typed_slot[k] = (int32_t)order_cvx.size(); order_cvx.push_back(g - n_sph_end); }
        }
        if (!dev_wide) gnodes.resize((size_t)s->n_nodes * 14);
        for (int64_t k = 0; k < (dev_wide ? 0 : s->n_nodes); k++) {
            const RefNode& r = s->ref_nodes[k];
            float* f = reinterpret_cast<float*>(&gnodes[(size_t)k * 14]);
            // an empty slot gets an inverted box (+inf, −inf): its slab test fails
            // by itself on the traversal's fast path
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 8; c++) {
                    bool empty = r.ch[c] == INT32_MIN;
                    f[a * 8 + c] = empty ? INFINITY : r.mn[a][c];
                    f[24 + a * 8 + c] = empty ? -INFINITY : r.mx[a][c];
                }
            uint32_t* ch = reinterpret_cast<uint32_t*>(f + 48);
            for (int c = 0; c < 8; c++) {
                int32_t v = r.ch[c];
                if (v == INT32_MIN) ch[c] = RT_EMPTY_REF;
                else if (v >= 0) ch[c] = (uint32_t)v;
                else {
                    int64_t slot = -(int64_t)v - 1;
                    int64_t g = s->leaf_gids[slot];
                    uint32_t type = g < d->n_tris ? RT_PRIM_TRI : (g < d->n_tris + d->n_quads ? RT_PRIM_QUAD
                                                                  : (g < n_sph_end ? RT_PRIM_SPHERE : RT_PRIM_CONVEX));
                    ch[c] = RT_LEAF_BIT | (type << 28) | (uint32_t)typed_slot[slot];
                }
            }
        }
        if (!dev_wide) s->sah_cost = sah_cost_of(s->ref_nodes);
        // primitive records in leaf order
        gtri.resize(order_tri.size() * 3);
        bool has_n = d->tri_n != nullptr;
        if (has_n) gtri_n.resize(order_tri.size() * 3);
        bool has_uv = d->tri_uv != nullptr;
        if (has_uv) { gtri_uv.resize(order_tri.size() * 2); gtri_tan.resize(order_tri.size() * 3); }
        for (size_t k = 0; k < order_tri.size(); k++) {
            int64_t g = order_tri[k];
            if (has_uv) {
                const float* u = d->tri_uv + g * 6;
                gtri_uv[k * 2] = make_float4(u[0], u[1], u[2], u[3]);
                gtri_uv[k * 2 + 1] = make_float4(u[4], u[5], 0.f, 0.f);
                const float* t = d->tri_tangent + g * 9;
                gtri_tan[k * 3] = make_float4(t[0], t[1], t[2], t[3]);
                gtri_tan[k * 3 + 1] = make_float4(t[4], t[5], t[6], t[7]);
                gtri_tan[k * 3 + 2] = make_float4(t[8], 0.f, 0.f, 0.f);
            }
            const float* v = d->tri_v + g * 9;
            H3 a = h3(v[0], v[1], v[2]);
            H3 e1 = h3(v[3], v[4], v[5]) - a, e2 = h3(v[6], v[7], v[8]) - a;
            gtri[k * 3] = make_float4(a.x, a.y, a.z, e1.x);
            gtri[k * 3 + 1] = make_float4(e1.y, e1.z, e2.x, e2.y);
            int32_t gi = (int32_t)g, mi = d->tri_mat[g], hn = has_n ? 1 : 0;
            float fg, fm, fh;
            memcpy(&fg, &gi, 4); memcpy(&fm, &mi, 4); memcpy(&fh, &hn, 4);
            gtri[k * 3 + 2] = make_float4(e2.z, fg, fm, fh);
            if (has_n) {
                const float* nn = d->tri_n + g * 9;
                gtri_n[k * 3] = make_float4(nn[0], nn[1], nn[2], nn[3]);
                gtri_n[k * 3 + 1] = make_float4(nn[4], nn[5], nn[6], nn[7]);
                gtri_n[k * 3 + 2] = make_float4(nn[8], 0.f, 0.f, 0.f);
            }
        }
        auto quad_rec = [&](int64_t qi, float4* out5, int32_t gid) {
            const float* q = d->quad_quv + qi * 9;
            out5[0] = make_float4(qn[qi * 3], qn[qi * 3 + 1], qn[qi * 3 + 2], qd[qi]);
            out5[1] = make_float4(q[0], q[1], q[2], q[3]);
            out5[2] = make_float4(q[4], q[5], q[6], q[7]);
            out5[3] = make_float4(q[8], qw[qi * 3], qw[qi * 3 + 1], qw[qi * 3 + 2]);
            int32_t mi = d->quad_mat[qi];
            float fg, fm;
            memcpy(&fg, &gid, 4); memcpy(&fm, &mi, 4);
            out5[4] = make_float4(fg, fm, qarea[qi], 0.f);
        };
        gquad.resize(order_quad.size() * 5);
        for (size_t k = 0; k < order_quad.size(); k++)
            quad_rec(order_quad[k], &gquad[k * 5], (int32_t)(d->n_tris + order_quad[k]));
        gsph.resize(order_sph.size() * 2);
        for (size_t k = 0; k < order_sph.size(); k++) {
            int64_t si = order_sph[k];
            const float* p = d->sphere + si * 4;
            int32_t gi = (int32_t)(d->n_tris + d->n_quads + si), mi = d->sphere_mat[si];
            float fg, fm;
            memcpy(&fg, &gi, 4); memcpy(&fm, &mi, 4);
            gsph[k * 2] = make_float4(p[0], p[1], p[2], p[3]);
            gsph[k * 2 + 1] = make_float4(fg, fm, 0.f, 0.f);
        }
        // lights
        std::vector<DevLight> lights(d->n_lights);
        for (int32_t i = 0; i < d->n_lights; i++) {
            int64_t g = d->light_prims[i];
            DevLight& L = lights[i];
            memset(&L, 0, sizeof(L));
            if (g < d->n_tris + d->n_quads) {
                int64_t qi = g - d->n_tris;
                L.type = RT_PRIM_QUAD;
                L.mat = d->quad_mat[qi];
                quad_rec(qi, L.g, (int32_t)g);
            } else {
                int64_t si = g - d->n_tris - d->n_quads;
                const float* p = d->sphere + si * 4;
                L.type = RT_PRIM_SPHERE;
                L.mat = d->sphere_mat[si];
                L.g[0] = make_float4(p[0], p[1], p[2], p[3]);
            }
        }
        // convex solids in leaf order, pointing at their world-space planes
        // (shapes share the leaf type: their count field is −1 − RT_SHAPE_*, the
        // offset indexes shape_par)
        std::vector<float4> gcvx(std::max<size_t>(order_cvx.size() * 2, 2));
        for (size_t k = 0; k < order_cvx.size(); k++) {
            int64_t j = order_cvx[k];
            int32_t gi = (int32_t)(n_sph_end + j);
            if (j < d->n_convex) {
                const RtConvex& c = d->convex[j];
                gcvx[k * 2] = make_float4(__int_as_float_h(wofs[j]), __int_as_float_h(c.n_planes),
                                          __int_as_float_h(c.mat), c.polish);
            } else {
                const RtShape& q = d->shapes[j - d->n_convex];
                gcvx[k * 2] = make_float4(__int_as_float_h((int32_t)((j - d->n_convex) * 8)),
                                          __int_as_float_h(-1 - q.type), __int_as_float_h(q.mat), 0.f);
            }
            gcvx[k * 2 + 1] = make_float4(__int_as_float_h(gi), 0.f, 0.f, 0.f);
        }
        int rc;
        if ((rc = upload(s, gshape.data(), gshape.size(), &s->S.shape_par))) return bail(rc);
        s->S.n_analytic = (int)(d->n_convex + d->n_shapes);
        if ((rc = upload(s, gcvx.data(), gcvx.size(), &s->S.cvx))) return bail(rc);
        if ((rc = upload(s, wpl.data(), wpl.size(), &s->S.cvx_planes))) return bail(rc);
        if ((rc = upload(s, wsh.data(), wsh.size(), &s->S.cvx_shade))) return bail(rc);
        if (dev_wide) {
            s->S.nodes = W.nodes;
            s->S.qnodes = W.qnodes;
            s->qnodes_ok = W.qnodes != nullptr;
            s->S.nodes4 = W.nodes4;
            s->wide4_ok = W.nodes4 != nullptr;
            s->S.node_format = RT_NODES_FULL;
        } else if ((rc = upload(s, gnodes.data(), gnodes.size(), &s->S.nodes))) {
            return bail(rc);
        } else {   // the quantised copy of the nodes (rt_set_tuning node_format RT_NODES_QUANTISED)
            std::vector<float4> qn((size_t)s->n_nodes * 8);
            bool qok = true;
            for (int64_t k = 0; k < s->n_nodes && qok; k++)
                qok = encode_qnode(s->ref_nodes[k], &gnodes[(size_t)k * 14], &qn[(size_t)k * 8]);
            if (qok) {
                if ((rc = upload(s, qn.data(), qn.size(), &s->S.qnodes))) return bail(rc);
                s->qnodes_ok = true;
            }
            s->S.node_format = RT_NODES_FULL;
        }
        if ((rc = upload(s, gtri.data(), gtri.size(), &s->S.tri))) return bail(rc);
        if ((rc = upload(s, gtri_n.data(), gtri_n.size(), &s->S.tri_n))) return bail(rc);
        if (!gtri_uv.empty()) {
            if ((rc = upload(s, gtri_uv.data(), gtri_uv.size(), &s->S.tri_uv))) return bail(rc);
            if ((rc = upload(s, gtri_tan.data(), gtri_tan.size(), &s->S.tri_tan))) return bail(rc);
        }
        if ((rc = upload(s, gquad.data(), gquad.size(), &s->S.quad))) return bail(rc);
        if ((rc = upload(s, gsph.data(), gsph.size(), &s->S.sphere))) return bail(rc);
        if ((rc = upload(s, lights.data(), lights.size(), &s->S.lights))) return bail(rc);
        s->h_lights = lights;
        s->S.n_lights = d->n_lights;
        s->empty = false;
    }

    // ── spectral tables (spectrum.rs:78-177) ────────────────────────────────
    int nspec = d->spectral_range ? RT_CIE_N + RT_CIE_EXT_N : RT_CIE_N;
    std::vector<float4> cmf(nspec);
    float sum[3] = {0, 0, 0}, fsum[3] = {0, 0, 0};
    for (int i = 0; i < nspec; i++) {
        const float* x = i < RT_CIE_N ? RT_CIE_XYZ[i] : RT_CIE_XYZ_EXT[i - RT_CIE_N];
        cmf[i] = make_float4(x[0], x[1], x[2], 0.f);
        float rgb[3], fc[3];
        xyz_srgb_h(x[0], x[1], x[2], rgb);
        fire_h(x[0], x[1], x[2], fc);
        for (int k = 0; k < 3; k++) { sum[k] += rgb[k]; fsum[k] += fc[k]; }
    }
    for (int k = 0; k < 3; k++) {
        s->S.norms[k] = (float)nspec / std::fmax(sum[k], 1e-6f);
        s->S.fire_norms[k] = (float)nspec / std::fmax(fsum[k], 1e-6f);
    }
    s->S.n_spec = nspec;
    s->S.lam_lo = 380.0f;
    s->S.lam_range = d->spectral_range ? 400.0f : 320.0f;
    int rc;
    if ((rc = upload(s, cmf.data(), cmf.size(), &s->S.cmf))) return bail(rc);

    // ── materials (+ blackbody constants, material.rs:47-62) ─────────────────
    std::vector<DevMaterial> mats(std::max(d->n_mats, 1));
    int n_pbr = 0;
    for (int32_t i = 0; i < d->n_mats; i++) {
        const RtMaterial& m = d->mats[i];
        DevMaterial& g = mats[i];
        memset(&g, 0, sizeof(g));
        g.type = m.type;
        g.metal = m.metal;
        for (int k = 0; k < 3; k++) { g.albedo[k] = m.albedo[k]; g.odd[k] = m.odd[k]; g.absorption[k] = m.absorption[k]; }
        g.checker_scale = m.checker_scale;
        g.cauchy_b = m.cauchy_b;
        g.cauchy_c = m.cauchy_c;
        g.roughness = m.roughness;
        g.temp_k = m.temp_k;
        g.intensity = m.intensity;
        if (m.type == RT_MAT_SPECTRAL_METAL) {
            if (m.metal == RT_METAL_CUSTOM) {
                g.nk_count = m.nk_count; g.nk_start = m.nk_start; g.nk_step = m.nk_step;
                for (int k = 0; k < m.nk_count; k++) { g.nk_n[k] = m.nk_n[k]; g.nk_k[k] = m.nk_k[k]; }
            } else {
                g.nk_count = RT_METAL_NK_N; g.nk_start = RT_METAL_NK_START; g.nk_step = RT_METAL_NK_STEP;
                for (int k = 0; k < RT_METAL_NK_N; k++) { g.nk_n[k] = RT_METAL_NK[m.metal][0][k]; g.nk_k[k] = RT_METAL_NK[m.metal][1][k]; }
            }
        }
        g.albedo_tex = m.albedo_tex; g.roughness_tex = m.roughness_tex; g.metallic_tex = m.metallic_tex;
        g.ao_tex = m.ao_tex; g.normal_tex = m.normal_tex;
        if (m.type == RT_MAT_PBR) {                                                 // material.rs:790-800
            g.metallic = m.metallic;
            g.aniso_c = std::cos(m.anisotropy_angle);
            g.aniso_s = std::sin(m.anisotropy_angle);
            g.aspect = std::sqrt(std::fmax(1.0f - 0.9f * std::fmin(std::fmax(m.anisotropy, 0.0f), 1.0f), 0.001f));
            g.clearcoat = m.clearcoat;
            g.clearcoat_roughness = m.clearcoat_roughness;
            g.film_thickness = m.film_thickness;
            g.film_ior = m.film_ior;
            g.sheen = m.sheen;
            g.sheen_tint = m.sheen_tint;
            for (int c = 0; c < 3; c++) g.emission[c] = m.emission[c] * m.emission_strength;
            n_pbr++;
        }
        if (m.type == RT_MAT_BLACKBODY_LIGHT) {
            std::vector<float> raw(nspec);
            float su = 0.0f;
            for (int k = 0; k < nspec; k++) { raw[k] = planck_h(380.0f + (float)k * 5.0f, m.temp_k); su += raw[k]; }
            float norm = 1.0f / std::fmax(su / (float)nspec, 1e-30f);
            float acc[3] = {0, 0, 0};
            for (int k = 0; k < nspec; k++) {
                // spectral_to_rgb at the grid wavelength: t is exact, frac = 0
                int kk = std::min(k, nspec - 2);
                float frac = (float)k - (float)kk;
                float xyz[3];
                const float4 a = cmf[kk], b = cmf[kk + 1];
                xyz[0] = a.x + frac * (b.x - a.x);
                xyz[1] = a.y + frac * (b.y - a.y);
                xyz[2] = a.z + frac * (b.z - a.z);
                float rgb[3];
                xyz_srgb_h(xyz[0], xyz[1], xyz[2], rgb);
                for (int c = 0; c < 3; c++) acc[c] = acc[c] + (rgb[c] * s->S.norms[c]) * (raw[k] * norm);
            }
            g.bb_norm = norm;
            for (int c = 0; c < 3; c++) g.bb_avg[c] = acc[c] / (float)nspec * m.intensity;
        }
    }
    if ((rc = upload(s, mats.data(), mats.size(), &s->S.mats))) return bail(rc);
    // the emission colour of every material, for photon emitters built from lights
    s->h_emission.assign(mats.size() * 3, 0.0f);
    for (size_t i = 0; i < (size_t)d->n_mats; i++) {
        const DevMaterial& g = mats[i];
        for (int c = 0; c < 3; c++)
            s->h_emission[i * 3 + c] = g.type == RT_MAT_DIFFUSE_LIGHT ? g.albedo[c]
                                     : g.type == RT_MAT_BLACKBODY_LIGHT ? g.bb_avg[c]
                                     : g.type == RT_MAT_PBR ? g.emission[c] : 0.0f;
    }
    s->S.n_pbr = n_pbr;
    s->S.n_mats = d->n_mats;
    std::vector<uint8_t> codes(mats.size(), 1);
    for (int32_t i = 0; i < d->n_mats; i++) {
        int t = d->mats[i].type;
        codes[i] = (t == RT_MAT_DIFFUSE_LIGHT || t == RT_MAT_BLACKBODY_LIGHT) ? 0
                 : t == RT_MAT_SPECTRAL_METAL ? 2
                 : (t == RT_MAT_DIELECTRIC || t == RT_MAT_SPECTRAL_DIELECTRIC) ? 3
                 : t == RT_MAT_PBR ? 4 : 1;
    }
    if ((rc = upload(s, codes.data(), codes.size(), &s->S.mat_code))) return bail(rc);
    // shading classes the scene can produce: a miss always, a hit's class from
    // its material's code (launches of the other classes' kernels are skipped)
    s->S.class_mask = 1u << CLS_MISS;
    for (int32_t i = 0; i < d->n_mats; i++) s->S.class_mask |= 1u << (CLS_EMIT + codes[i]);
    if (d->n_media > 0) s->S.class_mask |= 1u << CLS_MEDIUM;

    // ── participating media (scene_file.rs:962-983, volume.rs:88-97, 170-186) ─
    if (d->n_media < 0 || (d->n_media > 0 && !d->media)) return bail(fail(s, RT_ERR_INVALID, "bad media list"));
    if (d->n_media > 0) {
        std::vector<DevMedium> dm(d->n_media);
        for (int32_t i = 0; i < d->n_media; i++) {
            const RtMedium& m = d->media[i];
            bool ok = (m.type == RT_MEDIUM_CONSTANT || m.type == RT_MEDIUM_NOISE || m.type == RT_MEDIUM_GRID) &&
                      (m.boundary == RT_BOUND_SPHERE || m.boundary == RT_BOUND_BOX) && std::isfinite(m.density) &&
                      m.density >= 0.0f && (m.boundary != RT_BOUND_SPHERE || m.radius > 0.0f);
            if (!ok) return bail(fail(s, RT_ERR_INVALID, "invalid medium " + std::to_string(i)));
            if (m.type == RT_MEDIUM_GRID) {
                bool gok = m.boundary == RT_BOUND_BOX && m.grid != nullptr;
                for (int a = 0; a < 3; a++) gok = gok && m.grid_res[a] >= 1 && m.grid_res[a] <= RT_GRID_MAX_RES;
                if (!gok)
                    return bail(fail(s, RT_ERR_INVALID, "grid medium " + std::to_string(i) +
                                                            " needs a box boundary, a grid and 1 .. 1024 voxels per axis"));
            }
            DevMedium& g = dm[i];
            memset(&g, 0, sizeof(g));
            g.type = m.type;
            g.boundary = m.boundary;
            g.sphere = make_float4(m.center[0], m.center[1], m.center[2], m.radius);
            g.density = m.type == RT_MEDIUM_NOISE ? std::fmax(m.density, FLT_EPSILON) : m.density;
            g.g = m.g;
            g.noise_scale = m.noise_scale;
            g.threshold = std::fmin(std::fmax(m.threshold, 0.0f), 0.99f);
            g.color = make_float3(m.color[0], m.color[1], m.color[2]);
            Box mb;
            if (m.boundary == RT_BOUND_BOX) {                                        // quad.rs:201-215
                H3 mn = h3(std::fmin(m.p_min[0], m.p_max[0]), std::fmin(m.p_min[1], m.p_max[1]), std::fmin(m.p_min[2], m.p_max[2]));
                H3 mx = h3(std::fmax(m.p_min[0], m.p_max[0]), std::fmax(m.p_min[1], m.p_max[1]), std::fmax(m.p_min[2], m.p_max[2]));
                H3 dx = h3(mx.x - mn.x, 0, 0), dy = h3(0, mx.y - mn.y, 0), dz = h3(0, 0, mx.z - mn.z);
                H3 nz = h3(-dz.x, -dz.y, -dz.z), nx = h3(-dx.x, -dx.y, -dx.z);
                H3 faces[6][3] = {{h3(mn.x, mn.y, mx.z), dx, dy}, {h3(mx.x, mn.y, mx.z), nz, dy},
                                  {h3(mx.x, mn.y, mn.z), nx, dy}, {h3(mn.x, mn.y, mn.z), dz, dy},
                                  {h3(mn.x, mx.y, mx.z), dx, nz}, {h3(mn.x, mn.y, mn.z), dx, dz}};
                for (int f = 0; f < 6; f++) {
                    H3 Q = faces[f][0], u = faces[f][1], v = faces[f][2];
                    H3 nn = hcross(u, v);
                    float ar = hlen(nn);
                    if (!(ar > 0.0f)) return bail(fail(s, RT_ERR_INVALID, "degenerate medium box " + std::to_string(i)));
                    H3 nrm = nn / ar, w = nn / hdot(nn, nn);
                    g.face[f].g[0] = make_float4(nrm.x, nrm.y, nrm.z, hdot(nrm, Q));
                    g.face[f].g[1] = make_float4(Q.x, Q.y, Q.z, u.x);
                    g.face[f].g[2] = make_float4(u.y, u.z, v.x, v.y);
                    g.face[f].g[3] = make_float4(v.z, w.x, w.y, w.z);
                }
                mb = Box{mn, mx};
            } else {
                H3 c = h3(m.center[0], m.center[1], m.center[2]), r = h3(m.radius, m.radius, m.radius);
                mb = Box{c - r, c + r};
            }
            std::vector<float4> vec(256);
            for (int k = 0; k < 256; k++) vec[k] = make_float4(m.perlin_vec[k * 3], m.perlin_vec[k * 3 + 1], m.perlin_vec[k * 3 + 2], 0.f);
            std::vector<int32_t> perm(768);
            for (int k = 0; k < 768; k++) {
                if (m.type == RT_MEDIUM_NOISE && (m.perlin_perm[k] < 0 || m.perlin_perm[k] > 255))
                    return bail(fail(s, RT_ERR_INVALID, "Perlin permutation entry out of 0..255 in medium " + std::to_string(i)));
                perm[k] = m.perlin_perm[k] & 255;
            }
            if ((rc = upload(s, vec.data(), vec.size(), &g.vec))) return bail(rc);
            if ((rc = upload(s, perm.data(), perm.size(), &g.perm))) return bail(rc);
            if (m.type == RT_MEDIUM_GRID) {
                // voxels, and per brick of RT_GRID_BRICK³ voxels the largest value its
                // trilinear lookups read: voxels 8b − 1 .. 8b + 8 on each axis
                const int R[3] = {m.grid_res[0], m.grid_res[1], m.grid_res[2]};
                size_t nv = (size_t)R[0] * R[1] * R[2];
                for (size_t v = 0; v < nv; v++)
                    if (!(m.grid[v] >= 0.0f) || !std::isfinite(m.grid[v]))
                        return bail(fail(s, RT_ERR_INVALID, "grid medium " + std::to_string(i) +
                                                                ": voxel values must be finite and ≥ 0"));
                int NB[3];
                for (int a = 0; a < 3; a++) NB[a] = (R[a] + RT_GRID_BRICK - 1) / RT_GRID_BRICK;
                std::vector<float> major((size_t)NB[0] * NB[1] * NB[2], 0.0f);
                for (int bz = 0; bz < NB[2]; bz++)
                    for (int by = 0; by < NB[1]; by++)
                        for (int bx = 0; bx < NB[0]; bx++) {
                            const int b[3] = {bx, by, bz};
                            int lo[3], hi[3];
                            for (int a = 0; a < 3; a++) {
                                lo[a] = std::max(b[a] * RT_GRID_BRICK - 1, 0);
                                hi[a] = std::min(b[a] * RT_GRID_BRICK + RT_GRID_BRICK, R[a] - 1);
                            }
                            float mx = 0.0f;
                            for (int z = lo[2]; z <= hi[2]; z++)
                                for (int y = lo[1]; y <= hi[1]; y++)
                                    for (int x = lo[0]; x <= hi[0]; x++)
                                        mx = std::fmax(mx, m.grid[((size_t)z * R[1] + y) * R[0] + x]);
                            // enlarged by 2^-20 so the interpolation's rounding stays below it
                            major[((size_t)bz * NB[1] + by) * NB[0] + bx] = mx * 1.00000095367431640625f;
                        }
                if ((rc = upload(s, m.grid, nv, &g.grid))) return bail(rc);
                if ((rc = upload(s, major.data(), major.size(), &g.major))) return bail(rc);
                H3 mn = h3(std::fmin(m.p_min[0], m.p_max[0]), std::fmin(m.p_min[1], m.p_max[1]), std::fmin(m.p_min[2], m.p_max[2]));
                H3 mx = h3(std::fmax(m.p_min[0], m.p_max[0]), std::fmax(m.p_min[1], m.p_max[1]), std::fmax(m.p_min[2], m.p_max[2]));
                H3 ext = mx - mn;
                for (int a = 0; a < 3; a++) { g.res[a] = R[a]; g.nb[a] = NB[a]; }
                g.lo = make_float3(mn.x, mn.y, mn.z);
                g.inv_vox = make_float3((float)R[0] / ext.x, (float)R[1] / ext.y, (float)R[2] / ext.z);
                g.bw = make_float3(ext.x / (float)R[0] * RT_GRID_BRICK, ext.y / (float)R[1] * RT_GRID_BRICK,
                                   ext.z / (float)R[2] * RT_GRID_BRICK);
                g.inv_bw = make_float3(1.0f / g.bw.x, 1.0f / g.bw.y, 1.0f / g.bw.z);
            }
            // media join the photon bounds (volume.rs:152-154)
            for (int a = 0; a < 3; a++) {
                bool first = s->empty && i == 0;
                s->world_lo[a] = first ? hc(mb.mn, a) : std::fmin(s->world_lo[a], hc(mb.mn, a));
                s->world_hi[a] = first ? hc(mb.mx, a) : std::fmax(s->world_hi[a], hc(mb.mx, a));
            }
        }
        if ((rc = upload(s, dm.data(), dm.size(), &s->S.media))) return bail(rc);
        s->S.n_media = d->n_media;
    }

    std::call_once(g_elut_once, build_elut);
    if ((rc = upload(s, g_elut, (size_t)64 * 64, &s->S.elut))) return bail(rc);
    std::call_once(g_nacre_once, build_nacre);
    if ((rc = upload(s, g_nacre, (size_t)256, &s->S.nacre))) return bail(rc);

    // ── textures (texture.rs, output.rs:90-96 sRGB decode table) ─────────────
    {
        float lut[256];
        for (int c = 0; c < 256; c++) {
            float v = (float)c / 255.0f;
            lut[c] = v <= 0.04045f ? v / 12.92f : std::pow((v + 0.055f) / 1.055f, 2.4f);
        }
        if ((rc = upload(s, lut, (size_t)256, &s->S.srgb_lut))) return bail(rc);
        std::vector<DevTexture> dt(std::max(d->n_textures, 1));
        for (int32_t i = 0; i < d->n_textures; i++) {
            const RtTexture& t = d->textures[i];
            DevTexture& g = dt[i];
            memset(&g, 0, sizeof(g));
            g.type = t.type; g.w = t.width; g.h = t.height; g.scale = t.scale;
            g.lo = make_float3(t.lo[0], t.lo[1], t.lo[2]);
            g.hi = make_float3(t.hi[0], t.hi[1], t.hi[2]);
            if (t.type == RT_TEX_IMAGE) {
                if ((rc = upload(s, t.rgb8, (size_t)t.width * t.height * 3, &g.px))) return bail(rc);
            } else {
                std::vector<float4> vec(256);
                for (int k = 0; k < 256; k++)
                    vec[k] = make_float4(t.perlin_vec[k * 3], t.perlin_vec[k * 3 + 1], t.perlin_vec[k * 3 + 2], 0.f);
                if ((rc = upload(s, vec.data(), vec.size(), &g.vec))) return bail(rc);
                if ((rc = upload(s, t.perlin_perm, (size_t)768, &g.perm))) return bail(rc);
            }
        }
        if ((rc = upload(s, dt.data(), dt.size(), &s->S.tex))) return bail(rc);
    }

    // ── background + env alias table (renderer.rs:32-74) ────────────────────
    const RtBackground& bg = d->bg;
    if (bg.type < RT_BG_SOLID || bg.type > RT_BG_PHYSICAL) return bail(fail(s, RT_ERR_INVALID, "unknown background type"));
    s->S.bg_type = bg.type;
    s->S.vis_type = bg.type == RT_BG_ENVMAP ? bg.visible_type : -1;
    if (bg.type == RT_BG_PHYSICAL) {
        float3 sd = make_float3(bg.sun_dir[0], bg.sun_dir[1], bg.sun_dir[2]);
        float l2 = sd.x * sd.x + sd.y * sd.y + sd.z * sd.z;
        if (!(l2 > 0.0f) || !std::isfinite(l2) || !std::isfinite(bg.turbidity))
            return bail(fail(s, RT_ERR_INVALID, "Physical sky needs a finite non-zero sun direction and turbidity"));
        float l = std::sqrt(l2);
        s->S.sun_dir = make_float3(sd.x / l, sd.y / l, sd.z / l);
        s->S.turbidity = bg.turbidity;
        s->S.has_sun = bg.sun_dir[1] > 0.0f;
    }
    for (int k = 0; k < 3; k++) {
        s->S.bg_color[k] = bg.color[k]; s->S.bg_top[k] = bg.top[k]; s->S.bg_bottom[k] = bg.bottom[k];
        s->S.vis_color[k] = bg.visible_color[k]; s->S.vis_top[k] = bg.visible_top[k]; s->S.vis_bottom[k] = bg.visible_bottom[k];
    }
    if (bg.type == RT_BG_ENVMAP) {
        int W = bg.env_w, Hh = bg.env_h;
        size_t N = (size_t)W * Hh;
        std::vector<float4> env(N);
        std::vector<double> wgt(N);
        const float PI = 3.14159265358979323846f;
        float total = 0.0f;
        for (int j = 0; j < Hh; j++) {
            float sin_j = std::sin(PI * ((float)j + 0.5f) / (float)Hh);
            float rs = 0.0f;
            for (int i = 0; i < W; i++) {
                const float* p = bg.env_rgb + ((size_t)j * W + i) * 3;
                float lum = 0.2126f * p[0] + 0.7152f * p[1] + 0.0722f * p[2];
                env[(size_t)j * W + i] = make_float4(p[0], p[1], p[2], lum);
                rs += lum * sin_j;
                wgt[(size_t)j * W + i] = (double)lum * (double)sin_j;
            }
            total += rs;
        }
        // Vose's alias method over the texel weights lum·sinθ.
        std::vector<float2> alias(N);
        double wsum = 0.0;
        for (double x : wgt) wsum += x;
        if (!(wsum > 0.0)) { for (auto& x : wgt) x = 1.0; wsum = (double)N; }
        std::vector<double> q(N);
        std::vector<uint32_t> small, large;
        small.reserve(N); large.reserve(N);
        for (size_t k = 0; k < N; k++) {
            q[k] = wgt[k] * (double)N / wsum;
            (q[k] < 1.0 ? small : large).push_back((uint32_t)k);
        }
        std::vector<uint32_t> al(N);
        for (size_t k = 0; k < N; k++) al[k] = (uint32_t)k;
        while (!small.empty() && !large.empty()) {
            uint32_t sm = small.back(); small.pop_back();
            uint32_t lg = large.back();
            al[sm] = lg;
            q[lg] = (q[lg] + q[sm]) - 1.0;
            if (q[lg] < 1.0) { large.pop_back(); small.push_back(lg); }
        }
        for (uint32_t k : large) q[k] = 1.0;
        for (uint32_t k : small) q[k] = 1.0;
        for (size_t k = 0; k < N; k++) {
            float fa;
            uint32_t a = al[k];
            memcpy(&fa, &a, 4);
            alias[k] = make_float2((float)q[k], fa);
        }
        if ((rc = upload(s, env.data(), env.size(), &s->S.env))) return bail(rc);
        if ((rc = upload(s, alias.data(), alias.size(), &s->S.env_alias))) return bail(rc);
        s->S.has_env = 1;
        s->S.env_w = W;
        s->S.env_h = Hh;
        s->S.env_inv_total = total > 0.0f ? 1.0f / total : 0.0f;
        float rot = bg.env_rot_y_deg * (PI / 180.0f);
        s->S.env_sin_r = std::sin(rot);
        s->S.env_cos_r = std::cos(rot);
    }
    if (cudaMalloc(&s->d_err, sizeof(int)) != cudaSuccess) return bail(fail(s, RT_ERR_NOMEM, "cudaMalloc"));
    cudaMemset(s->d_err, 0, sizeof(int));
    if (cudaMalloc(&s->d_R, sizeof(RenderLaunch)) != cudaSuccess || cudaMalloc(&s->d_gstat, 2 * sizeof(uint32_t)) != cudaSuccess ||
        cudaHostAlloc((void**)&s->h_tot, 4 * sizeof(uint64_t), cudaHostAllocDefault) != cudaSuccess)
        return bail(fail(s, RT_ERR_NOMEM, "cudaMalloc"));
    *out = s;
    return RT_OK;
}

int32_t rt_scene_bvh_stats(const RtScene* s, int64_t* n_nodes, int64_t* n_leaves, int32_t* max_depth, double* sah) {
    if (!s) return RT_ERR_INVALID;
    if (sah) if (int rc = ensure_ref_nodes(s)) return rc;
    if (n_nodes) *n_nodes = s->n_nodes;
    if (n_leaves) *n_leaves = s->n_leaves;
    if (max_depth) *max_depth = s->max_depth;
    if (sah) *sah = s->sah_cost;
    return RT_OK;
}

int32_t rt_scene_bvh_export(const RtScene* s, float* nodes, int64_t* n_nodes, int32_t* leaf, int64_t* n_leaves) {
    if (!s) return RT_ERR_INVALID;
    if (nodes) if (int rc = ensure_ref_nodes(s)) return rc;
    if (n_nodes) *n_nodes = s->n_nodes;
    if (n_leaves) *n_leaves = s->n_leaves;
    if (nodes) memcpy(nodes, s->ref_nodes.data(), s->ref_nodes.size() * sizeof(RefNode));
    if (leaf) memcpy(leaf, s->leaf_gids.data(), s->leaf_gids.size() * sizeof(int32_t));
    return RT_OK;
}

}  // extern "C"

// ── helpers for the API calls ───────────────────────────────────────────────
static int ensure_stage(RtScene* s, size_t bytes) {
    if (s->stage_bytes >= bytes) return RT_OK;
    free_dev(s->stage);
    s->stage_bytes = 0;
    if (cudaMalloc(&s->stage, bytes) != cudaSuccess) return fail(s, RT_ERR_NOMEM, "cudaMalloc staging");
    s->stage_bytes = bytes;
    return RT_OK;
}
static int check_err(RtScene* s) {
    int h = 0;
    CK(cudaMemcpyAsync(&h, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (h) {
        cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream);
        return fail(s, h, h == RT_ERR_CAPACITY ? "traversal stack overflow"
                          : h == RT_ERR_TIMEOUT ? "wavefront did not drain within its iteration bound"
                                                : "device error");
    }
    return RT_OK;
}

extern "C" int32_t rt_trace_closest(RtScene* s, const float* rays, int64_t n, RtHit* hits, int32_t mem) {
    if (!s || (n > 0 && (!rays || !hits))) return RT_ERR_INVALID;
    if (n <= 0) return RT_OK;
    if (n > (1ll << 31)) return fail(s, RT_ERR_CAPACITY, "more than 2^31 rays per call");
    ENTER(s);
    bool media = s->S.n_media > 0;
    if (s->empty && !media) {
        if (mem == RT_MEM_DEVICE) { CK(cudaMemsetAsync(hits, 0xFF, n * sizeof(RtHit), s->stream)); return RT_OK; }
        for (int64_t i = 0; i < n; i++) hits[i] = RtHit{-1, 0.f, 0.f, 0.f};
        return RT_OK;
    }
    const float* drays = rays;
    int4* dout = reinterpret_cast<int4*>(hits);
    size_t rb = (size_t)n * 8 * sizeof(float), hb = (size_t)n * sizeof(RtHit);
    if (mem != RT_MEM_DEVICE) {
        int rc = ensure_stage(s, rb + hb + 256);
        if (rc) return rc;
        drays = (const float*)s->stage;
        dout = (int4*)((char*)s->stage + ((rb + 255) & ~(size_t)255));
        CK(cudaMemcpyAsync((void*)drays, rays, rb, cudaMemcpyHostToDevice, s->stream));
    }
    if (!s->counters) {
        if (cudaMalloc(&s->counters, sizeof(uint32_t) * RT_CTR_WORDS) != cudaSuccess)
            return fail(s, RT_ERR_NOMEM, "cudaMalloc counters");
    }
    if (!s->empty) {
        CK(cudaMemsetAsync(s->counters, 0, sizeof(uint32_t), s->stream));
        rth::launch_trace_closest_api(s->S, drays, (uint32_t)n, dout, s->counters, s->d_err, s->sms, s->stream);
    }
    if (media)
        rth::launch_media_api(s->S, drays, (uint32_t)n, dout, (int32_t)s->n_prims, s->empty ? 1 : 0, s->sms, s->stream);
    CK(cudaGetLastError());
    if (mem != RT_MEM_DEVICE) CK(cudaMemcpyAsync(hits, dout, hb, cudaMemcpyDeviceToHost, s->stream));
    return check_err(s);
}

// any-hit flags into `dout` (device); no primitives → all clear
static int any_hit_device(RtScene* s, const float* drays, int64_t n, uint8_t* dout) {
    if (s->empty) { CK(cudaMemsetAsync(dout, 0, n, s->stream)); return RT_OK; }
    if (!s->counters) {
        if (cudaMalloc(&s->counters, sizeof(uint32_t) * RT_CTR_WORDS) != cudaSuccess)
            return fail(s, RT_ERR_NOMEM, "cudaMalloc counters");
    }
    CK(cudaMemsetAsync(s->counters, 0, sizeof(uint32_t), s->stream));
    rth::launch_trace_any_api(s->S, drays, (uint32_t)n, dout, s->counters, s->d_err, s->sms, s->stream);
    return RT_OK;
}

extern "C" int32_t rt_trace_any(RtScene* s, const float* rays, int64_t n, uint8_t* occ, int32_t mem) {
    if (!s || (n > 0 && (!rays || !occ))) return RT_ERR_INVALID;
    if (n <= 0) return RT_OK;
    if (n > (1ll << 31)) return fail(s, RT_ERR_CAPACITY, "more than 2^31 rays per call");
    ENTER(s);
    const float* drays = rays;
    uint8_t* dout = occ;
    size_t rb = (size_t)n * 8 * sizeof(float);
    if (mem != RT_MEM_DEVICE) {
        int rc = ensure_stage(s, rb + n + 256);
        if (rc) return rc;
        drays = (const float*)s->stage;
        dout = (uint8_t*)((char*)s->stage + ((rb + 255) & ~(size_t)255));
        CK(cudaMemcpyAsync((void*)drays, rays, rb, cudaMemcpyHostToDevice, s->stream));
    }
    int rc = any_hit_device(s, drays, n, dout);
    if (rc) return rc;
    CK(cudaGetLastError());
    if (mem != RT_MEM_DEVICE) CK(cudaMemcpyAsync(occ, dout, n, cudaMemcpyDeviceToHost, s->stream));
    return check_err(s);
}

extern "C" int32_t rt_trace_transmittance(RtScene* s, const float* rays, int64_t n, float* tr, int32_t mem) {
    if (!s || (n > 0 && (!rays || !tr))) return RT_ERR_INVALID;
    if (n <= 0) return RT_OK;
    if (n > (1ll << 31)) return fail(s, RT_ERR_CAPACITY, "more than 2^31 rays per call");
    ENTER(s);
    size_t rb = (size_t)n * 8 * sizeof(float), ob = (size_t)n * sizeof(float);
    size_t off_out = (rb + 255) & ~(size_t)255, off_occ = (off_out + ob + 255) & ~(size_t)255;
    int rc = ensure_stage(s, off_occ + n + 256);
    if (rc) return rc;
    const float* drays = rays;
    float* dout = tr;
    uint8_t* docc = (uint8_t*)s->stage + off_occ;
    if (mem != RT_MEM_DEVICE) {
        drays = (const float*)s->stage;
        dout = (float*)((char*)s->stage + off_out);
        CK(cudaMemcpyAsync((void*)drays, rays, rb, cudaMemcpyHostToDevice, s->stream));
    }
    if ((rc = any_hit_device(s, drays, n, docc))) return rc;
    rth::launch_transmittance_api(s->S, drays, (uint32_t)n, docc, dout, s->sms, s->stream);
    CK(cudaGetLastError());
    if (mem != RT_MEM_DEVICE) CK(cudaMemcpyAsync(tr, dout, ob, cudaMemcpyDeviceToHost, s->stream));
    return check_err(s);
}

// ── render loop ─────────────────────────────────────────────────────────────
static const uint32_t MAX_PATHS = 1u << 23;   // 8M paths in flight

// every path buffer of the scene, for allocation and release
template <class F>
static void for_path_buffers(RtScene* s, F f) {
    PathState* sets[3] = {&s->P, &s->P2, &s->Rt};
    for (PathState* P : sets) {
        float4** f4[] = {&P->ray_o, &P->ray_d, &P->thr, &P->wts, (float4**)&P->meta, &P->L, &P->pend0, &P->pend1,
                         &P->pendC};
        for (int i = 0; i < 9; i++)
            if (P != &s->Rt || i >= 4) f((void**)f4[i], sizeof(float4));
        f((void**)&P->rec, sizeof(uint32_t));
    }
    f((void**)&s->P.hit, sizeof(float4));
    f((void**)&s->P.gq, 2 * sizeof(float4));
    f((void**)&s->queue[0], sizeof(uint32_t));
    f((void**)&s->queue[1], sizeof(uint32_t));
    f((void**)&s->sq, 2 * 2 * sizeof(float4));
    for (int c = 0; c < CLS_N; c++) f((void**)&s->cq.q[c], sizeof(uint32_t));
}

static void free_paths(RtScene* s) {
    s->P2.hit = s->P2.gq = nullptr;
    for_path_buffers(s, [](void** p, size_t) { if (*p) cudaFree(*p); *p = nullptr; });
    s->cap = 0;
}

static int ensure_paths(RtScene* s, uint32_t cap) {
    if (s->cap >= cap) return RT_OK;
    free_paths(s);
    bool ok = true;
    for_path_buffers(s, [&](void** p, size_t per) {
        if (ok && cudaMalloc(p, (size_t)cap * per) != cudaSuccess) ok = false;
    });
    if (!ok) { free_paths(s); return fail(s, RT_ERR_NOMEM, "cudaMalloc path state"); }
    s->P2.hit = s->P.hit;
    s->P2.gq = s->P.gq;
    if (!s->counters && cudaMalloc(&s->counters, sizeof(uint32_t) * RT_CTR_WORDS) != cudaSuccess)
        return fail(s, RT_ERR_NOMEM, "cudaMalloc counters");
    if (!s->d_bins && cudaMalloc(&s->d_bins, sizeof(uint32_t) * 2 * RT_NBINS) != cudaSuccess)
        return fail(s, RT_ERR_NOMEM, "cudaMalloc ray bins");
    s->cap = cap;
    return RT_OK;
}

// Device buffers of one wavefront run: the scene's own (grown on demand) or
// the fixed array of rt_render_pass_noalloc.
struct WaveBufs {
    PathState set[2]{};
    PathState Rt{};
    ClassQueues cq{};
    float4* sq = nullptr;
    uint32_t* counters = nullptr;
    int* derr = nullptr;
    uint32_t cap = 0;
    bool guide = false;               // the scene's guide may run (not the no-alloc array)
    bool graphable = false;           // the scene's own buffers: the call may run as the captured graph
    uint32_t* binq = nullptr;         // extend order after ray binning (RT_RAY_BINS), or null
    uint32_t* bins = nullptr;         // its histogram and cursors
};

static WaveBufs scene_bufs(const RtScene* s) {
    WaveBufs W;
    W.guide = true;
    W.graphable = true;
    W.set[0] = s->P; W.set[1] = s->P2; W.Rt = s->Rt;
    W.cq = s->cq; W.sq = s->sq; W.counters = s->counters; W.derr = s->d_err;
    W.cap = std::min(s->cap, s->max_paths);
    // the photon tracer's queue is free while a render runs
    W.binq = s->queue[0];
    W.bins = s->d_bins;
    return W;
}

// Samples sample_idx .. sample_idx+nsamp−1 of the `nactive` active pixels
// (`active` = null: all pixels) into dscratch (nsamp × npix × 3).
//
// The path pool (min(samples, W.cap) slots) is filled once; then each
// iteration runs extend → classify/shade → photon gather → shadow → retire,
// and the retire kernel hands every slot whose path ended to the next
// ungenerated sample.  While samples remain, the pool stays full, so every
// launch but those of the final drain works on a full wavefront.  The host
// does not wait per iteration: it reads the next-iteration ray count of the
// iteration launched STATUS_LAG iterations earlier (copied to pinned memory)
// and stops at the first zero; the at most STATUS_LAG iterations launched
// after it find empty queues.
static const uint32_t STATUS_RING = 8, STATUS_LAG = 2;

// End of iteration k in a graph: records the next iteration's ray count and
// the iterations run, arms the next iteration's conditional node while rays
// remain and the bound allows, and reports a bound reached with rays left.
__global__ void k_wave_next(const uint32_t* __restrict__ cnt_next, const RenderLaunch* __restrict__ R, uint64_t k,
                            cudaGraphConditionalHandle next, int has_next, uint32_t* gstat, int* derr) {
    uint32_t c = *cnt_next;
    gstat[0] = c;
    gstat[1] = (uint32_t)(k + 1);
    bool more = c > 0 && k + 1 < R->max_it;
    if (has_next) cudaGraphSetConditional(next, more ? 1u : 0u);
    if (c > 0 && !more) atomicCAS(derr, 0, RT_ERR_TIMEOUT);
}

static void wave_graph_free(RtScene* s) {
    if (s->wg.exec) cudaGraphExecDestroy(s->wg.exec);
    if (s->wg.graph) cudaGraphDestroy(s->wg.graph);
    s->wg = RtScene::WaveGraph{};
}

// What a captured wavefront graph depends on besides the device RenderLaunch
// (which carries the pool size, the bound and the batch table): the scene
// state and buffers its launches were given, the pool's capacity and the
// flags that choose its kernels.
static std::vector<uint8_t> wave_key(const RtScene* s, const WaveBufs& W, const RenderLaunch& R) {
    std::vector<uint8_t> k;
    auto put = [&](const void* p, size_t n) { const uint8_t* b = (const uint8_t*)p; k.insert(k.end(), b, b + n); };
    put(&s->S, sizeof(s->S));
    put(&W.set[0], sizeof(PathState));
    put(&W.set[1], sizeof(PathState));
    put(&W.Rt, sizeof(PathState));
    put(&W.cq, sizeof(W.cq));
    const void* ptrs[3] = {W.sq, W.counters, W.derr};
    put(ptrs, sizeof(ptrs));
    int64_t v[5] = {W.cap, R.photons, R.guide.mode, s->sms, R.photons ? (int64_t)s->photons.generation : -1};
    put(v, sizeof(v));
    return k;
}

// Capture (or keep) the graph of a wavefront call: the prologue as a child
// graph, then K ≥ max_it conditional IF nodes in a chain, node k holding
// iteration k's launches and k_wave_next.  Node 0 always runs; node k + 1
// runs when iteration k left rays and the call's bound allows — a chain of
// IF nodes cannot run past K, whatever the device state.
template <class Pro, class It>
static int wave_graph_ensure(RtScene* s, const WaveBufs& W, const RenderLaunch& R, uint64_t max_it, uint64_t kmin,
                             Pro&& prologue, It&& iteration) {
    std::vector<uint8_t> key = wave_key(s, W, R);
    if (s->wg.exec && s->wg.K >= max_it && key == s->wg.key) return RT_OK;
    wave_graph_free(s);
    const uint64_t K = (std::max(max_it, kmin) + 31) / 32 * 32;
    cudaGraph_t G = nullptr;
    cudaError_t e = cudaGraphCreate(&G, 0);
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess && r != cudaSuccess) e = r; return e == cudaSuccess; };
    cudaGraphNode_t prev = nullptr;
    if (ok(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal))) {
        int rc = prologue();
        cudaGraph_t gp = nullptr;
        ok(cudaStreamEndCapture(s->stream, &gp));
        if (rc && e == cudaSuccess) e = cudaErrorUnknown;
        if (gp) {
            ok(cudaGraphAddChildGraphNode(&prev, G, nullptr, 0, gp));
            cudaGraphDestroy(gp);
        }
    }
    std::vector<cudaGraphConditionalHandle> h(K);
    for (uint64_t k = 0; k < K && e == cudaSuccess; k++)
        ok(cudaGraphConditionalHandleCreate(&h[k], G, k == 0 ? 1u : 0u, cudaGraphCondAssignDefault));
    for (uint64_t k = 0; k < K && e == cudaSuccess; k++) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h[k];
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        if (!ok(cudaGraphAddNode(&node, G, &prev, 1, &cp))) break;
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        if (!ok(cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)))
            break;
        int rc = iteration(k);
        const uint32_t* cnt_next = W.counters + CTR_HDR_WORDS + ((k + 1) % RT_CTR_RING) * RT_CTR_STRIDE + CTR_COUNT;
        k_wave_next<<<1, 1, 0, s->stream>>>(cnt_next, s->d_R, k, k + 1 < K ? h[k + 1] : 0, k + 1 < K ? 1 : 0,
                                            s->d_gstat, W.derr);
        ok(cudaGetLastError());
        ok(cudaStreamEndCapture(s->stream, &body));
        if (rc && e == cudaSuccess) e = cudaErrorUnknown;
        prev = node;
    }
    if (e == cudaSuccess) ok(cudaGraphInstantiate(&s->wg.exec, G, 0));
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (s->wg.exec) cudaGraphExecDestroy(s->wg.exec);
        s->wg.exec = nullptr;
        if (G) cudaGraphDestroy(G);
        return fail(s, RT_ERR_CUDA, std::string("wavefront graph: ") + cudaGetErrorString(e));
    }
    s->wg.graph = G;
    s->wg.key = std::move(key);
    s->wg.K = K;
    return RT_OK;
}

static int run_wavefront(RtScene* s, const WaveBufs& W, const RtCamera* cam, const RtPassParams* p, uint32_t sample_idx,
                         uint32_t nsamp, float* dscratch, const uint32_t* active, uint32_t nactive, int64_t* ext_rays,
                         int64_t* sh_rays, int64_t* launches, const JobDev* jobs = nullptr, uint32_t n_jobs = 0,
                         uint64_t jobs_total = 0, bool async = false, uint64_t graph_kmin = 0) {
    uint64_t total = n_jobs ? jobs_total : (uint64_t)nsamp * nactive;
    if (total == 0) return RT_OK;
    uint32_t pool = (uint32_t)std::min<uint64_t>(total, W.cap);
    uint32_t maxd = std::min<uint32_t>(p->max_depth, RT_MAX_DEPTH);
    RenderLaunch R{};
    R.width = p->width; R.height = p->height; R.npix = p->width * p->height;
    R.nsamp = nsamp;
    R.sample_idx = sample_idx;
    R.strata = p->strata;
    R.max_depth = maxd;
    R.hero = std::max<uint32_t>(1, std::min<uint32_t>(p->hero_count, 4));
    R.bg_scale = p->bg_scale;
    R.seed = p->seed;
    R.cam = *cam;
    R.active = active;
    R.nactive = nactive;
    R.total = total;
    R.gen_next = (unsigned long long*)(W.counters + HDR_GEN);
    R.scratch = dscratch;
    R.photons = s->photons.present && s->photons.n > 0;
    if (W.guide && s->guide && rtgh::mode(s->guide) != RT_GUIDE_OFF) R.guide = rtgh::view(s->guide);
    R.jobs = jobs;
    R.n_jobs = n_jobs;
    R.dev = s->d_R;
    // every iteration with samples left advances `pool` path segments, and a
    // sample has at most maxd segments; the drain takes at most maxd more.  A
    // call whose samples all fit in the pool is never refilled: its paths all
    // start at depth 0 and none goes on past depth maxd − 1, so maxd
    // iterations (at least one) drain it, and the host queues no empty ones
    uint64_t max_it = total <= pool ? std::max<uint64_t>(maxd, 1) : total * maxd / pool + maxd + 2;
    if (s->max_iterations) max_it = std::min<uint64_t>(max_it, s->max_iterations);
    R.max_it = max_it;
    R.pool = pool;
    // stream-ordered: the previous call's kernels have read the old copy
    CK(cudaMemcpyAsync(s->d_R, &R, sizeof(R), cudaMemcpyHostToDevice, s->stream));
    uint32_t* hdr = W.counters;
    auto blk = [&](uint64_t it) { return W.counters + CTR_HDR_WORDS + (it % RT_CTR_RING) * RT_CTR_STRIDE; };
    size_t ev_used = 0;
    const bool graph = (s->graph_mode || async) && !s->profiling && !(s->cap_out && s->cap_depth >= 0) && W.graphable;
    auto mark = [&](int kind) {
        if (!s->profiling || graph) return;
        if (ev_used >= s->pev.size()) { cudaEvent_t e; cudaEventCreate(&e); s->pev.push_back(e); s->pkind.push_back(0); }
        s->pkind[ev_used] = kind;
        cudaEventRecord(s->pev[ev_used++], s->stream);
    };
    // launches per iteration: extend, classify, shadow, retire, one shading
    // kernel per class the scene's materials produce (the medium class counted
    // with the media pair), the guide pair and the photon gather
    const int64_t per_it = 4 + __builtin_popcount(s->S.class_mask & ~(1u << CLS_MEDIUM)) +
                           (R.guide.mode != 0 ? 2 : 0) + (s->S.n_media > 0 ? 2 : 0) + (R.photons ? 1 : 0);
    auto prologue = [&]() {
        CK(cudaMemsetAsync(W.counters, 0, sizeof(uint32_t) * RT_CTR_WORDS, s->stream));
        mark(0);
        // a captured first fill serves every pool size up to the capacity
        rth::launch_generate(s->S, W.set[0], R, graph ? W.cap : pool, blk(0) + CTR_COUNT, s->stream);
        return RT_OK;
    };
    // the launches of iteration `it`
    auto iteration = [&](uint64_t it) {
        uint32_t* c = blk(it);
        uint32_t* cn = blk(it + 1);
        const PathState& A = W.set[it & 1];
        const PathState& B = W.set[(it + 1) & 1];
        PendTargets T{{B.pend0, B.pend1, W.Rt.pend0, W.Rt.pend1}, {B.pendC, W.Rt.pendC}};
        mark(1);
        const uint32_t* xq = nullptr;
#if RT_RAY_BINS
        if (W.binq && W.bins) {
            float3 lo = make_float3(s->world_lo[0], s->world_lo[1], s->world_lo[2]);
            auto sc = [&](int a) { return (float)RT_BIN_CELLS / std::max(s->world_hi[a] - s->world_lo[a], 1e-6f); };
            rth::launch_bin_rays(A, c + CTR_COUNT, W.cap, lo, make_float3(sc(0), sc(1), sc(2)), W.bins, W.binq,
                                 s->stream);
            xq = W.binq;
        }
#endif
        rth::launch_extend(s->S, A, xq, c + CTR_COUNT, c + CTR_EXTEND_NEXT, W.derr, s->sms, s->stream);
        if (s->S.n_media > 0) rth::launch_media(s->S, A, nullptr, c + CTR_COUNT, s->sms, s->stream);
        if (!graph && (int64_t)it == s->cap_depth && s->cap_out) {
            // diagnostics: copy this iteration's rays out (origin, direction)
            CK(cudaStreamSynchronize(s->stream));
            uint32_t cnt = 0;
            CK(cudaMemcpy(&cnt, c + CTR_COUNT, 4, cudaMemcpyDeviceToHost));
            int64_t m = std::min<int64_t>(cnt, s->cap_max);
            std::vector<float4> ro(m), rd(m);
            CK(cudaMemcpy(ro.data(), A.ray_o, (size_t)m * 16, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(rd.data(), A.ray_d, (size_t)m * 16, cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < m; i++) {
                float* r = s->cap_out + i * 8;
                float4 a = ro[i], b = rd[i];
                r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = b.x; r[4] = b.y; r[5] = b.z; r[6] = 0.001f; r[7] = INFINITY;
            }
            s->cap_n = m;
        }
        mark(2);
        rth::launch_shade(s->S, A, B, W.Rt, R, c, W.cq, cn + CTR_COUNT, W.sq, s->sms, s->stream, &s->fk);
        if (R.photons) {
            // the caustic lookup scales the parked pendC terms and the shadow
            // rays cancel pend0 / pend1: disjoint writes, so the lookup runs
            // on a side stream beside the shadow rays (joined before retire)
            CK(cudaEventRecord(s->fk.fork, s->stream));
            CK(cudaStreamWaitEvent(s->fk.side[0], s->fk.fork, 0));
            rth::launch_photon_gather_paths(s->photons, T, A.gq, c + CTR_GATHER_COUNT, s->sms, s->fk.side[0]);
            CK(cudaEventRecord(s->fk.join[0], s->fk.side[0]));
        }
        mark(3);
        rth::launch_shadow(s->S, T, W.sq, c + CTR_SHADOW_COUNT, c + CTR_SHADOW_NEXT, W.derr, s->sms, s->stream);
        if (R.photons) CK(cudaStreamWaitEvent(s->stream, s->fk.join[0], 0));
        mark(0);
        rth::launch_retire(s->S, B, W.Rt, R, c, hdr, blk(it + 2), cn + CTR_COUNT, s->sms, s->stream);
        return RT_OK;
    };
    int64_t nl = 0;
    uint64_t tot[3] = {0, 0, 0};
    if (graph) {
        // the call as one graph launch: the prologue, then one conditional node
        // per iteration up to the bound, each run only while rays remain (the
        // graph is captured once and kept while the buffers, scene state and
        // bound it was made for stay the same)
        if (int rc = wave_graph_ensure(s, W, R, max_it, graph_kmin, prologue, iteration)) return rc;
        CK(cudaGraphLaunch(s->wg.exec, s->stream));
        CK(cudaMemcpyAsync(s->h_status, s->d_gstat, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
        if (async) {
            CK(cudaMemcpyAsync(s->h_tot, W.counters, sizeof(tot), cudaMemcpyDeviceToHost, s->stream));
            s->async_pending = true;
            s->async_per_it = per_it;
            return RT_OK;
        }
        CK(cudaMemcpyAsync(tot, W.counters, sizeof(tot), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        nl = 1 + (int64_t)s->h_status[1] * (per_it + 1);
        // a bound reached with rays left sets RT_ERR_TIMEOUT in the error word
    } else {
        prologue();
        nl++;
        bool done = false;
        uint64_t it = 0;
        for (; it < max_it && !done; it++) {
            iteration(it);
            nl += per_it;
            uint32_t slot = (uint32_t)(it % STATUS_RING);
            CK(cudaMemcpyAsync(s->h_status + slot, blk(it + 1) + CTR_COUNT, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               s->stream));
            CK(cudaEventRecord(s->st_ev[slot], s->stream));
            if (it >= STATUS_LAG) {
                uint32_t js = (uint32_t)((it - STATUS_LAG) % STATUS_RING);
                CK(cudaEventSynchronize(s->st_ev[js]));
                if (((volatile uint32_t*)s->h_status)[js] == 0) done = true;
            }
        }
        mark(0);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(tot, W.counters, sizeof(tot), cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        if (!done) {
            // the bound was reached: the last iteration must have left no rays
            // (a count that reaches zero stays zero: no path is left to retire
            // and hand its slot a new sample)
            if (it > 0 && s->h_status[(uint32_t)((it - 1) % STATUS_RING)] != 0)
                return fail(s, RT_ERR_TIMEOUT, "wavefront did not drain within its iteration bound (" +
                                                   std::to_string(max_it) + " iterations)");
        }
    }
    if (ext_rays) *ext_rays += (int64_t)tot[HDR_EXT / 2];
    if (sh_rays) *sh_rays += (int64_t)tot[HDR_SHADOW / 2];
    if (launches) *launches += nl;
    if (s->profiling) {
        for (size_t e = 0; e + 1 < ev_used; e++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, s->pev[e], s->pev[e + 1]);
            int kind = s->pkind[e];
            s->kms[kind] += ms;
            if (!(kind == 0 && e > 0 && s->pkind[e - 1] == 0)) s->kcount[kind]++;
        }
    }
    return RT_OK;
}

// Renders params->n_samples samples of every pixel into the device buffer
// `dscratch` (n_samples × npix × 3).  Pixels set in the converged mask are
// not traced and get zero.
static int render_device(RtScene* s, const RtCamera* cam, const RtPassParams* p, float* dscratch, const uint8_t* dconv,
                         int64_t* ext_rays, int64_t* sh_rays, int64_t* launches, bool async = false) {
    uint32_t npix = p->width * p->height;
    uint32_t nsamp = std::max<uint32_t>(p->n_samples, 1);
    uint64_t total = (uint64_t)nsamp * npix;
    int rc = ensure_paths(s, (uint32_t)std::min<uint64_t>(total, s->max_paths));
    if (rc) return rc;
    if (ext_rays) *ext_rays = 0;
    if (sh_rays) *sh_rays = 0;
    if (launches) *launches = 0;
    const uint32_t* active = nullptr;
    uint32_t nactive = npix;
    if (dconv) {
        if (s->active_cap < npix + 1) {
            free_dev((void*&)s->d_active);
            s->active_cap = 0;
            if (cudaMalloc(&s->d_active, ((size_t)npix + 1) * 4) != cudaSuccess)
                return fail(s, RT_ERR_NOMEM, "cudaMalloc active pixel list");
            s->active_cap = npix + 1;
        }
        uint32_t* dcount = s->d_active + npix;
        CK(cudaMemsetAsync(dcount, 0, 4, s->stream));
        rth::launch_active_list(dconv, p->width, p->height, s->d_active, dcount, s->stream);
        rth::launch_zero_converged(dconv, npix, nsamp, dscratch, s->stream);
        CK(cudaMemcpyAsync(&nactive, dcount, 4, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
        active = s->d_active;
        if (launches) *launches += 2;
    }
    bool guided = s->guide && rtgh::mode(s->guide) != RT_GUIDE_OFF;
    if (guided) {
        if (rtgh::ensure_paths(s->guide, s->cap)) return fail(s, RT_ERR_NOMEM, "cudaMalloc guide mixtures");
        CK(rtgh::begin_pass(s->guide, s->stream));
    }
    rc = run_wavefront(s, scene_bufs(s), cam, p, p->sample_idx, nsamp, dscratch, active, nactive, ext_rays, sh_rays,
                       launches, nullptr, 0, 0, async);
    if (rc || !guided) return rc;
    int64_t tl = 0;
    CK(rtgh::train_pass(s->guide, s->sms, s->stream, &tl));
    if (launches) *launches += tl;
    return RT_OK;
}

static int validate_pass(RtScene* s, const RtCamera* cam, const RtPassParams* p) {
    if (!s || !cam || !p) return RT_ERR_INVALID;
    if (p->width == 0 || p->height == 0) return fail(s, RT_ERR_INVALID, "zero image size");
    if ((uint64_t)p->width * p->height > (1ull << 26)) return fail(s, RT_ERR_CAPACITY, "image larger than 2^26 pixels");
    if (p->max_depth == 0 || p->max_depth > RT_MAX_DEPTH) return fail(s, RT_ERR_INVALID, "max_depth must be in 1..256");
    if (s->empty) return fail(s, RT_ERR_INVALID, "scene has no primitives");
    return RT_OK;
}

static int stage_conv(RtScene* s, const uint8_t* conv, size_t npix, int32_t mem, const uint8_t** dconv) {
    *dconv = nullptr;
    if (!conv) return RT_OK;
    if (mem == RT_MEM_DEVICE) { *dconv = conv; return RT_OK; }
    if (s->conv_bytes < npix) {
        free_dev((void*&)s->d_conv);
        if (cudaMalloc(&s->d_conv, npix) != cudaSuccess) return fail(s, RT_ERR_NOMEM, "cudaMalloc converged mask");
        s->conv_bytes = npix;
    }
    CK(cudaMemcpyAsync(s->d_conv, conv, npix, cudaMemcpyHostToDevice, s->stream));
    *dconv = s->d_conv;
    return RT_OK;
}

extern "C" int32_t rt_render_pass(RtScene* s, const RtCamera* cam, const RtPassParams* p, float* scratch,
                                  const uint8_t* converged, int32_t mem) {
    int rc = validate_pass(s, cam, p);
    if (rc) return rc;
    if (!scratch) return fail(s, RT_ERR_INVALID, "null scratch");
    ENTER(s);
    size_t npix = (size_t)p->width * p->height;
    uint32_t nsamp = std::max<uint32_t>(p->n_samples, 1);
    size_t bytes = (size_t)nsamp * npix * 3 * sizeof(float);
    float* dst = scratch;
    if (mem != RT_MEM_DEVICE) {
        if (s->scratch_bytes < bytes) {
            free_dev((void*&)s->scratch);
            s->scratch_bytes = 0;
            if (cudaMalloc(&s->scratch, bytes) != cudaSuccess) return fail(s, RT_ERR_NOMEM, "cudaMalloc scratch");
            s->scratch_bytes = bytes;
        }
        dst = s->scratch;
    }
    const uint8_t* dconv;
    if ((rc = stage_conv(s, converged, npix, mem, &dconv))) return rc;
    for (int k = 0; k < 4; k++) { s->kms[k] = 0.0; s->kcount[k] = 0; }
    CK(cudaEventRecord(s->ev0, s->stream));
    rc = render_device(s, cam, p, dst, dconv, &s->last_ext, &s->last_shadow, &s->last_launches);
    if (rc) return rc;
    CK(cudaEventRecord(s->ev1, s->stream));
    if (mem != RT_MEM_DEVICE) CK(cudaMemcpyAsync(scratch, dst, bytes, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaEventSynchronize(s->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    s->last_ms = ms;
    return check_err(s);
}

// rt_render_accumulate and its asynchronous form: `async` queues the work
// after `caller` (device outputs only), signals `caller` when it is done and
// leaves the error word, the statistics and the timing to rt_sync.
static int accumulate_impl(RtScene* s, const RtCamera* cam, const RtPassParams* p, float clamp, uint32_t min_samples,
                           float floor_, int32_t reset, float* out_sum, float* out_m2, uint32_t* out_count, int32_t mem,
                           bool async, cudaStream_t caller) {
    int rc = validate_pass(s, cam, p);
    if (rc) return rc;
    uint32_t npix = p->width * p->height;
    uint32_t nsamp = std::max<uint32_t>(p->n_samples, 1);
    // samples per wavefront run: as many as fit a 2 GiB sample buffer
    uint32_t per = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(nsamp, (2ull << 30) / ((uint64_t)npix * 12)));
    if (async) {
        if (mem != RT_MEM_DEVICE) return fail(s, RT_ERR_INVALID, "asynchronous calls take device buffers only");
        if (per < nsamp)
            return fail(s, RT_ERR_INVALID, "asynchronous calls take at most " + std::to_string(per) +
                                               " samples per pixel at this size (one 2 GiB sample buffer)");
        if (s->guide && rtgh::mode(s->guide) == RT_GUIDE_TRAIN)
            return fail(s, RT_ERR_INVALID, "asynchronous calls do not train the guide");
        CK(cudaSetDevice(s->device));
        if (s->async_pending) {
            // the previous asynchronous call's statistics are folded first
            if (int r2 = fold_async(s)) return r2;
        }
        CK(cudaEventRecord(s->caller_ev, caller));
        CK(cudaStreamWaitEvent(s->stream, s->caller_ev, 0));
    } else {
        ENTER(s);
    }
    if (s->acc_npix != npix) {
        if (async) CK(cudaStreamSynchronize(s->stream));
        free_dev((void*&)s->acc); free_dev((void*&)s->m2); free_dev((void*&)s->cnt);
        if (cudaMalloc(&s->acc, (size_t)npix * 12) != cudaSuccess || cudaMalloc(&s->m2, (size_t)npix * 12) != cudaSuccess ||
            cudaMalloc(&s->cnt, (size_t)npix * 4) != cudaSuccess)
            return fail(s, RT_ERR_NOMEM, "cudaMalloc accumulators");
        s->acc_npix = npix;
        reset = 1;
    }
    if (reset) {
        CK(cudaMemsetAsync(s->acc, 0, (size_t)npix * 12, s->stream));
        CK(cudaMemsetAsync(s->m2, 0, (size_t)npix * 12, s->stream));
        CK(cudaMemsetAsync(s->cnt, 0, (size_t)npix * 4, s->stream));
    }
    size_t bytes = (size_t)per * npix * 3 * sizeof(float);
    if (s->scratch_bytes < bytes) {
        CK(cudaStreamSynchronize(s->stream));
        free_dev((void*&)s->scratch);
        s->scratch_bytes = 0;
        if (cudaMalloc(&s->scratch, bytes) != cudaSuccess) return fail(s, RT_ERR_NOMEM, "cudaMalloc scratch");
        s->scratch_bytes = bytes;
    }
    for (int k = 0; k < 4; k++) { s->kms[k] = 0.0; s->kcount[k] = 0; }
    CK(cudaEventRecord(s->ev0, s->stream));
    int64_t ext = 0, sh = 0, nl = 0;
    for (uint32_t k0 = 0; k0 < nsamp; k0 += per) {
        RtPassParams q = *p;
        q.sample_idx = p->sample_idx + k0;
        q.n_samples = std::min(per, nsamp - k0);
        int64_t e1, s1, l1;
        rc = render_device(s, cam, &q, s->scratch, nullptr, &e1, &s1, &l1, async);
        if (rc) return rc;
        rth::launch_accumulate(s->scratch, q.n_samples, npix, s->acc, s->m2, s->cnt, nullptr, clamp, min_samples, floor_,
                               s->stream);
        ext += e1; sh += s1; nl += l1 + 1;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(s->ev1, s->stream));
    auto kind = mem == RT_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (out_sum) CK(cudaMemcpyAsync(out_sum, s->acc, (size_t)npix * 12, kind, s->stream));
    if (out_m2) CK(cudaMemcpyAsync(out_m2, s->m2, (size_t)npix * 12, kind, s->stream));
    if (out_count) CK(cudaMemcpyAsync(out_count, s->cnt, (size_t)npix * 4, kind, s->stream));
    if (async) {
        // the caller's stream waits for the outputs; statistics at rt_sync
        CK(cudaEventRecord(s->caller_ev, s->stream));
        CK(cudaStreamWaitEvent(caller, s->caller_ev, 0));
        s->last_launches = nl;                        // without the iterations, known at rt_sync
        return RT_OK;
    }
    CK(cudaStreamSynchronize(s->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    s->last_ms = ms;
    s->last_ext = ext;
    s->last_shadow = sh;
    s->last_launches = nl;
    return check_err(s);
}

extern "C" int32_t rt_render_accumulate(RtScene* s, const RtCamera* cam, const RtPassParams* p, float clamp,
                                        uint32_t min_samples, float floor_, int32_t reset, float* out_sum,
                                        float* out_m2, uint32_t* out_count, int32_t mem) {
    return accumulate_impl(s, cam, p, clamp, min_samples, floor_, reset, out_sum, out_m2, out_count, mem, false, 0);
}

extern "C" int32_t rt_render_accumulate_async(RtScene* s, const RtCamera* cam, const RtPassParams* p, float clamp,
                                              uint32_t min_samples, float floor_, int32_t reset, float* out_sum,
                                              float* out_m2, uint32_t* out_count, void* cuda_stream) {
    if (!s) return RT_ERR_INVALID;
    return accumulate_impl(s, cam, p, clamp, min_samples, floor_, reset, out_sum, out_m2, out_count, RT_MEM_DEVICE,
                           true, (cudaStream_t)cuda_stream);
}

static int fold_async(RtScene* s) {
    CK(cudaStreamSynchronize(s->stream));
    if (s->async_pending) {
        s->async_pending = false;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        s->last_ms = ms;
        s->last_ext = (int64_t)s->h_tot[HDR_EXT / 2];
        s->last_shadow = (int64_t)s->h_tot[HDR_SHADOW / 2];
        s->last_launches += (int64_t)s->h_status[1] * (s->async_per_it + 1);
    }
    return RT_OK;
}

extern "C" int32_t rt_sync(RtScene* s) {
    if (!s) return RT_ERR_INVALID;
    CK(cudaSetDevice(s->device));
    if (int rc = fold_async(s)) return rc;
    return check_err(s);
}

// ── packed batches ──────────────────────────────────────────────────────────
extern "C" int32_t rt_render_batch(RtScene* s, const RtBatchJob* jobs, int32_t n_jobs, const RtPassParams* shared,
                                   uint32_t window, float* out_sum, float* out_m2, uint32_t* out_count, float* done_ms,
                                   int32_t mem) {
    if (!s || !jobs || !shared || n_jobs < 1) return RT_ERR_INVALID;
    if (n_jobs > 65535) return fail(s, RT_ERR_CAPACITY, "more than 65535 requests in one batch");
    if (shared->max_depth == 0 || shared->max_depth > RT_MAX_DEPTH) return fail(s, RT_ERR_INVALID, "max_depth must be in 1..256");
    if (s->empty) return fail(s, RT_ERR_INVALID, "scene has no primitives");
    std::vector<uint64_t> pix_off((size_t)n_jobs + 1, 0);
    for (int32_t j = 0; j < n_jobs; j++) {
        const RtBatchJob& b = jobs[j];
        if (b.width == 0 || b.height == 0 || b.spp == 0) return fail(s, RT_ERR_INVALID, "batch request with no pixels or samples");
        if ((uint64_t)b.width * b.height > (1ull << 26)) return fail(s, RT_ERR_CAPACITY, "batch request larger than 2^26 pixels");
        pix_off[j + 1] = pix_off[j] + (uint64_t)b.width * b.height;
    }
    const uint64_t tot_pix = pix_off[n_jobs];
    ENTER(s);
    // packed accumulators (sum, M2, count) of every request
    if (s->batch_pix < tot_pix) {
        free_dev((void*&)s->b_acc); free_dev((void*&)s->b_m2); free_dev((void*&)s->b_cnt); free_dev((void*&)s->d_jobs);
        s->batch_pix = 0;
        if (cudaMalloc(&s->b_acc, tot_pix * 12) != cudaSuccess || cudaMalloc(&s->b_m2, tot_pix * 12) != cudaSuccess ||
            cudaMalloc(&s->b_cnt, tot_pix * 4) != cudaSuccess)
            return fail(s, RT_ERR_NOMEM, "cudaMalloc batch accumulators");
        s->batch_pix = tot_pix;
    }
    if (s->jobs_cap < (uint32_t)n_jobs) {
        free_dev((void*&)s->d_jobs);
        s->jobs_cap = 0;
        if (cudaMalloc(&s->d_jobs, (size_t)n_jobs * sizeof(JobDev)) != cudaSuccess)
            return fail(s, RT_ERR_NOMEM, "cudaMalloc batch table");
        s->jobs_cap = (uint32_t)n_jobs;
    }
    CK(cudaMemsetAsync(s->b_acc, 0, tot_pix * 12, s->stream));
    CK(cudaMemsetAsync(s->b_m2, 0, tot_pix * 12, s->stream));
    CK(cudaMemsetAsync(s->b_cnt, 0, tot_pix * 4, s->stream));
    // samples per pixel per pass: as many as keep the pass's samples within 2 GiB
    // and, when the passes replay the captured wavefront graph, within
    // RT_GRAPH_PASS_POOLS pools, so that one chain of (RT_GRAPH_PASS_POOLS + 1)
    // × depth + 2 iterations bounds every pass and the graph captured for the
    // first pass serves the others
    const uint32_t maxd_b = std::min<uint32_t>(shared->max_depth, RT_MAX_DEPTH);
    const uint64_t budget = s->graph_mode ? std::min<uint64_t>((2ull << 30) / 12,
                                                               (uint64_t)RT_GRAPH_PASS_POOLS * s->max_paths)
                                          : (2ull << 30) / 12;
    uint32_t W = window;
    if (W == 0) {
        uint32_t mx = 0;
        for (int32_t j = 0; j < n_jobs; j++) mx = std::max(mx, jobs[j].spp);
        W = 1;
        for (uint32_t c = 2; c <= mx; c++) {
            uint64_t need = 0;
            for (int32_t j = 0; j < n_jobs; j++) need += (uint64_t)std::min(jobs[j].spp, c) * (pix_off[j + 1] - pix_off[j]);
            if (need > budget) break;
            W = c;
        }
    }
    std::vector<uint32_t> left((size_t)n_jobs);
    for (int32_t j = 0; j < n_jobs; j++) left[j] = jobs[j].spp;
    std::vector<int> pass_of((size_t)n_jobs, -1);
    std::vector<cudaEvent_t> evs;
    cudaEvent_t e0;
    CK(cudaEventCreate(&e0));
    evs.push_back(e0);
    CK(cudaEventRecord(e0, s->stream));
    for (int k = 0; k < 4; k++) { s->kms[k] = 0.0; s->kcount[k] = 0; }
    int64_t ext = 0, sh = 0, nl = 0;
    RtPassParams q = *shared;
    int rc = RT_OK;
    for (int pass = 0; rc == RT_OK; pass++) {
        std::vector<JobDev> tab;
        std::vector<int32_t> ids;
        uint64_t cursor = 0, floats = 0;
        for (int32_t j = 0; j < n_jobs; j++) {
            if (!left[j]) continue;
            const RtBatchJob& b = jobs[j];
            JobDev J{};
            J.cam = b.cam;
            J.width = b.width; J.height = b.height; J.npix = b.width * b.height; J.strata = b.strata;
            J.nsamp = std::min(left[j], W);
            J.sample_idx = b.sample_idx + (b.spp - left[j]);
            J.first = cursor;
            J.seed = b.seed;
            J.scratch = reinterpret_cast<float*>(floats);        // offset now, pointer below
            cursor += (uint64_t)J.nsamp * J.npix;
            floats += (uint64_t)J.nsamp * J.npix * 3;
            tab.push_back(J);
            ids.push_back(j);
        }
        if (tab.empty()) break;
        if (s->scratch_bytes < floats * 4) {
            free_dev((void*&)s->scratch);
            s->scratch_bytes = 0;
            if (cudaMalloc(&s->scratch, floats * 4) != cudaSuccess) { rc = fail(s, RT_ERR_NOMEM, "cudaMalloc scratch"); break; }
            s->scratch_bytes = floats * 4;
        }
        for (JobDev& J : tab) J.scratch = s->scratch + reinterpret_cast<uint64_t>(J.scratch);
        if ((rc = ensure_paths(s, (uint32_t)std::min<uint64_t>(cursor, s->max_paths)))) break;
        if (cudaMemcpyAsync(s->d_jobs, tab.data(), tab.size() * sizeof(JobDev), cudaMemcpyHostToDevice, s->stream) !=
            cudaSuccess) { rc = fail(s, RT_ERR_CUDA, "batch table upload"); break; }
        WaveBufs Wb = scene_bufs(s);
        Wb.guide = false;
        q.width = tab[0].width; q.height = tab[0].height;
        int64_t e1 = 0, s1 = 0, l1 = 0;
        rc = run_wavefront(s, Wb, &tab[0].cam, &q, 0, 1, s->scratch, nullptr, 1, &e1, &s1, &l1, s->d_jobs,
                           (uint32_t)tab.size(), cursor, false, (RT_GRAPH_PASS_POOLS + 1ull) * maxd_b + 2);
        if (rc) break;
        for (size_t t = 0; t < tab.size(); t++) {
            int32_t j = ids[t];
            const JobDev& J = tab[t];
            rth::launch_accumulate(J.scratch, J.nsamp, J.npix, s->b_acc + pix_off[j] * 3, s->b_m2 + pix_off[j] * 3,
                                   s->b_cnt + pix_off[j], nullptr, 0.0f, 4u, 5.0f, s->stream);
            left[j] -= J.nsamp;
            if (!left[j]) pass_of[j] = pass + 1;
        }
        ext += e1; sh += s1; nl += l1 + (int64_t)tab.size();
        cudaEvent_t ev;
        if (cudaEventCreate(&ev) != cudaSuccess) { rc = fail(s, RT_ERR_CUDA, "cudaEventCreate"); break; }
        evs.push_back(ev);
        cudaEventRecord(ev, s->stream);
    }
    if (rc == RT_OK) {
        auto kind = mem == RT_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (out_sum && cudaMemcpyAsync(out_sum, s->b_acc, tot_pix * 12, kind, s->stream) != cudaSuccess) rc = RT_ERR_CUDA;
        if (out_m2 && cudaMemcpyAsync(out_m2, s->b_m2, tot_pix * 12, kind, s->stream) != cudaSuccess) rc = RT_ERR_CUDA;
        if (out_count && cudaMemcpyAsync(out_count, s->b_cnt, tot_pix * 4, kind, s->stream) != cudaSuccess) rc = RT_ERR_CUDA;
        if (rc) rc = fail(s, rc, "batch output copy");
    }
    cudaStreamSynchronize(s->stream);
    if (rc == RT_OK) {
        std::vector<float> pass_ms(evs.size(), 0.0f);
        for (size_t e = 1; e < evs.size(); e++) cudaEventElapsedTime(&pass_ms[e], evs[0], evs[e]);
        if (done_ms)
            for (int32_t j = 0; j < n_jobs; j++) done_ms[j] = pass_of[j] > 0 ? pass_ms[pass_of[j]] : 0.0f;
        s->last_ms = pass_ms.back();
        s->last_ext = ext;
        s->last_shadow = sh;
        s->last_launches = nl;
    }
    for (auto e : evs) cudaEventDestroy(e);
    if (rc) return rc;
    return check_err(s);
}

extern "C" int32_t rt_scene_build_time(const RtScene* s, double* ms) {
    if (!s || !ms) return RT_ERR_INVALID;
    *ms = s->build_ms;
    return RT_OK;
}

extern "C" int32_t rt_develop(RtScene* s, const float* lin, const RtDevelopParams* p, uint8_t* rgb8, int32_t mem) {
    if (!s || !p || !rgb8) return RT_ERR_INVALID;
    if (mem != RT_MEM_HOST && mem != RT_MEM_DEVICE) return fail(s, RT_ERR_INVALID, "mem must be RT_MEM_HOST or RT_MEM_DEVICE");
    if (p->width == 0 || p->height == 0 || (uint64_t)p->width * p->height > (1ull << 31))
        return fail(s, RT_ERR_INVALID, "develop: bad image size");
    if (p->tonemapper != RT_TONEMAP_AGX && p->tonemapper != RT_TONEMAP_ACES)
        return fail(s, RT_ERR_INVALID, "develop: unknown tone mapper");
    if (!(p->vignette >= 0.0f && p->vignette <= 1.0f) || !(p->distortion >= 0.0f && p->distortion <= 1.0f) ||
        !std::isfinite(p->exposure))
        return fail(s, RT_ERR_INVALID, "develop: vignette and distortion in [0, 1], a finite exposure");
    uint32_t npix = p->width * p->height;
    if (!lin && s->acc_npix != npix) return fail(s, RT_ERR_INVALID, "develop: no accumulators of this size");
    ENTER(s);
    size_t in_bytes = lin && mem == RT_MEM_HOST ? (size_t)npix * 12 : 0;
    size_t out_bytes = mem == RT_MEM_HOST ? ((size_t)npix * 3 + 15) / 16 * 16 : 0;
    int rc = ensure_stage(s, in_bytes + out_bytes);
    if (rc) return rc;
    const float* d_lin = lin;
    uint8_t* d_out = rgb8;
    if (in_bytes) {
        CK(cudaMemcpyAsync(s->stage, lin, in_bytes, cudaMemcpyHostToDevice, s->stream));
        d_lin = (const float*)s->stage;
    }
    if (out_bytes) d_out = (uint8_t*)s->stage + in_bytes;
    rth::launch_develop(d_lin, s->acc, s->cnt, p->width, p->height, p->exposure, p->tonemapper, p->vignette,
                        p->distortion, d_out, s->sms, s->stream);
    CK(cudaGetLastError());
    if (out_bytes) CK(cudaMemcpyAsync(rgb8, d_out, (size_t)npix * 3, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return RT_OK;
}

extern "C" int32_t rt_rgbe_decode(const uint8_t* d, size_t n, int32_t W, int32_t H, float* rgb) {
    if (!d || !rgb || W <= 0 || H <= 0) return RT_ERR_INVALID;
    std::vector<uint8_t> row((size_t)W * 4);
    size_t pos = 0;
    for (int32_t y = 0; y < H; y++) {
        if (pos + 4 <= n && d[pos] == 2 && d[pos + 1] == 2 && ((d[pos + 2] << 8) | d[pos + 3]) == W) {
            pos += 4;
            for (int c = 0; c < 4; c++)                      // one run list per channel
                for (int32_t x = 0; x < W;) {
                    if (pos >= n) return RT_ERR_INVALID;
                    int cnt = d[pos++];
                    bool run = cnt > 128;
                    if (run) cnt -= 128;
                    if (cnt == 0 || x + cnt > W || pos + (run ? 1 : (size_t)cnt) > n) return RT_ERR_INVALID;
                    for (int k = 0; k < cnt; k++) row[(size_t)(x + k) * 4 + c] = run ? d[pos] : d[pos + k];
                    pos += run ? 1 : cnt;
                    x += cnt;
                }
        } else {
            if (pos + (size_t)W * 4 > n) return RT_ERR_INVALID;
            memcpy(row.data(), d + pos, (size_t)W * 4);
            pos += (size_t)W * 4;
        }
        for (int32_t x = 0; x < W; x++) {
            const uint8_t* q = row.data() + (size_t)x * 4;
            float sc = q[3] ? std::ldexp(1.0f, (int)q[3] - 136) : 0.0f;
            float* o = rgb + ((size_t)y * W + x) * 3;
            o[0] = (float)q[0] * sc; o[1] = (float)q[1] * sc; o[2] = (float)q[2] * sc;
        }
    }
    return RT_OK;
}

extern "C" int32_t rt_last_render_stats(const RtScene* s, double* ms, int64_t* ext, int64_t* sh, int64_t* launches) {
    if (!s) return RT_ERR_INVALID;
    if (ms) *ms = s->last_ms;
    if (ext) *ext = s->last_ext;
    if (sh) *sh = s->last_shadow;
    if (launches) *launches = s->last_launches;
    return RT_OK;
}

extern "C" int32_t rt_set_tuning(RtScene* s, const RtTuning* t) {
    if (!s || !t) return RT_ERR_INVALID;
    if (t->max_paths != 0 && (t->max_paths < (1u << 16) || t->max_paths > MAX_PATHS))
        return fail(s, RT_ERR_INVALID, "max_paths must be 0 or in 65536..8388608");
    if (t->trace_blocks_per_sm > RT_TRACE_BLOCKS_PER_SM || t->shade_blocks_per_sm > 32)
        return fail(s, RT_ERR_INVALID, "trace_blocks_per_sm must be in 0..8, shade_blocks_per_sm in 0..32");
    if (t->stack_ring != 0 && (t->stack_ring > RT_SHORT_STACK || (t->stack_ring & (t->stack_ring - 1)) != 0))
        return fail(s, RT_ERR_INVALID, "stack_ring must be 0 or a power of two up to " + std::to_string(RT_SHORT_STACK));
    if (t->node_format != RT_NODES_QUANTISED && t->node_format != RT_NODES_FULL && t->node_format != RT_NODES_WIDE4)
        return fail(s, RT_ERR_INVALID, "node_format must be RT_NODES_FULL, RT_NODES_QUANTISED or RT_NODES_WIDE4");
    if (t->node_format == RT_NODES_QUANTISED && !s->qnodes_ok && !s->empty)
        return fail(s, RT_ERR_INVALID, "the scene's extents exceed the quantised node layout");
    if (t->node_format == RT_NODES_WIDE4 && !s->wide4_ok && !s->empty)
        return fail(s, RT_ERR_INVALID, "4-wide nodes exist for trees built on the device only");
    if (t->stack_limit != 0 && (int64_t)t->stack_limit > s->stack_cap_built)
        return fail(s, RT_ERR_INVALID, "stack_limit must be 0 or at most " + std::to_string(s->stack_cap_built) +
                                           " (the entries the scene's stack columns hold)");
    if (t->graph > 1) return fail(s, RT_ERR_INVALID, "graph must be 0 or 1");
    ENTER(s);
    CK(cudaStreamSynchronize(s->stream));
    s->max_paths = t->max_paths ? t->max_paths : MAX_PATHS;
    s->S.trace_per_sm = (int)t->trace_blocks_per_sm;
    s->S.shade_per_sm = (int)t->shade_blocks_per_sm;
    s->max_iterations = t->max_iterations;
    s->S.stack_cap = t->stack_limit ? (int)t->stack_limit : s->stack_cap_built;
    s->S.stack_ring = t->stack_ring ? (int)t->stack_ring : RT_SHORT_STACK;
    s->S.node_format = (s->qnodes_ok && t->node_format == RT_NODES_QUANTISED) ? RT_NODES_QUANTISED
                     : (s->wide4_ok && t->node_format == RT_NODES_WIDE4)    ? RT_NODES_WIDE4
                                                                            : RT_NODES_FULL;
    s->graph_mode = t->graph != 0;
    return RT_OK;
}

extern "C" int32_t rt_set_caller_stream(RtScene* s, void* stream) {
    if (!s) return RT_ERR_INVALID;
    s->caller = (cudaStream_t)stream;
    return RT_OK;
}

extern "C" int32_t rt_get_tuning(const RtScene* s, RtTuning* t) {
    if (!s || !t) return RT_ERR_INVALID;
    t->max_paths = s->max_paths;
    t->trace_blocks_per_sm = (uint32_t)s->S.trace_per_sm;
    t->shade_blocks_per_sm = (uint32_t)s->S.shade_per_sm;
    t->max_iterations = (uint32_t)s->max_iterations;
    t->stack_limit = (uint32_t)s->S.stack_cap;
    t->stack_ring = (uint32_t)s->S.stack_ring;
    t->node_format = (uint32_t)s->S.node_format;
    t->graph = s->graph_mode ? 1u : 0u;
    return RT_OK;
}

extern "C" int32_t rt_set_profiling(RtScene* s, int32_t enable) {
    if (!s) return RT_ERR_INVALID;
    s->profiling = enable != 0;
    return RT_OK;
}

extern "C" int32_t rt_kernel_times(const RtScene* s, double* ms, int64_t* launches) {
    if (!s) return RT_ERR_INVALID;
    for (int k = 0; k < 4; k++) {
        if (ms) ms[k] = s->kms[k];
        if (launches) launches[k] = s->kcount[k];
    }
    return RT_OK;
}

extern "C" int32_t rt_capture_rays(RtScene* s, const RtCamera* cam, const RtPassParams* p, uint32_t depth, float* rays,
                                   int64_t max_rays, int64_t* n_rays) {
    int rc = validate_pass(s, cam, p);
    if (rc) return rc;
    if (!rays || max_rays < 0) return fail(s, RT_ERR_INVALID, "null ray buffer");
    ENTER(s);
    RtPassParams q = *p;
    q.n_samples = 1;
    size_t bytes = (size_t)q.width * q.height * 3 * sizeof(float);
    if (s->scratch_bytes < bytes) {
        free_dev((void*&)s->scratch);
        s->scratch_bytes = 0;
        if (cudaMalloc(&s->scratch, bytes) != cudaSuccess) return fail(s, RT_ERR_NOMEM, "cudaMalloc scratch");
        s->scratch_bytes = bytes;
    }
    s->cap_depth = (int32_t)depth;
    s->cap_out = rays;
    s->cap_max = max_rays;
    s->cap_n = 0;
    int64_t e, sh, l;
    rc = render_device(s, cam, &q, s->scratch, nullptr, &e, &sh, &l);
    s->cap_depth = -1;
    s->cap_out = nullptr;
    if (n_rays) *n_rays = s->cap_n;
    if (rc) return rc;
    return check_err(s);
}

// ── allocation-free sample pass ─────────────────────────────────────────────
// Some hosts cannot let a library allocate device memory once they are
// running: a render loop that must not stall on cudaMalloc (it synchronises
// the device), a process whose device memory is already handed out by its
// framework's caching allocator so a direct cudaMalloc would fail or fragment
// the pool, or a plugin host that passes only buffers it allocated itself.
// rt_render_pass_noalloc serves them: its wavefront scratch (path state, ray
// and shadow queues, counters, error word) lives in the file-scope device array
// below instead of memory obtained at call time.  Every GPU that loads the
// library holds this array (RT_NOALLOC_SCRATCH_BYTES = 15 MB) until the
// process exits.
// path pool of the fixed array (positions are refilled with new samples as paths end):
// two path sets of 8 float4 fields, hit, retire records (4 float4), class
// queues and shadow rays
#define RT_NOALLOC_PATHS 32768u
static constexpr size_t kNaF4 = (size_t)RT_NOALLOC_PATHS * sizeof(float4);
static constexpr size_t kNaQueue = (size_t)RT_NOALLOC_PATHS * sizeof(uint32_t);
static constexpr size_t kNaShadow = (size_t)RT_NOALLOC_PATHS * 2 * 2 * sizeof(float4);
static constexpr size_t kNaCounters = (size_t)RT_CTR_WORDS * sizeof(uint32_t);
static constexpr size_t kNaBytes = 21 * kNaF4 + CLS_N * kNaQueue + kNaShadow + kNaCounters + 256;
static_assert(kNaBytes <= RT_NOALLOC_SCRATCH_BYTES, "no-alloc scratch size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[RT_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[64] = {};

// Device address of g_noalloc_scratch on `device` (the current device).  The
// symbol's host-side name is only a stand-in, so its address must come from
// cudaGetSymbolAddress, once per device.
static int noalloc_base(RtScene* s, void** out) {
    if (s->device < 0 || s->device >= 64) return fail(s, RT_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[s->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(s, RT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_addr[s->device] = p;
    }
    *out = g_noalloc_addr[s->device];
    return RT_OK;
}

extern "C" int32_t rt_render_pass_noalloc(RtScene* s, const RtCamera* cam, const RtPassParams* p,
                                          float* scratch_rgb) {
    int rc = validate_pass(s, cam, p);
    if (rc) return rc;
    if (!scratch_rgb) return fail(s, RT_ERR_INVALID, "null output buffer");
    uint64_t npix = (uint64_t)p->width * p->height;
    if (npix > RT_NOALLOC_MAX_PIXELS)
        return fail(s, RT_ERR_CAPACITY, "rt_render_pass_noalloc: width*height = " + std::to_string(npix) +
                                            " exceeds the fixed scratch limit of " +
                                            std::to_string(RT_NOALLOC_MAX_PIXELS) + " pixels");
    if (s->photons.present && s->photons.n > 0)
        return fail(s, RT_ERR_INVALID, "rt_render_pass_noalloc does not render scenes with a photon map");
    ENTER(s);
    void* base = nullptr;
    if ((rc = noalloc_base(s, &base))) return rc;
    unsigned char* b = (unsigned char*)base;
    WaveBufs W;
    size_t off = 0;
    auto take_f4 = [&]() { float4* q = (float4*)(b + off); off += kNaF4; return q; };
    for (int k = 0; k < 2; k++) {
        PathState& P = W.set[k];
        P.ray_o = take_f4(); P.ray_d = take_f4(); P.thr = take_f4(); P.wts = take_f4();
        P.meta = (uint4*)take_f4(); P.L = take_f4(); P.pend0 = take_f4(); P.pend1 = take_f4();
    }
    W.set[0].hit = W.set[1].hit = take_f4();
    W.Rt.meta = (uint4*)take_f4(); W.Rt.L = take_f4(); W.Rt.pend0 = take_f4(); W.Rt.pend1 = take_f4();
    for (int c = 0; c < CLS_N; c++) W.cq.q[c] = (uint32_t*)(b + off + c * kNaQueue);
    off += CLS_N * kNaQueue;
    W.sq = (float4*)(b + off);
    off += kNaShadow;
    W.counters = (uint32_t*)(b + off);
    off += kNaCounters;
    W.derr = (int*)(b + ((off + 255) & ~(size_t)255));
    W.cap = RT_NOALLOC_PATHS;
    CK(cudaMemsetAsync(W.derr, 0, sizeof(int), s->stream));
    uint32_t nsamp = std::max<uint32_t>(p->n_samples, 1);
    // the run clears the counters it uses: the array keeps the last call's contents
    rc = run_wavefront(s, W, cam, p, p->sample_idx, nsamp, scratch_rgb, nullptr, (uint32_t)npix, nullptr, nullptr,
                       nullptr);
    if (rc) return rc;
    int h = 0;
    CK(cudaMemcpyAsync(&h, W.derr, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (h) return fail(s, h, "traversal stack overflow");
    return RT_OK;
}

// ── photon map entry points ──────────────────────────────────────────────────
// Emitter set-up of PhotonMap::build / build_from_quad (photon.rs:41-135):
// 40 floats per emitter, consumed by the emission kernel.
static void emitter_setup(const RtScene* s, const RtPhotonEmitter& e0, float* f) {
    const float PI = 3.14159265358979323846f;
    RtPhotonEmitter e = e0;
    if (e.type == RT_EMIT_LIGHT) {
        // a quad of the light list, coloured by its material's emission; the quad
        // record is (normal, d) (Q.xyz, u.x) (u.yz, v.xy) (v.z, w.xyz) (gid, mat, area, -)
        const DevLight& L = s->h_lights[e.light];
        const float4* g = L.g;
        e.type = RT_EMIT_QUAD;
        e.corner[0] = g[1].x; e.corner[1] = g[1].y; e.corner[2] = g[1].z;
        e.u[0] = g[1].w; e.u[1] = g[2].x; e.u[2] = g[2].y;
        e.v[0] = g[2].z; e.v[1] = g[2].w; e.v[2] = g[3].x;
        for (int c = 0; c < 3; c++) e.color[c] = s->h_emission[(size_t)L.mat * 3 + c];
    }
    if (e.type == RT_EMIT_SUN) {
        // rebuild_caustics with a Physical sky (scene.rs:40-52): a disk facing the
        // sun, coloured by the sky radiance 0.04 off the sun direction, ×π
        float3 sun = s->S.sun_dir;
        float3 perp = std::fabs(sun.x) < 0.9f ? rtd::sky_unit(make_float3(0.0f, -sun.z, sun.y))
                                              : rtd::sky_unit(make_float3(-sun.z, 0.0f, sun.x));
        float3 pd = rtd::sky_unit(make_float3(sun.x + perp.x * 0.04f, sun.y + perp.y * 0.04f, sun.z + perp.z * 0.04f));
        float3 col = rtd::preetham_sky_eval(pd, sun, s->S.turbidity);
        e.type = RT_EMIT_DISK;
        e.dir[0] = sun.x; e.dir[1] = sun.y; e.dir[2] = sun.z;
        e.color[0] = col.x * PI; e.color[1] = col.y * PI; e.color[2] = col.z * PI;
    }
    memset(f, 0, 40 * sizeof(float));
    auto put = [&](int at, H3 v) { f[at] = v.x; f[at + 1] = v.y; f[at + 2] = v.z; };
    if (e.type == RT_EMIT_DISK) {
        H3 sun = h3(e.dir[0], e.dir[1], e.dir[2]);
        H3 ms = h3(-sun.x, -sun.y, -sun.z);
        H3 sd = ms / hlen(ms);
        H3 up = std::fabs(sd.x) < 0.999f ? h3(1, 0, 0) : h3(0, 1, 0);
        H3 t = hcross(sd, up);
        t = t / hlen(t);
        H3 b = hcross(sd, t);
        const float CLIP = 1.0e3f;
        auto clip = [&](float x) { return std::min(std::max(x, -CLIP), CLIP); };
        H3 mn = h3(clip(s->world_lo[0]), clip(s->world_lo[1]), clip(s->world_lo[2]));
        H3 mx = h3(clip(s->world_hi[0]), clip(s->world_hi[1]), clip(s->world_hi[2]));
        H3 c = (mn + mx) * 0.5f;
        float r = std::fmax(hlen(mx - mn) * 0.5f, 1.0e-3f);
        H3 su = sun / hlen(sun);
        float area = PI * r * r;
        put(0, t); put(3, b); put(6, c + su * r); put(9, sd);
        put(30, h3(e.color[0], e.color[1], e.color[2]) * (area / ((float)e.n_photons * PI)));
        f[33] = r;
        f[34] = 15.0f * area / (PI * 20.0f * 20.0f);
    } else {
        H3 u = h3(e.u[0], e.u[1], e.u[2]), v = h3(e.v[0], e.v[1], e.v[2]);
        H3 cr = hcross(u, v);
        float area = hlen(cr);
        H3 nrm = cr / area;
        H3 up = std::fabs(nrm.y) < 0.9f ? h3(0, 1, 0) : h3(1, 0, 0);
        H3 ta = hcross(nrm, up);
        ta = ta / hlen(ta);
        H3 ba = hcross(nrm, ta);
        put(12, nrm); put(15, h3(e.corner[0], e.corner[1], e.corner[2])); put(18, u); put(21, v);
        put(24, ta); put(27, ba);
        put(30, h3(e.color[0], e.color[1], e.color[2]) * (area * PI / (float)e.n_photons));
        f[34] = 15.0f;
        put(35, h3(e.target[0], e.target[1], e.target[2]));
        f[38] = e.target[3] > 0.0f ? e.target[3] : 0.0f;
    }
}

extern "C" int32_t rt_photon_build(RtScene* s, const RtPhotonParams* p, int64_t* n_stored) {
    if (!s || !p) return RT_ERR_INVALID;
    if (p->n_emitters < 1 || p->n_emitters > RT_MAX_EMITTERS) return fail(s, RT_ERR_INVALID, "1..8 photon emitters");
    if (!(p->gather_radius > 0.0f)) return fail(s, RT_ERR_INVALID, "gather radius must be positive");
    if (p->knn_k > 4096) return fail(s, RT_ERR_INVALID, "knn_k must be ≤ 4096");
    if (s->empty) return fail(s, RT_ERR_INVALID, "scene has no primitives");
    uint64_t total = 0;
    for (int i = 0; i < p->n_emitters; i++) {
        const RtPhotonEmitter& e = p->emitters[i];
        if (e.type != RT_EMIT_DISK && e.type != RT_EMIT_QUAD && e.type != RT_EMIT_SUN && e.type != RT_EMIT_LIGHT)
            return fail(s, RT_ERR_INVALID, "unknown emitter type");
        if (e.type == RT_EMIT_SUN && s->S.bg_type != RT_BG_PHYSICAL)
            return fail(s, RT_ERR_INVALID, "a sun emitter needs a Physical sky background");
        if (e.type == RT_EMIT_LIGHT &&
            (e.light < 0 || e.light >= (int32_t)s->h_lights.size() || s->h_lights[e.light].type != RT_PRIM_QUAD))
            return fail(s, RT_ERR_INVALID, "a light emitter must name a quad of the light list");
        if (e.n_photons == 0) return fail(s, RT_ERR_INVALID, "emitter with zero photons");
        total += e.n_photons;
    }
    if (total > 0xFFFFFFFFull) return fail(s, RT_ERR_CAPACITY, "more than 2^32 - 1 photons");
    uint64_t first = p->first_photon, count = p->shard_photons ? p->shard_photons : total;
    if (first + count > total) return fail(s, RT_ERR_INVALID, "photon shard beyond the emitters' photons");
    if (count > MAX_PATHS) return fail(s, RT_ERR_CAPACITY, "more than 8M photons traced per build");
    ENTER(s);
    int rc = ensure_paths(s, (uint32_t)std::max<uint64_t>(count, s->cap));
    if (rc) return rc;
    std::vector<float> setup((size_t)p->n_emitters * 40);
    for (int i = 0; i < p->n_emitters; i++) emitter_setup(s, p->emitters[i], &setup[(size_t)i * 40]);
    cudaError_t e = rth::photon_build(s->S, s->photons, s->P, s->queue[0], s->queue[1], s->counters, *p, setup.data(),
                                      (uint32_t)first, (uint32_t)count, s->sms, s->stream, n_stored,
                                      s->photon_stage_ms);
    if (e != cudaSuccess) return fail(s, RT_ERR_CUDA, std::string("photon build: ") + cudaGetErrorString(e));
    return check_err(s);
}

extern "C" int32_t rt_photon_build_times(const RtScene* s, float* ms) {
    if (!s || !ms) return RT_ERR_INVALID;
    for (int k = 0; k < 3; k++) ms[k] = s->photon_stage_ms[k];
    return RT_OK;
}

extern "C" int32_t rt_photon_set(RtScene* s, const float* pos, const float* power, const float* nor,
                                 const int32_t* index, int64_t n, float radius, uint32_t k) {
    if (!s || n < 0 || (n > 0 && (!pos || !power || !nor))) return RT_ERR_INVALID;
    if (!(radius > 0.0f)) return fail(s, RT_ERR_INVALID, "gather radius must be positive");
    if (n > (int64_t)MAX_PATHS) return fail(s, RT_ERR_CAPACITY, "more than 8M photons");
    ENTER(s);
    std::vector<float4> a(n), b(n), c(n);
    for (int64_t i = 0; i < n; i++) {
        int32_t id = index ? index[i] : (int32_t)i;
        float fid;
        memcpy(&fid, &id, 4);
        a[i] = make_float4(pos[i * 3], pos[i * 3 + 1], pos[i * 3 + 2], fid);
        b[i] = make_float4(power[i * 3], power[i * 3 + 1], power[i * 3 + 2], 0.f);
        c[i] = make_float4(nor[i * 3], nor[i * 3 + 1], nor[i * 3 + 2], 0.f);
    }
    cudaError_t e = rth::photon_set(s->photons, a.data(), b.data(), c.data(), (uint32_t)n, radius, k, s->stream);
    if (e != cudaSuccess) return fail(s, RT_ERR_CUDA, std::string("photon set: ") + cudaGetErrorString(e));
    return RT_OK;
}

extern "C" int32_t rt_photon_clear(RtScene* s) {
    if (!s) return RT_ERR_INVALID;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    s->photons.release();
    return RT_OK;
}

extern "C" int32_t rt_photon_export(const RtScene* s, float* pos, float* power, float* nor, int32_t* index, int64_t* n) {
    if (!s) return RT_ERR_INVALID;
    uint32_t m = s->photons.present ? s->photons.n : 0;
    if (n) *n = m;
    if (!pos || m == 0) return RT_OK;
    cudaSetDevice(s->device);
    std::vector<float4> a(m), b(m), c(m);
    cudaMemcpy(a.data(), s->photons.exp_pos, (size_t)m * 16, cudaMemcpyDeviceToHost);
    cudaMemcpy(b.data(), s->photons.exp_pow, (size_t)m * 16, cudaMemcpyDeviceToHost);
    cudaMemcpy(c.data(), s->photons.exp_nor, (size_t)m * 16, cudaMemcpyDeviceToHost);
    for (uint32_t i = 0; i < m; i++) {
        pos[i * 3] = a[i].x; pos[i * 3 + 1] = a[i].y; pos[i * 3 + 2] = a[i].z;
        power[i * 3] = b[i].x; power[i * 3 + 1] = b[i].y; power[i * 3 + 2] = b[i].z;
        nor[i * 3] = c[i].x; nor[i * 3 + 1] = c[i].y; nor[i * 3 + 2] = c[i].z;
        if (index) memcpy(&index[i], &a[i].w, 4);
    }
    return RT_OK;
}

extern "C" int32_t rt_photon_gather(RtScene* s, const float* q, int64_t n, float* irr, int32_t mem) {
    if (!s || n < 0 || (n > 0 && (!q || !irr))) return RT_ERR_INVALID;
    if (n == 0) return RT_OK;
    ENTER(s);
    if (!s->photons.present || s->photons.n == 0) {
        if (mem == RT_MEM_DEVICE) { CK(cudaMemsetAsync(irr, 0, n * 12, s->stream)); return RT_OK; }
        memset(irr, 0, n * 12);
        return RT_OK;
    }
    const float* dq = q;
    float* dout = irr;
    size_t qb = (size_t)n * 24, ob = (size_t)n * 12;
    if (mem != RT_MEM_DEVICE) {
        int rc = ensure_stage(s, qb + ob + 256);
        if (rc) return rc;
        dq = (const float*)s->stage;
        dout = (float*)((char*)s->stage + ((qb + 255) & ~(size_t)255));
        CK(cudaMemcpyAsync((void*)dq, q, qb, cudaMemcpyHostToDevice, s->stream));
    }
    rth::launch_photon_gather_api(s->photons, dq, (uint32_t)n, dout, s->sms, s->stream);
    CK(cudaGetLastError());
    if (mem != RT_MEM_DEVICE) CK(cudaMemcpyAsync(irr, dout, ob, cudaMemcpyDeviceToHost, s->stream));
    return check_err(s);
}

extern "C" int32_t rt_knn(RtScene* s, const float* q, int64_t n, int32_t k, float rmax, int32_t* idx, float* d2,
                          int32_t mem) {
    if (!s || n < 0 || k <= 0 || (n > 0 && (!q || !idx || !d2))) return RT_ERR_INVALID;
    if (k > 256) return fail(s, RT_ERR_INVALID, "k must be ≤ 256");
    if (n == 0) return RT_OK;
    ENTER(s);
    if (!s->photons.present || s->photons.n == 0) {
        std::vector<int32_t> mi((size_t)n * k, -1);
        std::vector<float> md((size_t)n * k, INFINITY);
        auto kind = mem == RT_MEM_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost;
        CK(cudaMemcpy(idx, mi.data(), mi.size() * 4, kind));
        CK(cudaMemcpy(d2, md.data(), md.size() * 4, kind));
        return RT_OK;
    }
    const float* dq = q;
    int32_t* di = idx;
    float* dd = d2;
    size_t qb = (size_t)n * 12, ob = (size_t)n * k * 4;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    if (mem != RT_MEM_DEVICE) {
        int rc = ensure_stage(s, al(qb) + 2 * al(ob) + 256);
        if (rc) return rc;
        dq = (const float*)s->stage;
        di = (int32_t*)((char*)s->stage + al(qb));
        dd = (float*)((char*)s->stage + al(qb) + al(ob));
        CK(cudaMemcpyAsync((void*)dq, q, qb, cudaMemcpyHostToDevice, s->stream));
    }
    rth::launch_knn_api(s->photons, dq, (uint32_t)n, k, rmax * rmax, di, dd, s->d_err, s->sms, s->stream);
    CK(cudaGetLastError());
    if (mem != RT_MEM_DEVICE) {
        CK(cudaMemcpyAsync(idx, di, ob, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaMemcpyAsync(d2, dd, ob, cudaMemcpyDeviceToHost, s->stream));
    }
    return check_err(s);
}

// ── path guiding ────────────────────────────────────────────────────────────
namespace {
// device copies for the rt_guide_* test entry points (freed on scope exit)
struct Tmp {
    void* p = nullptr;
    ~Tmp() { if (p) cudaFree(p); }
};
int guide_ready(RtScene* s) {
    if (!s) return RT_ERR_INVALID;
    if (!s->guide) return fail(s, RT_ERR_INVALID, "no guide: call rt_guide_init first");
    return RT_OK;
}
// in: host or device input of `bytes`; returns a device pointer
int stage_in(RtScene* s, const void* in, size_t bytes, int32_t mem, Tmp& t, const void** d) {
    if (mem == RT_MEM_DEVICE || bytes == 0) { *d = in; return RT_OK; }
    if (cudaMalloc(&t.p, bytes) != cudaSuccess) return fail(s, RT_ERR_NOMEM, "cudaMalloc guide staging");
    CK(cudaMemcpyAsync(t.p, in, bytes, cudaMemcpyHostToDevice, s->stream));
    *d = t.p;
    return RT_OK;
}
int stage_out(RtScene* s, void* out, size_t bytes, int32_t mem, Tmp& t, void** d) {
    if (mem == RT_MEM_DEVICE || bytes == 0) { *d = out; return RT_OK; }
    if (cudaMalloc(&t.p, bytes) != cudaSuccess) return fail(s, RT_ERR_NOMEM, "cudaMalloc guide staging");
    *d = t.p;
    return RT_OK;
}
int guide_api(RtScene* s, const float* q, const float* dirs, const float* u, int64_t n, float* raw, float* out,
              size_t out_per, int32_t mem) {
    int rc = guide_ready(s);
    if (rc) return rc;
    if (n < 0 || n > (1ll << 28) || (n > 0 && !q)) return fail(s, RT_ERR_INVALID, "guide query count or pointer");
    if (n == 0) return RT_OK;
    ENTER(s);
    Tmp tq, td, tu, tr, to;
    const void *dq = nullptr, *dd = nullptr, *du = nullptr;
    void *dr = nullptr, *dout = nullptr;
    if ((rc = stage_in(s, q, (size_t)n * 36, mem, tq, &dq))) return rc;
    if (dirs && (rc = stage_in(s, dirs, (size_t)n * 12, mem, td, &dd))) return rc;
    if (u && (rc = stage_in(s, u, (size_t)n * 16, mem, tu, &du))) return rc;
    if (raw && (rc = stage_out(s, raw, (size_t)n * rtg::NOUT * 4, mem, tr, &dr))) return rc;
    if (out && (rc = stage_out(s, out, (size_t)n * out_per * 4, mem, to, &dout))) return rc;
    rtgh::eval(s->guide, (const float*)dq, (uint32_t)n, (const float*)dd, (const float*)du, (float*)dr, (float*)dout,
               s->sms, s->stream);
    CK(cudaGetLastError());
    if (mem != RT_MEM_DEVICE) {
        if (raw) CK(cudaMemcpyAsync(raw, dr, (size_t)n * rtg::NOUT * 4, cudaMemcpyDeviceToHost, s->stream));
        if (out) CK(cudaMemcpyAsync(out, dout, (size_t)n * out_per * 4, cudaMemcpyDeviceToHost, s->stream));
    }
    CK(cudaStreamSynchronize(s->stream));
    return check_err(s);
}
// host samples (n × 13: position, normal, ω_o, ω_i, weight) → device training
// samples (3 float4 each: (p, w), (n, θ_o/π), (ω_i, φ_o/2π))
int stage_samples(RtScene* s, const float* smp, int64_t n, Tmp& t, const float4** d) {
    std::vector<float4> h((size_t)n * 3);
    for (int64_t i = 0; i < n; i++) {
        const float* r = smp + i * 13;
        float th = std::acos(std::fmin(std::fmax(r[8], -1.0f), 1.0f)) * 0.318309886f;
        float ph = (std::atan2(r[7], r[6]) + 3.14159265f) * 0.159154943f;
        h[i * 3] = make_float4(r[0], r[1], r[2], r[12]);
        h[i * 3 + 1] = make_float4(r[3], r[4], r[5], th);
        h[i * 3 + 2] = make_float4(r[9], r[10], r[11], ph);
    }
    if (cudaMalloc(&t.p, h.size() * sizeof(float4)) != cudaSuccess) return fail(s, RT_ERR_NOMEM, "cudaMalloc samples");
    CK(cudaMemcpy(t.p, h.data(), h.size() * sizeof(float4), cudaMemcpyHostToDevice));
    *d = (const float4*)t.p;
    return RT_OK;
}
}  // namespace

extern "C" int32_t rt_guide_init(RtScene* s, const RtGuideParams* p) {
    if (!s || !p) return RT_ERR_INVALID;
    if (p->batch == 0 || p->batch % 1024 || p->batch > (1u << 22))
        return fail(s, RT_ERR_INVALID, "guide batch must be a positive multiple of 1024, at most 2^22");
    if (p->record_capacity == 0 || p->record_capacity > (1u << 27))
        return fail(s, RT_ERR_INVALID, "guide record capacity must be in 1..2^27");
    if (!(p->learning_rate > 0.0f) || !(p->beta1 >= 0.0f && p->beta1 < 1.0f) || !(p->beta2 >= 0.0f && p->beta2 < 1.0f) ||
        !(p->epsilon > 0.0f))
        return fail(s, RT_ERR_INVALID, "guide Adam parameters");
    if (!(p->alpha_max > 0.0f && p->alpha_max < 1.0f) || !(p->log_kappa_max > rtg::LOGK_LO && p->log_kappa_max <= 20.0f))
        return fail(s, RT_ERR_INVALID, "guide caps: alpha_max in (0, 1), log_kappa_max in (-5, 20]");
    if (p->min_resolution < 2 || !(p->level_scale >= 1.0f) ||
        (double)p->min_resolution * std::pow((double)p->level_scale, rtg::LEVELS - 1) > (double)(1u << 20))
        return fail(s, RT_ERR_INVALID, "guide grid resolutions must be in 2..2^20");
    for (int a = 0; a < 3; a++)
        if (!std::isfinite(p->domain_min[a]) || !std::isfinite(p->domain_max[a]) || p->domain_max[a] < p->domain_min[a])
            return fail(s, RT_ERR_INVALID, "guide domain");
    ENTER(s);
    CK(cudaStreamSynchronize(s->stream));
    rtgh::destroy(s->guide);
    s->guide = nullptr;
    std::string err;
    s->guide = rtgh::create(*p, s->world_lo, s->world_hi, &err);
    if (!s->guide) return fail(s, RT_ERR_NOMEM, err);
    return RT_OK;
}

extern "C" int32_t rt_guide_mode(RtScene* s, int32_t mode) {
    if (!s) return RT_ERR_INVALID;
    if (mode < RT_GUIDE_OFF || mode > RT_GUIDE_TRAIN) return fail(s, RT_ERR_INVALID, "guide mode must be 0, 1 or 2");
    if (mode != RT_GUIDE_OFF && !s->guide) return fail(s, RT_ERR_INVALID, "no guide: call rt_guide_init first");
    if (s->guide) rtgh::set_mode(s->guide, mode);
    return RT_OK;
}

extern "C" int32_t rt_guide_params(RtScene* s, float* params, int32_t write) {
    int rc = guide_ready(s);
    if (rc) return rc;
    if (!params) return fail(s, RT_ERR_INVALID, "null parameter buffer");
    ENTER(s);
    CK(cudaStreamSynchronize(s->stream));
    CK(rtgh::params_io(s->guide, params, write, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return RT_OK;
}

extern "C" int32_t rt_guide_eval(RtScene* s, const float* q, int64_t n, float* raw, int32_t mem) {
    if (!raw && n > 0) return s ? fail(s, RT_ERR_INVALID, "null output") : RT_ERR_INVALID;
    return guide_api(s, q, nullptr, nullptr, n, raw, nullptr, 0, mem);
}

extern "C" int32_t rt_guide_pdf(RtScene* s, const float* q, const float* dirs, int64_t n, float* pdf, int32_t mem) {
    if ((!dirs || !pdf) && n > 0) return s ? fail(s, RT_ERR_INVALID, "null direction or output") : RT_ERR_INVALID;
    return guide_api(s, q, dirs, nullptr, n, nullptr, pdf, 1, mem);
}

extern "C" int32_t rt_guide_sample(RtScene* s, const float* q, const float* u, int64_t n, float* out, int32_t mem) {
    if ((!u || !out) && n > 0) return s ? fail(s, RT_ERR_INVALID, "null random numbers or output") : RT_ERR_INVALID;
    return guide_api(s, q, nullptr, u, n, nullptr, out, 4, mem);
}

extern "C" int32_t rt_guide_loss_grad(RtScene* s, const float* samples, int64_t n, float* loss, float* grad) {
    int rc = guide_ready(s);
    if (rc) return rc;
    if (n <= 0 || n > (1ll << 22) || !samples) return fail(s, RT_ERR_INVALID, "guide samples: 1..2^22 rows");
    ENTER(s);
    Tmp t;
    const float4* d = nullptr;
    if ((rc = stage_samples(s, samples, n, t, &d))) return rc;
    CK(rtgh::train_explicit(s->guide, d, (uint32_t)n, 0, loss, s->sms, s->stream));
    if (grad) CK(rtgh::grad_out(s->guide, grad, s->stream));
    return check_err(s);
}

extern "C" int32_t rt_guide_train(RtScene* s, const float* samples, int64_t n, int32_t steps, float* loss) {
    int rc = guide_ready(s);
    if (rc) return rc;
    if (n <= 0 || n > (1ll << 22) || !samples) return fail(s, RT_ERR_INVALID, "guide samples: 1..2^22 rows");
    if (steps < 1) return fail(s, RT_ERR_INVALID, "steps must be at least 1");
    ENTER(s);
    Tmp t;
    const float4* d = nullptr;
    if ((rc = stage_samples(s, samples, n, t, &d))) return rc;
    CK(rtgh::train_explicit(s->guide, d, (uint32_t)n, steps, loss, s->sms, s->stream));
    return check_err(s);
}

extern "C" int32_t rt_guide_stats(const RtScene* s, int64_t* records, int64_t* samples, int64_t* steps,
                                  double* train_ms) {
    if (!s || !s->guide) return RT_ERR_INVALID;
    rtgh::stats(s->guide, records, samples, steps, train_ms);
    return RT_OK;
}
