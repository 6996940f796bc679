// rt_build.cu — the BVH built on the device: the binary SAH tree, then its
// collapse to 8-wide nodes (full and quantised copies).
//
// The same tree as the host builder (SahBuilder in rt_host.cu), which restates
// BvhTree::sah_partition (bvh.rs:290-323): at every node the centroid bounds,
// 12 bins per axis, the prefix / suffix surface-area sweep with
// cost = 1 + (SA_l·N_l + SA_r·N_r)/SA_node, the cheapest (axis, bin) split,
// a stable counting sort of the node's primitives by bin on that axis, and a
// split at half the span when one side would be empty.  The internal node
// that splits [lo, hi) at mid is numbered mid − 1 (a bijection onto
// [0, n − 1)), so the tree does not depend on the order nodes are processed.
//
// Large nodes are split level by level: atomics (order-independent min / max
// and counts) gather the node box, centroid bounds and bin statistics, one
// thread per node chooses the split, and a segmented stable radix sort by bin
// reorders the primitives.  Nodes below SMALL primitives are finished by one
// thread each with the sequential algorithm.  Compiled without FMA
// contraction so every comparison sees the host's values.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "rt_internal.h"

namespace {

constexpr int NB = 12;           // bins per axis (bvh.rs:295)
constexpr int SMALL = 192;       // nodes below this many primitives: one thread
constexpr int CHUNK = 4096;      // primitives per block in the level kernels

struct Seg { int32_t lo, hi, parent, side; };   // side 0: parent's left child, 1: right, −1: root

// ordered-integer images of floats for atomicMin / atomicMax
__device__ __forceinline__ int f2o(float f) { int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7FFFFFFF; }
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

__device__ __forceinline__ float area6(const float* b) {                          // aabb surface area
    float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}
__device__ __forceinline__ void unite6(float* a, const float* b) {
    for (int k = 0; k < 3; k++) { a[k] = fminf(a[k], b[k]); a[3 + k] = fmaxf(a[3 + k], b[3 + k]); }
}
__device__ __forceinline__ int bin_of(float c, float cmn, float ext) {
    float t = (c - cmn) / ext;
    return min((int)((float)NB * t), NB - 1);
}

// node statistics: box (6), centroid bounds (6), then per axis per bin a count
// and a box (7 words): 12 + 3·NB·7 ints
constexpr int ST_WORDS = 12 + 3 * NB * 7;

__global__ void k_centroids(const float* __restrict__ box, int32_t n, float* __restrict__ cen, int32_t* idx) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* b = box + (size_t)i * 6;
        for (int a = 0; a < 3; a++) cen[(size_t)i * 3 + a] = (b[a] + b[3 + a]) * 0.5f;
        idx[i] = i;
    }
}

__global__ void k_stats_init(int32_t* st, int32_t nseg) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nseg * ST_WORDS; i += gridDim.x * blockDim.x) {
        int w = i % ST_WORDS;
        bool is_min;
        if (w < 12) is_min = (w % 6) < 3;
        else {
            int r = (w - 12) % 7;
            if (r == 0) { st[i] = 0; continue; }                 // count
            is_min = r <= 3;
        }
        st[i] = is_min ? 0x7F800000 : (int)0xFF800000 ^ 0x7FFFFFFF;   // +inf / −inf images
    }
}

// pass 1: node box and centroid bounds (chunk c of segment chunk_seg[c])
__global__ void k_stats_bounds(const Seg* __restrict__ segs, const int32_t* __restrict__ chunk_seg,
                               const int32_t* __restrict__ chunk_lo, int32_t nchunks, const int32_t* __restrict__ idx,
                               const float* __restrict__ box, const float* __restrict__ cen, int32_t* st) {
    __shared__ int sh[12];
    for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        if (threadIdx.x < 12) sh[threadIdx.x] = (threadIdx.x % 6) < 3 ? 0x7F800000 : (int)0xFF800000 ^ 0x7FFFFFFF;
        __syncthreads();
        const Seg s = segs[chunk_seg[c]];
        int32_t lo = chunk_lo[c], hi = min(lo + CHUNK, s.hi);
        float v[12];
        for (int k = 0; k < 3; k++) { v[k] = INFINITY; v[3 + k] = -INFINITY; v[6 + k] = INFINITY; v[9 + k] = -INFINITY; }
        for (int32_t k = lo + threadIdx.x; k < hi; k += blockDim.x) {
            int32_t o = idx[k];
            const float* b = box + (size_t)o * 6;
            for (int a = 0; a < 3; a++) {
                v[a] = fminf(v[a], b[a]); v[3 + a] = fmaxf(v[3 + a], b[3 + a]);
                float cc = cen[(size_t)o * 3 + a];
                v[6 + a] = fminf(v[6 + a], cc); v[9 + a] = fmaxf(v[9 + a], cc);
            }
        }
        for (int w = 0; w < 12; w++) {
            if ((w % 6) < 3) atomicMin(&sh[w], f2o(v[w])); else atomicMax(&sh[w], f2o(v[w]));
        }
        __syncthreads();
        if (threadIdx.x < 12) {
            int32_t* g = st + (size_t)chunk_seg[c] * ST_WORDS;
            if ((threadIdx.x % 6) < 3) atomicMin(&g[threadIdx.x], sh[threadIdx.x]);
            else atomicMax(&g[threadIdx.x], sh[threadIdx.x]);
        }
        __syncthreads();
    }
}

// pass 2: per axis with a non-degenerate centroid extent, bin counts and boxes
__global__ void k_stats_bins(const Seg* __restrict__ segs, const int32_t* __restrict__ chunk_seg,
                             const int32_t* __restrict__ chunk_lo, int32_t nchunks, const int32_t* __restrict__ idx,
                             const float* __restrict__ box, const float* __restrict__ cen, int32_t* st) {
    __shared__ int sh[3 * NB * 7];
    for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        for (int w = threadIdx.x; w < 3 * NB * 7; w += blockDim.x) {
            int r = w % 7;
            sh[w] = r == 0 ? 0 : (r <= 3 ? 0x7F800000 : (int)0xFF800000 ^ 0x7FFFFFFF);
        }
        __syncthreads();
        int32_t s = chunk_seg[c];
        const int32_t* g = st + (size_t)s * ST_WORDS;
        float cmn[3], ext[3];
        for (int a = 0; a < 3; a++) { cmn[a] = o2f(g[6 + a]); ext[a] = o2f(g[9 + a]) - cmn[a]; }
        int32_t lo = chunk_lo[c], hi = min(lo + CHUNK, segs[s].hi);
        for (int32_t k = lo + threadIdx.x; k < hi; k += blockDim.x) {
            int32_t o = idx[k];
            const float* b = box + (size_t)o * 6;
            for (int a = 0; a < 3; a++) {
                if (ext[a] < 1e-6f) continue;
                int bi = bin_of(cen[(size_t)o * 3 + a], cmn[a], ext[a]);
                int* bw = sh + (a * NB + bi) * 7;
                atomicAdd(bw, 1);
                for (int q = 0; q < 3; q++) { atomicMin(bw + 1 + q, f2o(b[q])); atomicMax(bw + 4 + q, f2o(b[3 + q])); }
            }
        }
        __syncthreads();
        int32_t* gw = st + (size_t)s * ST_WORDS + 12;
        for (int w = threadIdx.x; w < 3 * NB * 7; w += blockDim.x) {
            int r = w % 7;
            if (r == 0) { if (sh[w]) atomicAdd(gw + w, sh[w]); }
            else if (r <= 3) atomicMin(gw + w, sh[w]);
            else atomicMax(gw + w, sh[w]);
        }
        __syncthreads();
    }
}

// the split of one node from its statistics (SahBuilder::partition's sweep);
// *bax, *ext_ok: the axis the primitives are binned on; returns the split
// offset within the node
__device__ int32_t choose_split(const int32_t* g, int32_t span, int* bax_out, bool* binned) {
    float nb[6];
    for (int w = 0; w < 6; w++) nb[w] = o2f(g[w]);
    float nsa = area6(nb);
    float best = INFINITY;
    int bax = 0, bsp = 0;
    for (int ax = 0; ax < 3; ax++) {
        float ext = o2f(g[9 + ax]) - o2f(g[6 + ax]);
        if (ext < 1e-6f) continue;
        const int32_t* bw = g + 12 + ax * NB * 7;
        float lsa[NB];
        uint32_t ln[NB];
        bool ah = false;
        float acc[6];
        uint32_t an = 0;
        for (int i = 0; i < NB; i++) {
            const int32_t* q = bw + i * 7;
            an += (uint32_t)q[0];
            if (q[0]) {
                float b[6];
                for (int w = 0; w < 6; w++) b[w] = o2f(q[1 + w]);
                if (ah) unite6(acc, b); else for (int w = 0; w < 6; w++) acc[w] = b[w];
                ah = true;
            }
            ln[i] = an;
            lsa[i] = ah ? area6(acc) : 0.0f;
        }
        ah = false;
        an = 0;
        for (int sp = NB - 2; sp >= 0; sp--) {
            const int32_t* q = bw + (sp + 1) * 7;
            an += (uint32_t)q[0];
            if (q[0]) {
                float b[6];
                for (int w = 0; w < 6; w++) b[w] = o2f(q[1 + w]);
                if (ah) unite6(acc, b); else for (int w = 0; w < 6; w++) acc[w] = b[w];
                ah = true;
            }
            uint32_t nl = ln[sp], nr = an;
            if (nl == 0 || nr == 0) continue;
            float rsa = ah ? area6(acc) : 0.0f;
            float cost = 1.0f + (lsa[sp] * (float)nl + rsa * (float)nr) / nsa;
            if (cost < best) { best = cost; bax = ax; bsp = sp; }
        }
    }
    float ext = o2f(g[9 + bax]) - o2f(g[6 + bax]);
    *bax_out = bax;
    *binned = !(ext < 1e-6f);
    uint32_t mid_off = 0;
    if (*binned) {
        const int32_t* bw = g + 12 + bax * NB * 7;
        for (int b = 0; b <= bsp; b++) mid_off += (uint32_t)bw[b * 7];
    } else {
        mid_off = (uint32_t)span;                            // every primitive in bin 0
    }
    return (mid_off == 0 || mid_off == (uint32_t)span) ? span / 2 : (int32_t)mid_off;
}

struct LevelOut {
    Seg* next; int32_t* n_next;          // large children
    Seg* small; int32_t* n_small;        // small children
};

__device__ void link(int32_t* bl, int32_t* br, int32_t* root, const Seg& s, int32_t ref) {
    if (s.side < 0) *root = ref;
    else if (s.side == 0) bl[s.parent] = ref;
    else br[s.parent] = ref;
}
__device__ void emit_child(const Seg& c, const float* box, const int32_t* idx, int32_t* bl, int32_t* br,
                           int32_t* root, float* bbox, LevelOut out) {
    int32_t len = c.hi - c.lo;
    if (len == 1) { link(bl, br, root, c, -c.lo - 1); return; }
    if (len < SMALL) out.small[atomicAdd(out.n_small, 1)] = c;
    else out.next[atomicAdd(out.n_next, 1)] = c;
}

// one thread per large node: choose the split, write the bin keys' axis, the
// node box, and queue the two children
__global__ void k_split(const Seg* __restrict__ segs, int32_t nseg, const int32_t* __restrict__ st, int32_t* mids,
                        int32_t* axes, int32_t* bl, int32_t* br, int32_t* root, float* bbox) {
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
        const int32_t* g = st + (size_t)s * ST_WORDS;
        int bax;
        bool binned;
        int32_t span = segs[s].hi - segs[s].lo;
        int32_t mid = choose_split(g, span, &bax, &binned);
        mids[s] = segs[s].lo + mid;
        axes[s] = binned ? bax : -1;
        int32_t id = segs[s].lo + mid - 1;
        for (int w = 0; w < 6; w++) bbox[(size_t)id * 6 + w] = o2f(g[w]);
        link(bl, br, root, segs[s], id);
    }
}

__global__ void k_keys(const Seg* __restrict__ segs, const int32_t* __restrict__ chunk_seg,
                       const int32_t* __restrict__ chunk_lo, int32_t nchunks, const int32_t* __restrict__ idx,
                       const float* __restrict__ cen, const int32_t* __restrict__ st, const int32_t* __restrict__ axes,
                       uint8_t* keys) {
    for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        int32_t s = chunk_seg[c];
        int ax = axes[s];
        const int32_t* g = st + (size_t)s * ST_WORDS;
        float cmn = ax >= 0 ? o2f(g[6 + ax]) : 0.0f, ext = ax >= 0 ? o2f(g[9 + ax]) - cmn : 1.0f;
        int32_t lo = chunk_lo[c], hi = min(lo + CHUNK, segs[s].hi);
        for (int32_t k = lo + threadIdx.x; k < hi; k += blockDim.x)
            keys[k] = ax >= 0 ? (uint8_t)bin_of(cen[(size_t)idx[k] * 3 + ax], cmn, ext) : (uint8_t)0;
    }
}

__global__ void k_copy_back(const Seg* __restrict__ segs, const int32_t* __restrict__ chunk_seg,
                            const int32_t* __restrict__ chunk_lo, int32_t nchunks, const int32_t* __restrict__ from,
                            int32_t* to) {
    for (int32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        int32_t lo = chunk_lo[c], hi = min(lo + CHUNK, segs[chunk_seg[c]].hi);
        for (int32_t k = lo + threadIdx.x; k < hi; k += blockDim.x) to[k] = from[k];
    }
}

__global__ void k_children(const Seg* __restrict__ segs, int32_t nseg, const int32_t* __restrict__ mids,
                           const float* box, const int32_t* idx, int32_t* bl, int32_t* br, int32_t* root, float* bbox,
                           LevelOut out) {
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
        int32_t id = mids[s] - 1;
        emit_child(Seg{segs[s].lo, mids[s], id, 0}, box, idx, bl, br, root, bbox, out);
        emit_child(Seg{mids[s], segs[s].hi, id, 1}, box, idx, bl, br, root, bbox, out);
    }
}

// one thread finishes a small node: the sequential partition over its range,
// an explicit stack instead of recursion
__global__ void k_small(const Seg* __restrict__ segs, int32_t nseg, const float* __restrict__ box,
                        const float* __restrict__ cen, int32_t* idx, int32_t* tmp, uint8_t* bid, int32_t* bl,
                        int32_t* br, int32_t* root, float* bbox) {
    for (int32_t si = blockIdx.x * blockDim.x + threadIdx.x; si < nseg; si += gridDim.x * blockDim.x) {
        Seg stack[SMALL + 1];   // pending ranges are disjoint and non-empty: at most SMALL of them
        int sp = 0;
        stack[sp++] = segs[si];
        while (sp > 0) {
            Seg s = stack[--sp];
            int32_t lo = s.lo, hi = s.hi, span = hi - lo;
            if (span == 1) { link(bl, br, root, s, -lo - 1); continue; }
            float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
            float nb[6];
            for (int w = 0; w < 6; w++) nb[w] = box[(size_t)idx[lo] * 6 + w];
            for (int32_t k = lo; k < hi; k++) {
                int32_t o = idx[k];
                for (int a = 0; a < 3; a++) { cmn[a] = fminf(cmn[a], cen[(size_t)o * 3 + a]); cmx[a] = fmaxf(cmx[a], cen[(size_t)o * 3 + a]); }
                if (k > lo) unite6(nb, box + (size_t)o * 6);
            }
            float nsa = area6(nb);
            float best = INFINITY;
            int bax = 0, bsp = 0;
            for (int ax = 0; ax < 3; ax++) {
                float ext = cmx[ax] - cmn[ax];
                if (ext < 1e-6f) continue;
                bool has[NB];
                float bb[NB][6];
                uint32_t cnt[NB];
                for (int i = 0; i < NB; i++) { has[i] = false; cnt[i] = 0; }
                for (int32_t k = lo; k < hi; k++) {
                    int32_t o = idx[k];
                    int bi = bin_of(cen[(size_t)o * 3 + ax], cmn[ax], ext);
                    cnt[bi]++;
                    if (has[bi]) unite6(bb[bi], box + (size_t)o * 6);
                    else for (int w = 0; w < 6; w++) bb[bi][w] = box[(size_t)o * 6 + w];
                    has[bi] = true;
                }
                float lsa[NB];
                uint32_t ln[NB];
                bool ah = false;
                float acc[6];
                uint32_t an = 0;
                for (int i = 0; i < NB; i++) {
                    an += cnt[i];
                    if (has[i]) { if (ah) unite6(acc, bb[i]); else for (int w = 0; w < 6; w++) acc[w] = bb[i][w]; ah = true; }
                    ln[i] = an;
                    lsa[i] = ah ? area6(acc) : 0.0f;
                }
                ah = false;
                an = 0;
                for (int q = NB - 2; q >= 0; q--) {
                    an += cnt[q + 1];
                    if (has[q + 1]) { if (ah) unite6(acc, bb[q + 1]); else for (int w = 0; w < 6; w++) acc[w] = bb[q + 1][w]; ah = true; }
                    uint32_t nl = ln[q], nr = an;
                    if (nl == 0 || nr == 0) continue;
                    float rsa = ah ? area6(acc) : 0.0f;
                    float cost = 1.0f + (lsa[q] * (float)nl + rsa * (float)nr) / nsa;
                    if (cost < best) { best = cost; bax = ax; bsp = q; }
                }
            }
            float ext = cmx[bax] - cmn[bax];
            uint32_t cnt[NB];
            for (int i = 0; i < NB; i++) cnt[i] = 0;
            for (int32_t k = lo; k < hi; k++) {
                int bi = ext < 1e-6f ? 0 : bin_of(cen[(size_t)idx[k] * 3 + bax], cmn[bax], ext);
                bid[k] = (uint8_t)bi;
                cnt[bi]++;
            }
            uint32_t off[NB], run = 0;
            int32_t mid_off = 0;
            for (int b = 0; b < NB; b++) { off[b] = run; run += cnt[b]; if (b == bsp) mid_off = (int32_t)run; }
            for (int32_t k = lo; k < hi; k++) tmp[lo + off[bid[k]]++] = idx[k];
            for (int32_t k = lo; k < hi; k++) idx[k] = tmp[k];
            int32_t mid = lo + ((mid_off == 0 || mid_off == span) ? span / 2 : mid_off);
            int32_t id = mid - 1;
            for (int w = 0; w < 6; w++) bbox[(size_t)id * 6 + w] = nb[w];
            link(bl, br, root, s, id);
            stack[sp++] = Seg{mid, hi, id, 1};
            stack[sp++] = Seg{lo, mid, id, 0};
        }
    }
}

// ── the collapse to 8-wide nodes on the device ──────────────────────────────
// The host collapse (SahBuilder::collapse) builds a wide node from binary node
// b by opening the inner child of largest surface area (the first of equal
// ones) until 8 children (or only leaves) remain, and numbers the wide nodes
// in preorder, leaves in the order the preorder meets them.  Here: every
// binary node's opening is computed in parallel; the wide nodes are found
// level by level from the root; subtree node and leaf counts are summed
// bottom-up and the preorder indices handed down; then one thread per wide
// node writes it.

// kids of the wide node rooted at binary node b (≥ 0 binary node, < 0 leaf)
__global__ void k_wide_kids(const int32_t* __restrict__ bl, const int32_t* __restrict__ br,
                            const float* __restrict__ bbox, int32_t nn, int32_t* kids, int32_t* nk, int width) {
    for (int32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nn; b += gridDim.x * blockDim.x) {
        int32_t k[8];
        int n = 2;
        k[0] = bl[b]; k[1] = br[b];
        for (int c = 2; c < 8; c++) k[c] = 0;
        while (n < width) {
            int best = -1;
            float ba = -1.0f;
            for (int i = 0; i < n; i++)
                if (k[i] >= 0) { float a = area6(bbox + (size_t)k[i] * 6); if (a > ba) { ba = a; best = i; } }
            if (best < 0) break;
            int32_t o = k[best];
            k[best] = bl[o];
            k[n++] = br[o];
        }
        for (int c = 0; c < 8; c++) kids[(size_t)b * 8 + c] = k[c];
        nk[b] = n;
    }
}

__global__ void k_count_inner(const int32_t* __restrict__ lvl, int32_t m, const int32_t* __restrict__ kids,
                              const int32_t* __restrict__ nk, int32_t* cnt) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int32_t b = lvl[i], c = 0;
        for (int j = 0; j < nk[b]; j++) c += kids[(size_t)b * 8 + j] >= 0;
        cnt[i] = c;
    }
}
__global__ void k_next_level(const int32_t* __restrict__ lvl, int32_t m, const int32_t* __restrict__ kids,
                             const int32_t* __restrict__ nk, const int32_t* __restrict__ pos, int32_t* next) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int32_t b = lvl[i], o = pos[i];
        for (int j = 0; j < nk[b]; j++) {
            int32_t k = kids[(size_t)b * 8 + j];
            if (k >= 0) next[o++] = k;
        }
    }
}
// wide nodes (S) and leaves (L) in the wide subtree of every node of a level
__global__ void k_subtree_sizes(const int32_t* __restrict__ lvl, int32_t m, const int32_t* __restrict__ kids,
                                const int32_t* __restrict__ nk, int32_t* S, int32_t* L) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int32_t b = lvl[i], sn = 1, sl = 0;
        for (int j = 0; j < nk[b]; j++) {
            int32_t k = kids[(size_t)b * 8 + j];
            if (k >= 0) { sn += S[k]; sl += L[k]; } else sl += 1;
        }
        S[b] = sn;
        L[b] = sl;
    }
}
// preorder index (P) and first leaf slot (LB) of every inner kid of a level's nodes
__global__ void k_preorder(const int32_t* __restrict__ lvl, int32_t m, const int32_t* __restrict__ kids,
                           const int32_t* __restrict__ nk, const int32_t* __restrict__ S,
                           const int32_t* __restrict__ L, int32_t* P, int32_t* LB) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int32_t b = lvl[i], on = P[b] + 1, ol = LB[b];
        for (int j = 0; j < nk[b]; j++) {
            int32_t k = kids[(size_t)b * 8 + j];
            if (k >= 0) { P[k] = on; LB[k] = ol; on += S[k]; ol += L[k]; } else ol += 1;
        }
    }
}
// the node of every wide root: child boxes (empty slots inverted), inner
// children by preorder index, leaves for now as RT_LEAF_BIT | leaf slot
__global__ void k_write_nodes(const int32_t* __restrict__ order, int32_t m, const int32_t* __restrict__ kids,
                              const int32_t* __restrict__ nk, const int32_t* __restrict__ P,
                              const int32_t* __restrict__ LB, const int32_t* __restrict__ L, const float* __restrict__ bbox,
                              const float* __restrict__ box, const int32_t* __restrict__ idx, float4* nodes,
                              int32_t* export_ch, int32_t* leaf_gid) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int32_t b = order[i], me = P[b], ol = LB[b];
        float f[56];
        for (int c = 0; c < 8; c++) {
            int32_t k = c < nk[b] ? kids[(size_t)b * 8 + c] : INT32_MIN;
            uint32_t ref;
            int32_t ex;
            const float* cb = nullptr;
            if (c >= nk[b]) {
                ref = RT_EMPTY_REF; ex = INT32_MIN;
            } else if (k >= 0) {
                ref = (uint32_t)P[k]; ex = P[k]; cb = bbox + (size_t)k * 6;
                ol += L[k];                                  // the inner kid's leaves come first
            } else {
                int32_t slot = ol++, prim = idx[-k - 1];
                leaf_gid[slot] = prim;
                ref = RT_LEAF_BIT | (uint32_t)slot; ex = -(slot + 1); cb = box + (size_t)prim * 6;
            }
            for (int a = 0; a < 3; a++) {
                f[a * 8 + c] = cb ? cb[a] : INFINITY;
                f[24 + a * 8 + c] = cb ? cb[3 + a] : -INFINITY;
            }
            f[48 + c] = __uint_as_float(ref);
            export_ch[(size_t)me * 8 + c] = ex;
        }
        float4* out = nodes + (size_t)me * 14;
        for (int q = 0; q < 14; q++) out[q] = make_float4(f[q * 4], f[q * 4 + 1], f[q * 4 + 2], f[q * 4 + 3]);
    }
}
// 4-wide nodes (7 float4: lower x, y, z and upper x, y, z planes of the 4
// children, then their references).  The leaves keep the 8-wide tree's leaf
// order, in which the primitive records are stored: a leaf kid's reference is
// its primitive's typed slot there (inv8: primitive → 8-wide leaf slot).
__global__ void k_write_nodes4(const int32_t* __restrict__ order, int32_t m, const int32_t* __restrict__ kids,
                               const int32_t* __restrict__ nk, const int32_t* __restrict__ P,
                               const float* __restrict__ bbox, const float* __restrict__ box,
                               const int32_t* __restrict__ idx, const int32_t* __restrict__ inv8,
                               const int32_t* __restrict__ scans, int32_t n, int64_t e0, int64_t e1, int64_t e2,
                               float4* nodes4) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        int32_t b = order[i], me = P[b];
        float f[28];
        for (int c = 0; c < 4; c++) {
            int32_t k = c < nk[b] ? kids[(size_t)b * 8 + c] : INT32_MIN;
            uint32_t ref;
            const float* cb = nullptr;
            if (c >= nk[b]) {
                ref = RT_EMPTY_REF;
            } else if (k >= 0) {
                ref = (uint32_t)P[k]; cb = bbox + (size_t)k * 6;
            } else {
                int32_t prim = idx[-k - 1], slot = inv8[prim];
                uint32_t t = prim < e0 ? RT_PRIM_TRI : prim < e1 ? RT_PRIM_QUAD : prim < e2 ? RT_PRIM_SPHERE : RT_PRIM_CONVEX;
                ref = RT_LEAF_BIT | (t << 28) | (uint32_t)scans[(size_t)t * n + slot];
                cb = box + (size_t)prim * 6;
            }
            for (int a = 0; a < 3; a++) {
                f[a * 4 + c] = cb ? cb[a] : INFINITY;
                f[12 + a * 4 + c] = cb ? cb[3 + a] : -INFINITY;
            }
            f[24 + c] = __uint_as_float(ref);
        }
        float4* out = nodes4 + (size_t)me * 7;
        for (int q = 0; q < 7; q++) out[q] = make_float4(f[q * 4], f[q * 4 + 1], f[q * 4 + 2], f[q * 4 + 3]);
    }
}
__global__ void k_invert(const int32_t* __restrict__ leaf_gid, int32_t n, int32_t* inv) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) inv[leaf_gid[i]] = i;
}
// leaf type of every slot: one flag array per type for the typed-slot scans
__global__ void k_leaf_types(const int32_t* __restrict__ leaf_gid, int32_t n, int64_t e0, int64_t e1, int64_t e2,
                             int32_t* flags) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int64_t g = leaf_gid[i];
        int t = g < e0 ? RT_PRIM_TRI : g < e1 ? RT_PRIM_QUAD : g < e2 ? RT_PRIM_SPHERE : RT_PRIM_CONVEX;
        for (int k = 0; k < 4; k++) flags[(size_t)k * n + i] = t == k;
    }
}
// leaf references: type in bits 28-30, the slot among leaves of that type
__global__ void k_fix_leaf_refs(float4* nodes, int64_t n_nodes, const int32_t* __restrict__ leaf_gid, int32_t n,
                                int64_t e0, int64_t e1, int64_t e2, const int32_t* __restrict__ scans) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_nodes * 8; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t* ch = reinterpret_cast<uint32_t*>(nodes + (size_t)(i / 8) * 14 + 12) + (i % 8);
        uint32_t v = *ch;
        if (v == RT_EMPTY_REF || !(v & RT_LEAF_BIT)) continue;
        int32_t slot = (int32_t)(v & ~RT_LEAF_BIT);
        int64_t g = leaf_gid[slot];
        uint32_t t = g < e0 ? RT_PRIM_TRI : g < e1 ? RT_PRIM_QUAD : g < e2 ? RT_PRIM_SPHERE : RT_PRIM_CONVEX;
        *ch = RT_LEAF_BIT | (t << 28) | (uint32_t)scans[(size_t)t * n + slot];
    }
}
// the quantised copy of every node, as encode_qnode does on the host: the
// directed-rounding subtractions are the exact ones the host forms from
// TwoSum; a node whose extent needs a step beyond 2^60 sets *fail
__global__ void k_encode_qnodes(const float4* __restrict__ nodes, int64_t n_nodes, float4* qnodes, int* fail) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const float4* N = nodes + (size_t)i * 14;
        float f[56];
        for (int q = 0; q < 14; q++) { float4 v = N[q]; f[q * 4] = v.x; f[q * 4 + 1] = v.y; f[q * 4 + 2] = v.z; f[q * 4 + 3] = v.w; }
        uint32_t valid = 0;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int c = 0; c < 8; c++) {
            if (__float_as_uint(f[48 + c]) == RT_EMPTY_REF) continue;
            valid |= 1u << c;
            for (int a = 0; a < 3; a++) { lo[a] = fminf(lo[a], f[a * 8 + c]); hi[a] = fmaxf(hi[a], f[24 + a * 8 + c]); }
        }
        if (!valid) for (int a = 0; a < 3; a++) lo[a] = hi[a] = 0.0f;
        int e[3];
        bool flat[3];
        int e_any = -60;
        for (int a = 0; a < 3; a++) {
            float ext = __fsub_ru(hi[a], lo[a]);
            flat[a] = !(ext > 0.0f);
            if (flat[a]) continue;
            int ex;
            frexpf(ext / 255.0f, &ex);
            while (ex > -60 && ldexpf(255.0f, ex - 1) >= ext) ex--;
            while (ldexpf(255.0f, ex) < ext) ex++;
            e[a] = max(ex, -60);
            e_any = max(e_any, e[a]);
        }
        bool ok = true;
        for (int a = 0; a < 3; a++) {
            if (flat[a]) e[a] = e_any;
            if (e[a] > 60) ok = false;
        }
        if (!ok) { atomicExch(fail, 1); continue; }
        uint32_t w[3][4] = {};
        for (int a = 0; a < 3; a++) {
            float sa = ldexpf(1.0f, e[a]);
            for (int c = 0; c < 8; c++) {
                uint32_t ql = 255, qh = 0;
                if ((valid >> c) & 1u) {
                    float dl = __fsub_rd(f[a * 8 + c], lo[a]), dh = __fsub_ru(f[24 + a * 8 + c], lo[a]);
                    ql = (uint32_t)fminf(fmaxf(floorf(dl / sa), 0.0f), 255.0f);
                    qh = (uint32_t)fminf(fmaxf(ceilf(dh / sa), 0.0f), 255.0f);
                }
                w[a][c >> 2] |= ql << (8 * (c & 3));
                w[a][2 + (c >> 2)] |= qh << (8 * (c & 3));
            }
        }
        uint32_t meta = (uint32_t)(e[0] + 127) | (uint32_t)(e[1] + 127) << 8 | (uint32_t)(e[2] + 127) << 16 | valid << 24;
        float4* Q = qnodes + (size_t)i * 8;
        Q[0] = make_float4(lo[0], lo[1], lo[2], __uint_as_float(meta));
        for (int a = 0; a < 3; a++)
            Q[1 + a] = make_float4(__uint_as_float(w[a][0]), __uint_as_float(w[a][1]), __uint_as_float(w[a][2]),
                                   __uint_as_float(w[a][3]));
        Q[4] = N[12];
        Q[5] = N[13];
        Q[6] = Q[7] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

}  // namespace

namespace rth {

// the device collapse: bl / br / bbox / box / idx and root are the device
// arrays of the binary tree
static cudaError_t collapse_wide(const int32_t* bl, const int32_t* br, const float* bbox, const float* box,
                                 const int32_t* idx, int32_t root, int32_t n, int sms, cudaStream_t st, WideOut* W) {
    const int32_t nn = n - 1;
    int32_t *kids = nullptr, *nk = nullptr, *order = nullptr, *cnt = nullptr, *pos = nullptr;
    int32_t *S = nullptr, *L = nullptr, *P = nullptr, *LB = nullptr, *leaf_gid = nullptr, *flags = nullptr, *scans = nullptr;
    int* fail = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess && r != cudaSuccess) e = r; return e == cudaSuccess; };
    auto scan = [&](const int32_t* in, int32_t* out, int32_t m) {
        size_t need = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, need, in, out, m, st);
        if (need > tmp_bytes) {
            if (tmp) cudaFree(tmp);
            tmp = nullptr;
            if (!ok(cudaMalloc(&tmp, need))) return;
            tmp_bytes = need;
        }
        ok(cub::DeviceScan::ExclusiveSum(tmp, need, in, out, m, st));
    };
    ok(cudaMalloc(&kids, (size_t)nn * 8 * 4)); ok(cudaMalloc(&nk, (size_t)nn * 4));
    ok(cudaMalloc(&order, ((size_t)nn + 1) * 4)); ok(cudaMalloc(&cnt, ((size_t)nn + 1) * 4));
    ok(cudaMalloc(&pos, ((size_t)nn + 1) * 4));
    ok(cudaMalloc(&S, (size_t)nn * 4)); ok(cudaMalloc(&L, (size_t)nn * 4));
    ok(cudaMalloc(&P, (size_t)nn * 4)); ok(cudaMalloc(&LB, (size_t)nn * 4));
    ok(cudaMalloc(&leaf_gid, (size_t)n * 4)); ok(cudaMalloc(&flags, (size_t)n * 16)); ok(cudaMalloc(&scans, (size_t)n * 16));
    ok(cudaMalloc(&fail, 4));
    int grid = sms * 8;
    std::vector<int32_t> lvl_off;
    // the wide nodes of one width: each binary node's opening, the wide roots
    // level by level (in `order`), subtree sizes bottom-up and preorder indices
    // top-down; returns the node count (0 on an error) and the depth in *depth
    auto plan = [&](int width, int32_t* depth) -> int32_t {
        lvl_off.assign({0, 1});
        if (e != cudaSuccess) return 0;
        k_wide_kids<<<grid, 256, 0, st>>>(bl, br, bbox, nn, kids, nk, width);
        ok(cudaMemcpyAsync(order, &root, 4, cudaMemcpyHostToDevice, st));
        while (e == cudaSuccess) {
            int32_t off = lvl_off[lvl_off.size() - 2], m = lvl_off.back() - off;
            k_count_inner<<<std::max(1, std::min((m + 255) / 256, grid)), 256, 0, st>>>(order + off, m, kids, nk, cnt);
            scan(cnt, pos, m);
            int32_t tail[2] = {0, 0};
            ok(cudaMemcpyAsync(&tail[0], pos + m - 1, 4, cudaMemcpyDeviceToHost, st));
            ok(cudaMemcpyAsync(&tail[1], cnt + m - 1, 4, cudaMemcpyDeviceToHost, st));
            ok(cudaStreamSynchronize(st));
            int32_t nxt = tail[0] + tail[1];
            if (nxt == 0 || e != cudaSuccess) break;
            if (lvl_off.back() + nxt > nn) { e = cudaErrorUnknown; break; }
            k_next_level<<<std::max(1, std::min((m + 255) / 256, grid)), 256, 0, st>>>(order + off, m, kids, nk, pos,
                                                                                   order + lvl_off.back());
            lvl_off.push_back(lvl_off.back() + nxt);
        }
        const int nlev = (int)lvl_off.size() - 1;
        if (e != cudaSuccess) return 0;
        for (int l = nlev - 1; l >= 0; l--) {
            int32_t m = lvl_off[l + 1] - lvl_off[l];
            k_subtree_sizes<<<std::max(1, std::min((m + 255) / 256, grid)), 256, 0, st>>>(order + lvl_off[l], m, kids,
                                                                                       nk, S, L);
        }
        ok(cudaMemsetAsync(P + root, 0, 4, st));
        ok(cudaMemsetAsync(LB + root, 0, 4, st));
        for (int l = 0; l < nlev; l++) {
            int32_t m = lvl_off[l + 1] - lvl_off[l];
            k_preorder<<<std::max(1, std::min((m + 255) / 256, grid)), 256, 0, st>>>(order + lvl_off[l], m, kids, nk,
                                                                                  S, L, P, LB);
        }
        int32_t total = 0;
        ok(cudaMemcpyAsync(&total, S + root, 4, cudaMemcpyDeviceToHost, st));
        ok(cudaStreamSynchronize(st));
        if (e == cudaSuccess && total != lvl_off.back()) e = cudaErrorUnknown;   // every wide root counted once
        *depth = nlev - 1;
        return e == cudaSuccess ? total : 0;
    };
    if (e == cudaSuccess) W->n_nodes = plan(8, &W->max_depth);
    if (e == cudaSuccess) {
        ok(cudaMalloc(&W->nodes, (size_t)W->n_nodes * 14 * 16));
        ok(cudaMalloc(&W->qnodes, (size_t)W->n_nodes * 8 * 16));
        ok(cudaMalloc(&W->export_ch, (size_t)W->n_nodes * 8 * 4));
    }
    if (e == cudaSuccess) {
        int32_t m = lvl_off.back();
        k_write_nodes<<<std::max(1, std::min((m + 127) / 128, grid)), 128, 0, st>>>(
            order, m, kids, nk, P, LB, L, bbox, box, idx, W->nodes, W->export_ch, leaf_gid);
        k_leaf_types<<<grid, 256, 0, st>>>(leaf_gid, n, W->type_end[0], W->type_end[1], W->type_end[2], flags);
        for (int t = 0; t < 4; t++) scan(flags + (size_t)t * n, scans + (size_t)t * n, n);
        k_fix_leaf_refs<<<grid, 256, 0, st>>>(W->nodes, W->n_nodes, leaf_gid, n, W->type_end[0], W->type_end[1],
                                             W->type_end[2], scans);
        ok(cudaMemsetAsync(fail, 0, 4, st));
        k_encode_qnodes<<<grid, 128, 0, st>>>(W->nodes, W->n_nodes, W->qnodes, fail);
        int hfail = 0;
        ok(cudaMemcpyAsync(W->leaf_gids_h, leaf_gid, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
        ok(cudaMemcpyAsync(&hfail, fail, 4, cudaMemcpyDeviceToHost, st));
        ok(cudaStreamSynchronize(st));
        ok(cudaGetLastError());
        if (e == cudaSuccess && hfail) { cudaFree(W->qnodes); W->qnodes = nullptr; }
    }
    // the 4-wide tree over the same binary tree (RT_NODES_WIDE4), its leaves
    // referring to the primitive records in the 8-wide leaf order
    if (e == cudaSuccess) {
        int32_t* inv8 = cnt;                         // n + 1 ≥ n entries, free now
        W->n_nodes4 = plan(4, &W->max_depth4);
        if (e == cudaSuccess) ok(cudaMalloc(&W->nodes4, (size_t)W->n_nodes4 * 7 * 16));
        if (e == cudaSuccess) {
            k_invert<<<grid, 256, 0, st>>>(leaf_gid, n, inv8);
            int32_t m = lvl_off.back();
            k_write_nodes4<<<std::max(1, std::min((m + 127) / 128, grid)), 128, 0, st>>>(
                order, m, kids, nk, P, bbox, box, idx, inv8, scans, n, W->type_end[0], W->type_end[1], W->type_end[2],
                W->nodes4);
            ok(cudaStreamSynchronize(st));
            ok(cudaGetLastError());
        }
    }
    void* all[] = {kids, nk, order, cnt, pos, S, L, P, LB, leaf_gid, flags, scans, fail, tmp};
    for (void* p : all) if (p) cudaFree(p);
    if (e != cudaSuccess) {
        void* outs[] = {W->nodes, W->qnodes, W->export_ch, W->nodes4};
        for (void* p : outs) if (p) cudaFree(p);
        W->nodes = W->qnodes = W->nodes4 = nullptr;
        W->export_ch = nullptr;
    }
    return e;
}

// Build the binary SAH tree of n primitive boxes (host, 6 floats each) on the
// device; idx (n), bl / br (n − 1 child refs: ≥ 0 node, < 0 leaf −(pos + 1))
// and bbox ((n − 1) × 6) are written on the host.  Returns 0 or a CUDA error.
int gpu_build_binary(const float* boxes_h, int32_t n, int32_t* idx_h, int32_t* bl_h, int32_t* br_h, float* bbox_h,
                     int32_t* root_h, int sms, cudaStream_t st, WideOut* wide) {
    float *box = nullptr, *cen = nullptr, *bbox = nullptr;
    int32_t *idx = nullptr, *tmp = nullptr, *bl = nullptr, *br = nullptr, *root = nullptr, *cnt = nullptr;
    int32_t *stats = nullptr, *mids = nullptr, *axes = nullptr, *chunk_seg = nullptr, *chunk_lo = nullptr;
    uint8_t *keys = nullptr, *keys2 = nullptr;
    Seg *cur = nullptr, *nxt = nullptr, *small = nullptr;
    int32_t *beg = nullptr, *end = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int32_t nn = std::max(n - 1, 1);
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess && r != cudaSuccess) e = r; return e == cudaSuccess; };
    size_t max_chunks = (size_t)n / CHUNK + (size_t)n / SMALL + 2;
    size_t max_segs = (size_t)n / SMALL + 2;
    ok(cudaMalloc(&box, (size_t)n * 24)); ok(cudaMalloc(&cen, (size_t)n * 12)); ok(cudaMalloc(&bbox, (size_t)nn * 24));
    ok(cudaMalloc(&idx, (size_t)n * 4)); ok(cudaMalloc(&tmp, (size_t)n * 4));
    ok(cudaMalloc(&bl, (size_t)nn * 4)); ok(cudaMalloc(&br, (size_t)nn * 4)); ok(cudaMalloc(&root, 4));
    ok(cudaMalloc(&cnt, 8)); ok(cudaMalloc(&keys, (size_t)n)); ok(cudaMalloc(&keys2, (size_t)n));
    ok(cudaMalloc(&stats, max_segs * ST_WORDS * 4)); ok(cudaMalloc(&mids, max_segs * 4)); ok(cudaMalloc(&axes, max_segs * 4));
    ok(cudaMalloc(&chunk_seg, max_chunks * 4)); ok(cudaMalloc(&chunk_lo, max_chunks * 4));
    ok(cudaMalloc(&cur, max_segs * sizeof(Seg))); ok(cudaMalloc(&nxt, max_segs * sizeof(Seg)));
    ok(cudaMalloc(&small, ((size_t)n / 2 + 2) * sizeof(Seg)));
    ok(cudaMalloc(&beg, max_segs * 4)); ok(cudaMalloc(&end, max_segs * 4));
    if (e == cudaSuccess) {
        ok(cudaMemcpyAsync(box, boxes_h, (size_t)n * 24, cudaMemcpyHostToDevice, st));
        k_centroids<<<sms * 8, 256, 0, st>>>(box, n, cen, idx);
        ok(cudaMemsetAsync(cnt, 0, 8, st));
        ok(cudaMemsetAsync(root, 0, 4, st));
    }
    // the root: large, small or a single leaf
    std::vector<Seg> level;
    int32_t n_small = 0;
    Seg r0{0, n, -1, -1};
    if (n == 1) {
        int32_t leaf = -1;
        ok(cudaMemcpyAsync(root, &leaf, 4, cudaMemcpyHostToDevice, st));
    } else if (n < SMALL) {
        ok(cudaMemcpyAsync(small, &r0, sizeof(Seg), cudaMemcpyHostToDevice, st));
        n_small = 1;
    } else {
        level.push_back(r0);
    }
    std::vector<int32_t> cs, cl, bh, eh;
    while (e == cudaSuccess && !level.empty()) {
        int32_t ns = (int32_t)level.size();
        cs.clear(); cl.clear(); bh.clear(); eh.clear();
        for (int32_t s = 0; s < ns; s++) {
            for (int32_t lo = level[s].lo; lo < level[s].hi; lo += CHUNK) { cs.push_back(s); cl.push_back(lo); }
            bh.push_back(level[s].lo); eh.push_back(level[s].hi);
        }
        int32_t nch = (int32_t)cs.size();
        ok(cudaMemcpyAsync(cur, level.data(), ns * sizeof(Seg), cudaMemcpyHostToDevice, st));
        ok(cudaMemcpyAsync(chunk_seg, cs.data(), nch * 4, cudaMemcpyHostToDevice, st));
        ok(cudaMemcpyAsync(chunk_lo, cl.data(), nch * 4, cudaMemcpyHostToDevice, st));
        ok(cudaMemcpyAsync(beg, bh.data(), ns * 4, cudaMemcpyHostToDevice, st));
        ok(cudaMemcpyAsync(end, eh.data(), ns * 4, cudaMemcpyHostToDevice, st));
        int grid = std::min(nch, sms * 16);
        k_stats_init<<<std::min((ns * ST_WORDS + 255) / 256, sms * 8), 256, 0, st>>>(stats, ns);
        k_stats_bounds<<<grid, 256, 0, st>>>(cur, chunk_seg, chunk_lo, nch, idx, box, cen, stats);
        k_stats_bins<<<grid, 256, 0, st>>>(cur, chunk_seg, chunk_lo, nch, idx, box, cen, stats);
        k_split<<<(ns + 127) / 128, 128, 0, st>>>(cur, ns, stats, mids, axes, bl, br, root, bbox);
        k_keys<<<grid, 256, 0, st>>>(cur, chunk_seg, chunk_lo, nch, idx, cen, stats, axes, keys);
        // stable sort of every large node's primitives by bin (the counting sort)
        size_t need = 0;
        cub::DeviceSegmentedRadixSort::SortPairs(nullptr, need, keys, keys2, idx, tmp, n, ns, beg, end, 0, 4, st);
        if (need > cub_bytes) {
            if (cub_tmp) cudaFree(cub_tmp);
            cub_tmp = nullptr;
            if (!ok(cudaMalloc(&cub_tmp, need))) break;
            cub_bytes = need;
        }
        ok(cub::DeviceSegmentedRadixSort::SortPairs(cub_tmp, need, keys, keys2, idx, tmp, n, ns, beg, end, 0, 4, st));
        k_copy_back<<<grid, 256, 0, st>>>(cur, chunk_seg, chunk_lo, nch, tmp, idx);
        ok(cudaMemsetAsync(cnt, 0, 4, st));
        LevelOut out{nxt, cnt, small + n_small, cnt + 1};
        k_children<<<(ns + 127) / 128, 128, 0, st>>>(cur, ns, mids, box, idx, bl, br, root, bbox, out);
        int32_t counts[2];
        ok(cudaMemcpyAsync(counts, cnt, 8, cudaMemcpyDeviceToHost, st));
        ok(cudaStreamSynchronize(st));
        ok(cudaMemsetAsync(cnt + 1, 0, 4, st));
        n_small += counts[1];
        level.resize(counts[0]);
        if (counts[0]) ok(cudaMemcpyAsync(level.data(), nxt, counts[0] * sizeof(Seg), cudaMemcpyDeviceToHost, st));
        ok(cudaStreamSynchronize(st));
    }
    if (e == cudaSuccess && n_small > 0)
        k_small<<<(n_small + 63) / 64, 64, 0, st>>>(small, n_small, box, cen, idx, tmp, keys, bl, br, root, bbox);
    ok(cudaGetLastError());
    if (e == cudaSuccess && wide) {
        // the collapse on the device; the host gets the leaf order, not the tree
        int32_t rt = 0;
        ok(cudaMemcpyAsync(&rt, root, 4, cudaMemcpyDeviceToHost, st));
        ok(cudaStreamSynchronize(st));
        if (e == cudaSuccess) {
            if (rt < 0 || n < 2) e = cudaErrorInvalidValue;       // one primitive: the host builds that node
            else ok(collapse_wide(bl, br, bbox, box, idx, rt, n, sms, st, wide));
        }
        if (root_h) *root_h = rt;
    } else if (e == cudaSuccess) {
        ok(cudaMemcpyAsync(idx_h, idx, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
        if (n > 1) {
            ok(cudaMemcpyAsync(bl_h, bl, (size_t)(n - 1) * 4, cudaMemcpyDeviceToHost, st));
            ok(cudaMemcpyAsync(br_h, br, (size_t)(n - 1) * 4, cudaMemcpyDeviceToHost, st));
            ok(cudaMemcpyAsync(bbox_h, bbox, (size_t)(n - 1) * 24, cudaMemcpyDeviceToHost, st));
        }
        ok(cudaMemcpyAsync(root_h, root, 4, cudaMemcpyDeviceToHost, st));
        ok(cudaStreamSynchronize(st));
    }
    void* all[] = {box, cen, bbox, idx, tmp, bl, br, root, cnt, keys, keys2, stats, mids, axes, chunk_seg, chunk_lo,
                   cur, nxt, small, beg, end, cub_tmp};
    for (void* p : all) if (p) cudaFree(p);
    return (int)e;
}

}  // namespace rth
