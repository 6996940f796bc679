// rt_internal.h — declarations shared by the CUDA translation units of
// librtb200.so (not part of the public ABI; that is include/rt_api.h).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rt_api.h"
#include "rt_device.cuh"
#include "rt_guide.cuh"

#define RT_TRACE_BLOCK 128
#define RT_TRACE_BLOCKS_PER_SM 8
// resident blocks per SM of the persistent traversal kernels (their launch
// bound and the most blocks per SM a traversal grid has): 6 blocks of 128
// threads cap the kernels at 80 registers (measured faster than 5 blocks at
// 96 registers and than 8 blocks at 64)
#ifndef RT_TRACE_MINB
#define RT_TRACE_MINB 6
#endif
// the traversal stack's ring in local memory (1) or shared memory (0): a
// shared ring reserves 8 KB per block of the SM's L1 / shared storage, and the
// node fetches lose more to the smaller L1 than the stack gains (measured on
// the icosphere workload: extend 67.5 ms shared, 62.8 ms local)
#ifndef RT_STACK_LOCAL
#define RT_STACK_LOCAL 1
#endif
// traversal stack: RT_SHORT_STACK entries per thread in a ring (local or
// shared memory), deeper entries spilled to a per-thread column of global memory
// sized from the tree depth at scene creation (7 per level: a visit pushes
// at most 7 of its 8 children), so a traversal never runs out of stack
#define RT_SHORT_STACK 16
#define RT_SHADE_BLOCK 128
#define RT_SHADE_BLOCKS_PER_SM 8
#define RT_MAX_DEPTH 256
// samples of one rt_render_batch pass, in path pools, when the passes replay
// the captured wavefront graph (the chain it captures grows with it)
#ifndef RT_RAY_BINS
#define RT_RAY_BINS 0
#endif
#define RT_BIN_CELLS 4
#define RT_NBINS (8 * RT_BIN_CELLS * RT_BIN_CELLS * RT_BIN_CELLS)
#ifndef RT_GRAPH_PASS_POOLS
#define RT_GRAPH_PASS_POOLS 32
#endif

// Counter block of one wavefront iteration (RT_CTR_STRIDE uint32): ray count,
// fetch cursors of the persistent kernels, shadow-ray count, per-material-class
// path counts and cursors, photon-gather requests and retired paths.
#define RT_CTR_STRIDE 32
#define CTR_COUNT          0
#define CTR_EXTEND_NEXT    1
#define CTR_SHADOW_COUNT   3
#define CTR_SHADOW_NEXT    4
#define CTR_CLS_COUNT      5   // CLS_N entries
#define CTR_GATHER_COUNT   15  // photon-gather requests of the iteration
#define CTR_RETIRE_COUNT   16  // paths that ended in the iteration

// Render counters: a header of 64-bit totals, then a ring of RT_CTR_RING
// iteration blocks (iteration it uses block it % RT_CTR_RING; the retire
// kernel of iteration it clears block it + 2, whose last user, it − 2, is done).
#define RT_CTR_RING        4
#define CTR_HDR_WORDS      32
#define HDR_GEN            0   // u64: next sample index to generate
#define HDR_EXT            2   // u64: extension rays traced
#define HDR_SHADOW         4   // u64: shadow rays traced
#define RT_CTR_WORDS       512 // allocation (the photon build uses 14 blocks)
static_assert(CTR_HDR_WORDS + RT_CTR_RING * RT_CTR_STRIDE <= RT_CTR_WORDS, "counter layout");
static_assert(14 * RT_CTR_STRIDE <= RT_CTR_WORDS, "photon counter layout");

// material classes shaded by separate kernels
enum { CLS_MISS = 0, CLS_EMIT = 1, CLS_DIFFUSE = 2, CLS_METAL = 3, CLS_DIELEC = 4, CLS_PBR = 5, CLS_MEDIUM = 6, CLS_N = 7 };
struct ClassQueues { uint32_t* q[CLS_N]; };
static_assert(CTR_CLS_COUNT + CLS_N <= CTR_GATHER_COUNT, "counter slots");

// Streams the shading kernels of one iteration fan out to.  The class kernels
// read disjoint class queues and append to the shared queues (next set, retire
// records, shadow and gather requests) by atomic reservation, so they may run
// at the same time: `fork` is recorded after classification and every class
// but the diffuse one waits on it from a side stream of its own; each `join`
// orders the launching stream after its class before the shadow rays.
struct ShadeFork {
    static constexpr int N = CLS_N - 1;
    cudaStream_t side[N];
    cudaEvent_t fork;
    cudaEvent_t join[N];
};

// Per-path wavefront state, structure of arrays.  The render loop keeps two
// dense sets (iteration it reads set it&1 at positions 0..count−1 and writes
// the paths that go on, compacted, into the other set), plus a set of
// retire records for the paths that ended (L, pend*, meta only).  `hit` and
// `gq` are shared by the sets.
struct PathState {
    float4* ray_o;     // origin xyz
    float4* ray_d;     // direction xyz
    float4* hit;       // (leaf ref bits, t, b1, b2) written by extend
    float4* thr;       // throughput T.rgb, prev_mis_w_brdf
    float4* wts;       // per-wavelength weights w0..w3
    uint4*  meta;      // pixel, sample slot, flags, lam0 bits
    float4* L;         // accumulated radiance rgb
    float4* pend0;     // parked area-light NEE contribution (cancelled if occluded)
    float4* pend1;     // parked env-map NEE contribution
    float4* pendC;     // parked caustic (photon-map) contribution, folded before pend0/pend1
    float4* gq;        // photon-gather requests of the bounce: (p, pid) (n, -)
    uint32_t* rec;     // newest guide training record of the path (guide training only)
};

// Where a contribution parked this iteration lives, for the shadow and gather
// kernels: target tag = index << 2 | retired << 1 | (1 for the env-NEE slot).
struct PendTargets {
    float4* pend[4];    // [retired * 2 + which]: pend0 / pend1 of the next set, then of the retire records
    float4* pendC[2];   // [retired]
};
#define PT_RETIRED 2u

// meta.z flag layout
#define PF_DEPTH_MASK   0xFFu
#define PF_PREV_SPEC    (1u << 8)
#define PF_TINT_SHIFT   9
#define PF_TINT_MASK    (3u << 9)
#define PF_SEC_ALIVE    (1u << 11)
#define PF_REC_OPEN     (1u << 12)   // the newest guide record waits for its base radiance

namespace rtph { struct Map; }

// Uniform cell grid over the photons' box: cubic cells of at least twice the
// gather radius (so a gather ball meets at most 2 cells per axis), at most
// 1024 per axis and RT_PH_GRID_MAX_CELLS in all.
#define RT_PH_GRID_MAX_CELLS (1u << 22)
struct PhotonGrid {
    float lo[3];
    float inv;           // 1 / cell size
    int n[3];            // cells per axis (1 × 1 × 1 when the map has no grid)
    float r2;            // the squared radius the grid serves (< 0: none)
};

// Device photon map: photons sorted by (grid cell, Morton code) — every cell a
// contiguous run — with the [start, end) table of the cells, a box heap over
// 32-photon leaves of the same order, and an emission-order copy.  Its arrays
// and the build's work buffers grow on demand and are kept across builds, so a
// rebuild of a map no larger than before allocates and frees nothing
// (release() only drops the map).
struct PhotonMapDev {
    float4 *pos = nullptr, *pow = nullptr, *nor = nullptr, *blo = nullptr, *bhi = nullptr;
    float4 *exp_pos = nullptr, *exp_pow = nullptr, *exp_nor = nullptr;
    uint32_t n = 0, nleaf_pow2 = 1, knn_k = 0;
    float r2 = 0.0f;
    bool present = false;
    uint64_t generation = 0;                                  // bumped by every build, set and release
    PhotonGrid grid{{0.f, 0.f, 0.f}, 0.f, {1, 1, 1}, -1.f};
    uint2* cells = nullptr;                                   // [start, end) per grid cell
    // capacities (elements) of the map arrays, the heap, the cell table and the build's work buffers
    size_t cap_map = 0, cap_heap = 0, cap_cells = 0, cap_work = 0, cap_tmp = 0;
    uint8_t* flags = nullptr;                                 // stored flag per traced photon
    float4 *st_pos = nullptr, *st_pow = nullptr, *st_nor = nullptr;   // stored record per traced photon
    uint32_t *fl32 = nullptr, *scan = nullptr;                // compaction
    uint64_t *key = nullptr, *key2 = nullptr;                 // sort keys: cell code << 30 | Morton code
    uint32_t *val = nullptr, *val2 = nullptr;
    float* bounds = nullptr;
    void* tmp = nullptr;                                      // CUB temporary storage
    ~PhotonMapDev();
    void release();
    void free_all();
    rtph::Map view() const;
};

// One request of a packed batch pass: its camera and frame, the samples of
// this pass (sample_idx .. sample_idx + nsamp − 1 of every pixel), where they
// start in the pass's sample cursor, and where they are written.
struct JobDev {
    RtCamera cam;
    uint32_t width, height, npix, strata, sample_idx, nsamp;
    uint64_t first;            // first cursor value of this request
    uint64_t seed;
    float*   scratch;          // nsamp × npix × 3, slot-major
};
#define PF_JOB_SHIFT 16        // meta.z bits 16-31: the request of a packed batch path

// One sample group of a render call: samples sample_idx .. sample_idx+nsamp−1
// of every active pixel, traced by a pool of paths that is refilled with new
// samples as paths end (sample g ↦ slot k = g / nactive, pixel active[g % nactive]).
struct RenderLaunch {
    uint32_t width, height, npix, nsamp;
    uint32_t sample_idx, strata, max_depth, hero;
    float    bg_scale;
    uint64_t seed;
    RtCamera cam;
    const uint32_t* active;                // active pixel list (device), or null: every pixel
    uint32_t nactive;
    uint64_t total;                        // nsamp × nactive samples to trace
    unsigned long long* gen_next;          // device cursor over [0, total)
    float*   scratch;                      // nsamp × npix × 3 (device), slot-major
    int      photons;                      // a photon map feeds the diffuse vertices
    rtg::GuideDev guide;                   // learned proposal at diffuse vertices (mode 0: off)
    // packed batch (n_jobs > 0): the requests, ascending in `first`; the cursor
    // runs over all of them and width / height / cam / scratch above are unused
    const JobDev* jobs;
    uint32_t n_jobs;
    // the device copy of this struct, which the kernels read (uploaded once per
    // call, so a captured graph of the call's launches serves every call)
    const RenderLaunch* dev;
    uint64_t max_it;                       // the call's wavefront iteration bound
    uint32_t pool;                         // paths of the pool's first fill (read on the device, so a
                                           // captured graph serves calls of any pool size)
};

namespace rth {
void launch_trace_closest_api(const rtd::DevScene& S, const float* rays, uint32_t n, int4* out, uint32_t* next,
                              int* err, int sms, cudaStream_t st);
void launch_trace_any_api(const rtd::DevScene& S, const float* rays, uint32_t n, uint8_t* out, uint32_t* next,
                          int* err, int sms, cudaStream_t st);
// media events after the closest hit: queue = NULL for the dense path set
// (wavelength in meta.w), else queued photons (wavelength in ray_d.w)
void launch_media(const rtd::DevScene& S, const PathState& P, const uint32_t* queue, const uint32_t* count, int sms,
                  cudaStream_t st);
void launch_media_api(const rtd::DevScene& S, const float* rays, uint32_t n, int4* out, int32_t n_prims,
                      int fill_miss, int sms, cudaStream_t st);
void launch_transmittance_api(const rtd::DevScene& S, const float* rays, uint32_t n, const uint8_t* occ, float* out,
                              int sms, cudaStream_t st);
void launch_extend(const rtd::DevScene& S, const PathState& P, const uint32_t* queue, const uint32_t* count,
                   uint32_t* next, int* err, int sms, cudaStream_t st);
void launch_shadow(const rtd::DevScene& S, const PendTargets& T, const float4* sq, const uint32_t* count,
                   uint32_t* next, int* err, int sms, cudaStream_t st);

// ray binning before extend (RT_RAY_BINS): a counting sort of set A's rays
// by direction octant and an RT_BIN_CELLS³ cell of the origin in the box
// (lo, lo + RT_BIN_CELLS / scale); `out` receives the path positions in bin
// order, `bins` holds 2 × RT_NBINS words of scratch (cleared here)
void launch_bin_rays(const PathState& A, const uint32_t* count, uint32_t capacity, float3 lo, float3 scale,
                     uint32_t* bins, uint32_t* out, cudaStream_t st);
// first fill of the path pool: samples 0 .. R.pool−1 into positions 0 .. R.pool−1 of set A
// (R.pool read on the device; `capacity` ≥ R.pool only sizes the grid)
void launch_generate(const rtd::DevScene& S, const PathState& A, const RenderLaunch& R, uint32_t capacity,
                     uint32_t* count0, cudaStream_t st);
// classify + one shading kernel per material class: paths that go on are
// compacted into B (count `cout`), ended paths into the retire records Rt
// (side by side on the streams of `fk` when it is given, else in turn on `st`)
void launch_shade(const rtd::DevScene& S, const PathState& A, const PathState& B, const PathState& Rt,
                  const RenderLaunch& R, uint32_t* ctr, const ClassQueues& Q, uint32_t* cout, float4* sq, int sms,
                  cudaStream_t st, const ShadeFork* fk = nullptr);
// write the ended paths' samples and append new samples, one per ended path
// while samples remain, to B; add the iteration's ray counts to the header;
// clear the counter block of iteration it + 2
void launch_retire(const rtd::DevScene& S, const PathState& B, const PathState& Rt, const RenderLaunch& R,
                   uint32_t* ctr, uint32_t* hdr, uint32_t* clear_block, uint32_t* cout, int sms, cudaStream_t st);
// active-pixel list of a converged mask, and zero output for converged pixels
void launch_active_list(const uint8_t* conv, uint32_t width, uint32_t height, uint32_t* list, uint32_t* count,
                        cudaStream_t st);
void launch_zero_converged(const uint8_t* conv, uint32_t npix, uint32_t nsamp, float* scratch, cudaStream_t st);

// traces photons first .. first + count − 1 of the emission order (the emitters'
// photons one after the other) and builds the map of those stored
cudaError_t photon_build(const rtd::DevScene& S, PhotonMapDev& map, const PathState& P, uint32_t* qa, uint32_t* qb,
                         uint32_t* counters, const RtPhotonParams& prm, const float* emit_setup, uint32_t first,
                         uint32_t count, int sms, cudaStream_t st, int64_t* n_stored, float stage_ms[3]);
cudaError_t photon_set(PhotonMapDev& map, const float4* pos, const float4* pow, const float4* nor, uint32_t n,
                       float radius, uint32_t k, cudaStream_t st);
void launch_photon_gather_api(const PhotonMapDev& map, const float* q, uint32_t n, float* out, int sms, cudaStream_t st);
void launch_knn_api(const PhotonMapDev& map, const float* q, uint32_t n, int k, float rmax2, int* idx, float* d2,
                    int* err, int sms, cudaStream_t st);
void launch_photon_gather_paths(const PhotonMapDev& map, const PendTargets& T, const float4* gq, const uint32_t* count,
                                int sms, cudaStream_t st);
void launch_accumulate(const float* scratch, uint32_t nsamp, uint32_t npix, float* acc, float* m2, uint32_t* cnt,
                       const uint8_t* conv, float clamp, uint32_t min_samples, float floor_, cudaStream_t st);
// The 8-wide tree collapsed on the device from the binary tree (the host
// collapse's greedy rule and preorder numbering): full and quantised node
// arrays in device memory (the caller owns them), the leaf order, the node
// count and depth, and per node the children in the reference's export form
// (≥ 0 node, −(leaf slot + 1), INT32_MIN empty) for rt_scene_bvh_export.
struct WideOut {
    int64_t type_end[3];          // canonical ids below [0] are triangles, below [1] quads, below [2] spheres
    float4* nodes = nullptr;      // 14 float4 per node
    float4* qnodes = nullptr;     // 8 float4 per node (null when an extent is beyond the quantised range)
    int32_t* export_ch = nullptr; // 8 per node
    int64_t n_nodes = 0;
    int32_t max_depth = 0;
    int32_t* leaf_gids_h = nullptr;   // host, n entries
    float4* nodes4 = nullptr;     // 4-wide nodes of the same binary tree, 7 float4 per node
    int64_t n_nodes4 = 0;
    int32_t max_depth4 = 0;
};
// binary tree on the device, then (wide == null) its arrays copied to the host
// or (wide != null) the device collapse into *wide
int gpu_build_binary(const float* boxes_h, int32_t n, int32_t* idx_h, int32_t* bl_h, int32_t* br_h, float* bbox_h,
                     int32_t* root_h, int sms, cudaStream_t st, WideOut* wide = nullptr);
// guide mixture of every path in the diffuse queue (before its shading kernel)
void launch_guide_infer(const rtd::DevScene& S, const PathState& A, const RenderLaunch& R, const uint32_t* queue,
                        const uint32_t* count, int sms, cudaStream_t st);
void launch_develop(const float* lin, const float* sum, const uint32_t* cnt, uint32_t w, uint32_t h, float exposure,
                    int tm, float vignette, float distortion, uint8_t* out, int sms, cudaStream_t st);
}  // namespace rth

// host state of the path-guiding network (rt_guide.cu)
#include <string>
namespace rtgh {
struct Guide;
Guide* create(const RtGuideParams& p, const float scene_lo[3], const float scene_hi[3], std::string* err);
void destroy(Guide* g);
void set_mode(Guide* g, int mode);
int mode(const Guide* g);
rtg::GuideDev view(const Guide* g);
int ensure_paths(Guide* g, uint32_t cap);
cudaError_t params_io(Guide* g, float* host, int write, cudaStream_t st);
void eval(Guide* g, const float* q, uint32_t n, const float* dirs, const float* u, float* raw, float* out, int sms,
          cudaStream_t st);
cudaError_t train_explicit(Guide* g, const float4* samples, uint32_t n, int steps, float* loss_host, int sms,
                           cudaStream_t st);
cudaError_t grad_out(Guide* g, float* host, cudaStream_t st);
cudaError_t begin_pass(Guide* g, cudaStream_t st);
cudaError_t train_pass(Guide* g, int sms, cudaStream_t st, int64_t* launches);
void stats(const Guide* g, int64_t* records, int64_t* samples, int64_t* steps, double* ms);
}  // namespace rtgh
