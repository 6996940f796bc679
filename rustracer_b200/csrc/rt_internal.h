// rt_internal.h — declarations shared by the CUDA translation units of
// librtb200.so (not part of the public ABI; that is include/rt_api.h).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rt_api.h"
#include "rt_device.cuh"

#define RT_TRACE_BLOCK 128
#define RT_TRACE_BLOCKS_PER_SM 8
#define RT_SHADE_BLOCK 128
#define RT_SHADE_BLOCKS_PER_SM 8
#define RT_MAX_DEPTH 256

// Counter block of one bounce (RT_CTR_STRIDE uint32 per bounce): ray count,
// fetch cursors of the persistent kernels, shadow-ray count, and per-material-
// class path counts and cursors.
#define RT_CTR_STRIDE 16
#define CTR_COUNT          0
#define CTR_EXTEND_NEXT    1
#define CTR_CLASSIFY_NEXT  2
#define CTR_SHADOW_COUNT   3
#define CTR_SHADOW_NEXT    4
#define CTR_CLS_COUNT      5   // 5 entries
#define CTR_CLS_NEXT       10  // 5 entries
#define CTR_GATHER_COUNT   15  // photon-gather requests of the bounce

// material classes shaded by separate kernels
enum { CLS_MISS = 0, CLS_EMIT = 1, CLS_DIFFUSE = 2, CLS_METAL = 3, CLS_DIELEC = 4, CLS_N = 5 };
struct ClassQueues { uint32_t* q[CLS_N]; };

// Per-path wavefront state, structure of arrays, indexed by path id.
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
};

// meta.z flag layout
#define PF_DEPTH_MASK   0xFFu
#define PF_PREV_SPEC    (1u << 8)
#define PF_TINT_SHIFT   9
#define PF_TINT_MASK    (3u << 9)
#define PF_SEC_ALIVE    (1u << 11)

namespace rtph { struct Map; }

// Device photon map: Morton-ordered photons, box heap, and an emission-order copy.
struct PhotonMapDev {
    float4 *pos = nullptr, *pow = nullptr, *nor = nullptr, *blo = nullptr, *bhi = nullptr;
    float4 *exp_pos = nullptr, *exp_pow = nullptr, *exp_nor = nullptr;
    uint32_t n = 0, nleaf_pow2 = 1, knn_k = 0;
    float r2 = 0.0f;
    bool present = false;
    ~PhotonMapDev();
    void release();
    rtph::Map view() const;
};

struct RenderLaunch {
    uint32_t width, height, npix, nsamp;   // this chunk: nsamp consecutive samples
    uint32_t sample_idx, strata, max_depth, hero;
    float    bg_scale;
    uint64_t seed;
    RtCamera cam;
    const uint8_t* converged;              // device, nullable
    float*   scratch;                      // nsamp × npix × 3 (device)
    int      photons;                      // a photon map feeds the diffuse vertices
};

namespace rth {
void launch_trace_closest_api(const rtd::DevScene& S, const float* rays, uint32_t n, int4* out, uint32_t* next,
                              int* err, int sms, cudaStream_t st);
void launch_trace_any_api(const rtd::DevScene& S, const float* rays, uint32_t n, uint8_t* out, uint32_t* next,
                          int* err, int sms, cudaStream_t st);
void launch_extend(const rtd::DevScene& S, const PathState& P, const uint32_t* queue, const uint32_t* count,
                   uint32_t* next, int* err, int sms, cudaStream_t st);
void launch_shadow(const rtd::DevScene& S, const PathState& P, const float4* sq, const uint32_t* count,
                   uint32_t* next, int* err, int sms, cudaStream_t st);

void launch_generate(const rtd::DevScene& S, const PathState& P, const RenderLaunch& R, uint32_t* queue0,
                     uint32_t* count0, cudaStream_t st);
void launch_shade(const rtd::DevScene& S, const PathState& P, const RenderLaunch& R, uint32_t depth,
                  const uint32_t* qin, const uint32_t* cin, uint32_t* ctr, const ClassQueues& Q, uint32_t* qout,
                  uint32_t* cout, float4* sq, uint32_t* scount, int sms, cudaStream_t st);
void launch_finalize(const PathState& P, const RenderLaunch& R, cudaStream_t st);

cudaError_t photon_build(const rtd::DevScene& S, PhotonMapDev& map, const PathState& P, uint32_t* qa, uint32_t* qb,
                         uint32_t* counters, const RtPhotonParams& prm, const float* emit_setup, int sms,
                         cudaStream_t st, int64_t* n_stored);
cudaError_t photon_set(PhotonMapDev& map, const float4* pos, const float4* pow, const float4* nor, uint32_t n,
                       float radius, uint32_t k, cudaStream_t st);
void launch_photon_gather_api(const PhotonMapDev& map, const float* q, uint32_t n, float* out, int sms, cudaStream_t st);
void launch_knn_api(const PhotonMapDev& map, const float* q, uint32_t n, int k, float rmax2, int* idx, float* d2,
                    int* err, int sms, cudaStream_t st);
void launch_photon_gather_paths(const PhotonMapDev& map, const PathState& P, const float4* gq, const uint32_t* count,
                                int sms, cudaStream_t st);
void launch_accumulate(const float* scratch, uint32_t nsamp, uint32_t npix, float* acc, float* m2, uint32_t* cnt,
                       const uint8_t* conv, float clamp, uint32_t min_samples, float floor_, cudaStream_t st);
}  // namespace rth
