/*
 * rt_api.h — C ABI of the B200 render hot path (librtb200.so).
 *
 * This is the drop-in boundary for the reference renderer's sample-pass entry
 * point.  The reference exposes (src/renderer.rs:655-669)
 *
 *     render_tiles(scratch, converged, sample_idx, strata, width, height,
 *                  camera, world, background, lights, bg_scale, photon_map,
 *                  frame_time)
 *
 * with trait objects (&dyn Hittable, &dyn Material) that cannot cross an FFI.
 * Here the scene is handed over once as flat structure-of-arrays buffers
 * (RtSceneDesc), flattened on the host exactly as the reference's loader builds
 * it (src/scene_file.rs:899-1132), and rendering calls take plain pointers.
 *
 * Conventions
 *  - Every function returns an int32 status: RT_OK (0) or an RT_ERR_* code.
 *    rt_last_error() returns the message of the last failure on a handle.
 *  - The caller owns every buffer it passes; the library copies what it keeps.
 *  - Buffers flagged RT_MEM_DEVICE are CUDA device pointers on the scene's
 *    device; otherwise they are host pointers (pageable or pinned).
 *  - One handle per thread; calls on one handle are serialised on its own
 *    (non-blocking) stream.  Every call first makes that stream wait for the
 *    work already queued on the caller's stream (rt_set_caller_stream; the
 *    legacy default stream unless set), so device buffers written by the
 *    caller's kernels are complete before the library reads them, and every
 *    call has finished its device work when it returns.
 *  - All arithmetic is IEEE-754 binary32 ("f32" in the reference).
 */
#ifndef RT_API_H
#define RT_API_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RT_API_VERSION 1

/* ── status codes ─────────────────────────────────────────────────────────── */
#define RT_OK            0
#define RT_ERR_INVALID   1   /* degenerate or malformed input (replaces the reference's asserts, e.g. src/quad.rs:27-28) */
#define RT_ERR_CAPACITY  2   /* a queue, stack or table limit was exceeded */
#define RT_ERR_TIMEOUT   3   /* a bounded device loop ran out of iterations */
#define RT_ERR_CUDA      4   /* a CUDA runtime call failed */
#define RT_ERR_NOMEM     5   /* a device allocation failed */

#define RT_MEM_HOST      0
#define RT_MEM_DEVICE    1

/* ── materials (src/material.rs, src/texture.rs) ─────────────────────────── */
#define RT_MAT_LAMBERTIAN          0  /* material.rs:85-102, texture Solid */
#define RT_MAT_CHECKER             1  /* Lambertian with texture.rs:32-37 checker */
#define RT_MAT_DIELECTRIC          2  /* material.rs:323-332 */
#define RT_MAT_SPECTRAL_DIELECTRIC 3  /* material.rs:357-403 */
#define RT_MAT_SPECTRAL_METAL      4  /* material.rs:427-554 */
#define RT_MAT_DIFFUSE_LIGHT       5  /* material.rs:14-25 */
#define RT_MAT_BLACKBODY_LIGHT     6  /* material.rs:40-83 */
#define RT_MAT_PBR                 7  /* PbrMaterial with scalar parameters, material.rs:680-1050 */

/* conductor n,k tables built into the library (src/spectrum.rs:213-240) */
#define RT_METAL_GOLD    0
#define RT_METAL_COPPER  1
#define RT_METAL_SILVER  2
#define RT_METAL_CUSTOM  3  /* uses RtMaterial.nk_* (a uniform wavelength grid) */
#define RT_MAX_NK        16

typedef struct RtMaterial {
    int32_t type;            /* RT_MAT_* */
    float   albedo[3];       /* Lambertian colour, checker "even", DiffuseLight colour */
    float   odd[3];          /* checker "odd" colour */
    float   checker_scale;   /* checker tile frequency (texture.rs:32-37) */
    float   cauchy_b;        /* Dielectric: ior; SpectralDielectric: Cauchy B (µm²) */
    float   cauchy_c;        /* SpectralDielectric: Cauchy C (µm²) */
    float   absorption[3];   /* SpectralDielectric Beer-Lambert sigma per unit length */
    float   roughness;       /* SpectralMetal roughness (alpha = max(r², 1e-4)) */
    int32_t metal;           /* RT_METAL_* */
    float   temp_k;          /* BlackbodyLight temperature (K) */
    float   intensity;       /* BlackbodyLight intensity */
    int32_t nk_count;        /* RT_METAL_CUSTOM: samples on the grid */
    float   nk_start;        /* RT_METAL_CUSTOM: first wavelength (nm) */
    float   nk_step;         /* RT_METAL_CUSTOM: grid step (nm) */
    float   nk_n[RT_MAX_NK];
    float   nk_k[RT_MAX_NK];
    /* RT_MAT_PBR (albedo, roughness above): metallic workflow GGX with an
     * anisotropic base lobe, a clearcoat with optional thin film, a sheen lobe
     * and an emission (material.rs:680-1050) */
    float   metallic;            /* 0 dielectric .. 1 conductor */
    float   anisotropy;          /* 0 .. 1 */
    float   anisotropy_angle;    /* radians, in the tangent plane */
    float   clearcoat;           /* coat weight 0 .. 1 */
    float   clearcoat_roughness;
    float   film_thickness;      /* nm; 0 = no thin film on the coat */
    float   film_ior;
    float   sheen;               /* 0 .. 1 */
    float   sheen_tint;          /* 0 white .. 1 albedo */
    float   emission[3];         /* linear RGB, times emission_strength */
    float   emission_strength;
    /* texture maps, 1-based indices into RtSceneDesc.textures (0 = none):
     * RT_MAT_LAMBERTIAN takes albedo_tex (texture.rs Image / Mottle); RT_MAT_PBR
     * takes all five (material.rs:758-786) */
    int32_t albedo_tex, roughness_tex, metallic_tex, ao_tex, normal_tex;
} RtMaterial;

/* ── textures (src/texture.rs, material.rs:633-671) ──────────────────────────
 * IMAGE: 8-bit RGB texels, row 0 = top.  A Lambertian albedo samples the
 * nearest texel and decodes sRGB (texture.rs:34-43); PBR maps sample bilinear
 * (albedo sRGB-decoded; roughness / metallic / ao the red channel / 255;
 * normal maps rgb / 255 → 2x − 1).  UVs: triangles carry tri_uv (else the
 * reference's defaults (0,0) (1,0) (0.5,1)), quads their (α, β), spheres
 * sphere.rs's (φ, θ) map; convex solids and shapes have (0, 0).
 * MOTTLE: lerp(lo, hi, clamp(2·turb(p·scale, 7), 0, 1)) (texture.rs:52-55). */
#define RT_TEX_IMAGE   0
#define RT_TEX_MOTTLE  1
typedef struct RtTexture {
    int32_t        type;          /* RT_TEX_* */
    int32_t        width, height; /* IMAGE */
    const uint8_t* rgb8;          /* IMAGE: height × width × 3 */
    float          scale;         /* MOTTLE */
    float          lo[3], hi[3];  /* MOTTLE */
    float          perlin_vec[256 * 3];   /* MOTTLE: the Perlin tables (perlin.rs:4-33) */
    int32_t        perlin_perm[3 * 256];
} RtTexture;

/* ── background (src/renderer.rs:183-223) ────────────────────────────────── */
#define RT_BG_SOLID     0
#define RT_BG_GRADIENT  1
#define RT_BG_ENVMAP    2   /* EnvMap, or EnvMapSplit when visible_type >= 0 */
#define RT_BG_PHYSICAL  3   /* Preetham sky with a sun disc (renderer.rs:231-337): sun NEE at
                               diffuse and rough-conductor vertices (renderer.rs:421-456, 495-518) */

typedef struct RtBackground {
    int32_t      type;            /* RT_BG_* */
    float        color[3];        /* Solid */
    float        top[3];          /* Gradient */
    float        bottom[3];
    /* env map: equirectangular, row-major H×W×3 float RGB, top row = +Y */
    int32_t      env_w, env_h;
    const float* env_rgb;
    float        env_rot_y_deg;   /* EnvMapData::with_rotation (renderer.rs:78-81) */
    /* EnvMapSplit visible backdrop: -1 = none, else RT_BG_SOLID / RT_BG_GRADIENT */
    int32_t      visible_type;
    float        visible_color[3];
    float        visible_top[3];
    float        visible_bottom[3];
    /* RT_BG_PHYSICAL: unit direction towards the sun and the turbidity
     * (scene_file.rs:917-927 builds sun_dir from azimuth and elevation) */
    float        sun_dir[3];
    float        turbidity;
} RtBackground;

/* ── scene description ───────────────────────────────────────────────────── *
 * Primitives are world-space (object transforms of transform.rs are applied on
 * the host before the call).  The canonical primitive id used for hit records
 * and tie-breaking is: triangles [0, n_tris), then quads, then spheres, each in
 * the order given. */
#define RT_PRIM_TRI    0
#define RT_PRIM_QUAD   1
#define RT_PRIM_SPHERE 2

/* ── participating media (volume.rs:39-263, scene_file.rs:297-336, 962-983) ─
 * A medium is not a BVH primitive: its scatter distance depends only on the
 * ray (the reference seeds the medium's random stream from the ray's bits,
 * volume.rs:114-120), so each ray's medium candidates are computed next to the
 * BVH traversal and the nearer event wins (medium ids follow the primitives'
 * canonical ids; an exact tie goes to the surface). */
#define RT_MEDIUM_CONSTANT 0   /* ConstantMedium: exponential free flight, Beer–Lambert shadows */
#define RT_MEDIUM_NOISE    1   /* NoiseMedium: delta tracking against density·max, 16-point shadow quadrature */
#define RT_MEDIUM_GRID     2   /* no counterpart in the reference: a voxel grid of σ_t in a box boundary,
                                  trilinear between voxel centres; delta tracking and ratio-tracked
                                  shadows against per-brick majorants (8³ voxels per brick) */
#define RT_GRID_MAX_RES    1024
#define RT_BOUND_SPHERE    0
#define RT_BOUND_BOX       1   /* axis-aligned box of 6 quads (quad.rs:201-215) */

typedef struct RtMedium {
    int32_t type;               /* RT_MEDIUM_* */
    int32_t boundary;           /* RT_BOUND_* */
    float   center[3], radius;  /* sphere boundary */
    float   p_min[3], p_max[3]; /* box boundary */
    float   density;            /* σ (constant) or density scale = majorant (noise) */
    float   color[3];           /* single-scattering albedo of the HG phase function */
    float   g;                  /* Henyey–Greenstein asymmetry */
    float   noise_scale;        /* noise: turbulence frequency */
    float   threshold;          /* noise: density = max(turb(7)·0.5 − threshold, 0)·density */
    /* noise: the Perlin tables of this medium (perlin.rs:4-33): 256 unit
     * vectors and three permutations of 0..255 */
    float   perlin_vec[256 * 3];
    int32_t perlin_perm[3 * 256];
    /* grid: grid_res[0] × grid_res[1] × grid_res[2] values (x fastest), each
     * 1 .. RT_GRID_MAX_RES, over the box p_min..p_max (box boundary only);
     * σ_t(x) = density × trilinear(grid) ≥ 0.  The library copies the grid. */
    const float* grid;
    int32_t grid_res[3];
} RtMedium;

/* ── analytic convex solids (diamond.rs:198-253) ─────────────────────────────
 * A gem is a convex polyhedron: the intersection of outward half-spaces
 * n·x ≤ d (`convex_planes`, 4 floats per plane, in the solid's OBJECT space).
 * Each solid carries the placement the reference wraps around a gem
 * (scene_file.rs:924-930): a uniform scale about the origin
 * (transform.rs:15-27), a rotation about `pivot` (transform.rs:218-224) and a
 * translation, i.e. x_world = rot·(scale·x − pivot) + pivot + translate.
 * Identity: scale 1, rot = I, pivot = translate = 0.  Several solids may share
 * one run of planes.  Canonical ids follow the spheres.  Materials must not
 * be emissive. */
#define RT_PRIM_CONVEX 3
typedef struct RtConvex {
    int32_t plane_offset;       /* first plane in convex_planes */
    int32_t n_planes;           /* 4 .. 1024 */
    int32_t mat;
    float   polish;             /* per-facet micro-tilt amplitude in radians (hittable.rs:261-270), 0 .. 0.25 */
    float   box_lo[3], box_hi[3]; /* object-space box that contains the solid */
    float   scale;              /* > 0 */
    float   rot[9];             /* row-major world-from-object rotation */
    float   pivot[3];
    float   translate[3];
} RtConvex;

/* ── other analytic shapes (cylinder.rs, cone.rs, disk.rs, plane.rs) ─────────
 * In object space: the cylinder and the cone stand on the y axis with their
 * base centre at `center` (cylinder: closed caps at y = 0 and height; cone: a
 * base disk at y = 0 and the apex at height); the disk and the infinite plane
 * (with its optional two-sine wave bump of the shading normal) are given by
 * a point and a normal.  The placement is the objects' SRT wrapper
 * (scene_file.rs:1036-1042): x_world = rot·(scale·x) + translate.  Canonical
 * ids follow the convex solids.  Shapes are not NEE lights; an infinite
 * plane is bounded by the reference's ±1e5 proxy box and stays out of the
 * photon-emitter bounds. */
#define RT_SHAPE_CYLINDER 0
#define RT_SHAPE_CONE     1
#define RT_SHAPE_DISK     2
#define RT_SHAPE_PLANE    3
typedef struct RtShape {
    int32_t type;               /* RT_SHAPE_* */
    int32_t mat;
    float   center[3];          /* base centre (cylinder, cone), centre (disk), point (plane) */
    float   normal[3];          /* disk / plane normal, any length > 0 */
    float   radius;             /* cylinder, cone, disk */
    float   height;             /* cylinder, cone */
    float   wave_amplitude;     /* plane: 0 = flat */
    float   wave_scale;
    float   scale;              /* > 0 */
    float   rot[9];             /* row-major rotation */
    float   translate[3];
} RtShape;

typedef struct RtSceneDesc {
    int64_t        n_tris;
    const float*   tri_v;         /* n_tris × 9  : v0, v1, v2 */
    const float*   tri_n;         /* n_tris × 9  : per-vertex normals (NULL → face normal) */
    const int32_t* tri_mat;       /* n_tris      : material index */
    int64_t        n_quads;
    const float*   quad_quv;      /* n_quads × 9 : corner Q, edge u, edge v (quad.rs:21-33) */
    const int32_t* quad_mat;
    int64_t        n_spheres;
    const float*   sphere;        /* n_spheres × 4 : centre xyz, radius */
    const int32_t* sphere_mat;
    int32_t        n_mats;
    const RtMaterial* mats;
    /* NEE light list (hittable.rs:138-225): canonical prim ids of the light
     * copies (quads or spheres).  The reference inserts each [[lights]] quad in
     * the world AND in the light list (scene_file.rs:1065-1066). */
    int32_t        n_lights;
    const int32_t* light_prims;
    RtBackground   bg;
    /* spectral sampling: 0 = reference range 380–700 nm (65-entry CIE table),
     * 1 = 380–780 nm (table extended past 700 nm) */
    int32_t        spectral_range;
    /* participating media (may be 0 / NULL) */
    int32_t        n_media;
    const RtMedium* media;
    /* analytic convex solids (may be 0 / NULL); ids follow the spheres, media ids follow them */
    int64_t        n_convex;
    const RtConvex* convex;
    const float*   convex_planes;  /* planes × 4: outward unit normal xyz, offset d (object space) */
    /* cylinders, cones, disks, infinite planes (may be 0 / NULL); ids follow the convex solids */
    int64_t        n_shapes;
    const RtShape* shapes;
    /* textures and the triangles' texture coordinates and tangents (all may be 0 / NULL) */
    int32_t          n_textures;
    const RtTexture* textures;
    const float*     tri_uv;        /* n_tris × 6: (u, v) at v0, v1, v2 */
    const float*     tri_tangent;   /* n_tris × 9: per-vertex tangents (mesh.rs:33-54) */
    int32_t          bvh_builder;   /* RT_BVH_DEVICE (0, default) or RT_BVH_HOST: where the binary SAH tree is built */
} RtSceneDesc;

#define RT_BVH_DEVICE 0   /* the binary SAH tree on the GPU (same tree as the host builder) */
#define RT_BVH_HOST   1   /* the binary SAH tree on host threads */

/* ── camera (src/camera.rs:24-59) ────────────────────────────────────────── */
typedef struct RtCamera {
    float   origin[3];
    float   lower_left[3];
    float   horizontal[3];
    float   vertical[3];
    float   u[3], v[3];
    float   lens_radius;
    int32_t aperture_blades;  /* 0 = round lens; polygonal bokeh is not supported */
} RtCamera;

/* ── one sample pass (render_tiles, renderer.rs:655-730) ─────────────────── */
typedef struct RtPassParams {
    uint32_t width, height;
    uint32_t sample_idx;     /* first sample index of this call */
    uint32_t n_samples;      /* consecutive sample passes rendered by this call (≥1) */
    uint32_t strata;         /* ⌊√spp⌋ stratification grid (main.rs:64) */
    uint32_t max_depth;      /* reference constant MAX_DEPTH = 50 (renderer.rs:16) */
    uint32_t hero_count;     /* wavelengths per path: 1 (reference) or 4 */
    uint32_t use_frame_time; /* 0: time ~ U[0,1) (camera.rs:57); 1: t0 + U·(t1-t0) */
    float    t0, t1;
    float    bg_scale;       /* multiplies the background on a miss only (renderer.rs:402) */
    uint64_t seed;           /* per-pixel RNG streams are keyed on (seed, pixel, sample) */
} RtPassParams;

/* ── hit record for the ray-level test entry points ──────────────────────── */
typedef struct RtHit {
    int32_t prim;      /* canonical primitive id, -1 = miss */
    float   t;
    float   b1, b2;    /* triangle barycentrics / quad (alpha, beta) / sphere (u, v) */
} RtHit;

typedef struct RtScene RtScene;

/* Library / device information. */
int32_t rt_version(void);
int32_t rt_device_count(int32_t* count);

/* Create a scene on CUDA device `device`: copies the descriptor's arrays,
 * builds the 8-wide SAH BVH with the cost model of src/bvh.rs:52-174 and the
 * environment sampling tables (renderer.rs:32-74).  Replaces
 * scene_file::build (scene_file.rs:899-1132) + BvhTree::from_list (bvh.rs:199). */
int32_t rt_scene_create(const RtSceneDesc* desc, int32_t device, RtScene** out);
int32_t rt_scene_destroy(RtScene* scene);
int32_t rt_last_error(const RtScene* scene, char* buf, size_t len);

/* BVH statistics of the built tree: node count, leaf count, max depth, SAH cost. */
/* Wall time of the BVH build at scene creation (binary SAH tree + collapse to 8-wide), ms. */
int32_t rt_scene_build_time(const RtScene* scene, double* ms);
int32_t rt_scene_bvh_stats(const RtScene* scene, int64_t* n_nodes, int64_t* n_leaves,
                           int32_t* max_depth, double* sah_cost);
/* Export the 8-wide node array in the reference layout (bvh.rs:25-32, 224 B per
 * node: min[3][8], max[3][8], children[8]; leaf = -(leaf_slot+1), INT32_MIN =
 * empty) and the canonical prim id of every leaf slot.  Pass NULL to query sizes. */
int32_t rt_scene_bvh_export(const RtScene* scene, float* nodes_224B, int64_t* n_nodes,
                            int32_t* leaf_prims, int64_t* n_leaves);

/* Closest hit for n rays.  rays: n × 8 floats (origin xyz, dir xyz, t_min, t_max).
 * Replaces BvhTree::hit_index (bvh.rs:229-288).  Ties on t go to the smaller
 * canonical prim id.  With media, a medium scatter event nearer than the
 * surface hit is returned as prim = n_prims + medium index (b1 = b2 = 0); the
 * ray's wavelength, which keys the medium's random stream, is 550 nm. */
int32_t rt_trace_closest(RtScene* scene, const float* rays, int64_t n, RtHit* hits, int32_t mem);
/* Any hit for n rays (bvh.rs:487-530); occluded[i] = 1 when an opaque hit
 * exists (media never occlude). */
int32_t rt_trace_any(RtScene* scene, const float* rays, int64_t n, uint8_t* occluded, int32_t mem);
/* Transmittance for n rays over [t_min, t_max] (bvh.rs:532-575 with
 * volume.rs:140-146, 239-252): 0 if an opaque primitive is hit, else the
 * product of the media's transmittances. */
int32_t rt_trace_transmittance(RtScene* scene, const float* rays, int64_t n, float* tr, int32_t mem);

/* One call = params->n_samples consecutive sample passes of render_tiles.
 * scratch_rgb receives n_samples × height × width × 3 floats (linear radiance,
 * row 0 = top image row), the per-pass output of render_tiles.  converged
 * (nullable, height × width bytes) skips pixels like renderer.rs:695-698. */
int32_t rt_render_pass(RtScene* scene, const RtCamera* cam, const RtPassParams* params,
                       float* scratch_rgb, const uint8_t* converged, int32_t mem);

/* Render params->n_samples passes and fold them into device-resident
 * accumulators in sample order with the semantics of accumulate_sample
 * (main.rs:603-643): non-finite samples dropped, optional luminance clamp
 * max(firefly_clamp·mean_lum, firefly_floor) after firefly_min_samples, per-
 * channel Welford.  With reset != 0 the accumulators are cleared first.
 * out_sum (h×w×3), out_m2 (h×w×3), out_count (h×w) are written when non-NULL. */
int32_t rt_render_accumulate(RtScene* scene, const RtCamera* cam, const RtPassParams* params,
                             float firefly_clamp, uint32_t firefly_min_samples,
                             float firefly_floor, int32_t reset,
                             float* out_sum, float* out_m2, uint32_t* out_count, int32_t mem);

/* Asynchronous form of rt_render_accumulate, with the explicit stream of the
 * replacement contract's threading rule (the reference's render_tiles,
 * src/renderer.rs:655-669, is synchronous): the work is queued on the scene's
 * stream after the work already on `cuda_stream` (a cudaStream_t; NULL = the
 * legacy default stream), `cuda_stream` is made to wait for its end, and the
 * call returns without waiting.  The wavefront runs as one CUDA graph (see
 * RtTuning.graph).  Outputs are RT_MEM_DEVICE buffers (or NULL) that must
 * stay valid until the work is done; at most one 2 GiB sample buffer of
 * samples per call (W·H·n_samples·12 bytes), no guide training.  Errors of
 * the device work (RT_ERR_TIMEOUT, RT_ERR_CAPACITY) come from the next
 * rt_sync, or from the next call on the handle that checks the device's
 * status, whichever comes first; the statistics of rt_last_render_stats from
 * rt_sync (a later call on the handle first waits for the queued work). */
int32_t rt_render_accumulate_async(RtScene* scene, const RtCamera* cam, const RtPassParams* params,
                                   float firefly_clamp, uint32_t firefly_min_samples,
                                   float firefly_floor, int32_t reset,
                                   float* out_sum, float* out_m2, uint32_t* out_count, void* cuda_stream);
/* Waits for the handle's queued work; returns the device status of the last
 * asynchronous call (RT_OK, RT_ERR_TIMEOUT, RT_ERR_CAPACITY) and makes its
 * statistics those of rt_last_render_stats. */
int32_t rt_sync(RtScene* scene);

/* ── output (src/output.rs, src/main.rs:571-583) ─────────────────────────── */
#define RT_TONEMAP_AGX   0   /* Blender AgX with the "Punchy" look (output.rs:34-80), the default */
#define RT_TONEMAP_ACES  1   /* Narkowicz ACES fit in AP1 (output.rs:7-31) */

typedef struct RtDevelopParams {
    uint32_t width, height;
    float    exposure;       /* linear multiplier (default 1) */
    int32_t  tonemapper;     /* RT_TONEMAP_* */
    float    vignette;       /* 0 .. 1: corners × (1 − vignette) */
    float    distortion;     /* 0 .. 1: barrel coefficient k */
} RtDevelopParams;

/* Develop linear radiance into 8-bit sRGB, replacing apply_optics + save_png's
 * tone_map (output.rs:84-190): optics in linear light (vignette, barrel
 * distortion with bilinear resampling), exposure, AgX or ACES, the sRGB
 * curve and the quantisation (x.clamp(0, 0.999)·256 truncated).  linear_rgb
 * (height × width × 3 per-sample means, row 0 = top) may be NULL: the scene's
 * accumulators are developed (sum / max(count, 1), main.rs:571-583).
 * rgb8 receives height × width × 3 bytes.  mem applies to both buffers. */
int32_t rt_develop(RtScene* scene, const float* linear_rgb, const RtDevelopParams* params, uint8_t* rgb8,
                   int32_t mem);

/* Decode the scanlines of a Radiance RGBE image (flat or new-style RLE rows,
 * the part of `image`'s HDR decoder the reference's env maps go through,
 * renderer.rs:32-74) into height × width × 3 linear floats.  Host only; no
 * device is touched. */
int32_t rt_rgbe_decode(const uint8_t* scanlines, size_t n_bytes, int32_t width, int32_t height, float* rgb);

/* ── caustic photon map (src/photon.rs, src/scene.rs:35-74) ──────────────── */
#define RT_EMIT_DISK     0   /* directional disk facing `dir` (PhotonMap::build, photon.rs:41-94) */
#define RT_EMIT_QUAD     1   /* cosine-weighted quad (PhotonMap::build_from_quad, photon.rs:97-135) */
#define RT_EMIT_SUN      2   /* the Physical sky's sun: a disk facing sun_dir with the sky radiance at
                                the sun direction nudged by 0.04, ×π (scene.rs:40-52); dir/color unused */
#define RT_EMIT_LIGHT    3   /* a quad of the scene's NEE light list as a cosine-weighted quad source
                                (build_from_quad) coloured by its material's emission: a diffuse light's
                                colour, a blackbody's time-averaged RGB × intensity (material.rs:53-59);
                                the reference's rebuild_caustics picks the env disk over the lights when
                                both exist (scene.rs:52-73), this type lets a caller emit from the lights */
#define RT_MAX_EMITTERS  8

typedef struct RtPhotonEmitter {
    int32_t  type;          /* RT_EMIT_* */
    float    dir[3];        /* DISK: direction toward the source (sun_dir) */
    float    color[3];      /* DISK: sun colour (radiance · π); QUAD: emission colour */
    float    corner[3];     /* QUAD corner, edges u and v */
    float    u[3], v[3];
    uint32_t n_photons;     /* photons emitted by this source */
    int32_t  light;         /* LIGHT: index into the scene's light list (RtSceneDesc.light_prims), a quad */
    /* QUAD / LIGHT: a sphere (centre xyz, radius) around the specular objects
     * the caustics come from, or radius 0.  With a radius, every photon leaves
     * toward the sphere (uniform in the cone it subtends) and its power is
     * scaled by the cosine-density ratio 2·cosθ·(1 − cos θ_max), zero below the
     * light's plane; photons whose first hit is diffuse are never stored
     * (trace_photon, photon.rs:232-277), so the expected map is that of the
     * full hemisphere while almost every photon reaches the stones (a
     * projection map).  The reference emits over the whole hemisphere. */
    float    target[4];
} RtPhotonEmitter;

typedef struct RtPhotonParams {
    int32_t  n_emitters;
    RtPhotonEmitter emitters[RT_MAX_EMITTERS];
    float    gather_radius; /* Epanechnikov radius (photon.rs:137-157), or the k-NN maximum radius */
    uint32_t knn_k;         /* 0: fixed-radius gather (the reference); k > 0: k nearest within the radius */
    uint64_t seed;
    /* A shard of the emission: trace only the photons with emission index
     * first_photon .. first_photon + shard_photons − 1 (indices run over the
     * emitters in order; shard_photons 0: all of them).  Photon power stays
     * normalised by each emitter's full n_photons, so the stored photons of
     * all shards together are the photons of one unsharded build (ranks of
     * a multi-GPU render each trace a shard and exchange what they store). */
    uint32_t first_photon;
    uint32_t shard_photons;
} RtPhotonParams;

/* Emit, trace and store photons on the device, then build the gather
 * structure (Morton-sorted photons under an implicit box tree).  Replaces
 * SceneData::rebuild_caustics → PhotonMap::build/_from_quad (scene.rs:35-74,
 * photon.rs:41-135, trace_photon :232-277, kd_build :165-191).  The map then
 * feeds every diffuse vertex of later render calls (renderer.rs:461-467). */
int32_t rt_photon_build(RtScene* scene, const RtPhotonParams* params, int64_t* n_stored);

/* Device time of the last rt_photon_build's stages (diagnostics, no reference
 * counterpart), from CUDA events on the scene's stream: ms[0] emission and
 * tracing, ms[1] compaction of the stored photons, ms[2] the gather
 * structure (Morton sort and box heap). */
int32_t rt_photon_build_times(const RtScene* scene, float* ms);
/* Replace the map with caller-given photons (n × 3 positions, powers, normals;
 * indices = emission index used to break distance ties). */
int32_t rt_photon_set(RtScene* scene, const float* pos, const float* power, const float* nor,
                      const int32_t* index, int64_t n, float gather_radius, uint32_t knn_k);
int32_t rt_photon_clear(RtScene* scene);
/* Stored photons in emission order (NULL arrays query the count). */
int32_t rt_photon_export(const RtScene* scene, float* pos, float* power, float* nor, int32_t* index,
                         int64_t* n);
/* Irradiance estimate at n queries (n × 6: position, surface normal) → n × 3
 * (PhotonMap::irradiance, photon.rs:148-157, or the k-NN estimate). */
int32_t rt_photon_gather(RtScene* scene, const float* queries, int64_t n, float* irr, int32_t mem);
/* k nearest photons of n query points with d² ≤ rmax²: emission indices and
 * d², sorted by (d², index); -1 / INFINITY pad when fewer exist. */
int32_t rt_knn(RtScene* scene, const float* queries, int64_t n, int32_t k, float rmax,
               int32_t* idx, float* d2, int32_t mem);

/* ── packed batches of render requests (no counterpart in the reference,
 * whose renderer serves one frame at a time, renderer.rs:655-730) ───────────
 * Many requests on one scene — each with its own camera, size, samples per
 * pixel, first sample and seed — render together: one wavefront pool draws
 * samples from all of them (a cursor over the concatenated requests), so the
 * GPU stays full however small each frame is.  Every request's samples are
 * those of an rt_render_accumulate call with the same camera and
 * RtPassParams (width, height, sample_idx, n_samples = spp, strata, seed;
 * max_depth, hero_count and bg_scale from `shared`), accumulated in the same
 * sample order, so the results are bit-identical to rendering the requests
 * one at a time.  Samples are taken in passes of at most `window` samples
 * per pixel of every unfinished request (0: as many as fit a 2 GiB sample
 * buffer).  Outputs are packed request after request: out_sum / out_m2
 * (Σ w·h·3 floats), out_count (Σ w·h), and done_ms[j], the device time from
 * the start of the call to the end of the pass that finished request j.
 * No converged masks, no guide. */
typedef struct RtBatchJob {
    RtCamera cam;
    uint32_t width, height;
    uint32_t spp;            /* samples per pixel of the request (≥ 1) */
    uint32_t strata;         /* ⌊√spp⌋ unless the caller says otherwise */
    uint32_t sample_idx;     /* first sample index */
    uint32_t pad;
    uint64_t seed;
} RtBatchJob;
int32_t rt_render_batch(RtScene* scene, const RtBatchJob* jobs, int32_t n_jobs, const RtPassParams* shared,
                        uint32_t window, float* out_sum, float* out_m2, uint32_t* out_count, float* done_ms,
                        int32_t mem);

/* Device timing of the last render call: total milliseconds and ray counts. */
int32_t rt_last_render_stats(const RtScene* scene, double* ms, int64_t* ext_rays,
                             int64_t* shadow_rays, int64_t* kernel_launches);

/* Per-stage device timing (diagnostics, no reference counterpart): with
 * profiling enabled every launch of the render loop is bracketed by CUDA
 * events on the launching stream.  ms[4] / launches[4] receive the totals of
 * the last render call for: 0 generate+finalize, 1 extend (closest hit),
 * 2 shade, 3 shadow (any hit). */
int32_t rt_set_profiling(RtScene* scene, int32_t enable);
int32_t rt_kernel_times(const RtScene* scene, double* ms, int64_t* launches);

/* Extension rays of bounce `depth` of sample pass params->sample_idx (diagnostics,
 * no reference counterpart): renders one pass and copies up to max_rays of that
 * bounce's queued rays as n × 8 floats (origin, direction, t_min, t_max) into
 * host memory.  Used to count the reference traversal's work on the rays the
 * GPU actually traces. */
int32_t rt_capture_rays(RtScene* scene, const RtCamera* cam, const RtPassParams* params,
                        uint32_t depth, float* rays, int64_t max_rays, int64_t* n_rays);

/* rt_render_pass without any device allocation (no counterpart in the
 * reference).  For hosts that may not allocate device memory while they run —
 * a real-time loop that must not stall on cudaMalloc, a process whose device
 * memory is already owned by its framework's caching allocator, a plugin host
 * that hands over only its own buffers — the wavefront scratch comes from a
 * fixed device array inside the library (RT_NOALLOC_SCRATCH_BYTES, held on
 * every GPU that loads the library until exit) instead of cudaMalloc.
 *  - scratch_rgb must be DEVICE memory: n_samples × height × width × 3 floats.
 *  - The array holds a pool of 32,768 paths that is refilled with new samples
 *    as paths end, so any frame fits it; but 32,768 paths fill a small part of
 *    the GPU, so width × height is capped at RT_NOALLOC_MAX_PIXELS (a chosen
 *    limit, RT_ERR_CAPACITY beyond it): larger frames belong on
 *    rt_render_pass, whose pool grows to 8,388,608 paths.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress); make that first call before any stream capture.
 *  - Like every call here, it waits for its device work before returning.
 *  - All calls share the one array: calls that overlap on the GPU (two
 *    streams, two threads, two scenes on one device) race and must be
 *    serialised by the caller.
 *  - No converged mask (every pixel is rendered). */
#define RT_NOALLOC_MAX_PIXELS     65536
#define RT_NOALLOC_SCRATCH_BYTES  (15u << 20)
int32_t rt_render_pass_noalloc(RtScene* scene, const RtCamera* cam, const RtPassParams* params,
                               float* scratch_rgb);

/* ── launch tuning (no counterpart in the reference) ─────────────────────────
 * The path-pool capacity and the grids of the persistent traversal kernels and
 * of the shading kernels.  Every path draws its random numbers from (pixel,
 * sample), so a tuning changes speed and memory, never the image.  Zero fields
 * select the built-in values (8,388,608 paths; the traversal's resident limit;
 * 8 shading blocks per SM).  rustracer_b200/autotune.py times candidates on a
 * short render and sets the fastest. */
typedef struct RtTuning {
    uint32_t max_paths;            /* 0 or 65536 .. 8388608 */
    uint32_t trace_blocks_per_sm;  /* 0 or 1 .. 8 (capped at the kernels' resident blocks) */
    uint32_t shade_blocks_per_sm;  /* 0 or 1 .. 32 */
    /* Limits of the device loops (0: the built-in ones, which a render of the
     * scene never reaches).  Lower values exist to exercise the error paths:
     * a render call whose wavefront has not drained after max_iterations
     * iterations returns RT_ERR_TIMEOUT; a traversal that needs more than
     * stack_limit stack entries stops and the call returns RT_ERR_CAPACITY.
     * rt_get_tuning reports the stack entries in force (7 per tree level). */
    uint32_t max_iterations;       /* 0 or ≥ 1 */
    uint32_t stack_limit;          /* 0 or 1 .. the built-in capacity */
    /* Traversal stack entries kept in a per-thread ring (local memory) before the
     * rest spills to global memory (0: 16; else a power of two ≤ 16).  The
     * results never depend on it; small rings make every traversal take the
     * spill path. */
    uint32_t stack_ring;
    /* Node layout the traversal reads: RT_NODES_FULL (0, the default), the
     * reference's 224-byte float layout (bvh.rs:25-32); RT_NODES_QUANTISED
     * (1, when the scene's extents allow it), 128-byte nodes whose child boxes
     * are 8-bit offsets rounded outward; RT_NODES_WIDE4 (2, scenes whose tree
     * was built on the device), 4-wide nodes of 112 bytes over the same binary
     * SAH tree — the reference's BVH width choice (bvh.rs:10-14).  The hits do
     * not depend on it. */
    uint32_t node_format;
    /* 1: every render call runs its wavefront as one CUDA graph — the path
     * pool's first fill, then one conditional node per iteration up to the
     * call's bound, each run only while rays remain — captured on the first
     * call and replayed while the scene state, buffers and pool stay the
     * same (every pass of an rt_render_batch call included: its job table
     * is read from device memory); 0 (the default): the host queues each
     * iteration's launches and stops two iterations after the pool drains.
     * rt_render_pass_noalloc always runs the host-driven loop.  The images
     * are the same. */
    uint32_t graph;
} RtTuning;
#define RT_NODES_FULL      0
#define RT_NODES_QUANTISED 1
#define RT_NODES_WIDE4     2
int32_t rt_set_tuning(RtScene* scene, const RtTuning* tuning);

/* The stream the caller queues its own work on (a cudaStream_t; NULL = the
 * legacy default stream, the initial setting).  No counterpart in the
 * reference, whose render_tiles works on host memory only: a host that passes
 * RT_MEM_DEVICE buffers written by its own kernels names the stream they were
 * queued on, and every later call on this handle waits for that stream's work
 * so far before its first kernel. */
int32_t rt_set_caller_stream(RtScene* scene, void* cuda_stream);
int32_t rt_get_tuning(const RtScene* scene, RtTuning* tuning);

/* ── path guiding: a learned proposal at diffuse vertices (no counterpart in
 * the reference, whose diffuse bounce is the cosine lobe of pdf.rs:12-41 and
 * renderer.rs:545-571).
 *
 * A 16-level hash grid of the hit position (2 features per level, 2^19
 * entries per level) and a one-blob encoding of the outgoing direction ω_o
 * (toward the previous path vertex) feed a
 * 64-64-64 ReLU MLP (BF16 weights and activations, FP32 accumulation) whose
 * 41 outputs are 8 von Mises–Fisher lobes (mean, log κ, mixture logit) and a
 * guide fraction α ≤ alpha_max.  With guiding on, a Lambertian bounce is drawn with
 * probability α from the lobes and otherwise from the cosine lobe, weighted
 * by the exact mixture density; NEE and bounce MIS use the same density, so
 * the estimator stays unbiased.  In training mode every render call records
 * (position, normal, direction, f·L·cos/p) at its guided vertices and, after
 * the call, takes `steps_per_pass` Adam steps on minibatches of them: the
 * lobes minimise −w·log p_vmf (the KL divergence from the product
 * distribution), α minimises −w·log p_mix with the lobes held fixed.
 * rt_render_pass_noalloc never guides. */
typedef struct RtGuideParams {
    float    domain_min[3], domain_max[3]; /* hash-grid box in world space; min == max: the scene bounds */
    float    learning_rate;                /* Adam step size (1e-2) */
    float    beta1, beta2, epsilon;        /* Adam moment decays and ε (0.9, 0.99, 1e-8) */
    uint32_t batch;                        /* training minibatch rows, a multiple of 1024 (65536) */
    uint32_t steps_per_pass;               /* Adam steps after each training render call */
    uint32_t record_capacity;              /* training records kept per render call */
    uint32_t min_resolution;               /* grid resolution of the coarsest level (4) */
    float    level_scale;                  /* resolution growth per level (1.32: 4 → ≈257) */
    float    alpha_max;                    /* cap of the guide fraction α, in (0, 1); the cosine lobe keeps the rest */
    float    log_kappa_max;                /* cap of log κ of a lobe, in (−5, 20] */
    uint64_t seed;                         /* initial parameters and minibatch draws */
} RtGuideParams;

#define RT_GUIDE_OFF    0   /* plain cosine bounces (the reference's estimator) */
#define RT_GUIDE_SAMPLE 1   /* guided bounces, network frozen */
#define RT_GUIDE_TRAIN  2   /* guided bounces, records, Adam steps after each render call */
#define RT_GUIDE_PARAMS 16792576   /* 15360 weights (4 layers, [out][in]; W3 48×64) + 16×2^19×2 table */

/* Create (or re-create) the scene's guide with fresh parameters; mode RT_GUIDE_OFF. */
int32_t rt_guide_init(RtScene* scene, const RtGuideParams* params);
int32_t rt_guide_mode(RtScene* scene, int32_t mode);
/* Copy the RT_GUIDE_PARAMS fp32 parameters out (write = 0) or in (write = 1;
 * also clears the Adam moments and step count).  Host memory. */
int32_t rt_guide_params(RtScene* scene, float* params, int32_t write);
/* Network outputs at q (n × 9: position, unit normal, unit ω_o) into raw (n × 41). */
int32_t rt_guide_eval(RtScene* scene, const float* q, int64_t n, float* raw, int32_t mem);
/* Mixture density (guide and cosine lobe) at unit directions dirs (n × 3). */
int32_t rt_guide_pdf(RtScene* scene, const float* q, const float* dirs, int64_t n, float* pdf, int32_t mem);
/* One-sample draw with u (n × 4: strategy, lobe, two direction numbers) →
 * out (n × 4: direction, mixture density), the draw the shading kernel makes. */
int32_t rt_guide_sample(RtScene* scene, const float* q, const float* u, int64_t n, float* out, int32_t mem);
/* Loss Σ −w·log p over samples (n × 13: position, normal, ω_o, direction, weight)
 * and its gradient (RT_GUIDE_PARAMS floats, the loss divided by n) — no
 * update.  Host memory. */
int32_t rt_guide_loss_grad(RtScene* scene, const float* samples, int64_t n, float* loss, float* grad);
/* `steps` Adam steps, each on all n samples; loss of the last step's forward
 * pass.  Host memory. */
int32_t rt_guide_train(RtScene* scene, const float* samples, int64_t n, int32_t steps, float* loss);
/* Training totals: records, weighted samples, Adam steps, GPU time of the training kernels. */
int32_t rt_guide_stats(const RtScene* scene, int64_t* records, int64_t* samples, int64_t* steps, double* train_ms);

#ifdef __cplusplus
}
#endif
#endif /* RT_API_H */
