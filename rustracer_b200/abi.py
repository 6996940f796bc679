"""ctypes mirror of include/rt_api.h (the C ABI of librtb200.so).

Field order and types follow the header exactly; keep them in sync.
"""
import ctypes as C

RT_OK, RT_ERR_INVALID, RT_ERR_CAPACITY, RT_ERR_TIMEOUT, RT_ERR_CUDA, RT_ERR_NOMEM = 0, 1, 2, 3, 4, 5
RT_MEM_HOST, RT_MEM_DEVICE = 0, 1

RT_MAT_LAMBERTIAN = 0
RT_MAT_CHECKER = 1
RT_MAT_DIELECTRIC = 2
RT_MAT_SPECTRAL_DIELECTRIC = 3
RT_MAT_SPECTRAL_METAL = 4
RT_MAT_DIFFUSE_LIGHT = 5
RT_MAT_BLACKBODY_LIGHT = 6
RT_MAT_PBR = 7

RT_METAL_GOLD, RT_METAL_COPPER, RT_METAL_SILVER, RT_METAL_CUSTOM = 0, 1, 2, 3
RT_MAX_NK = 16

RT_BG_SOLID, RT_BG_GRADIENT, RT_BG_ENVMAP, RT_BG_PHYSICAL = 0, 1, 2, 3
RT_PRIM_TRI, RT_PRIM_QUAD, RT_PRIM_SPHERE, RT_PRIM_CONVEX = 0, 1, 2, 3

F3 = C.c_float * 3


class RtMaterial(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("albedo", F3),
        ("odd", F3),
        ("checker_scale", C.c_float),
        ("cauchy_b", C.c_float),
        ("cauchy_c", C.c_float),
        ("absorption", F3),
        ("roughness", C.c_float),
        ("metal", C.c_int32),
        ("temp_k", C.c_float),
        ("intensity", C.c_float),
        ("nk_count", C.c_int32),
        ("nk_start", C.c_float),
        ("nk_step", C.c_float),
        ("nk_n", C.c_float * RT_MAX_NK),
        ("nk_k", C.c_float * RT_MAX_NK),
        ("metallic", C.c_float),
        ("anisotropy", C.c_float),
        ("anisotropy_angle", C.c_float),
        ("clearcoat", C.c_float),
        ("clearcoat_roughness", C.c_float),
        ("film_thickness", C.c_float),
        ("film_ior", C.c_float),
        ("sheen", C.c_float),
        ("sheen_tint", C.c_float),
        ("emission", F3),
        ("emission_strength", C.c_float),
        ("albedo_tex", C.c_int32),
        ("roughness_tex", C.c_int32),
        ("metallic_tex", C.c_int32),
        ("ao_tex", C.c_int32),
        ("normal_tex", C.c_int32),
    ]


RT_TEX_IMAGE = 0
RT_TEX_MOTTLE = 1


class RtTexture(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("rgb8", C.POINTER(C.c_uint8)),
        ("scale", C.c_float),
        ("lo", F3),
        ("hi", F3),
        ("perlin_vec", C.c_float * 768),
        ("perlin_perm", C.c_int32 * 768),
    ]


class RtBackground(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("color", F3),
        ("top", F3),
        ("bottom", F3),
        ("env_w", C.c_int32),
        ("env_h", C.c_int32),
        ("env_rgb", C.POINTER(C.c_float)),
        ("env_rot_y_deg", C.c_float),
        ("visible_type", C.c_int32),
        ("visible_color", F3),
        ("visible_top", F3),
        ("visible_bottom", F3),
        ("sun_dir", F3),
        ("turbidity", C.c_float),
    ]


RT_MEDIUM_CONSTANT, RT_MEDIUM_NOISE, RT_MEDIUM_GRID = 0, 1, 2
RT_BOUND_SPHERE, RT_BOUND_BOX = 0, 1


class RtMedium(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("boundary", C.c_int32),
        ("center", F3),
        ("radius", C.c_float),
        ("p_min", F3),
        ("p_max", F3),
        ("density", C.c_float),
        ("color", F3),
        ("g", C.c_float),
        ("noise_scale", C.c_float),
        ("threshold", C.c_float),
        ("perlin_vec", C.c_float * (256 * 3)),
        ("perlin_perm", C.c_int32 * (3 * 256)),
        ("grid", C.c_void_p),
        ("grid_res", C.c_int32 * 3),
    ]


class RtConvex(C.Structure):
    _fields_ = [
        ("plane_offset", C.c_int32),
        ("n_planes", C.c_int32),
        ("mat", C.c_int32),
        ("polish", C.c_float),
        ("box_lo", F3),
        ("box_hi", F3),
        ("scale", C.c_float),
        ("rot", C.c_float * 9),
        ("pivot", F3),
        ("translate", F3),
    ]


RT_SHAPE_CYLINDER = 0
RT_SHAPE_CONE = 1
RT_SHAPE_DISK = 2
RT_SHAPE_PLANE = 3


class RtShape(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("mat", C.c_int32),
        ("center", F3),
        ("normal", F3),
        ("radius", C.c_float),
        ("height", C.c_float),
        ("wave_amplitude", C.c_float),
        ("wave_scale", C.c_float),
        ("scale", C.c_float),
        ("rot", C.c_float * 9),
        ("translate", F3),
    ]


class RtSceneDesc(C.Structure):
    _fields_ = [
        ("n_tris", C.c_int64),
        ("tri_v", C.POINTER(C.c_float)),
        ("tri_n", C.POINTER(C.c_float)),
        ("tri_mat", C.POINTER(C.c_int32)),
        ("n_quads", C.c_int64),
        ("quad_quv", C.POINTER(C.c_float)),
        ("quad_mat", C.POINTER(C.c_int32)),
        ("n_spheres", C.c_int64),
        ("sphere", C.POINTER(C.c_float)),
        ("sphere_mat", C.POINTER(C.c_int32)),
        ("n_mats", C.c_int32),
        ("mats", C.POINTER(RtMaterial)),
        ("n_lights", C.c_int32),
        ("light_prims", C.POINTER(C.c_int32)),
        ("bg", RtBackground),
        ("spectral_range", C.c_int32),
        ("n_media", C.c_int32),
        ("media", C.POINTER(RtMedium)),
        ("n_convex", C.c_int64),
        ("convex", C.POINTER(RtConvex)),
        ("convex_planes", C.POINTER(C.c_float)),
        ("n_shapes", C.c_int64),
        ("shapes", C.POINTER(RtShape)),
        ("n_textures", C.c_int32),
        ("textures", C.POINTER(RtTexture)),
        ("tri_uv", C.POINTER(C.c_float)),
        ("tri_tangent", C.POINTER(C.c_float)),
        ("bvh_builder", C.c_int32),
    ]


RT_BVH_DEVICE = 0
RT_BVH_HOST = 1


class RtCamera(C.Structure):
    _fields_ = [
        ("origin", F3),
        ("lower_left", F3),
        ("horizontal", F3),
        ("vertical", F3),
        ("u", F3),
        ("v", F3),
        ("lens_radius", C.c_float),
        ("aperture_blades", C.c_int32),
    ]


RT_TONEMAP_AGX = 0
RT_TONEMAP_ACES = 1


class RtDevelopParams(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("exposure", C.c_float),
        ("tonemapper", C.c_int32),
        ("vignette", C.c_float),
        ("distortion", C.c_float),
    ]


class RtTuning(C.Structure):
    """RtTuning (include/rt_api.h): path-pool capacity, launch grids and the
    device loops' limits (0 = built-in)."""
    _fields_ = [("max_paths", C.c_uint32), ("trace_blocks_per_sm", C.c_uint32), ("shade_blocks_per_sm", C.c_uint32),
                ("max_iterations", C.c_uint32), ("stack_limit", C.c_uint32), ("stack_ring", C.c_uint32),
                ("node_format", C.c_uint32), ("graph", C.c_uint32)]


class RtGuideParams(C.Structure):
    """RtGuideParams (include/rt_api.h): the path-guiding network's set-up."""
    _fields_ = [
        ("domain_min", C.c_float * 3),
        ("domain_max", C.c_float * 3),
        ("learning_rate", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("epsilon", C.c_float),
        ("batch", C.c_uint32),
        ("steps_per_pass", C.c_uint32),
        ("record_capacity", C.c_uint32),
        ("min_resolution", C.c_uint32),
        ("level_scale", C.c_float),
        ("alpha_max", C.c_float),
        ("log_kappa_max", C.c_float),
        ("seed", C.c_uint64),
    ]


RT_GUIDE_OFF, RT_GUIDE_SAMPLE, RT_GUIDE_TRAIN = 0, 1, 2
RT_GUIDE_PARAMS = 16792576
GUIDE_N_MLP = 15360


class RtPassParams(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("sample_idx", C.c_uint32),
        ("n_samples", C.c_uint32),
        ("strata", C.c_uint32),
        ("max_depth", C.c_uint32),
        ("hero_count", C.c_uint32),
        ("use_frame_time", C.c_uint32),
        ("t0", C.c_float),
        ("t1", C.c_float),
        ("bg_scale", C.c_float),
        ("seed", C.c_uint64),
    ]


class RtBatchJob(C.Structure):
    """RtBatchJob (include/rt_api.h): one request of a packed batch."""
    _fields_ = [("cam", RtCamera), ("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("strata", C.c_uint32), ("sample_idx", C.c_uint32), ("pad", C.c_uint32), ("seed", C.c_uint64)]


class RtHit(C.Structure):
    _fields_ = [("prim", C.c_int32), ("t", C.c_float), ("b1", C.c_float), ("b2", C.c_float)]


def fptr(a):
    """Pointer to a contiguous float32 numpy array (None → NULL)."""
    if a is None:
        return C.POINTER(C.c_float)()
    return a.ctypes.data_as(C.POINTER(C.c_float))


def iptr(a):
    if a is None:
        return C.POINTER(C.c_int32)()
    return a.ctypes.data_as(C.POINTER(C.c_int32))


RT_EMIT_DISK, RT_EMIT_QUAD, RT_EMIT_SUN, RT_EMIT_LIGHT = 0, 1, 2, 3
RT_NODES_FULL, RT_NODES_QUANTISED, RT_NODES_WIDE4 = 0, 1, 2
RT_MAX_EMITTERS = 8


class RtPhotonEmitter(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("dir", F3),
        ("color", F3),
        ("corner", F3),
        ("u", F3),
        ("v", F3),
        ("n_photons", C.c_uint32),
        ("light", C.c_int32),
        ("target", C.c_float * 4),
    ]


class RtPhotonParams(C.Structure):
    _fields_ = [
        ("n_emitters", C.c_int32),
        ("emitters", RtPhotonEmitter * RT_MAX_EMITTERS),
        ("gather_radius", C.c_float),
        ("knn_k", C.c_uint32),
        ("seed", C.c_uint64),
        ("first_photon", C.c_uint32),
        ("shard_photons", C.c_uint32),
    ]
