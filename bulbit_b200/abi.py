"""ctypes mirror of the C ABI declared in include/bbg.h.

Plain structure and enum definitions only; loading the shared library is done
by bulbit_b200.lib. Field order and types follow the header one for one.
"""
import ctypes as C

BBG_OK = 0
BBG_ERR_INVALID_ARG = 1
BBG_ERR_OOM = 2
BBG_ERR_TIMEOUT = 3
BBG_ERR_QUEUE_OVERFLOW = 4
BBG_ERR_STACK_OVERFLOW = 5
BBG_ERR_CUDA = 6
BBG_ERR_BAD_BVH = 7
BBG_ERR_UNSUPPORTED = 8
BBG_ERR_NO_DEVICE = 9

STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "TIMEOUT", 4: "QUEUE_OVERFLOW",
    5: "STACK_OVERFLOW", 6: "CUDA", 7: "BAD_BVH", 8: "UNSUPPORTED", 9: "NO_DEVICE",
}

BBG_MEM_HOST = 0
BBG_MEM_DEVICE = 1

BBG_PRIM_TRIANGLE = 0
BBG_PRIM_SPHERE = 1

BBG_MAT_NONE = -1
BBG_MAT_DIFFUSE = 0
BBG_MAT_CONDUCTOR = 1
BBG_MAT_DIELECTRIC = 2
BBG_MAT_METALLIC_ROUGHNESS = 3

BBG_TRAVERSAL_ORDERED = 0
BBG_TRAVERSAL_REFERENCE = 1
BBG_TRAVERSAL_WIDE = 2
BBG_SHADE_SORTED = 0
BBG_SHADE_QUEUE = 1

BBG_FILTER_BOX = 0
BBG_FILTER_TENT = 1
BBG_FILTER_GAUSSIAN = 2

BBG_SAMPLER_INDEPENDENT = 0
BBG_SAMPLER_STRATIFIED = 1

BBG_LIGHT_POINT = 0
BBG_LIGHT_SPOT = 1
BBG_LIGHT_UNIFORM_INFINITE = 2
BBG_LIGHT_DIFFUSE_AREA = 3

f3 = C.c_float * 3


class BvhNode(C.Structure):
    _fields_ = [("bmin", f3), ("bmax", f3), ("offset", C.c_int32),
                ("count", C.c_uint16), ("axis", C.c_uint8), ("pad", C.c_uint8)]


class Bvh(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("nodes", C.c_void_p),
                ("n_slots", C.c_int32), ("slot_prims", C.c_void_p)]


class Sphere(C.Structure):
    _fields_ = [("p", f3), ("q", C.c_float * 4), ("s", f3), ("radius", C.c_float)]


class Geometry(C.Structure):
    _fields_ = [("n_vertices", C.c_int32), ("positions", C.c_void_p), ("normals", C.c_void_p),
                ("tangents", C.c_void_p), ("uvs", C.c_void_p),
                ("n_triangles", C.c_int32), ("tri_indices", C.c_void_p),
                ("n_spheres", C.c_int32), ("spheres", C.c_void_p),
                ("n_prims", C.c_int32), ("prim_kind", C.c_void_p), ("prim_index", C.c_void_p)]


class Ray(C.Structure):
    _fields_ = [("o", f3), ("d", f3), ("t_min", C.c_float), ("t_max", C.c_float)]


class Hit(C.Structure):
    _fields_ = [("prim", C.c_int32), ("t", C.c_float), ("u", C.c_float), ("v", C.c_float)]


class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("conductor_from_r", C.c_int32), ("reflectance", f3),
                ("eta", f3), ("k", f3), ("roughness", C.c_float * 2), ("metallic", C.c_float),
                ("energy_compensation", C.c_int32)]


class Light(C.Structure):
    _fields_ = [("type", C.c_int32), ("prim", C.c_int32), ("two_sided", C.c_int32),
                ("position", f3), ("direction", f3), ("intensity", f3), ("scale", C.c_float),
                ("angle_max", C.c_float), ("angle_falloff_start", C.c_float)]


class CameraSpec(C.Structure):
    _fields_ = [("position", f3), ("target", f3), ("up", f3), ("vfov_deg", C.c_float),
                ("aperture_radius", C.c_float), ("focus_distance", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32), ("filter_extent", C.c_float),
                ("filter_type", C.c_int32), ("filter_sigma", C.c_float)]


class Camera(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("origin", f3), ("lower_left", f3),
                ("horizontal", f3), ("vertical", f3), ("u", f3), ("v", f3),
                ("lens_radius", C.c_float), ("filter_extent", C.c_float),
                ("filter_type", C.c_int32), ("filter_sigma", C.c_float)]


class RenderParams(C.Structure):
    _fields_ = [("spp", C.c_int32), ("seed", C.c_int32), ("wave_paths", C.c_int64),
                ("use_graph", C.c_int32), ("light_alias", C.c_int32), ("guide", C.c_void_p),
                ("guide_train", C.c_int32), ("guide_batch", C.c_int32), ("guide_lr", C.c_float),
                ("guide_select", C.c_float), ("guide_steps", C.c_int32),
                ("sampler", C.c_int32), ("x_samples", C.c_int32), ("jitter", C.c_int32),
                ("shade_order", C.c_int32), ("pass_through_levels", C.c_int32)]


class Tuning(C.Structure):
    _fields_ = [("block", C.c_int32), ("short_stack", C.c_int32), ("wave_paths", C.c_int64),
                ("probe_ms", C.c_double), ("from_cache", C.c_int32)]


class Film(C.Structure):
    _fields_ = [("rgb_sum", C.c_void_p), ("count", C.c_void_p), ("moments", C.c_void_p),
                ("path_L", C.c_void_p)]


class RenderStats(C.Structure):
    _fields_ = [("paths", C.c_int64), ("closest_rays", C.c_int64), ("shadow_rays", C.c_int64),
                ("device_ms", C.c_double)]


# (name, restype, argtypes) of every exported entry point of include/bbg.h.
P = C.c_void_p
I32, I64 = C.c_int32, C.c_int64
EXPORTS = [
    ("bbg_bvh_build", I32, [P, I32, P, P, P]),
    ("bbg_prim_aabbs", I32, [P, P]),
    ("bbg_accel_create", I32, [P, P, P]),
    ("bbg_accel_create_device_build", I32, [P, P]),
    ("bbg_accel_create_device_sah", I32, [P, P]),
    ("bbg_accel_destroy", I32, [P]),
    ("bbg_accel_bounds", I32, [P, P]),
    ("bbg_accel_export", I32, [P, P, P, P, P]),
    ("bbg_intersect", I32, [P, P, I64, P, I32, P]),
    ("bbg_intersect_any", I32, [P, P, I64, P, I32, P]),
    ("bbg_intersect_submit", I32, [P, P, I64, P, I32]),
    ("bbg_intersect_any_submit", I32, [P, P, I64, P, I32]),
    ("bbg_accel_synchronize", I32, [P]),
    ("bbg_accel_export_wide8", I32, [P, P, P]),
    ("bbg_intersect_static", I32, [P, P, I64, P]),
    ("bbg_accel_set_traversal", I32, [P, I32]),
    ("bbg_accel_set_counting", I32, [P, I32]),
    ("bbg_accel_last_counts", I32, [P, P, P]),
    ("bbg_camera_perspective", I32, [P, P]),
    ("bbg_integrator_create", I32, [P, P, P, I32, P, I32, I32, I32, I32, P]),
    ("bbg_integrator_destroy", I32, [P]),
    ("bbg_integrator_light_pmf", I32, [P, P]),
    ("bbg_render", I32, [P, P, P, P, I32, P]),
    ("bbg_sampler_draws", I32, [I32, I32, I32, I32, I32, P]),
    ("bbg_bsdf_probe", I32, [P, I32, I32, P, P, P, P]),
    ("bbg_ggx_energy_tables", I32, [P, P]),
    ("bbg_dielectric_energy_tables", I32, [P, P, P, P]),
    ("bbg_accel_create_split", I32, [P, C.c_float, P]),
    ("bbg_accel_create_device_split", I32, [P, C.c_float, P]),
    ("bbg_split_references", I32, [P, C.c_float, I32, P, P, P]),
    ("bbg_batch_create", I32, [P]),
    ("bbg_batch_destroy", I32, [P]),
    ("bbg_batch_render", I32, [P, I32, P, P, P, P, I32, P]),
    ("bbg_integrator_autotune", I32, [P, P, P, P]),
    ("bbg_integrator_set_tuning", I32, [P, P]),
    ("bbg_batch_autotune", I32, [P, I32, P, P, P, P]),
    ("bbg_guide_create", I32, [P, C.c_uint64, P]),
    ("bbg_guide_destroy", I32, [P]),
    ("bbg_guide_get_params", I32, [P, P]),
    ("bbg_guide_set_params", I32, [P, P]),
    ("bbg_guide_forward", I32, [P, P, I64, P]),
    ("bbg_guide_gradient", I32, [P, P, P, P, I64, P, P]),
    ("bbg_guide_train_step", I32, [P, P, P, P, I64, C.c_float, P]),
    ("bbg_guide_mixture_sample", I32, [P, P, I64, P, P]),
    ("bbg_guide_mixture_pdf", I32, [P, P, I64, P]),
    ("bbg_last_error", C.c_char_p, []),
    ("bbg_version", C.c_char_p, []),
]
