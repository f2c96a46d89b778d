"""ctypes binding of libcolvillea_b200.so (C ABI: include/colvillea_b200.h).

There is no fallback: if the library is missing, loading fails loudly.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcolvillea_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "colvillea_b200.h")

CL_OK, CL_ERR_CUDA, CL_ERR_OOM, CL_ERR_QUEUE_OVERFLOW, CL_ERR_TIMEOUT, CL_ERR_INVALID_ARG, CL_ERR_STATE = range(7)
STATUS_NAMES = {0: "CL_OK", 1: "CL_ERR_CUDA", 2: "CL_ERR_OOM", 3: "CL_ERR_QUEUE_OVERFLOW", 4: "CL_ERR_TIMEOUT",
                5: "CL_ERR_INVALID_ARG", 6: "CL_ERR_STATE"}

CL_INTEGRATOR_DIRECT_LIGHTING = 1
CL_INTEGRATOR_PATH_TRACING = 2

CL_COMPAT_PDF = 1 << 0
CL_COMPAT_FRAME = 1 << 1
CL_COMPAT_ESCAPE = 1 << 2
CL_COMPAT_ALL = CL_COMPAT_PDF | CL_COMPAT_FRAME | CL_COMPAT_ESCAPE
CL_DOME_ALIAS = 1 << 4
CL_FILM_FP64 = 1 << 5
CL_PROFILE_STAGES = 1 << 6
CL_TRACE_STATS = 1 << 7
CL_TWO_LEVEL = 1 << 8

CL_BVH_UPDATE_AUTO, CL_BVH_UPDATE_REFIT, CL_BVH_UPDATE_REBUILD = range(3)

vp = ctypes.c_void_p
u32 = ctypes.c_uint32


class RenderConfig(ctypes.Structure):
    _fields_ = [("max_depth", u32), ("rr_start_depth", u32), ("flags", u32), ("path_slots", u32)]


class MeshDesc(ctypes.Structure):
    _fields_ = [("positions", vp), ("normals", vp), ("tangents", vp), ("uvs", vp), ("num_vertices", u32),
                ("indices", vp), ("num_triangles", u32)]


class InstanceDesc(ctypes.Structure):
    _fields_ = [("mesh_id", u32), ("material_index", u32), ("transform", ctypes.c_float * 12)]


class MaterialDesc(ctypes.Structure):
    _fields_ = [("type", u32), ("reflectance", ctypes.c_float * 3), ("roughness", ctypes.c_float),
                ("interior_ior", ctypes.c_float), ("eta", ctypes.c_float * 3), ("k", ctypes.c_float * 3),
                ("reflectance_texture", u32), ("roughness_texture", u32), ("normal_texture", u32)]


CL_TEXTURE_RGBA8, CL_TEXTURE_RGBA32F = 0, 1


class TextureDesc(ctypes.Structure):
    _fields_ = [("format", u32), ("width", u32), ("height", u32), ("srgb", u32), ("texels", vp)]


class EmitterDesc(ctypes.Structure):
    _fields_ = [("type", u32), ("intensity", ctypes.c_float * 3), ("direction", ctypes.c_float * 3),
                ("angular_radius", ctypes.c_float), ("texels", vp), ("width", u32), ("height", u32)]


class Camera(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_float * 3), ("d00", ctypes.c_float * 3), ("ddu", ctypes.c_float * 3),
                ("ddv", ctypes.c_float * 3)]


class Stats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_uint64), ("rays_closest", ctypes.c_uint64), ("rays_shadow", ctypes.c_uint64),
                ("iteration", u32), ("spp", u32), ("bvh_nodes", u32), ("bvh_depth", u32), ("triangles", u32),
                ("waves", u32), ("ms_bvh_build", ctypes.c_float), ("ms_dome_build", ctypes.c_float),
                ("ms_last_render", ctypes.c_float), ("ms_trace", ctypes.c_float), ("ms_shade", ctypes.c_float),
                ("ms_shadow", ctypes.c_float), ("launches", u32), ("pad", u32), ("trace_nodes", ctypes.c_uint64),
                ("trace_tris", ctypes.c_uint64), ("shadow_nodes", ctypes.c_uint64), ("shadow_tris", ctypes.c_uint64),
                ("last_rays_closest", ctypes.c_uint64), ("last_rays_shadow", ctypes.c_uint64),
                ("ms_bvh_update", ctypes.c_float), ("ms_bvh_refit", ctypes.c_float), ("bvh_refits", u32),
                ("bvh_rebuilds", u32),
                ("bvh_sah", ctypes.c_double), ("bvh_sah_build", ctypes.c_double),
                ("ms_bvh_build_wall", ctypes.c_float), ("ms_bvh_build_alloc", ctypes.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GuideConfig(ctypes.Structure):
    _fields_ = [("log2_table", u32), ("resolutions", u32 * 16), ("n_min", ctypes.c_float), ("n_max", ctypes.c_float),
                ("learning_rate", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("epsilon", ctypes.c_float), ("bsdf_fraction", ctypes.c_float), ("batch", u32),
                ("train_spp", u32), ("class_mask", u32), ("seed", u32), ("learn_selection", u32),
                ("weight_clamp", ctypes.c_float), ("min_depth", u32),
                ("min_alpha", ctypes.c_float)]


class RadianceCacheConfig(ctypes.Structure):
    _fields_ = [("network", GuideConfig), ("prefix_bounces", u32), ("train_log2_fraction", u32), ("train_spp", u32)]


class GuideStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_uint64), ("samples_trained", ctypes.c_uint64), ("records_last", ctypes.c_uint64),
                ("inferred", ctypes.c_uint64), ("last_loss", ctypes.c_double), ("ms_train", ctypes.c_float),
                ("ms_infer", ctypes.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# name -> argtypes (every entry point returns cl_status unless listed in _VOID)
_SIGS = {
    "cl_integrator_create": [u32, u32, u32, ctypes.POINTER(RenderConfig), ctypes.POINTER(vp)],
    "cl_integrator_destroy": [vp],
    "cl_build_meshes": [vp, ctypes.POINTER(MeshDesc), u32],
    "cl_build_instances": [vp, ctypes.POINTER(InstanceDesc), u32],
    "cl_update_mesh_vertices": [vp, u32, vp, vp, vp, u32, u32],
    "cl_get_bvh": [vp, vp, ctypes.c_size_t, vp, ctypes.c_size_t],
    "cl_build_materials": [vp, ctypes.POINTER(MaterialDesc), u32],
    "cl_build_textures": [vp, ctypes.POINTER(TextureDesc), u32],
    "cl_unit_normal_frame": [vp, vp, u32],
    "cl_unit_tc_wait_timeout": [ctypes.POINTER(ctypes.c_uint64)],
    "cl_unit_binary_version": [ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
    "cl_unit_texture_lookup": [ctypes.POINTER(TextureDesc), vp, vp, u32],
    "cl_build_emitters": [vp, ctypes.POINTER(EmitterDesc), u32],
    "cl_update_camera": [vp, ctypes.POINTER(Camera)],
    "cl_render": [vp, u32],
    "cl_readback_film": [vp, vp, ctypes.c_size_t],
    "cl_readback_film_async": [vp, vp, ctypes.c_size_t],
    "cl_readback_wait": [vp],
    "cl_readback_film_stats": [vp, vp, vp, ctypes.c_size_t],
    "cl_resize": [vp, u32, u32],
    "cl_get_film_size": [vp, ctypes.POINTER(u32), ctypes.POINTER(u32)],
    "cl_reset_iteration": [vp],
    "cl_set_iteration": [vp, u32],
    "cl_get_stats": [vp, ctypes.POINTER(Stats)],
    "cl_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "cl_trace_rays": [vp, vp, u32, vp, vp, vp, vp],
    "cl_occluded_rays": [vp, vp, u32, vp],
    "cl_trace_stats": [vp, vp, u32, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)],
    "cl_get_dome_tables": [vp, vp, vp, vp, vp],
    "cl_get_dome_alias_tables": [vp, vp, vp],
    "cl_get_wave_rays": [vp, vp, u32, ctypes.POINTER(ctypes.c_uint32)],
    "cl_integrator_guide_probe": [vp, u32, vp, ctypes.POINTER(ctypes.c_uint32)],
    "cl_dome_alias_sample": [vp, vp, vp, vp, vp, u32],
    "cl_unit_bsdf_eval": [u32, vp, vp, vp, vp, u32],
    "cl_unit_bsdf_pdf": [u32, vp, vp, vp, vp, u32, u32],
    "cl_unit_bsdf_sample": [u32, vp, vp, vp, vp, vp, vp, u32],
    "cl_unit_ggx_eval": [vp, vp, vp, vp, vp, vp, vp, vp, u32],
    "cl_unit_ggx_sample": [vp, vp, vp, vp, u32],
    "cl_unit_fresnel_conductor": [vp, vp, vp, vp, u32],
    "cl_unit_fresnel_dielectric": [vp, vp, vp, vp, u32],
    "cl_unit_warp": [vp, vp, vp, u32],
    "cl_unit_make_frame": [vp, vp, vp, u32],
    "cl_unit_frame": [vp, vp, vp, vp, vp, vp, u32],
    "cl_unit_pcg4d": [vp, vp, u32],
    "cl_unit_sampler_sequence": [vp, u32, u32, vp],
    "cl_unit_dome_sample": [vp, u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, u32],
    "cl_unit_dome_pdf_eval": [vp, u32, u32, vp, vp, vp, vp, vp, u32],
    "cl_unit_directional_sample": [vp, vp, vp, vp, vp, u32],
    "cl_dome_build_tables_noalloc": [vp, u32, u32, vp, vp, vp, vp, vp, vp, vp],
    "cl_guide_default_config": [ctypes.POINTER(GuideConfig)],
    "cl_guide_default_resolutions": [ctypes.c_float, ctypes.c_float, vp],
    "cl_guide_create": [ctypes.POINTER(GuideConfig), ctypes.POINTER(vp)],
    "cl_guide_destroy": [vp],
    "cl_guide_param_count": [vp, ctypes.POINTER(ctypes.c_uint64)],
    "cl_guide_get_resolutions": [vp, vp],
    "cl_guide_set_params": [vp, vp, ctypes.c_uint64],
    "cl_guide_get_params": [vp, vp, ctypes.c_uint64],
    "cl_guide_forward": [vp, vp, u32, vp],
    "cl_guide_gradient": [vp, vp, u32, ctypes.POINTER(ctypes.c_double), vp],
    "cl_guide_train_step": [vp, vp, u32, ctypes.POINTER(ctypes.c_double)],
    "cl_guide_sample": [vp, vp, vp, u32, vp, vp],
    "cl_guide_pdf": [vp, vp, vp, u32, vp],
    "cl_integrator_set_guiding": [vp, ctypes.POINTER(GuideConfig)],
    "cl_integrator_get_guide": [vp, ctypes.POINTER(vp)],
    "cl_integrator_guide_stats": [vp, ctypes.POINTER(GuideStats)],
}
_SIGS.update({
    "cl_radiance_cache_default_config": [ctypes.POINTER(RadianceCacheConfig)],
    "cl_cache_create": [ctypes.POINTER(GuideConfig), ctypes.POINTER(vp)],
    "cl_cache_destroy": [vp],
    "cl_cache_param_count": [vp, ctypes.POINTER(ctypes.c_uint64)],
    "cl_cache_get_resolutions": [vp, vp],
    "cl_cache_set_params": [vp, vp, ctypes.c_uint64],
    "cl_cache_get_params": [vp, vp, ctypes.c_uint64],
    "cl_cache_forward": [vp, vp, u32, vp],
    "cl_cache_gradient": [vp, vp, u32, ctypes.POINTER(ctypes.c_double), vp],
    "cl_cache_train_step": [vp, vp, u32, ctypes.POINTER(ctypes.c_double)],
    "cl_integrator_set_radiance_cache": [vp, ctypes.POINTER(RadianceCacheConfig)],
    "cl_integrator_get_cache": [vp, ctypes.POINTER(vp)],
    "cl_integrator_cache_stats": [vp, ctypes.POINTER(GuideStats)],
})
_SIGS.update({
    "cl_obj_load": [ctypes.c_char_p, ctypes.POINTER(vp)],
    "cl_obj_mesh_count": [vp, ctypes.POINTER(u32)],
    "cl_obj_get_mesh": [vp, u32, ctypes.POINTER(MeshDesc)],
    "cl_obj_free": [vp],
    "cl_image_load_hdr": [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(ctypes.c_float)), ctypes.POINTER(u32),
                          ctypes.POINTER(u32)],
    "cl_image_free": [vp],
    "cl_image_write_pfm": [ctypes.c_char_p, vp, u32, u32],
    "cl_image_read_pfm": [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(ctypes.c_float)), ctypes.POINTER(u32),
                          ctypes.POINTER(u32)],
})
_VOID = {"cl_guide_default_config", "cl_radiance_cache_default_config"}

_lib = None


class ClError(RuntimeError):
    def __init__(self, fn, status, msg):
        super().__init__(f"{fn} -> {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    """The loaded library.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"colvillea_b200 native library missing ({LIB_PATH}); "
                               "build it with `python -m colvillea_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.restype = None if name in _VOID else ctypes.c_int32
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(4096)
    lib().cl_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(fn, status):
    if status != CL_OK:
        raise ClError(fn, status, last_error())


def call(name, *args):
    check(name, getattr(lib(), name)(*args))
