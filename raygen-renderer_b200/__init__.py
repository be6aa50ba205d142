"""raygen-renderer_b200: B200 wavefront path tracer behind RayGen's renderer interface.

Python host mirror of the reference's C++ surface (src/raygen/rayrenderer.h):

* ``RendererSettings``   <- RendererSettings (rayrenderer.h:98-153), same field names
* ``RayRenderer``        <- RayRenderer: ``set_scene`` / ``render`` /
  ``get_render_result`` / ``get_hdr_result`` / ``progress_callback`` / ``cancel``
* ``Scene``              <- a flattened scene description (procedural workloads,
  the reference JSON schema, or caller arrays)

Every call goes through the C ABI of ``librg_b200.so`` (include/raygen_b200.h);
there is no CPU fallback: without the library or a CUDA device the calls fail
with ``RayGenError``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field, fields
from typing import Callable, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librg_b200.so")

RG_OK = 0
RG_ERR_INVALID_ARGUMENT = -1
RG_ERR_NO_SCENE = -2
RG_ERR_UNSUPPORTED = -3
RG_ERR_CUDA = -4
RG_ERR_OUT_OF_MEMORY = -5
RG_ERR_CANCELLED = -6
RG_ERR_DEVICE_STATUS = -7
RG_ERR_IO = -8
RG_ERR_PARSE = -9
RG_ERR_BUSY = -10
RG_ERR_NO_DEVICE = -11

RG_ADAPTIVE_PIXEL = 0
RG_ADAPTIVE_TILE = 1

# occluder predicates of rg_trace_any
PRED_AREA, PRED_POINT, PRED_AO, PRED_ALL, PRED_VOLUME = 0, 1, 2, 3, 4

# medium emission modes and density fields (rg_medium)
RG_EMISSION_CONSTANT, RG_EMISSION_CONE, RG_EMISSION_PATH = 0, 1, 2
RG_DENSITY_NONE, RG_DENSITY_FBM = 0, 1


class RayGenError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rg status {code}: {msg}")
        self.code = code


# ------------------------------------------------------------------ ABI types
class rg_settings(C.Structure):
    _fields_ = [
        ("resolution_width", C.c_int32), ("resolution_height", C.c_int32),
        ("threads", C.c_int32), ("samples", C.c_int32), ("shader_provider", C.c_int32),
        ("enable_antialias", C.c_int32), ("enable_point_light_antialias", C.c_int32),
        ("enable_color_sampling", C.c_int32), ("enable_rendering_postprocess", C.c_int32),
        ("enable_denoise", C.c_int32), ("cull_back_face", C.c_int32),
        ("denoise_levels", C.c_int32),
        ("denoise_sigma_color", C.c_float), ("denoise_sigma_normal", C.c_float),
        ("denoise_sigma_depth", C.c_float), ("denoise_intensity", C.c_float),
        ("firefly_clamp", C.c_float),
        ("enable_adaptive_sampling", C.c_int32), ("adaptive_base_samples", C.c_int32),
        ("adaptive_threshold", C.c_float), ("adaptive_mode", C.c_int32),
        ("bloom_threshold", C.c_float), ("bloom_strength", C.c_float), ("bloom_radius", C.c_float),
        ("bloom_size_aspect", C.c_float), ("bloom_curve", C.c_float),
        ("world_color", C.c_float * 3), ("back_color", C.c_float * 4),
        ("seed", C.c_uint32), ("max_depth", C.c_int32), ("rr_depth", C.c_int32),
        ("light_pick_fix", C.c_int32), ("paths_per_wave", C.c_int32), ("bvh_bins", C.c_int32),
        ("bvh_width", C.c_int32),
    ]


class rg_material(C.Structure):
    _fields_ = [
        ("color", C.c_float * 3),
        ("diffuse", C.c_float), ("glossy", C.c_float), ("roughness", C.c_float),
        ("transparency", C.c_float), ("refraction", C.c_float), ("refraction_ratio", C.c_float),
        ("chroma_dispersion", C.c_float), ("metallic", C.c_float), ("anisotropy", C.c_float),
        ("aniso_rotation", C.c_float), ("emission", C.c_float), ("spot_range", C.c_float),
        ("texture", C.c_int32), ("tex_tiling", C.c_float * 2),
    ]


class rg_medium_path_point(C.Structure):
    _fields_ = [("p", C.c_float * 3), ("radius", C.c_float), ("t", C.c_float)]


class rg_medium(C.Structure):
    _fields_ = [("sigma_a", C.c_float * 3), ("sigma_s", C.c_float * 3), ("sigma_e", C.c_float * 3),
                ("g", C.c_float), ("density", C.c_float),
                ("emission_mode", C.c_int32),
                ("cone_origin", C.c_float * 3), ("cone_axis", C.c_float * 3),
                ("cone_length", C.c_float), ("cone_radius", C.c_float),
                ("cone_inner", C.c_float * 3), ("cone_outer", C.c_float * 3),
                ("cone_intensity", C.c_float), ("cone_peak_axial", C.c_float), ("cone_peak_sharpness", C.c_float),
                ("cone_emission_samples", C.c_int32),
                ("num_path_points", C.c_int32), ("path_points", C.POINTER(rg_medium_path_point)),
                ("path_inner", C.c_float * 3), ("path_outer", C.c_float * 3),
                ("path_intensity", C.c_float), ("path_falloff_power", C.c_float),
                ("path_emission_samples", C.c_int32),
                ("density_field", C.c_int32), ("noise_frequency", C.c_float), ("noise_octaves", C.c_int32),
                ("noise_gain", C.c_float), ("noise_lacunarity", C.c_float), ("noise_amplitude", C.c_float),
                ("noise_bias", C.c_float), ("noise_offset", C.c_float * 3),
                ("heat_haze", C.c_int32), ("ior_amplitude", C.c_float), ("ior_frequency", C.c_float),
                ("ior_octaves", C.c_int32), ("ior_gain", C.c_float), ("ior_lacunarity", C.c_float),
                ("ior_march_steps", C.c_int32), ("ior_offset", C.c_float * 3), ("ior_falloff", C.c_float)]


class rg_object(C.Structure):
    _fields_ = [("material", C.c_int32), ("interior_medium", C.c_int32), ("location", C.c_float * 3)]


class rg_point_light(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("normal", C.c_float * 3), ("material", C.c_int32)]


class rg_camera(C.Structure):
    _fields_ = [
        ("location", C.c_float * 3), ("angle", C.c_float * 3), ("field_of_view", C.c_float),
        ("view_near", C.c_float), ("view_far", C.c_float), ("depth_of_field", C.c_float),
        ("aperture", C.c_float), ("aperture_blades", C.c_int32), ("aperture_rotation", C.c_float),
        ("exposure", C.c_float),
    ]


class rg_texture(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("is_hdr", C.c_int32),
                ("rgba", C.POINTER(C.c_float))]


class rg_scene_desc(C.Structure):
    _fields_ = [
        ("num_triangles", C.c_int32), ("positions", C.POINTER(C.c_float)),
        ("normals", C.POINTER(C.c_float)), ("uvs", C.POINTER(C.c_float)),
        ("tri_mesh", C.POINTER(C.c_int32)), ("num_meshes", C.c_int32),
        ("mesh_object", C.POINTER(C.c_int32)), ("num_objects", C.c_int32),
        ("objects", C.POINTER(rg_object)), ("num_materials", C.c_int32),
        ("materials", C.POINTER(rg_material)), ("num_media", C.c_int32),
        ("media", C.POINTER(rg_medium)), ("global_medium", C.c_int32),
        ("num_point_lights", C.c_int32), ("point_lights", C.POINTER(rg_point_light)),
        ("num_textures", C.c_int32), ("textures", C.POINTER(rg_texture)),
        ("camera", rg_camera),
        ("has_envmap", C.c_int32), ("envmap_texture", C.c_int32),
        ("envmap_intensity", C.c_float), ("envmap_rotation", C.c_float),
        ("envmap_cube", C.c_int32), ("envmap_cube_faces", C.c_int32 * 6),
    ]


class rg_stats(C.Structure):
    _fields_ = [
        ("trace_ms", C.c_double), ("post_ms", C.c_double), ("build_ms", C.c_double),
        ("samples", C.c_uint64), ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
        ("nodes_visited", C.c_uint64), ("tris_tested", C.c_uint64),
        ("shadow_nodes_visited", C.c_uint64), ("shadow_tris_tested", C.c_uint64),
        ("extend_ms", C.c_double), ("shade_ms", C.c_double), ("connect_ms", C.c_double),
        ("bvh_nodes", C.c_int32), ("waves", C.c_int32), ("kernel_launches", C.c_int32),
        ("device_error", C.c_int32), ("host_setup_ms", C.c_double), ("host_total_ms", C.c_double),
    ]


class rg_server_config(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_resident_jobs", C.c_int32),
                ("paths_per_wave", C.c_int32), ("max_depth_cap", C.c_int32),
                ("shade_blocks_per_sm", C.c_int32), ("trace_blocks_per_sm", C.c_int32), ("wave_fill", C.c_int32)]


class rg_job_desc(C.Structure):
    _fields_ = [("scene", C.POINTER(rg_scene_desc)), ("width", C.c_int32), ("height", C.c_int32),
                ("samples", C.c_int32), ("max_depth", C.c_int32), ("rr_depth", C.c_int32),
                ("seed", C.c_uint32), ("denoise", C.c_int32)]


class rg_job_status(C.Structure):
    _fields_ = [("state", C.c_int32), ("error", C.c_int32), ("submit_ms", C.c_double), ("start_ms", C.c_double),
                ("done_ms", C.c_double), ("latency_ms", C.c_double), ("samples_issued", C.c_int64),
                ("samples_total", C.c_int64)]


class rg_server_stats(C.Structure):
    _fields_ = [("jobs_done", C.c_int64), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("max_ms", C.c_double), ("images_per_s", C.c_double), ("samples_done", C.c_uint64),
                ("device_ms", C.c_double), ("waves", C.c_int64), ("resident_peak", C.c_int32),
                ("pending", C.c_int32), ("bytes_peak", C.c_uint64)]


RG_JOB_QUEUED, RG_JOB_RESIDENT, RG_JOB_DONE, RG_JOB_FAILED = 0, 1, 2, 3

PROGRESS_FN = C.CFUNCTYPE(None, C.c_float, C.c_void_p)

_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load librg_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RayGenError(RG_ERR_IO, f"{path} is missing: run __graft_entry__.build()")
    lib = C.CDLL(path)
    P = C.POINTER
    sig = {
        "rg_settings_default": (None, [P(rg_settings)]),
        "rg_create": (C.c_int, [P(rg_settings), P(C.c_void_p)]),
        "rg_destroy": (C.c_int, [C.c_void_p]),
        "rg_update_settings": (C.c_int, [C.c_void_p, P(rg_settings)]),
        "rg_set_scene": (C.c_int, [C.c_void_p, P(rg_scene_desc)]),
        "rg_render": (C.c_int, [C.c_void_p]),
        "rg_set_progress_cb": (C.c_int, [C.c_void_p, PROGRESS_FN, C.c_void_p]),
        "rg_cancel": (C.c_int, [C.c_void_p]),
        "rg_render_async": (C.c_int, [C.c_void_p, P(C.c_void_p)]),
        "rg_poll": (C.c_int, [C.c_void_p, P(C.c_int32), P(C.c_float)]),
        "rg_wait": (C.c_int, [C.c_void_p, C.c_double]),
        "rg_job_free": (C.c_int, [C.c_void_p]),
        "rg_get_hdr": (C.c_int, [C.c_void_p, P(C.c_float), C.c_size_t]),
        "rg_get_ldr": (C.c_int, [C.c_void_p, P(C.c_float), C.c_size_t]),
        "rg_get_aovs": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), P(C.c_float), C.c_size_t]),
        "rg_get_sample_counts": (C.c_int, [C.c_void_p, P(C.c_int32), C.c_size_t]),
        "rg_get_stats": (C.c_int, [C.c_void_p, P(rg_stats)]),
        "rg_last_error": (C.c_char_p, []),
        "rg_version": (C.c_char_p, []),
        "rg_trace_closest": (C.c_int, [C.c_void_p, P(C.c_float), C.c_int32, P(C.c_float), P(C.c_int32)]),
        "rg_trace_any": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), C.c_int32, C.c_int32, P(C.c_uint8)]),
        "rg_get_view_matrix": (C.c_int, [C.c_void_p, P(C.c_float)]),
        "rg_denoise_atrous": (C.c_int, [C.c_int32, C.c_int32, P(C.c_float), P(C.c_float), P(C.c_float),
                                        P(C.c_float), P(C.c_float), C.c_int32, C.c_float, C.c_float,
                                        C.c_float, C.c_float, P(C.c_float)]),
        "rg_tonemap": (C.c_int, [C.c_int32, C.c_int32, P(C.c_float), P(C.c_float)]),
        "rg_bloom": (C.c_int, [C.c_int32, C.c_int32, P(C.c_float)] + [C.c_float] * 5 + [P(C.c_float)]),
        "rg_save_image": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, P(C.c_float)]),
        "rg_load_image": (C.c_int, [C.c_char_p, P(C.c_int32), P(C.c_int32), P(C.c_int32), P(C.c_float), C.c_size_t]),
        "rg_tc_gemm_bf16": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, P(C.c_uint16), P(C.c_uint16), P(C.c_float)]),
        "rg_denoiser_num_params": (C.c_int32, []),
        "rg_denoiser_create": (C.c_int, [C.c_uint32, P(C.c_void_p)]),
        "rg_denoiser_destroy": (C.c_int, [C.c_void_p]),
        "rg_denoiser_get_params": (C.c_int, [C.c_void_p, P(C.c_float), C.c_size_t]),
        "rg_denoiser_set_params": (C.c_int, [C.c_void_p, P(C.c_float), C.c_size_t]),
        "rg_denoiser_add_example": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32] + [P(C.c_float)] * 4
                                    + [C.c_float, P(C.c_float)]),
        "rg_denoiser_clear_examples": (C.c_int, [C.c_void_p]),
        "rg_denoiser_train": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_float, P(C.c_float)]),
        "rg_denoiser_gradients": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32] + [P(C.c_float)] * 4
                                  + [C.c_float] + [P(C.c_float)] * 3),
        "rg_denoiser_apply": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32] + [P(C.c_float)] * 4
                              + [C.c_float, P(C.c_float)]),
        "rg_set_denoiser": (C.c_int, [C.c_void_p, C.c_void_p]),
        "rg_denoiser_timing": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float)]),
        "rg_server_set_denoiser": (C.c_int, [C.c_void_p, C.c_void_p]),
        "rg_server_autotune": (C.c_int, [P(rg_settings), P(rg_job_desc), C.c_int32, P(rg_server_config),
                                         P(C.c_double)]),
        "rg_reapply_postprocess": (C.c_int, [C.c_void_p]),
        "rg_medium_defaults": (None, [P(rg_medium)]),
        "rg_medium_eval": (C.c_int, [C.c_void_p, C.c_int32, P(C.c_float), C.c_int32, P(C.c_float)]),
        "rg_probe_sampling": (C.c_int, [C.c_int32, P(C.c_float), C.c_int32, P(C.c_float)]),
        "rg_debug_set_traversal_step_cap": (C.c_int, [C.c_int32]),
        "rg_debug_set_tc_wait_limit": (C.c_int, [C.c_uint32]),
        "rg_medium_bend": (C.c_int, [C.c_void_p, C.c_int32, P(C.c_float), C.c_int32, P(C.c_float)]),
        "rg_scene_builtin": (C.c_int, [C.c_int32, C.c_uint32, P(C.c_int32), C.c_int32, P(P(rg_scene_desc))]),
        "rg_scene_free": (C.c_int, [P(rg_scene_desc)]),
        "rg_load_scene_json": (C.c_int, [C.c_char_p, P(P(rg_scene_desc))]),
        "rg_server_config_default": (None, [P(rg_server_config)]),
        "rg_server_create": (C.c_int, [P(rg_settings), P(rg_server_config), P(C.c_void_p)]),
        "rg_server_submit": (C.c_int, [C.c_void_p, P(rg_job_desc), P(C.c_int64)]),
        "rg_server_poll": (C.c_int, [C.c_void_p, C.c_int64, P(rg_job_status)]),
        "rg_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.c_double]),
        "rg_server_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
        "rg_server_add_scene": (C.c_int, [C.c_void_p, P(rg_scene_desc), P(C.c_int64)]),
        "rg_server_submit_scene": (C.c_int, [C.c_void_p, C.c_int64, P(rg_job_desc), P(C.c_int64)]),
        "rg_server_remove_scene": (C.c_int, [C.c_void_p, C.c_int64]),
        "rg_server_get_result": (C.c_int, [C.c_void_p, C.c_int64, P(C.c_float), C.c_size_t, C.c_int32]),
        "rg_server_snapshot": (C.c_int, [C.c_void_p, C.c_int64, P(C.c_float), C.c_size_t, C.c_double]),
        "rg_server_get_stats": (C.c_int, [C.c_void_p, P(rg_server_stats)]),
        "rg_server_destroy": (C.c_int, [C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def medium(path_points=(), **fields) -> rg_medium:
    """An rg_medium with the reference's defaults (rg_medium_defaults) and the
    given fields (sequences for the vector fields).  path_points: sequence of
    (xyz, radius, t); the array is kept alive by the returned structure."""
    m = rg_medium()
    load_library().rg_medium_defaults(C.byref(m))
    for k, v in fields.items():
        if not hasattr(m, k):
            raise AttributeError(f"rg_medium has no field {k}")
        cur = getattr(m, k)
        if isinstance(cur, C.Array):
            for i, x in enumerate(v):
                cur[i] = x
        else:
            setattr(m, k, v)
    if path_points:
        arr = (rg_medium_path_point * len(path_points))()
        for i, (p, radius, t) in enumerate(path_points):
            arr[i].p[:] = [float(c) for c in p]
            arr[i].radius = float(radius)
            arr[i].t = float(t)
        m.num_path_points = len(path_points)
        m.path_points = arr
        m._keep = arr
    return m


def _check(code: int) -> None:
    if code != RG_OK:
        msg = load_library().rg_last_error()
        raise RayGenError(code, msg.decode() if msg else "")


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def version() -> str:
    return load_library().rg_version().decode()


# --------------------------------------------------------------- settings
@dataclass
class RendererSettings:
    """Field-for-field mirror of the reference RendererSettings (rayrenderer.h:98-153)."""
    resolutionWidth: int = 800
    resolutionHeight: int = 600
    threads: int = 1
    samples: int = 100
    shaderProvider: int = 5
    enableAntialias: bool = True
    enablePointLightAntialias: bool = True
    enableColorSampling: bool = True
    enableRenderingPostProcess: bool = False
    enableDenoise: bool = False
    cullBackFace: bool = False
    denoiseLevels: int = 5
    denoiseSigmaColor: float = 0.4
    denoiseSigmaNormal: float = 128.0
    denoiseSigmaDepth: float = 0.1
    denoiseIntensity: float = 1.0
    fireflyClamp: float = 10.0
    enableAdaptiveSampling: bool = False
    adaptiveBaseSamples: int = 4
    adaptiveThreshold: float = 0.02
    adaptiveMode: int = RG_ADAPTIVE_TILE
    bloomThreshold: float = 1.0
    bloomStrength: float = 1.0
    bloomRadius: float = 0.03
    bloomSizeAspect: float = 0.15
    bloomCurve: float = 1.0
    worldColor: tuple = (0.1, 0.095, 0.09)
    backColor: tuple = (0.2, 0.19, 0.18, 0.0)
    # tracer knobs
    seed: int = 1
    maxDepth: int = 32
    rrDepth: int = 3
    lightPickFix: bool = False
    pathsPerWave: int = 0
    bvhBins: int = 32
    bvhWidth: int = 8

    _MAP = {
        "resolutionWidth": "resolution_width", "resolutionHeight": "resolution_height",
        "threads": "threads", "samples": "samples", "shaderProvider": "shader_provider",
        "enableAntialias": "enable_antialias", "enablePointLightAntialias": "enable_point_light_antialias",
        "enableColorSampling": "enable_color_sampling",
        "enableRenderingPostProcess": "enable_rendering_postprocess", "enableDenoise": "enable_denoise",
        "cullBackFace": "cull_back_face", "denoiseLevels": "denoise_levels",
        "denoiseSigmaColor": "denoise_sigma_color", "denoiseSigmaNormal": "denoise_sigma_normal",
        "denoiseSigmaDepth": "denoise_sigma_depth", "denoiseIntensity": "denoise_intensity",
        "fireflyClamp": "firefly_clamp", "enableAdaptiveSampling": "enable_adaptive_sampling",
        "adaptiveBaseSamples": "adaptive_base_samples", "adaptiveThreshold": "adaptive_threshold",
        "adaptiveMode": "adaptive_mode", "bloomThreshold": "bloom_threshold",
        "bloomStrength": "bloom_strength", "bloomRadius": "bloom_radius",
        "bloomSizeAspect": "bloom_size_aspect", "bloomCurve": "bloom_curve",
        "seed": "seed", "maxDepth": "max_depth", "rrDepth": "rr_depth",
        "lightPickFix": "light_pick_fix", "pathsPerWave": "paths_per_wave", "bvhBins": "bvh_bins",
        "bvhWidth": "bvh_width",
    }

    def to_c(self) -> rg_settings:
        s = rg_settings()
        for k, v in self._MAP.items():
            val = getattr(self, k)
            setattr(s, v, int(val) if isinstance(val, bool) else val)
        for i in range(3):
            s.world_color[i] = self.worldColor[i]
        for i in range(4):
            s.back_color[i] = self.backColor[i]
        return s


def default_settings_c() -> rg_settings:
    s = rg_settings()
    load_library().rg_settings_default(C.byref(s))
    return s


# ------------------------------------------------------------------ scenes
class Scene:
    """A flattened scene description (rg_scene_desc) owned by the library or by Python arrays."""

    def __init__(self, desc_ptr, owned_by_lib: bool, keepalive=None):
        self._ptr = desc_ptr
        self._owned = owned_by_lib
        self._keep = keepalive

    @property
    def desc(self) -> rg_scene_desc:
        """The rg_scene_desc; it keeps this Scene (and so the memory it points into) alive."""
        c = self._ptr.contents
        c._owner = self
        return c

    @property
    def ptr(self):
        return self._ptr

    @classmethod
    def builtin(cls, kind: int, seed: int = 1, iparams=None) -> "Scene":
        lib = load_library()
        out = C.POINTER(rg_scene_desc)()
        ip = (C.c_int32 * len(iparams))(*iparams) if iparams else None
        _check(lib.rg_scene_builtin(kind, seed, ip, len(iparams) if iparams else 0, C.byref(out)))
        return cls(out, True)

    @classmethod
    def from_json(cls, path: str) -> "Scene":
        lib = load_library()
        out = C.POINTER(rg_scene_desc)()
        _check(lib.rg_load_scene_json(path.encode(), C.byref(out)))
        return cls(out, True)

    @classmethod
    def from_arrays(cls, positions, normals, tri_mesh, mesh_object, objects, materials, camera,
                    media=(), global_medium=-1, point_lights=(), uvs=None, textures=(),
                    envmap=None, envmap_intensity=1.0, envmap_rotation=0.0, envmap_cube=None) -> "Scene":
        """Scene from arrays.  textures: sequence of (H x W x 4 float32 RGBA, is_hdr);
        envmap: index of the equirectangular environment texture (None = no environment);
        envmap_cube: texture indices of six square cubemap faces (+X -X +Y -Y +Z -Z)."""
        pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 9)
        nrm = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 9)
        tm = np.ascontiguousarray(tri_mesh, dtype=np.int32)
        mo = np.ascontiguousarray(mesh_object, dtype=np.int32)
        objs = (rg_object * max(1, len(objects)))(*objects)
        mats = (rg_material * max(1, len(materials)))(*materials)
        meds = (rg_medium * max(1, len(media)))(*media)
        pls = (rg_point_light * max(1, len(point_lights)))(*point_lights)
        d = rg_scene_desc()
        d.num_triangles = pos.shape[0]
        d.positions = _fptr(pos)
        d.normals = _fptr(nrm)
        uv = None
        if uvs is not None:
            uv = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 6)
            d.uvs = _fptr(uv)
        d.tri_mesh = tm.ctypes.data_as(C.POINTER(C.c_int32))
        d.num_meshes = len(mo)
        d.mesh_object = mo.ctypes.data_as(C.POINTER(C.c_int32))
        d.num_objects = len(objects)
        d.objects = objs
        d.num_materials = len(materials)
        d.materials = mats
        d.num_media = len(media)
        d.media = meds
        d.global_medium = global_medium
        d.num_point_lights = len(point_lights)
        d.point_lights = pls
        d.camera = camera
        texs = []
        if textures:
            tarr = (rg_texture * len(textures))()
            for i, (img, is_hdr) in enumerate(textures):
                a = np.ascontiguousarray(img, dtype=np.float32)
                if a.ndim != 3 or a.shape[2] != 4:
                    raise ValueError("textures must be H x W x 4 RGBA arrays")
                texs.append(a)
                tarr[i].height, tarr[i].width = a.shape[0], a.shape[1]
                tarr[i].is_hdr = int(bool(is_hdr))
                tarr[i].rgba = _fptr(a)
            d.num_textures = len(textures)
            d.textures = tarr
            texs.append(tarr)
        if envmap is not None:
            d.has_envmap = 1
            d.envmap_texture = int(envmap)
        if envmap_cube is not None:  # texture indices of the faces +X -X +Y -Y +Z -Z
            d.envmap_cube = 1
            d.envmap_cube_faces[:] = [int(i) for i in envmap_cube]
        if envmap is not None or envmap_cube is not None:
            d.envmap_intensity = float(envmap_intensity)
            d.envmap_rotation = float(envmap_rotation)
        keep = (pos, nrm, tm, mo, objs, mats, meds, pls, uv, d, texs,
                [getattr(m, "_keep", None) for m in media])
        return cls(C.pointer(d), False, keep)

    def arrays(self):
        """numpy views of the triangle arrays (positions n x 9, normals n x 9, tri_mesh n)."""
        d = self.desc
        n = d.num_triangles
        pos = np.ctypeslib.as_array(d.positions, shape=(n, 9)) if n else np.zeros((0, 9), np.float32)
        nrm = np.ctypeslib.as_array(d.normals, shape=(n, 9)) if n else np.zeros((0, 9), np.float32)
        tm = np.ctypeslib.as_array(d.tri_mesh, shape=(n,)) if n else np.zeros((0,), np.int32)
        return pos, nrm, tm

    def close(self):
        if self._owned and self._ptr:
            load_library().rg_scene_free(self._ptr)
        self._ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- renderer
class RenderJob:
    """An asynchronous render (rg_render_async): poll(), wait(), then the
    renderer's result getters.  The job is freed when it is waited for and
    garbage collected, or by close()."""

    def __init__(self, renderer: "RayRenderer", job: C.c_void_p):
        self._r = renderer
        self._lib = renderer._lib
        self._job = job

    def poll(self):
        """(done, progress in [0, 1])."""
        done = C.c_int32()
        pr = C.c_float()
        _check(self._lib.rg_poll(self._job, C.byref(done), C.byref(pr)))
        return bool(done.value), float(pr.value)

    def wait(self, timeout_ms: float = -1.0) -> bool:
        """Wait for the render; False on timeout; raises RayGenError if the render failed
        (RG_ERR_CANCELLED after cancel())."""
        rc = self._lib.rg_wait(self._job, float(timeout_ms))
        if rc == RG_ERR_BUSY:
            return False
        _check(rc)
        return True

    def close(self) -> None:
        if self._job:
            self._lib.rg_job_free(self._job)
            self._job = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RayRenderer:
    """Mirror of the reference RayRenderer (rayrenderer.h:199-434) over the device tracer."""

    def __init__(self, settings: Optional[RendererSettings] = None):
        self.settings = settings or RendererSettings()
        self._lib = load_library()
        self._h = C.c_void_p()
        s = self.settings.to_c()
        _check(self._lib.rg_create(C.byref(s), C.byref(self._h)))
        self.progressCallback: Optional[Callable[[float], None]] = None
        self._cb = None
        self._scene: Optional[Scene] = None

    def _sync_settings(self):
        s = self.settings.to_c()
        _check(self._lib.rg_update_settings(self._h, C.byref(s)))

    def set_scene(self, scene: Scene) -> None:
        self._sync_settings()
        _check(self._lib.rg_set_scene(self._h, scene.ptr))
        self._scene = scene

    setScene = set_scene

    def _install_progress(self):
        if self.progressCallback is not None:
            user = self.progressCallback
            self._cb = PROGRESS_FN(lambda p, _u: user(float(p)))
            _check(self._lib.rg_set_progress_cb(self._h, self._cb, None))
        elif self._cb is not None:
            self._cb = None
            _check(self._lib.rg_set_progress_cb(self._h, PROGRESS_FN(0), None))

    def render(self) -> None:
        self._sync_settings()
        self._install_progress()
        _check(self._lib.rg_render(self._h))

    def render_async(self) -> "RenderJob":
        """Start the render on a host thread (the reference's threaded render();
        progressCallback is called from that thread).  Returns a RenderJob."""
        self._sync_settings()
        self._install_progress()
        job = C.c_void_p()
        _check(self._lib.rg_render_async(self._h, C.byref(job)))
        return RenderJob(self, job)

    def cancel(self) -> None:
        _check(self._lib.rg_cancel(self._h))

    def _size(self):
        return self.settings.resolutionHeight, self.settings.resolutionWidth

    def set_denoiser(self, denoiser) -> None:
        """Use a trained Denoiser when enableDenoise is set (None: back to A-Trous)."""
        self._denoiser = denoiser  # keep it alive while attached
        _check(self._lib.rg_set_denoiser(self._h, denoiser._h if denoiser is not None else None))

    def reapply_post_process(self) -> None:
        """RayRenderer::reapplyPostProcess: bloom + tonemap again from the last pre-bloom HDR
        with the current settings (e.g. after changing bloomStrength)."""
        self._sync_settings()
        _check(self._lib.rg_reapply_postprocess(self._h))

    def _result_buffer(self, out):
        h, w = self._size()
        if out is None:
            return np.empty((h, w, 4), np.float32)
        if out.dtype != np.float32 or out.shape != (h, w, 4) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float32 array of shape {(h, w, 4)}")
        return out

    def get_hdr_result(self, out: np.ndarray = None) -> np.ndarray:
        """Linear HDR result (H x W x 4); `out` may be a preallocated (e.g. page-locked) array."""
        out = self._result_buffer(out)
        _check(self._lib.rg_get_hdr(self._h, _fptr(out), out.size))
        return out

    def get_render_result(self, out: np.ndarray = None) -> np.ndarray:
        """Tonemapped result (H x W x 4); `out` may be a preallocated array."""
        out = self._result_buffer(out)
        _check(self._lib.rg_get_ldr(self._h, _fptr(out), out.size))
        return out

    getHdrResult = get_hdr_result
    getRenderResult = get_render_result

    def get_aovs(self):
        h, w = self._size()
        n = np.empty((h, w, 3), np.float32)
        a = np.empty((h, w, 3), np.float32)
        d = np.empty((h, w), np.float32)
        _check(self._lib.rg_get_aovs(self._h, _fptr(n), _fptr(a), _fptr(d), n.size))
        return n, a, d

    def get_sample_counts(self) -> np.ndarray:
        h, w = self._size()
        out = np.empty((h, w), np.int32)
        _check(self._lib.rg_get_sample_counts(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)), out.size))
        return out

    def stats(self) -> dict:
        s = rg_stats()
        _check(self._lib.rg_get_stats(self._h, C.byref(s)))
        return {f[0]: getattr(s, f[0]) for f in rg_stats._fields_}

    def view_matrix(self) -> np.ndarray:
        m = np.empty(16, np.float32)
        _check(self._lib.rg_get_view_matrix(self._h, _fptr(m)))
        return m.reshape(4, 4)

    def trace_closest(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        tuv = np.empty((n, 3), np.float32)
        prim = np.empty(n, np.int32)
        _check(self._lib.rg_trace_closest(self._h, _fptr(rays), n, _fptr(tuv),
                                          prim.ctypes.data_as(C.POINTER(C.c_int32))))
        return tuv, prim

    def trace_any(self, rays: np.ndarray, tmax: np.ndarray, predicate: int = PRED_AREA):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        tmax = np.ascontiguousarray(tmax, dtype=np.float32).reshape(-1)
        n = rays.shape[0]
        out = np.empty(n, np.uint8)
        _check(self._lib.rg_trace_any(self._h, _fptr(rays), _fptr(tmax), n, predicate,
                                      out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out.astype(bool)

    def medium_eval(self, medium: int, points: np.ndarray) -> np.ndarray:
        """Camera-space points n x 3 -> n x 5 (density, emission rgb, ior) of medium `medium`."""
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        out = np.empty((pts.shape[0], 5), np.float32)
        _check(self._lib.rg_medium_eval(self._h, medium, _fptr(pts), pts.shape[0], _fptr(out)))
        return out

    def medium_bend(self, medium: int, rays: np.ndarray) -> np.ndarray:
        """Rays n x 7 (origin, direction, march length) -> bent rays n x 6 (heat haze)."""
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 7)
        out = np.empty((r.shape[0], 6), np.float32)
        _check(self._lib.rg_medium_bend(self._h, medium, _fptr(r), r.shape[0], _fptr(out)))
        return out

    def close(self):
        if self._h:
            self._lib.rg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def denoise_atrous(color, normal, depth, albedo, albedo_alpha, levels=5, sigma_color=0.4,
                   sigma_normal=128.0, sigma_depth=0.1, intensity=1.0) -> np.ndarray:
    """Device A-Trous on host arrays (RayRenderer::denoiseImage, rayrenderer.cpp:2649-2772)."""
    lib = load_library()
    color = np.ascontiguousarray(color, np.float32)
    h, w = color.shape[:2]
    args = [np.ascontiguousarray(a, np.float32) for a in (normal, depth, albedo, albedo_alpha)]
    out = np.empty((h, w, 3), np.float32)
    _check(lib.rg_denoise_atrous(w, h, _fptr(color), _fptr(args[0]), _fptr(args[1]), _fptr(args[2]),
                                 _fptr(args[3]), levels, sigma_color, sigma_normal, sigma_depth,
                                 intensity, _fptr(out)))
    return out


# Output widths of rg_probe_sampling's rows (see the C header for the layouts).
PROBE_OUT_WIDTH = (3, 1, 1, 3, 6, 3, 3, 1, 3, 1, 1)
PROBE_VNDF, PROBE_SMITH, PROBE_SCHLICK, PROBE_REFRACT, PROBE_FRAME, PROBE_COSINE, PROBE_TRIANGLE_POINT, \
    PROBE_LDS, PROBE_PHASE_SAMPLE, PROBE_PHASE_PDF, PROBE_FREE_FLIGHT = range(11)


def probe_sampling(which: int, rows: np.ndarray) -> np.ndarray:
    """Run one of the shade kernel's sampling helpers on the device, one row per input."""
    lib = load_library()
    x = np.ascontiguousarray(rows, np.float32)
    out = np.empty((x.shape[0], PROBE_OUT_WIDTH[which]), np.float32)
    _check(lib.rg_probe_sampling(which, _fptr(x), x.shape[0], _fptr(out)))
    return out


def bloom(hdr_rgba: np.ndarray, threshold=1.0, strength=1.0, radius=0.03, size_aspect=0.15, curve=1.0) -> np.ndarray:
    """Device HDR bloom on a host RGBA image (RayRenderer::applyPostProcess, rayrenderer.cpp:598-696)."""
    lib = load_library()
    hdr = np.ascontiguousarray(hdr_rgba, np.float32)
    h, w = hdr.shape[:2]
    out = np.empty_like(hdr)
    _check(lib.rg_bloom(w, h, _fptr(hdr), threshold, strength, radius, size_aspect, curve, _fptr(out)))
    return out


def save_image(path: str, rgba: np.ndarray) -> None:
    """Write an H x W x 4 float image; the format follows the extension (.hdr .pfm .jpg .png .ppm)."""
    lib = load_library()
    a = np.ascontiguousarray(rgba, np.float32)
    _check(lib.rg_save_image(path.encode(), a.shape[1], a.shape[0], _fptr(a)))


def load_image(path: str):
    """Read an image file as a texture: (H x W x 4 float32, is_hdr).  Radiance .hdr and .pfm
    by name, JPEG and PNG by content; LDR values in [0, 1] as stored (not sRGB-decoded)."""
    lib = load_library()
    w, h, hdr = C.c_int32(), C.c_int32(), C.c_int32()
    _check(lib.rg_load_image(path.encode(), C.byref(w), C.byref(h), C.byref(hdr), None, 0))
    out = np.empty((h.value, w.value, 4), np.float32)
    _check(lib.rg_load_image(path.encode(), C.byref(w), C.byref(h), C.byref(hdr), _fptr(out), out.size))
    return out, bool(hdr.value)


def to_bf16_bits(a: np.ndarray) -> np.ndarray:
    """float32 -> BF16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def tc_gemm_bf16(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """Tensor-core BF16 GEMM (tcgen05, FP32 accumulation): A (M x K) @ B (N x K)^T."""
    lib = load_library()
    a = np.ascontiguousarray(to_bf16_bits(A))
    b = np.ascontiguousarray(to_bf16_bits(B))
    M, K = a.shape
    N = b.shape[0]
    d = np.empty((M, N), np.float32)
    P16 = C.POINTER(C.c_uint16)
    _check(lib.rg_tc_gemm_bf16(M, N, K, a.ctypes.data_as(P16), b.ctypes.data_as(P16), _fptr(d)))
    return d


class Denoiser:
    """Learned denoiser: a kernel-predicting CNN trained and run on the tensor cores.

    Images are H x W (x C) float arrays: noisy / ref RGBA, normal and albedo guides
    (as RayRenderer.get_aovs returns them), depth guide H x W.  Batched calls take
    N x H x W (x C) arrays.  `spp` is the noisy image's samples per pixel, an input
    of the network (its noise level); the renderer and the job server pass their
    per-pixel sample counts themselves."""

    def __init__(self, seed: int = 0, params=None):
        self._lib = load_library()
        h = C.c_void_p()
        _check(self._lib.rg_denoiser_create(int(seed) & 0xFFFFFFFF, C.byref(h)))
        self._h = h
        if params is not None:
            self.params = params

    WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kpcn_weights.bin")

    @classmethod
    def pretrained(cls, path: Optional[str] = None) -> "Denoiser":
        """The network trained by kpcn_train.py on tracer-rendered pairs (shipped weights)."""
        d = cls(seed=0)
        d.load(path or cls.WEIGHTS)
        return d

    @staticmethod
    def num_params() -> int:
        return int(load_library().rg_denoiser_num_params())

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.num_params(), np.float32)
        _check(self._lib.rg_denoiser_get_params(self._h, _fptr(out), out.size))
        return out

    @params.setter
    def params(self, p) -> None:
        a = np.ascontiguousarray(p, np.float32).ravel()
        _check(self._lib.rg_denoiser_set_params(self._h, _fptr(a), a.size))

    def save(self, path: str) -> None:
        self.params.tofile(path)

    def load(self, path: str) -> None:
        self.params = np.fromfile(path, np.float32)

    @staticmethod
    def _inputs(depth, noisy, normal, albedo, *rgba):
        """Contiguous float32 arrays of the shapes the C ABI reads: RGB images get an
        alpha channel of 1; every image must match depth's N x H x W."""
        depth = np.ascontiguousarray(depth, np.float32)
        out = [depth]
        for a, ch in [(noisy, 4), (normal, 3), (albedo, 3)] + [(r, 4) for r in rgba]:
            a = np.asarray(a, np.float32)
            if ch == 4 and a.shape[-1] == 3:
                a = np.concatenate([a, np.ones(a.shape[:-1] + (1,), np.float32)], -1)
            if a.shape != depth.shape + (ch,):
                raise ValueError(f"image of shape {a.shape}: expected {depth.shape + (ch,)}")
            out.append(np.ascontiguousarray(a))
        return out

    def add_example(self, noisy, normal, albedo, depth, ref, spp: float = 8.0) -> None:
        depth, noisy, normal, albedo, ref = self._inputs(depth, noisy, normal, albedo, ref)
        h, w = depth.shape
        _check(self._lib.rg_denoiser_add_example(self._h, w, h, _fptr(noisy), _fptr(normal), _fptr(albedo),
                                                 _fptr(depth), float(spp), _fptr(ref)))

    def clear_examples(self) -> None:
        _check(self._lib.rg_denoiser_clear_examples(self._h))

    def train(self, steps: int, batch: int = 8, lr: float = 1e-3) -> np.ndarray:
        losses = np.zeros(max(1, steps), np.float32)
        _check(self._lib.rg_denoiser_train(self._h, steps, batch, lr, _fptr(losses)))
        return losses[:steps]

    def gradients(self, noisy, normal, albedo, depth, ref, spp: float = 8.0):
        """(loss, gradient) for a batch N x H x W (relMSE against ref)."""
        depth, noisy, normal, albedo, ref = self._inputs(depth, noisy, normal, albedo, ref)
        n, h, w = depth.shape
        loss = np.zeros(1, np.float32)
        grad = np.zeros(self.num_params(), np.float32)
        _check(self._lib.rg_denoiser_gradients(self._h, n, w, h, _fptr(noisy), _fptr(normal), _fptr(albedo),
                                               _fptr(depth), float(spp), _fptr(ref), _fptr(loss), _fptr(grad)))
        return float(loss[0]), grad

    def apply(self, noisy, normal, albedo, depth, spp: float = 8.0) -> np.ndarray:
        depth, noisy, normal, albedo = self._inputs(depth, noisy, normal, albedo)
        h, w = depth.shape
        out = np.empty((h, w, 4), np.float32)
        _check(self._lib.rg_denoiser_apply(self._h, w, h, _fptr(noisy), _fptr(normal), _fptr(albedo), _fptr(depth),
                                           float(spp), _fptr(out)))
        return out

    def timing(self) -> dict:
        """Device ms of the last apply() and of the mean step of the last train()."""
        a, t = C.c_float(), C.c_float()
        _check(self._lib.rg_denoiser_timing(self._h, C.byref(a), C.byref(t)))
        return {"apply_ms": a.value, "train_step_ms": t.value}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.rg_denoiser_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tonemap(hdr_rgba: np.ndarray) -> np.ndarray:
    """Device Reinhard + gamma (RayRenderer::applyTonemapGamma, rayrenderer.cpp:2610-2647)."""
    lib = load_library()
    hdr = np.ascontiguousarray(hdr_rgba, np.float32)
    h, w = hdr.shape[:2]
    out = np.empty_like(hdr)
    _check(lib.rg_tonemap(w, h, _fptr(hdr), _fptr(out)))
    return out


class RenderServer:
    """Resident multi-job server: continuous batching of many render jobs on one GPU.

    Jobs are admitted under an HBM budget; waves mix paths of the resident jobs
    (shared evenly, or with wave_fill=1 filled from as few jobs as possible);
    finished jobs are resolved (optionally denoised) on the device.
    """

    def __init__(self, settings: Optional[RendererSettings] = None, hbm_budget_gb: float = 120.0,
                 max_resident_jobs: int = 256, paths_per_wave: int = 8 << 20, max_depth_cap: int = 10,
                 shade_blocks_per_sm: int = 0, trace_blocks_per_sm: int = 0, wave_fill: int = 0):
        self._lib = load_library()
        cfg = self._config(hbm_budget_gb, max_resident_jobs, paths_per_wave, max_depth_cap, shade_blocks_per_sm,
                           trace_blocks_per_sm, wave_fill)
        base = (settings or RendererSettings()).to_c()
        self._h = C.c_void_p()
        _check(self._lib.rg_server_create(C.byref(base), C.byref(cfg), C.byref(self._h)))
        self._jobs = {}

    @staticmethod
    def _config(hbm_budget_gb=120.0, max_resident_jobs=256, paths_per_wave=8 << 20, max_depth_cap=10,
                shade_blocks_per_sm=0, trace_blocks_per_sm=0, wave_fill=0):
        cfg = rg_server_config()
        load_library().rg_server_config_default(C.byref(cfg))
        cfg.hbm_budget_bytes = int(hbm_budget_gb * (1 << 30))
        cfg.max_resident_jobs = max_resident_jobs
        cfg.paths_per_wave = paths_per_wave
        cfg.max_depth_cap = max_depth_cap
        cfg.shade_blocks_per_sm = shade_blocks_per_sm
        cfg.trace_blocks_per_sm = trace_blocks_per_sm
        cfg.wave_fill = wave_fill
        return cfg

    @staticmethod
    def autotune(probe, settings: Optional[RendererSettings] = None, hbm_budget_gb: float = 120.0,
                 max_resident_jobs: int = 256, max_depth_cap: int = 10) -> dict:
        """Pick paths_per_wave / shade_blocks_per_sm / trace_blocks_per_sm / wave_fill for a job mix.

        probe: list of (scene, width, height, samples, max_depth, seed).  Returns the
        constructor keyword arguments of the fastest configuration plus its probe time."""
        lib = load_library()
        jobs = (rg_job_desc * len(probe))()
        for k, (sc, w, h, spp, depth, seed) in enumerate(probe):
            jobs[k].scene = sc.ptr
            jobs[k].width, jobs[k].height, jobs[k].samples = w, h, spp
            jobs[k].max_depth, jobs[k].rr_depth, jobs[k].seed, jobs[k].denoise = depth, 0, seed, 0
        cfg = RenderServer._config(hbm_budget_gb, max_resident_jobs, 8 << 20, max_depth_cap)
        base = (settings or RendererSettings()).to_c()
        best = C.c_double()
        _check(lib.rg_server_autotune(C.byref(base), jobs, len(probe), C.byref(cfg), C.byref(best)))
        return {"paths_per_wave": cfg.paths_per_wave, "shade_blocks_per_sm": cfg.shade_blocks_per_sm,
                "trace_blocks_per_sm": cfg.trace_blocks_per_sm, "wave_fill": cfg.wave_fill, "probe_ms": best.value}

    def add_scene(self, scene: Scene) -> int:
        """Upload and build a scene once; jobs submitted with its id reuse it."""
        sid = C.c_int64()
        _check(self._lib.rg_server_add_scene(self._h, scene.ptr, C.byref(sid)))
        return sid.value

    def remove_scene(self, scene_id: int) -> None:
        _check(self._lib.rg_server_remove_scene(self._h, scene_id))

    def submit(self, scene, width: int, height: int, samples: int, max_depth: int = 8, rr_depth: int = 3,
               seed: int = 1, denoise=False) -> int:
        """scene: a Scene (uploaded for this job) or the id of a resident scene (add_scene).
        denoise: False / 0 none, True / 1 A-Trous, 2 the learned denoiser (see set_denoiser)."""
        d = rg_job_desc()
        d.width, d.height, d.samples = width, height, samples
        d.max_depth, d.rr_depth, d.seed, d.denoise = max_depth, rr_depth, seed, int(denoise)
        jid = C.c_int64()
        if isinstance(scene, int):
            _check(self._lib.rg_server_submit_scene(self._h, scene, C.byref(d), C.byref(jid)))
        else:
            d.scene = scene.ptr
            _check(self._lib.rg_server_submit(self._h, C.byref(d), C.byref(jid)))
        self._jobs[jid.value] = (scene, width, height)  # keep the scene alive until done
        return jid.value

    def set_denoiser(self, denoiser) -> None:
        """Learned denoiser for jobs submitted with denoise=2 (None: A-Trous)."""
        self._denoiser = denoiser
        _check(self._lib.rg_server_set_denoiser(self._h, denoiser._h if denoiser is not None else None))

    def status(self, job: int) -> dict:
        st = rg_job_status()
        _check(self._lib.rg_server_poll(self._h, job, C.byref(st)))
        return {f[0]: getattr(st, f[0]) for f in rg_job_status._fields_}

    def wait(self, job: int, timeout_ms: float = 600000.0) -> None:
        _check(self._lib.rg_server_wait(self._h, job, timeout_ms))

    def cancel(self, job: int) -> int:
        """Cancel a queued, admitting or resident job (its slot and memory are freed
        between waves).  Returns RG_OK, or RG_ERR_BUSY when it finished rendering already."""
        rc = self._lib.rg_server_cancel(self._h, job)
        if rc not in (RG_OK, RG_ERR_BUSY):
            _check(rc)
        return rc

    def result(self, job: int, release: bool = True) -> np.ndarray:
        _, w, h = self._jobs[job]
        out = np.empty((h, w, 4), np.float32)
        _check(self._lib.rg_server_get_result(self._h, job, _fptr(out), out.size, int(release)))
        if release:
            self._jobs.pop(job, None)
        return out

    def snapshot(self, job: int, timeout_ms: float = 10000.0) -> np.ndarray:
        _, w, h = self._jobs[job]
        out = np.empty((h, w, 4), np.float32)
        _check(self._lib.rg_server_snapshot(self._h, job, _fptr(out), out.size, timeout_ms))
        return out

    def stats(self) -> dict:
        st = rg_server_stats()
        _check(self._lib.rg_server_get_stats(self._h, C.byref(st)))
        return {f[0]: getattr(st, f[0]) for f in rg_server_stats._fields_}

    def close(self):
        if self._h:
            self._lib.rg_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
