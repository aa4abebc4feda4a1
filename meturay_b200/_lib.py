"""ctypes binding of ``libmrb200.so`` (the C ABI declared in include/mrb200.h).

The library is the product: if it is missing the import fails loudly; there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libmrb200.so"


class MrbError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Material(C.Structure):
    _fields_ = [("type", C.c_uint32), ("albedo", C.c_float * 3), ("eta", C.c_float * 3),
                ("k", C.c_float * 3), ("specular", C.c_float * 3), ("roughness", C.c_float),
                ("metallic", C.c_float), ("medium", C.c_uint32), ("radiance", C.c_float * 3)]


class SceneDesc(C.Structure):
    _fields_ = [("vertex_count", C.c_uint32), ("triangle_count", C.c_uint32),
                ("positions", C.c_void_p), ("normals", C.c_void_p), ("uvs", C.c_void_p),
                ("indices", C.c_void_p), ("tri_material", C.c_void_p), ("tri_cull", C.c_void_p),
                ("material_count", C.c_uint32), ("materials", C.POINTER(Material)),
                ("medium_count", C.c_uint32), ("medium_ior", C.c_void_p),
                ("base_medium", C.c_uint32)]


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("gaze", C.c_float * 3), ("up", C.c_float * 3),
                ("near_far", C.c_float * 2), ("fov", C.c_float * 2)]


class PoolJob(C.Structure):
    _fields_ = [("camera", Camera), ("width", C.c_uint32), ("height", C.c_uint32),
                ("samples", C.c_uint32), ("frames", C.c_uint32), ("max_depth", C.c_uint32),
                ("rr_start", C.c_uint32), ("nee", C.c_uint32), ("mis", C.c_uint32),
                ("seed", C.c_uint64)]


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
            "g.build()'` (nvcc, sm_100a). There is no CPU fallback.")
    lib = C.CDLL(str(_LIB_PATH))
    vp, u32, u64, i32, sz = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_size_t
    sig = {
        "mrb_last_error": (C.c_char_p, []),
        "mrb_system_create": (i32, [i32, C.POINTER(vp)]),
        "mrb_system_destroy": (None, [vp]),
        "mrb_scene_create": (i32, [vp, C.POINTER(SceneDesc), C.POINTER(vp)]),
        "mrb_scene_destroy": (None, [vp]),
        "mrb_scene_counts": (i32, [vp, vp]),
        "mrb_scene_export": (i32, [vp] + [vp] * 8),
        "mrb_scene_export_ext": (i32, [vp, vp, vp, vp]),
        "mrb_accel_construct": (i32, [vp, vp]),
        "mrb_accel_export": (i32, [vp] + [vp] * 9),
        "mrb_accel_hit": (i32, [vp, vp, vp, u32, vp, vp, vp, vp, vp]),
        "mrb_accel_set_traversal": (i32, [vp, i32]),
        "mrb_accel_info": (i32, [vp, vp]),
        "mrb_accel_set_wide_tree": (i32, [vp, i32]),
        "mrb_accel_set_wide_collapse": (i32, [vp, i32]),
        "mrb_accel_wide_collapse": (i32, [vp, C.POINTER(i32), vp]),
        "mrb_accel_set_wide_order": (i32, [vp, i32]),
        "mrb_accel_wide_order": (i32, [vp, C.POINTER(C.c_int), vp]),
        "mrb_accel_info_ext": (i32, [vp, vp, vp]),
        "mrb_svo_build": (i32, [vp, u32, vp]),
        "mrb_svo_info": (i32, [vp, vp, vp]),
        "mrb_svo_export": (i32, [vp, vp, vp, vp, vp, vp, vp]),
        "mrb_svo_export_payload": (i32, [vp, vp, vp, vp, vp, vp]),
        "mrb_json_scene_load": (i32, [C.c_char_p, sz, C.POINTER(vp)]),
        "mrb_json_scene_load_file": (i32, [C.c_char_p, C.POINTER(vp)]),
        "mrb_json_scene_destroy": (None, [vp]),
        "mrb_json_scene_get": (i32, [vp, C.POINTER(SceneDesc), C.POINTER(u32)]),
        "mrb_json_scene_camera": (i32, [vp, u32, C.POINTER(Camera)]),
        "mrb_tracer_set_option_float": (i32, [vp, C.c_char_p, C.c_double]),
        "mrb_tracer_svo_info": (i32, [vp, vp, vp]),
        "mrb_tracer_svo_export": (i32, [vp] + [vp] * 11),
        "mrb_tracer_svo_guiding": (i32, [vp, vp, vp]),
        "mrb_tracer_guide_export": (i32, [vp, C.POINTER(u32), vp, vp, vp, vp]),
        "mrb_tracer_create": (i32, [vp, vp, C.c_char_p, C.POINTER(vp)]),
        "mrb_tracer_destroy": (None, [vp]),
        "mrb_tracer_set_option": (i32, [vp, C.c_char_p, u64]),
        "mrb_tracer_set_resolution": (i32, [vp, u32, u32]),
        "mrb_tracer_set_camera": (i32, [vp, C.POINTER(Camera)]),
        "mrb_camera_frame": (i32, [C.POINTER(Camera), vp]),
        "mrb_tracer_generate_work": (i32, [vp, u32]),
        "mrb_tracer_render": (i32, [vp]),
        "mrb_tracer_finalize": (i32, [vp]),
        "mrb_tracer_render_frame": (i32, [vp]),
        "mrb_tracer_get_image": (i32, [vp, vp]),
        "mrb_tracer_get_image_async": (i32, [vp, vp]),
        "mrb_tracer_wait_image": (i32, [vp]),
        "mrb_tracer_get_samples": (i32, [vp, vp]),
        "mrb_tracer_reset_image": (i32, [vp]),
        "mrb_tracer_stats": (i32, [vp, C.POINTER(u64), C.POINTER(u32)]),
        "mrb_tracer_stream": (vp, [vp]),
        "mrb_tracer_launches_per_frame": (i32, [vp]),
        "mrb_tracer_wide_orders": (i32, [vp, C.POINTER(C.c_int), u32]),
        "mrb_tracer_profile_frame": (i32, [vp, vp, vp]),
        "mrb_tracer_profile_stages": (i32, [vp, vp, u32, vp]),
        "mrb_morton_codes": (i32, [vp, vp, u32, vp, vp, vp, vp]),
        "mrb_radix_sort_temp_bytes": (sz, [u32, i32, i32, i32]),
        "mrb_radix_sort_pairs_u64": (i32, [vp, vp, u32, i32, i32, i32, vp, sz, vp]),
        "mrb_radix_sort_pairs_u32": (i32, [vp, vp, u32, i32, i32, i32, vp, sz, vp]),
        "mrb_radix_sort_pairs_u32_noalloc": (i32, [vp, vp, u32, i32, i32, i32, vp]),
        "mrb_lbvh_hierarchy": (i32, [vp, vp, vp, u32, vp, vp, vp, vp, vp, vp, vp, vp]),
        "mrb_partition_temp_bytes": (sz, [u32, u32]),
        "mrb_partition": (i32, [vp, u32, u32, vp, vp, vp, vp, vp, vp, sz, vp]),
        "mrb_debug_math": (i32, [vp, u32, vp, vp, vp, vp]),
        "mrb_recon_filter_create": (i32, [C.c_char_p, C.c_float, u32, C.POINTER(C.c_char_p),
                                          C.POINTER(C.c_float), C.POINTER(vp)]),
        "mrb_recon_filter_destroy": (None, [vp]),
        "mrb_recon_filter_type": (C.c_char_p, [vp]),
        "mrb_recon_filter_used_bytes": (sz, [vp]),
        "mrb_recon_filter_pixel_wh": (u32, [C.c_float]),
        "mrb_recon_filter_weight": (C.c_float, [vp] + [C.c_float] * 4),
        "mrb_recon_filter_to_img": (i32, [vp, vp, vp, u32, vp, u32, C.c_float, vp]),
        "mrb_image_create": (i32, [C.c_int32, C.c_int32, u32, C.POINTER(vp)]),
        "mrb_image_destroy": (None, [vp]),
        "mrb_image_reportion": (i32, [vp] + [C.c_int32] * 4),
        "mrb_image_resize": (i32, [vp, C.c_int32, C.c_int32]),
        "mrb_image_reset": (i32, [vp, vp]),
        "mrb_image_info": (i32, [vp, vp]),
        "mrb_image_device": (i32, [vp, C.POINTER(vp), C.POINTER(vp)]),
        "mrb_image_get": (i32, [vp, vp, vp, vp]),
        "mrb_tracer_set_filter": (i32, [vp, vp]),
        "mrb_tracer_set_option_string": (i32, [vp, C.c_char_p, C.c_char_p]),
        "mrb_pool_create": (i32, [vp, u32, u32, sz, C.POINTER(vp)]),
        "mrb_pool_destroy": (None, [vp]),
        "mrb_pool_set_launch": (i32, [vp, i32, i32]),
        "mrb_pool_submit": (i32, [vp, vp, C.POINTER(PoolJob), C.POINTER(u64)]),
        "mrb_pool_step": (i32, [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]),
        "mrb_pool_job_status": (i32, [vp, u64, C.POINTER(u32), C.POINTER(u32)]),
        "mrb_pool_job_image": (i32, [vp, u64, vp, i32]),
        "mrb_pool_stats": (i32, [vp, C.POINTER(u64), C.POINTER(u64), C.POINTER(sz),
                                 C.POINTER(sz)]),
        "mrb_pool_stream": (vp, [vp]),
        "mrb_mlp_param_count": (u32, []),
        "mrb_tracer_learned_params": (i32, [vp, vp]),
        "mrb_tracer_learned_loss": (i32, [vp, vp]),
        "mrb_mlp_create": (i32, [vp, C.POINTER(vp)]),
        "mrb_mlp_destroy": (None, [vp]),
        "mrb_mlp_set_params": (i32, [vp, vp]),
        "mrb_mlp_get_params": (i32, [vp, vp]),
        "mrb_mlp_encode": (i32, [vp, vp, vp, u32, vp, vp]),
        "mrb_mlp_forward": (i32, [vp, vp, u32, vp, vp]),
        "mrb_mlp_gradients": (i32, [vp, vp, vp, u32, vp, vp, vp]),
        "mrb_mlp_train_step": (i32, [vp, vp, vp, u32, C.c_float, vp, vp]),
        "mrb_tracer_svo_dump": (i32, [vp, vp, sz, C.POINTER(sz)]),
        "mrb_tracer_svo_load": (i32, [vp, vp, sz]),
        "mrb_tracer_write_image": (i32, [vp, C.c_char_p]),
        "mrb_image_write": (i32, [vp, C.c_char_p]),
        "mrb_write_exr": (i32, [C.c_char_p, vp, u32, u32, u32, i32]),
        "mrb_write_pfm": (i32, [C.c_char_p, vp, u32, u32, u32]),
        "mrb_read_image": (i32, [C.c_char_p, vp, sz, C.POINTER(u32), C.POINTER(u32),
                                 C.POINTER(u32)]),
        "mrb_accel_group_create": (i32, [vp, vp, u32, vp, vp, vp, vp, vp, u32, vp, u32,
                                         C.POINTER(vp)]),
        "mrb_accel_group_destroy": (None, [vp]),
        "mrb_accel_group_attach_transforms": (i32, [vp, vp, u32, u32]),
        "mrb_accel_group_construct": (i32, [vp, vp]),
        "mrb_accel_group_hit": (i32, [vp, vp, vp, vp, vp, u32, vp, vp, vp, u32, vp]),
        "mrb_accel_group_aabbs": (i32, [vp, vp, u32]),
        "mrb_accel_group_primitive_count": (u64, [vp]),
        "mrb_accel_group_accelerator_count": (u32, [vp]),
        "mrb_accel_group_total_area": (i32, [vp, C.POINTER(C.c_float), vp]),
        "mrb_accel_group_sample_points": (i32, [vp, vp, vp, u32, u64, vp]),
        "mrb_accel_group_voxel_counts": (i32, [vp, vp, u32, vp, vp]),
        "mrb_accel_group_voxelize": (i32, [vp, vp, vp, vp, vp, vp, u32, u32, vp, vp]),
        "mrb_base_accel_create": (i32, [vp, C.POINTER(vp)]),
        "mrb_base_accel_destroy": (None, [vp]),
        "mrb_base_accel_construct": (i32, [vp, vp, vp, u32]),
        "mrb_base_accel_get_ready": (i32, [vp, u32, vp]),
        "mrb_base_accel_hit": (i32, [vp, vp, vp, vp, u32, vp]),
        "mrb_base_accel_extents": (i32, [vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(code: int) -> int:
    """Raise MrbError for a negative status; return the status otherwise."""
    if code < 0:
        raise MrbError(code, lib.mrb_last_error().decode(errors="replace"))
    return code


def exported_symbols() -> list[str]:
    """Names of the entry points declared in include/mrb200.h."""
    import re
    hdr = Path(__file__).resolve().parent.parent / "include" / "mrb200.h"
    text = hdr.read_text()
    return sorted(set(re.findall(r"\b(mrb_[a-z0-9_]+)\s*\(", text)))
