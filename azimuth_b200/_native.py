"""ctypes view of the C-ABI in include/azimuth_gpu.h and include/azimuth_scenes.h.

The library is ``azimuth_b200/libazimuth_b200.so`` (built in-tree by
``azimuth_b200/build.py``).  Loading fails loudly when it is missing: there is
no Python or CPU fallback for the render path.
"""
import ctypes as C
import os

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libazimuth_b200.so")
_lib = None


class Vec2u(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32)]


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class Scissor(C.Structure):
    """az_scissor: {Max, Min}, rows/cols in [Min, Max) (src/azimuth_main.cpp:35-38)."""
    _fields_ = [("Max", Vec2u), ("Min", Vec2u)]


class Ray3(C.Structure):
    _fields_ = [("Origin", Vec3), ("Direction", Vec3), ("T", C.c_float)]


class GenParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("max_depth", C.c_uint32), ("detail", C.c_uint32), ("filter", C.c_int32),
                ("importance_sampling", C.c_int32), ("env_width", C.c_uint32),
                ("env_height", C.c_uint32), ("flags", C.c_uint32)]


class GeneratedScene(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", C.c_void_p), ("epsilons", C.c_void_p),
                ("filter_type", C.c_int32), ("backface_culling", C.c_uint32),
                ("perlin_gradients", C.c_void_p), ("triangle_count", C.c_uint64),
                ("sphere_count", C.c_uint64), ("owner", C.c_void_p), ("soup", C.c_void_p)]


class RenderOpts(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("perlin_gradients", C.c_void_p), ("stream", C.c_void_p),
                ("device", C.c_int32), ("flags", C.c_uint32), ("chunk_samples", C.c_uint32),
                ("bvh_width", C.c_uint32), ("block_size", C.c_uint32), ("variant", C.c_uint32),
                ("bvh_leaf", C.c_uint32), ("bvh_builder", C.c_uint32), ("sample_part", C.c_uint32),
                ("sample_parts", C.c_uint32)]


class Tonemap(C.Structure):
    _fields_ = [("KeyValue", C.c_float), ("BurnoutPercentage", C.c_float), ("Saturation", C.c_float),
                ("Operator", C.c_uint32)]


class Job(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("guide", C.c_void_p), ("film", C.c_void_p), ("camera", C.c_void_p),
                ("epsilons", C.c_void_p), ("scissor", Scissor), ("filter_type", C.c_int32),
                ("backface_culling", C.c_uint32), ("train", C.c_uint32), ("reserved0", C.c_uint32),
                ("seed", C.c_uint64), ("done_ms", C.c_float), ("status", C.c_int32), ("samples", C.c_uint64)]


class BatchOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("streams", C.c_uint32), ("flags", C.c_uint32), ("chunk_samples", C.c_uint32),
                ("largest_first", C.c_uint32), ("tiles", C.c_uint32), ("reserved", C.c_uint32 * 2)]


class BatchStats(C.Structure):
    _fields_ = [("samples", C.c_uint64), ("gpu_ms", C.c_float), ("p50_ms", C.c_float), ("p99_ms", C.c_float),
                ("jobs", C.c_uint32), ("failed", C.c_uint32), ("streams", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class GuideConfig(C.Structure):
    _fields_ = [("learning_rate", C.c_float), ("train_batch", C.c_uint32), ("record_samples", C.c_uint32),
                ("steps_per_wave", C.c_uint32), ("seed", C.c_uint64), ("kernels", C.c_uint32),
                ("queue_order_rows", C.c_uint32), ("reserved", C.c_uint32 * 4)]


class RenderStats(C.Structure):
    _fields_ = [("samples", C.c_uint64), ("extend_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("chunks", C.c_uint32), ("retries", C.c_uint32), ("kernel_launches", C.c_uint64),
                ("gpu_ms", C.c_float), ("extend_ms", C.c_float), ("shade_ms", C.c_float),
                ("shadow_ms", C.c_float), ("node_visits", C.c_uint64), ("prim_visits", C.c_uint64),
                ("extend_launches", C.c_uint32), ("reserved0", C.c_uint32),
                ("shadow_node_visits", C.c_uint64), ("shadow_prim_visits", C.c_uint64),
                ("reserved", C.c_uint32 * 2)]


class SceneInfo(C.Structure):
    _fields_ = [("triangles", C.c_uint64), ("spheres", C.c_uint64), ("wide_nodes", C.c_uint64),
                ("device_bytes", C.c_uint64), ("bvh_width", C.c_uint32), ("bvh_leaf", C.c_uint32),
                ("bvh_depth", C.c_uint32), ("hierarchies", C.c_uint32), ("flatten_ms", C.c_float),
                ("upload_ms", C.c_float), ("bvh_ms", C.c_float), ("total_ms", C.c_float),
                ("ingest_ms", C.c_float), ("bvh_builder", C.c_uint32), ("queue_order", C.c_uint32),
                ("variant", C.c_uint32), ("shadow_variant", C.c_uint32)]


class SceneArrays(C.Structure):
    _fields_ = [("wide_nodes", C.c_void_p), ("wide_node_count", C.c_uint64), ("triangles", C.c_void_p),
                ("triangle_count", C.c_uint64), ("tlas_root", C.c_uint32), ("single_group_root", C.c_uint32),
                ("reserved", C.c_uint32 * 4)]


class MeshDesc(C.Structure):
    _fields_ = [("face_base", C.c_uint32), ("face_count", C.c_uint32), ("uv_offset", C.c_int32),
                ("shading_mode", C.c_uint32), ("material_index", C.c_uint32), ("texture_index", C.c_uint32),
                ("is_emitter", C.c_uint32), ("unique_entity_id", C.c_uint32), ("motion", C.c_float * 3),
                ("radiance", C.c_float * 3), ("transform", C.c_float * 16), ("inv_transform", C.c_float * 16)]


class MeshSoup(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("faces", C.c_void_p), ("uvs", C.c_void_p), ("meshes", C.c_void_p),
                ("vertex_count", C.c_uint32), ("face_count", C.c_uint32), ("uv_count", C.c_uint32),
                ("mesh_count", C.c_uint32)]


def lib():
    """Load (once) and return the native library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError("azimuth_b200 native library missing: %s (run python -m azimuth_b200.build)"
                               % _LIB_PATH)
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def library_path():
    return _LIB_PATH


def _declare(L):
    vp, u32, i32, u64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64
    L.az_scene_generate.argtypes = [i32, u64, C.POINTER(GenParams), C.POINTER(GeneratedScene)]
    L.az_scene_generate.restype = i32
    L.az_scene_release.argtypes = [C.POINTER(GeneratedScene)]
    L.az_scene_release.restype = None
    if hasattr(L, "az_gpu_produce_image"):
        L.az_gpu_last_error.argtypes = []
        L.az_gpu_last_error.restype = C.c_char_p
        L.az_gpu_produce_image.argtypes = [vp, vp, vp, vp, Scissor, i32, u32, C.POINTER(RenderOpts)]
        L.az_gpu_produce_image.restype = i32
        L.az_gpu_scene_create.argtypes = [vp, C.POINTER(RenderOpts), C.POINTER(vp)]
        L.az_gpu_scene_create.restype = i32
        L.az_gpu_scene_destroy.argtypes = [vp]
        L.az_gpu_scene_destroy.restype = None
        L.az_gpu_scene_arrays.argtypes = [vp, C.POINTER(SceneArrays)]
        L.az_gpu_scene_arrays.restype = i32
        L.az_gpu_scene_info.argtypes = [vp, C.POINTER(SceneInfo)]
        L.az_gpu_scene_info.restype = i32
        L.az_gpu_scene_create_from_meshes.argtypes = [vp, vp, C.POINTER(RenderOpts), C.POINTER(vp)]
        L.az_gpu_scene_create_from_meshes.restype = i32
        L.az_gpu_mesh_postprocess.argtypes = [vp, vp, vp, vp, vp, C.POINTER(RenderOpts)]
        L.az_gpu_mesh_postprocess.restype = i32
        L.az_gpu_render.argtypes = [vp, vp, vp, vp, Scissor, i32, u32, C.POINTER(RenderOpts),
                                    C.POINTER(RenderStats)]
        L.az_gpu_render.restype = i32
        L.az_gpu_render_host.argtypes = [vp, vp, vp, vp, Scissor, i32, u32, C.POINTER(RenderOpts),
                                         C.POINTER(RenderStats)]
        L.az_gpu_render_host.restype = i32
        L.az_gpu_render_samples.argtypes = [vp, vp, vp, vp, Scissor, u32, C.POINTER(RenderOpts),
                                            C.POINTER(RenderStats)]
        L.az_gpu_render_samples.restype = i32
        L.az_gpu_autotune.argtypes = [vp, vp, vp, Scissor, i32, u32, C.POINTER(RenderOpts), vp, vp]
        L.az_gpu_autotune.restype = i32
        L.az_gpu_autotune_scene.argtypes = [vp, vp, vp, vp, Scissor, i32, u32, C.POINTER(RenderOpts), vp, vp, vp]
        L.az_gpu_autotune_scene.restype = i32
        L.az_gpu_render_noalloc.argtypes = [vp, vp, vp, vp, Scissor, i32, u32, C.POINTER(RenderOpts)]
        L.az_gpu_postprocess.argtypes = [vp, u32, u32, C.POINTER(Tonemap), C.c_float, u32, u32, vp, vp,
                                         C.POINTER(RenderOpts)]
        L.az_gpu_postprocess.restype = i32
        L.az_gpu_output_pixels_to_file.argtypes = [C.c_char_p, vp, u32, u32, C.POINTER(Tonemap), C.c_float, u32,
                                                    i32, u32, C.POINTER(RenderOpts)]
        L.az_gpu_output_pixels_to_file.restype = i32
        L.az_write_image.argtypes = [C.c_char_p, vp, u32, u32, i32]
        L.az_write_image.restype = i32
        L.az_write_jpg_quality.argtypes = [C.c_char_p, vp, u32, u32, i32]
        L.az_write_jpg_quality.restype = i32
        L.az_write_exr.argtypes = [C.c_char_p, vp, u32, u32]
        L.az_write_exr.restype = i32
        L.az_exr_sibling_path.argtypes = [C.c_char_p, C.c_char_p, u32]
        L.az_exr_sibling_path.restype = i32
        L.az_gpu_render_batch.argtypes = [vp, u32, C.POINTER(BatchOpts), C.POINTER(BatchStats)]
        L.az_gpu_render_batch.restype = i32
        L.az_gpu_render_tiles.argtypes = [vp, u32, C.POINTER(BatchOpts), C.POINTER(BatchStats)]
        L.az_gpu_render_tiles.restype = i32
        L.az_guide_create.argtypes = [vp, C.POINTER(GuideConfig), C.POINTER(vp)]
        L.az_guide_create.restype = i32
        L.az_guide_destroy.argtypes = [vp]
        L.az_guide_destroy.restype = None
        L.az_gpu_render_guided.argtypes = [vp, vp, vp, vp, vp, Scissor, i32, u32, u32, C.POINTER(RenderOpts), vp]
        L.az_gpu_render_guided.restype = i32
        L.az_guide_get_params.argtypes = [vp, vp, vp, vp]
        L.az_guide_get_params.restype = i32
        L.az_guide_set_params.argtypes = [vp, vp, vp, vp]
        L.az_guide_set_params.restype = i32
        L.az_guide_info.argtypes = [vp, vp, vp, vp, vp]
        L.az_guide_info.restype = i32
        L.az_guide_eval.argtypes = [vp, vp, u32, vp, vp, vp, vp, vp]
        L.az_guide_eval.restype = i32
        L.az_guide_train.argtypes = [vp, vp, u32, u32, vp]
        L.az_guide_train.restype = i32
        L.az_guide_infer.argtypes = [vp, vp, u32, vp]
        L.az_guide_infer.restype = i32
        L.az_gpu_render_noalloc.restype = i32
        L.az_gpu_closest_hit.argtypes = [vp, vp, u32, i32, C.c_float, vp, vp, vp, vp, vp]
        L.az_gpu_closest_hit.restype = i32
        L.az_gpu_device_info.argtypes = [i32, vp, u32]
        L.az_gpu_device_info.restype = i32
        L.az_rng_u01.argtypes = [u64, u32, u32, u32, u32, u32]
        L.az_rng_u01.restype = C.c_float
        L.az_rng_philox4x32_10.argtypes = [vp, u32, u32, vp]
        L.az_rng_philox4x32_10.restype = None
