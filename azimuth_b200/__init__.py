"""azimuth_b200: B200-native render path for azimuth scenes.

Python access to the C-ABI of ``libazimuth_b200.so`` (include/azimuth_gpu.h,
include/azimuth_scenes.h).  The render work runs only in the native library's
CUDA kernels; if the library or a GPU is missing, calls raise.

Typical use::

    from azimuth_b200 import generate_scene, GpuScene
    sc = generate_scene(0, seed=0, width=256, height=256, spp=16)
    with GpuScene(sc) as g:
        film = g.render(sc)              # numpy (H, W, 4): rgb sum, weight sum
"""
import ctypes as C
import os

import numpy as np

from . import _native
from ._native import (BatchOpts, BatchStats, GenParams, GeneratedScene, GuideConfig, Job, MeshDesc, MeshSoup,
                      RenderOpts, RenderStats, SceneArrays, SceneInfo, Scissor, Tonemap, Vec2u, Ray3, lib)

GEN_SOUP_ONLY = 1   # az_gen_params.flags: meshes left as the importer's soup

SCENE_CORNELL = 0
SCENE_DENSE_MESH = 1
SCENE_MOTION_ENV = 2
SCENE_INTERIOR = 3
SCENE_FEATURES = 100
SCENE_ENV_SPHERES = 101

FILTER_BOX = 0
FILTER_GAUSSIAN = 1

FLAG_COUNT_TRAVERSAL = 1
FLAG_NO_GRAPH = 2
FLAG_TIME_STAGES = 4
FLAG_ENV_IMPORTANCE = 8
FLAG_ORDER_SHADOW = 16     # visit shadow queues by origin cell
FLAG_ORDER_EXTEND = 32     # visit extension queues by origin cell and direction octant
FLAG_ORDER_NONE = 64       # queues in fill order
FLAG_SERIAL_LEVELS = 128   # visibility queries of a level before the next level's closest-hit queries
FLAG_WATERTIGHT = 256      # triangles by the watertight test (production mode) instead of azimuth's Cramer test
GUIDE_TCGEN05, GUIDE_MMA_SYNC = 0, 1   # az_guide_config.kernels
LAUNCH_VARIANTS = 20   # AZ_LAUNCH_VARIANTS

STATUS = {0: "AZ_OK", 1: "AZ_ERR_INVALID_ARGUMENT", 2: "AZ_ERR_INVALID_SCENE", 3: "AZ_ERR_OUT_OF_MEMORY",
          4: "AZ_ERR_CUDA", 5: "AZ_ERR_TIMEOUT", 6: "AZ_ERR_UNSUPPORTED", 7: "AZ_ERR_NO_DEVICE"}


class AzError(RuntimeError):
    def __init__(self, code, what):
        msg = lib().az_gpu_last_error().decode(errors="replace") if hasattr(lib(), "az_gpu_last_error") else ""
        super().__init__("%s failed: %s (%s)" % (what, STATUS.get(code, code), msg))
        self.code = code


def _check(code, what):
    if code != 0:
        raise AzError(code, what)


class Scene:
    """A generated azimuth scene (azimuth structs owned by the native library)."""

    def __init__(self, scene_id, seed=0, width=0, height=0, spp=0, max_depth=0, detail=0, filter=-1,
                 importance_sampling=-1, env_width=0, env_height=0, soup_only=False):
        self._g = GeneratedScene()
        p = GenParams(width, height, spp, max_depth, detail, filter, importance_sampling, env_width, env_height,
                      GEN_SOUP_ONLY if soup_only else 0)
        rc = lib().az_scene_generate(int(scene_id), int(seed), C.byref(p), C.byref(self._g))
        if rc != 0:
            raise RuntimeError("az_scene_generate(%d) failed with %d" % (scene_id, rc))
        self.scene_id = scene_id
        self.seed = seed

    @property
    def scene_ptr(self):
        return self._g.scene

    @property
    def soup_ptr(self):
        """The meshes before the importer's post-processing (az_mesh_soup*)."""
        return self._g.soup

    def soup_arrays(self):
        """Copies of the soup: (vertices (V, 3) f32, faces (F, 3) u32, uvs (U, 2) f32, mesh descs list)."""
        s = MeshSoup.from_address(self._g.soup)

        def arr(ptr, n, k, dt):
            if n == 0:
                return np.zeros((0, k), dt)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float if dt == np.float32 else C.c_uint32)),
                                         (n * k,)).reshape(n, k).copy()
        descs = [MeshDesc.from_address(s.meshes + i * C.sizeof(MeshDesc)) for i in range(s.mesh_count)]
        descs = [{k: (list(getattr(d, k)) if not isinstance(getattr(d, k), int) else getattr(d, k))
                  for k, _ in MeshDesc._fields_} for d in descs]
        return (arr(s.vertices, s.vertex_count, 3, np.float32), arr(s.faces, s.face_count, 3, np.uint32),
                arr(s.uvs, s.uv_count, 2, np.float32), descs)

    @property
    def camera_ptr(self):
        return self._g.camera

    @property
    def epsilons_ptr(self):
        return self._g.epsilons

    @property
    def filter_type(self):
        return self._g.filter_type

    @property
    def perlin_gradients(self):
        return self._g.perlin_gradients

    @property
    def triangle_count(self):
        return self._g.triangle_count

    @property
    def sphere_count(self):
        return self._g.sphere_count

    def resolution(self):
        # az_camera.Resolution at byte offset 340 (include/az_abi.h)
        buf = (C.c_uint32 * 2).from_address(self._g.camera + 340)
        return int(buf[0]), int(buf[1])

    def sample_count(self):
        return int(C.c_uint32.from_address(self._g.camera + 384).value)

    def max_depth(self):
        return int(C.c_uint32.from_address(self._g.scene + 2720).value)

    def close(self):
        if self._g.owner:
            lib().az_scene_release(C.byref(self._g))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_scene(scene_id, seed=0, **kw):
    return Scene(scene_id, seed, **kw)


def full_scissor(scene):
    w, h = scene.resolution()
    return Scissor(Vec2u(w, h), Vec2u(0, 0))


BVH_LBVH, BVH_PLOC = 1, 2   # az_render_opts.bvh_builder


def make_opts(scene=None, seed=0, stream=None, device=0, flags=0, chunk_samples=0, block_size=0, variant=0,
              bvh_width=0, bvh_leaf=0, bvh_builder=0, sample_part=0, sample_parts=0):
    o = RenderOpts()
    o.sample_part = sample_part
    o.sample_parts = sample_parts
    o.bvh_builder = bvh_builder
    o.variant = variant
    o.bvh_width = bvh_width
    o.bvh_leaf = bvh_leaf
    o.seed = seed
    o.perlin_gradients = scene.perlin_gradients if scene is not None else None
    o.stream = stream
    o.device = device
    o.flags = flags
    o.chunk_samples = chunk_samples
    o.block_size = block_size
    return o


def produce_image(scene, pixels=None, scissor=None, filter_type=None, backface_culling=0, seed=0, device=0):
    """az_gpu_produce_image on a host film (numpy float32 (H, W, 4)); returns the film."""
    w, h = scene.resolution()
    if pixels is None:
        pixels = np.zeros((h, w, 4), np.float32)
    assert pixels.dtype == np.float32 and pixels.shape == (h, w, 4) and pixels.flags.c_contiguous
    sc = scissor or full_scissor(scene)
    ft = scene.filter_type if filter_type is None else filter_type
    o = make_opts(scene, seed=seed, device=device)
    _check(lib().az_gpu_produce_image(pixels.ctypes.data, scene.scene_ptr, scene.camera_ptr, scene.epsilons_ptr,
                                      sc, ft, backface_culling, C.byref(o)), "az_gpu_produce_image")
    return pixels


class GpuScene:
    """A device-resident scene (az_gpu_scene_create / az_gpu_scene_destroy)."""

    def __init__(self, scene, device=0, bvh_width=0, bvh_leaf=0, from_soup=False, bvh_builder=0):
        """from_soup: build through az_gpu_scene_create_from_meshes from the scene's mesh soup (the meshes
        post-processed on the GPU) instead of azimuth's finished structs."""
        self.scene = scene
        self.device = device
        self._h = C.c_void_p()
        o = make_opts(scene, device=device, bvh_width=bvh_width, bvh_leaf=bvh_leaf, bvh_builder=bvh_builder)
        if from_soup:
            _check(lib().az_gpu_scene_create_from_meshes(scene.scene_ptr, scene.soup_ptr, C.byref(o),
                                                         C.byref(self._h)), "az_gpu_scene_create_from_meshes")
        else:
            _check(lib().az_gpu_scene_create(scene.scene_ptr, C.byref(o), C.byref(self._h)), "az_gpu_scene_create")

    def info(self):
        """az_gpu_scene_info: what the build made (triangles, spheres, wide nodes, depth, device bytes) and
        the time of its parts (host flattening, uploads, GPU BVH build) in ms."""
        si = SceneInfo()
        _check(lib().az_gpu_scene_info(self._h, C.byref(si)), "az_gpu_scene_info")
        return {k: getattr(si, k) for k, _ in SceneInfo._fields_}

    def arrays(self):
        """az_gpu_scene_arrays: device addresses and counts of the wide nodes and triangles, the top-level
        root and the root of a single top-level group."""
        sa = SceneArrays()
        _check(lib().az_gpu_scene_arrays(self._h, C.byref(sa)), "az_gpu_scene_arrays")
        return {k: getattr(sa, k) for k, _ in SceneArrays._fields_ if k != "reserved"}

    def autotune(self, seed=0, stream=None):
        """az_gpu_autotune: picks the traversal launch variant for this scene; returns (variant, ms)."""
        o = make_opts(self.scene, seed=seed, stream=stream, device=self.device)
        v = C.c_uint32()
        ms = C.c_float()
        _check(lib().az_gpu_autotune(self._h, self.scene.camera_ptr, self.scene.epsilons_ptr, full_scissor(self.scene),
                                     self.scene.filter_type, 0, C.byref(o), C.byref(v), C.byref(ms)),
               "az_gpu_autotune")
        return v.value, ms.value

    def autotune_scene(self, seed=0, stream=None):
        """az_gpu_autotune_scene: sweeps the hierarchy's shape (width 8/4/2, 1-3 triangles per leaf) and the
        launch variant, keeps the fastest build; returns (width, variant, ms)."""
        o = make_opts(self.scene, seed=seed, stream=stream, device=self.device)
        w = C.c_uint32()
        v = C.c_uint32()
        ms = C.c_float()
        _check(lib().az_gpu_autotune_scene(self.scene.scene_ptr, self._h, self.scene.camera_ptr,
                                           self.scene.epsilons_ptr, full_scissor(self.scene), self.scene.filter_type,
                                           0, C.byref(o), C.byref(w), C.byref(v), C.byref(ms)),
               "az_gpu_autotune_scene")
        return w.value, v.value, ms.value

    def render_device(self, film_ptr, camera_ptr=None, scissor=None, filter_type=None, seed=0, stream=None,
                      stats=False, flags=0, chunk_samples=0, variant=0, sample_part=0, sample_parts=0):
        """az_gpu_render into a DEVICE film pointer; returns az_render_stats as a dict if stats.
        sample_part / sample_parts: render one of that many equal ranges of the camera-sample sequence."""
        sc = scissor or full_scissor(self.scene)
        ft = self.scene.filter_type if filter_type is None else filter_type
        o = make_opts(self.scene, seed=seed, stream=stream, device=self.device, flags=flags,
                      chunk_samples=chunk_samples, variant=variant, sample_part=sample_part,
                      sample_parts=sample_parts)
        st = RenderStats() if stats else None
        _check(lib().az_gpu_render(self._h, film_ptr, camera_ptr or self.scene.camera_ptr, self.scene.epsilons_ptr,
                                   sc, ft, 0, C.byref(o), C.byref(st) if st is not None else None),
               "az_gpu_render")
        return _stats(st)

    def render_samples(self, samples_ptr, camera_ptr=None, scissor=None, seed=0, stream=None, stats=False, flags=0,
                       chunk_samples=0, variant=0):
        """az_gpu_render_samples: every camera sample's radiance (4 floats, DEVICE pointer) in the scissor's
        sample order (sample number * scissor pixels + pixel) instead of a film."""
        sc = scissor or full_scissor(self.scene)
        o = make_opts(self.scene, seed=seed, stream=stream, device=self.device, flags=flags,
                      chunk_samples=chunk_samples, variant=variant)
        st = RenderStats() if stats else None
        _check(lib().az_gpu_render_samples(self._h, samples_ptr, camera_ptr or self.scene.camera_ptr,
                                           self.scene.epsilons_ptr, sc, 0, C.byref(o),
                                           C.byref(st) if st is not None else None), "az_gpu_render_samples")
        return _stats(st)

    def render_host(self, pixels, camera_ptr=None, scissor=None, filter_type=None, seed=0, stream=None,
                    flags=0, chunk_samples=0):
        """az_gpu_render_host: HOST film (numpy float32 (H, W, 4), ideally pinned) in and out."""
        sc = scissor or full_scissor(self.scene)
        ft = self.scene.filter_type if filter_type is None else filter_type
        o = make_opts(self.scene, seed=seed, stream=stream, device=self.device, flags=flags,
                      chunk_samples=chunk_samples)
        st = RenderStats()
        ptr = pixels.ctypes.data if hasattr(pixels, "ctypes") else pixels
        _check(lib().az_gpu_render_host(self._h, ptr, camera_ptr or self.scene.camera_ptr, self.scene.epsilons_ptr,
                                        sc, ft, 0, C.byref(o), C.byref(st)), "az_gpu_render_host")
        return _stats(st)

    def closest_hit(self, rays, cull=0, eps=0.0, flags=0):
        """rays: numpy (N, 7) float32 [origin, direction, T]; returns (hit, uid, face, t).
        flags: FLAG_WATERTIGHT for the watertight triangle test."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        hit = np.zeros(n, np.uint32)
        uid = np.zeros(n, np.uint32)
        face = np.zeros(n, np.uint32)
        t = np.zeros(n, np.float32)
        o = make_opts(self.scene, device=self.device, flags=flags)
        _check(lib().az_gpu_closest_hit(self._h, rays.ctypes.data, n, cull, eps, hit.ctypes.data, uid.ctypes.data,
                                        face.ctypes.data, t.ctypes.data, C.byref(o)), "az_gpu_closest_hit")
        return hit, uid, face, t

    def close(self):
        if self._h:
            lib().az_gpu_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Guide:
    """A neural path guide for one GpuScene (az_guide_create / az_guide_destroy)."""

    LEVELS = 16
    TABLE = 1 << 19

    def __init__(self, gpu_scene, seed=0, learning_rate=0.0, train_batch=0, record_samples=0, steps_per_wave=0,
                 kernels=0, queue_order_rows=False):
        """kernels: GUIDE_TCGEN05 (default) or GUIDE_MMA_SYNC, the network kernels (proposals and training);
        queue_order_rows: the tcgen05 proposals visit rows in queue order instead of spatial order."""
        self.gs = gpu_scene
        cfg = GuideConfig()
        cfg.kernels = kernels
        cfg.queue_order_rows = 1 if queue_order_rows else 0
        cfg.learning_rate = learning_rate
        cfg.train_batch = train_batch
        cfg.record_samples = record_samples
        cfg.steps_per_wave = steps_per_wave
        cfg.seed = seed
        self._h = C.c_void_p()
        _check(lib().az_guide_create(gpu_scene._h, C.byref(cfg), C.byref(self._h)), "az_guide_create")

    def render(self, film_ptr, train=False, seed=0, stream=None, stats=True, flags=0, chunk_samples=0,
               camera_ptr=None, scissor=None):
        """az_gpu_render_guided into a DEVICE film pointer; returns az_render_stats as a dict if stats."""
        sc_ = self.gs.scene
        o = make_opts(sc_, seed=seed, stream=stream, device=self.gs.device, flags=flags, chunk_samples=chunk_samples)
        st = RenderStats() if stats else None
        _check(lib().az_gpu_render_guided(self.gs._h, self._h, film_ptr, camera_ptr or sc_.camera_ptr,
                                          sc_.epsilons_ptr, scissor or full_scissor(sc_), sc_.filter_type, 0,
                                          1 if train else 0, C.byref(o), C.byref(st) if st is not None else None),
               "az_gpu_render_guided")
        return _stats(st)

    def info(self):
        res = np.zeros(16, np.uint32)
        lo = np.zeros(3, np.float32)
        inv = np.zeros(3, np.float32)
        steps = C.c_uint32()
        _check(lib().az_guide_info(self._h, res.ctypes.data, lo.ctypes.data, inv.ctypes.data, C.byref(steps)),
               "az_guide_info")
        return {"res": res, "lo": lo, "inv_ext": inv, "steps": steps.value}

    def params(self, grid=True):
        mlp = np.zeros((4, 64, 64), np.float32)
        bias = np.zeros(64, np.float32)
        g = np.zeros((self.LEVELS, self.TABLE, 2), np.float32) if grid else None
        _check(lib().az_guide_get_params(self._h, mlp.ctypes.data, bias.ctypes.data,
                                         g.ctypes.data if grid else None), "az_guide_get_params")
        return mlp, bias, g

    def set_params(self, mlp=None, bias=None, grid=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (mlp, bias, grid)]
        _check(lib().az_guide_set_params(self._h, *[None if a is None else a.ctypes.data for a in arrs]),
               "az_guide_set_params")

    def eval(self, rows):
        """rows: (N, 16) float32 [pos, weight, normal, 0, wo, 0, wi, 0]; outputs, loss and gradients."""
        rows = np.ascontiguousarray(rows, np.float32)
        n = rows.shape[0]
        out = np.zeros((n, 64), np.float32)
        loss = np.zeros(1, np.float32)
        mg = np.zeros((4, 64, 64), np.float32)
        bg = np.zeros(64, np.float32)
        eg = np.zeros((n, 32), np.float32)
        _check(lib().az_guide_eval(self._h, rows.ctypes.data, n, out.ctypes.data, loss.ctypes.data, mg.ctypes.data,
                                   bg.ctypes.data, eg.ctypes.data), "az_guide_eval")
        return {"outputs": out, "loss": float(loss[0]), "mlp_grad": mg, "bias_grad": bg, "enc_grad": eg}

    def infer(self, rows):
        """az_guide_infer: raw outputs (N, 64) of rows by the tcgen05 inference kernel."""
        rows = np.ascontiguousarray(rows, np.float32)
        out = np.zeros((rows.shape[0], 64), np.float32)
        _check(lib().az_guide_infer(self._h, rows.ctypes.data, rows.shape[0], out.ctypes.data), "az_guide_infer")
        return out

    def train(self, rows, steps):
        rows = np.ascontiguousarray(rows, np.float32)
        losses = np.zeros(steps, np.float32)
        _check(lib().az_guide_train(self._h, rows.ctypes.data, rows.shape[0], steps, losses.ctypes.data),
               "az_guide_train")
        return losses

    def close(self):
        if self._h:
            lib().az_guide_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def postprocess(film_ptr, width, height, key_value=0.18, burnout=1.0, saturation=1.0, photographic=True,
                inv_gamma=1.0 / 2.2, srgb=True, linear=False, rgb_ptr=None, rgb8_ptr=None, stream=None, device=0):
    """az_gpu_postprocess: azimuth's normalisation, tone mapping and gamma of a DEVICE film into DEVICE
    outputs (rgb_ptr: width*height*3 float32; rgb8_ptr: width*height*3 uint8)."""
    tm = _tonemap(key_value, burnout, saturation, photographic)
    o = make_opts(stream=stream, device=device)
    _check(lib().az_gpu_postprocess(film_ptr, width, height, C.byref(tm), inv_gamma, 1 if srgb else 0,
                                    1 if linear else 0, rgb_ptr, rgb8_ptr, C.byref(o)), "az_gpu_postprocess")


FILE_PNG, FILE_BMP, FILE_TGA, FILE_JPG, FILE_EXR = 0, 1, 2, 3, 4   # azimuth's file_format values


def mesh_postprocess(scene, device=0):
    """az_gpu_mesh_postprocess of a generated scene's soup: dict of vertex_normals (V, 3), triangles (F, 12:
    P0, P1, P2, N), attrs (F, 15: N0, N1, N2, UV0, UV1, UV2), total_area (M,), all float32."""
    s = MeshSoup.from_address(scene.soup_ptr)
    vn = np.zeros((s.vertex_count, 3), np.float32)
    tris = np.zeros((s.face_count, 12), np.float32)
    attrs = np.zeros((s.face_count, 15), np.float32)
    area = np.zeros(s.mesh_count, np.float32)
    o = make_opts(device=device)
    _check(lib().az_gpu_mesh_postprocess(scene.soup_ptr, vn.ctypes.data, tris.ctypes.data, attrs.ctypes.data,
                                         area.ctypes.data, C.byref(o)), "az_gpu_mesh_postprocess")
    return {"vertex_normals": vn, "triangles": tris, "attrs": attrs, "total_area": area}


def _tonemap(key_value, burnout, saturation, photographic):
    tm = Tonemap()
    tm.KeyValue = key_value
    tm.BurnoutPercentage = burnout
    tm.Saturation = saturation
    tm.Operator = 1 if photographic else 0
    return tm


def output_pixels_to_file(path, film_ptr, width, height, file_format=FILE_PNG, key_value=0.18, burnout=1.0,
                          saturation=1.0, photographic=True, inv_gamma=1.0 / 2.2, srgb=True, save_exr=False,
                          stream=None, device=0):
    """az_gpu_output_pixels_to_file: azimuth's OutputPixelsToFile for a DEVICE film (post-process on the
    GPU, then this library's PNG/BMP/TGA/JPG/EXR writer)."""
    tm = _tonemap(key_value, burnout, saturation, photographic)
    o = make_opts(stream=stream, device=device)
    _check(lib().az_gpu_output_pixels_to_file(os.fsencode(path), film_ptr, width, height, C.byref(tm), inv_gamma,
                                              1 if srgb else 0, file_format, 1 if save_exr else 0, C.byref(o)),
           "az_gpu_output_pixels_to_file")


def write_image(path, rgb8, file_format=FILE_PNG, quality=None):
    """az_write_image (az_write_jpg_quality with quality): uint8 array (H, W, 3) to a file."""
    a = np.ascontiguousarray(rgb8, np.uint8)
    h, w = a.shape[:2]
    if quality is not None:
        _check(lib().az_write_jpg_quality(os.fsencode(path), a.ctypes.data, w, h, int(quality)), "az_write_jpg_quality")
    else:
        _check(lib().az_write_image(os.fsencode(path), a.ctypes.data, w, h, file_format), "az_write_image")


def write_exr(path, rgb):
    """az_write_exr: float array (H, W, 3) to an uncompressed half-float OpenEXR file."""
    a = np.ascontiguousarray(rgb, np.float32)
    h, w = a.shape[:2]
    _check(lib().az_write_exr(os.fsencode(path), a.ctypes.data, w, h), "az_write_exr")


def exr_sibling_path(path):
    """az_exr_sibling_path: the EXR name OutputPixelsToFile derives from `path`, or None."""
    buf = C.create_string_buffer(256)
    rc = lib().az_exr_sibling_path(os.fsencode(path), buf, 256)
    return buf.value.decode() if rc == 0 else None


def render_tiles(jobs, flags=0, chunk_samples=0, device=0):
    """az_gpu_render_tiles: jobs (same dict keys as render_batch, no guide; any GpuScenes of one device)
    rendered together in shared waves of 4096-sample tiles.  Returns (per-job list, stats dict)."""
    arr, o, st = _batch_args(jobs, 0, flags, chunk_samples, device, False)
    rc = lib().az_gpu_render_tiles(arr, len(jobs), C.byref(o), C.byref(st))
    per = [{"done_ms": arr[k].done_ms, "status": arr[k].status, "samples": arr[k].samples} for k in range(len(jobs))]
    _check(rc, "az_gpu_render_tiles")
    return per, {"samples": st.samples, "gpu_ms": st.gpu_ms, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
                 "jobs": st.jobs, "failed": st.failed, "streams": st.streams}


def _batch_args(jobs, streams, flags, chunk_samples, device, largest_first, tiles=False):
    arr = (Job * len(jobs))()
    for k, j in enumerate(jobs):
        gs = j["gpu_scene"]
        sc_ = gs.scene
        a = arr[k]
        a.scene = gs._h
        a.guide = j["guide"]._h if j.get("guide") is not None else None
        a.film = j["film_ptr"]
        a.camera = j.get("camera_ptr") or sc_.camera_ptr
        a.epsilons = j.get("epsilons_ptr") or sc_.epsilons_ptr
        a.scissor = j.get("scissor") or full_scissor(sc_)
        a.filter_type = j["filter_type"] if "filter_type" in j else sc_.filter_type
        a.backface_culling = 0
        a.train = 1 if j.get("train") else 0
        a.seed = j.get("seed", 0)
    o = BatchOpts()
    o.device = device
    o.streams = streams
    o.flags = flags
    o.chunk_samples = chunk_samples
    o.largest_first = 1 if largest_first else 0
    o.tiles = 1 if tiles else 0
    return arr, o, BatchStats()


def render_batch(jobs, streams=0, flags=0, chunk_samples=0, device=0, largest_first=False, tiles=False):
    """az_gpu_render_batch.  jobs: list of dicts with keys gpu_scene (GpuScene), film_ptr (device film of
    the scene's camera resolution) and optionally guide (Guide), train, seed, scissor, and camera_ptr,
    epsilons_ptr, filter_type (default: those of the GpuScene's host scene).  tiles: the plain jobs
    render together in tile waves on one stream while the other streams take the guided jobs.  Returns
    (per-job list of dicts done_ms/status/samples, batch stats dict)."""
    arr, o, st = _batch_args(jobs, streams, flags, chunk_samples, device, largest_first, tiles)
    rc = lib().az_gpu_render_batch(arr, len(jobs), C.byref(o), C.byref(st))
    per = [{"done_ms": arr[k].done_ms, "status": arr[k].status, "samples": arr[k].samples} for k in range(len(jobs))]
    _check(rc, "az_gpu_render_batch")
    return per, {"samples": st.samples, "gpu_ms": st.gpu_ms, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
                 "jobs": st.jobs, "failed": st.failed, "streams": st.streams}


def _stats(st):
    if st is None:
        return None
    return {"samples": st.samples, "extend_rays": st.extend_rays, "shadow_rays": st.shadow_rays,
            "chunks": st.chunks, "retries": st.retries, "kernel_launches": st.kernel_launches,
            "gpu_ms": st.gpu_ms, "extend_ms": st.extend_ms, "shade_ms": st.shade_ms, "shadow_ms": st.shadow_ms,
            "node_visits": st.node_visits, "prim_visits": st.prim_visits, "extend_launches": st.extend_launches,
            "shadow_node_visits": st.shadow_node_visits, "shadow_prim_visits": st.shadow_prim_visits}


def device_info(device=0):
    buf = C.create_string_buffer(256)
    rc = lib().az_gpu_device_info(device, buf, 256)
    return buf.value.decode() if rc == 0 else None
