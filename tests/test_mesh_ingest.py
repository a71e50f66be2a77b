"""Scene ingestion on the GPU: the importer's mesh post-processing
(src/azimuth_xml.cpp:3632-3750) as az_gpu_mesh_postprocess, bit for bit
against the numpy restatement in oracle/mesh_oracle.py, which is itself pinned
against the host scene builder's finished azimuth structs (the input of
azimuth's renderer in the render parity tests) and against azimuth's own
importer (tests/test_xml_import.py); and a device scene built from
the raw mesh soup (az_gpu_scene_create_from_meshes) against one built from
the finished structs."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mesh_oracle as mo  # noqa: E402

SCENES = [(az.SCENE_CORNELL, {}), (az.SCENE_DENSE_MESH, {"detail": 3}), (az.SCENE_INTERIOR, {"detail": 3}),
          (az.SCENE_FEATURES, {})]
IDS = ["cornell", "dense_mesh", "interior", "features"]

# byte offsets in azimuth's structs (include/az_abi.h; x86-64)
SCENE_MESHES, SCENE_MESH_COUNT = 1352, 2704
MESH_SIZE, MESH_BVH, MESH_TRIS, MESH_AREA, MESH_COUNT = 200, 152, 160, 168, 180
ENT_RIGHT, ENT_LEFT, ENT_ID, ENT_TYPE = 40, 48, 276, 284


def _u32(addr):
    return C.c_uint32.from_address(addr).value


def _ptr(addr):
    return C.c_void_p.from_address(addr).value


def _f32(addr, n):
    return np.ctypeslib.as_array((C.c_float * n).from_address(addr)).copy()


def _builder_meshes(scene):
    """Per mesh of the finished scene: triangles (F, 12), TotalArea, and the triangle entities' N0-N2 and
    UV0-UV2 (F, 15) by face id (entity.ID), from a walk of the mesh BVH."""
    base, n = _ptr(scene.scene_ptr + SCENE_MESHES), _u32(scene.scene_ptr + SCENE_MESH_COUNT)
    out = []
    for i in range(n):
        m = base + i * MESH_SIZE
        cnt = _u32(m + MESH_COUNT)
        tris = _f32(_ptr(m + MESH_TRIS), 12 * cnt).reshape(cnt, 12)
        area = np.float32(C.c_float.from_address(m + MESH_AREA).value)
        attrs = np.zeros((cnt, 15), np.float32)
        stack = [_ptr(m + MESH_BVH)]
        while stack:
            e = stack.pop()
            if _u32(e + ENT_TYPE) == 3:   # BVH node
                stack += [_ptr(e + ENT_RIGHT), _ptr(e + ENT_LEFT)]
                continue
            attrs[_u32(e + ENT_ID)] = _f32(e + 36, 15)   # N0, N1, N2 (36..72), skip FaceNormal, UVs (84..108)
            attrs[_u32(e + ENT_ID), 9:15] = _f32(e + 84, 6)
        out.append((tris, area, attrs))
    return out


def _oracle(scene):
    v, f, uv, descs = scene.soup_arrays()
    return mo.postprocess(v, f, uv, descs), descs


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("scene_id,kw", SCENES, ids=IDS)
def test_oracle_matches_the_scene_builder(scene_id, kw):
    sc = az.generate_scene(scene_id, seed=1, width=16, height=16, spp=1, **kw)
    try:
        o, descs = _oracle(sc)
        built = _builder_meshes(sc)
        assert len(built) == len(descs)
        for d, (tris, area, attrs) in zip(descs, built):
            b, n = d["face_base"], d["face_count"]
            assert np.array_equal(_bits(tris), _bits(o["triangles"][b:b + n]))
            assert _bits(area) == _bits(o["total_area"][descs.index(d)])
            assert np.array_equal(_bits(attrs), _bits(o["attrs"][b:b + n]))
    finally:
        sc.close()


def test_soup_only_scene_has_the_same_soup_and_no_mesh_structs():
    full = az.generate_scene(az.SCENE_DENSE_MESH, seed=2, width=16, height=16, spp=1, detail=2)
    soup = az.generate_scene(az.SCENE_DENSE_MESH, seed=2, width=16, height=16, spp=1, detail=2, soup_only=True)
    try:
        a, b = full.soup_arrays(), soup.soup_arrays()
        for x, y in zip(a[:3], b[:3]):
            assert np.array_equal(x, y)
        assert a[3] == b[3]
        base = _ptr(soup.scene_ptr + SCENE_MESHES)
        for i in range(_u32(soup.scene_ptr + SCENE_MESH_COUNT)):
            assert _ptr(base + i * MESH_SIZE + MESH_TRIS) is None and _ptr(base + i * MESH_SIZE + MESH_BVH) is None
    finally:
        full.close()
        soup.close()


def _soup_struct(v, f, uv, descs):
    """An az_mesh_soup over numpy arrays (kept alive by the returned tuple)."""
    v = np.ascontiguousarray(v, np.float32)
    f = np.ascontiguousarray(f, np.uint32)
    uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    md = (az.MeshDesc * max(1, len(descs)))()
    for i, d in enumerate(descs):
        md[i].face_base, md[i].face_count, md[i].uv_offset = d["face_base"], d["face_count"], d["uv_offset"]
        md[i].transform[0] = md[i].transform[5] = md[i].transform[10] = md[i].transform[15] = 1.0
        md[i].inv_transform[0] = md[i].inv_transform[5] = md[i].inv_transform[10] = md[i].inv_transform[15] = 1.0
    s = az.MeshSoup(v.ctypes.data, f.ctypes.data, uv.ctypes.data if uv.size else None, C.addressof(md),
                    v.shape[0], f.shape[0], uv.shape[0], len(descs))
    return s, (v, f, uv, md)


def _gpu_postprocess(s):
    vn = np.zeros((s.vertex_count, 3), np.float32)
    tris = np.zeros((s.face_count, 12), np.float32)
    attrs = np.zeros((s.face_count, 15), np.float32)
    area = np.zeros(s.mesh_count, np.float32)
    rc = az.lib().az_gpu_mesh_postprocess(C.addressof(s), vn.ctypes.data, tris.ctypes.data, attrs.ctypes.data,
                                          area.ctypes.data, C.byref(az.make_opts()))
    return rc, {"vertex_normals": vn, "triangles": tris, "attrs": attrs, "total_area": area}


def _same(a, b):
    # bit for bit, except that a NaN (the 0/0 normal of a zero-area face) may
    # carry another payload: x86 makes 0xFFC00000, the GPU 0x7FFFFFFF
    for k in ("vertex_normals", "triangles", "attrs", "total_area"):
        x, y = np.asarray(a[k], np.float32), np.asarray(b[k], np.float32)
        nan = np.isnan(x) & np.isnan(y)
        assert np.array_equal(_bits(x)[~nan], _bits(y)[~nan]) and np.array_equal(np.isnan(x), np.isnan(y)), k


@pytest.mark.gpu
@pytest.mark.parametrize("scene_id,kw", SCENES, ids=IDS)
def test_gpu_postprocess_is_bit_exact(gpu, scene_id, kw):
    sc = az.generate_scene(scene_id, seed=1, width=16, height=16, spp=1, **kw)
    try:
        o, _ = _oracle(sc)
        _same(az.mesh_postprocess(sc), o)
    finally:
        sc.close()


@pytest.mark.gpu
def test_gpu_postprocess_edge_cases(gpu):
    rng = np.random.default_rng(5)
    v = rng.normal(size=(40, 3)).astype(np.float32)
    f = rng.integers(0, 39, (60, 3)).astype(np.uint32)   # vertex 39 is used by no face
    f[3] = (7, 7, 9)                                    # a vertex twice in one face: zero area, NaN normal
    f[4] = (1, 1, 1)
    uv = rng.uniform(size=(30, 2)).astype(np.float32)
    descs = [{"face_base": 0, "face_count": 20, "uv_offset": -5},      # some UV indices negative
             {"face_base": 20, "face_count": 25, "uv_offset": 3},      # some past the end
             {"face_base": 50, "face_count": 10, "uv_offset": 0}]      # faces 45-49 in no mesh
    s, keep = _soup_struct(v, f, uv, descs)
    rc, g = _gpu_postprocess(s)
    assert rc == 0
    _same(g, mo.postprocess(v, f, uv, descs))
    assert not g["vertex_normals"][39].any()


@pytest.mark.gpu
def test_gpu_postprocess_rejects_bad_soups(gpu):
    v = np.zeros((3, 3), np.float32)
    s, keep = _soup_struct(v, [[0, 1, 3]], np.zeros((0, 2)), [{"face_base": 0, "face_count": 1, "uv_offset": 0}])
    assert _gpu_postprocess(s)[0] == 2            # vertex index past the array: AZ_ERR_INVALID_SCENE
    s, keep = _soup_struct(v, [[0, 1, 2]] * 4, np.zeros((0, 2)),
                           [{"face_base": 0, "face_count": 3, "uv_offset": 0},
                            {"face_base": 2, "face_count": 2, "uv_offset": 0}])
    assert _gpu_postprocess(s)[0] == 2            # overlapping meshes


def _rays(n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d, rng.uniform(0, 1, (n, 1)).astype(np.float32)], axis=1)


@pytest.mark.gpu
@pytest.mark.parametrize("scene_id,kw", SCENES, ids=IDS)
def test_scene_from_soup_renders_like_the_finished_scene(gpu, scene_id, kw):
    import torch
    full = az.generate_scene(scene_id, seed=4, width=48, height=32, spp=4, **kw)
    soup = az.generate_scene(scene_id, seed=4, width=48, height=32, spp=4, soup_only=True, **kw)
    try:
        span = (0.5, 3.5) if scene_id == az.SCENE_INTERIOR else (-1.0, 1.0)
        rays = _rays(1 << 14, scene_id, *span)
        with az.GpuScene(full) as a, az.GpuScene(soup, from_soup=True) as b:
            ha, hb = a.closest_hit(rays), b.closest_hit(rays)
            info = b.info()
            assert info["triangles"] == a.info()["triangles"] and info["ingest_ms"] > 0.0
            # the same primitives: identical nearest hits except exact ties, which the
            # two hierarchies may break differently
            same = (ha[0] == hb[0]) & (ha[1] == hb[1]) & (ha[2] == hb[2]) & (ha[3] == hb[3])
            assert same.mean() >= 0.999
            assert np.array_equal(ha[3][~same], hb[3][~same])   # a tie: same distance
            w, h = full.resolution()
            fa = torch.zeros((h, w, 4), device="cuda")
            fb = torch.zeros((h, w, 4), device="cuda")
            a.render_device(fa.data_ptr(), seed=9)
            b.render_device(fb.data_ptr(), seed=9)
            assert ol.film_compare(fa.cpu().numpy(), fb.cpu().numpy(), 1e-4)[0] >= 0.999
    finally:
        full.close()
        soup.close()
