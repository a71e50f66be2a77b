"""azimuth's own scene importer, ImportXML with its PLY loader
(src/azimuth_xml.cpp:3021-3930), run on a hand-written scene through the
header-only reader (include/az_xmlreader.h) in place of libxml2, then the
imported structs rendered and intersected by the GPU path against azimuth's
own render code.  tests/scenes/box.xml holds an inline mesh, a light mesh, a
point light, spheres, a smooth mesh from an ASCII PLY file with a quad face, a
transformed instance of it, and a cube from a binary PLY file with motion;
tests/scenes/features.xml the lights, materials, textures and indexing
options that box.xml leaves out."""
import ctypes as C
import os
import shutil
import struct
import sys
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import azimuth_b200 as az
import oracle_lib as ol

HERE = os.path.dirname(os.path.abspath(__file__))
SCENES = os.path.join(HERE, "scenes")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import mesh_oracle as mo  # noqa: E402

pytestmark = pytest.mark.skipif(not ol.have_ref(), reason="reference harness not built")


def _cube_ply(path, half=0.15):
    """A cube as a binary little-endian PLY file: 8 vertices of x y z nx ny nz u v, 6 quads."""
    v = np.array([[x, y, z] for x in (-half, half) for y in (-half, half) for z in (-half, half)], np.float32)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    for a, b, c, d in quads:   # outward windings, checked on both halves of the split
        for tri in ((a, b, c), (a, c, d)):
            n = np.cross(v[tri[1]] - v[tri[0]], v[tri[2]] - v[tri[0]])
            assert np.dot(n, v[list(tri)].mean(0)) > 0
    head = ("ply\nformat binary_little_endian 1.0\ncomment a cube for azimuth's PLY loader\n"
            "element vertex 8\nproperty float x\nproperty float y\nproperty float z\n"
            "property float nx\nproperty float ny\nproperty float nz\nproperty float u\nproperty float v\n"
            "element face 6\nproperty list uchar int vertex_indices\nend_header\n").encode()
    body = b"".join(struct.pack("<8f", *p, *(p / np.linalg.norm(p)), 0.5, 0.5) for p in v)
    body += b"".join(struct.pack("<B4i", 4, *q) for q in quads)
    with open(path, "wb") as f:
        f.write(head + body)


def write_box_scene(dirpath, xml_text=None):
    ascii_ply = os.path.join(dirpath, "pyramid.ply")
    binary_ply = os.path.join(dirpath, "cube.ply")
    shutil.copy(os.path.join(SCENES, "pyramid.ply"), ascii_ply)
    _cube_ply(binary_ply)
    text = xml_text if xml_text is not None else open(os.path.join(SCENES, "box.xml")).read()
    text = text.replace("@PLY_ASCII@", ascii_ply).replace("@PLY_BINARY@", binary_ply)
    path = os.path.join(dirpath, "box.xml")
    with open(path, "w") as f:
        f.write(text)
    return path


def write_features_scene(dirpath):
    """tests/scenes/features.xml with its image texture, a 16x12 PNG written by the library's writer."""
    y, x = np.mgrid[0:12, 0:16]
    rgb8 = np.stack([x * 16, y * 20, ((x // 4 + y // 4) % 2) * 200 + 30], -1).astype(np.uint8)
    image = os.path.join(dirpath, "checker.png")
    az.write_image(image, rgb8, az.FILE_PNG)
    text = open(os.path.join(SCENES, "features.xml")).read().replace("@IMAGE@", image)
    path = os.path.join(dirpath, "features.xml")
    with open(path, "w") as f:
        f.write(text)
    return path


class ImportedScene:
    """The scene, first camera and epsilons that ImportXML produced (azimuth's own structs)."""

    filter_type = az.FILTER_BOX       # RenderScene's filter (src/azimuth_main.cpp:1847)

    def __init__(self, path):
        L = ol.ref()
        L.azref_import_xml.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.azref_import_xml.restype = C.c_int
        L.azref_scene_summary.argtypes = [C.c_void_p, C.c_void_p]
        s, cams, eps = C.c_void_p(), C.c_void_p(), C.c_void_p()
        n = C.c_uint32()
        self.ok = L.azref_import_xml(os.fsencode(path), C.byref(s), C.byref(cams), C.byref(n), C.byref(eps)) == 1
        self.scene_ptr, self.camera_ptr, self.epsilons_ptr = s.value, cams.value, eps.value
        self.camera_count = n.value
        self.path = path
        self._soup = None
        # the Perlin gradient table the import filled (a process-wide table in azimuth)
        self._grad = np.zeros(768, np.float32)
        L.azref_get_perlin_gradients.argtypes = [C.c_void_p]
        L.azref_get_perlin_gradients(self._grad.ctypes.data)
        self.perlin_gradients = self._grad.ctypes.data if self.ok else None

    def resolution(self):
        buf = (C.c_uint32 * 2).from_address(self.camera_ptr + 340)   # az_camera.Resolution
        return int(buf[0]), int(buf[1])

    def sample_count(self):
        return int(C.c_uint32.from_address(self.camera_ptr + 384).value)

    def summary(self):
        out = (C.c_uint32 * 9)()
        ol.ref().azref_scene_summary(self.scene_ptr, out)
        keys = ("meshes", "materials", "lights", "triangles", "spheres", "instances", "emitters", "path_trace",
                "max_depth")
        return dict(zip(keys, (int(x) for x in out)))

    def mesh_arrays(self, m):
        """azimuth's finished mesh m: (triangles (F, 12), triangle entities (F, 24), TotalArea, MeshDesc)."""
        L = ol.ref()
        L.azref_mesh_arrays.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.azref_mesh_arrays.restype = C.c_int
        cap = 4096
        tris, ents = np.zeros((cap, 12), np.float32), np.zeros((cap, 24), np.float32)
        area, desc = C.c_float(), az.MeshDesc()
        n = L.azref_mesh_arrays(self.scene_ptr, m, tris.ctypes.data, ents.ctypes.data, C.byref(area), C.byref(desc))
        assert 0 <= n <= cap
        return tris[:n], ents[:n], np.float32(area.value), desc

    def soup(self):
        """The arrays ImportXML gathers before its mesh loop, rebuilt from the scene file: the XML
        vertices, then each PLY file's vertices (src/azimuth_xml.cpp:3498-3508); the inline faces in
        document order made 0-based (:2707-2735), then each PLY file's faces with its vertex offset,
        quads split as (a, b, c), (a, c, d) (:3514-3600); UVs from the PLY files; per mesh its face
        range and UVOffset (-vertex offset for a PLY mesh, :3606-3614).  Returns (vertices, faces,
        uvs, descs) with the other desc fields from azimuth's finished meshes."""
        root = ET.parse(self.path).getroot()
        verts = [np.array(root.find("VertexData").text.split(), np.float32).reshape(-1, 3)]
        zb = root.find("ZeroBasedIndexing")
        one_based = zb is None or zb.text.strip() != "true"
        tc = root.find("TexCoordData")
        faces, ranges, plys = [], [], []
        uvs = [np.array(tc.text.split(), np.float32).reshape(-1, 2) if tc is not None else np.zeros((0, 2), np.float32)]
        for m in (e for e in root.find("Objects") if e.tag in ("Mesh", "LightMesh")):
            fe = m.find("Faces")
            if fe.get("plyFile"):
                plys.append((len(ranges), fe.get("plyFile")))
                ranges.append(None)
            else:
                voff = int(fe.get("vertexOffset", 0))
                f = np.array(fe.text.split(), np.int64).reshape(-1, 3) + voff - (1 if one_based else 0)
                ranges.append((sum(len(x) for x in faces), len(f), int(fe.get("textureOffset", 0)) - voff))
                faces.append(f)
        nverts = len(verts[0])
        for mi, path in plys:
            v, f, uv = read_ply(path)
            ranges[mi] = (sum(len(x) for x in faces), len(f), -nverts)
            faces.append(f + nverts)
            verts.append(v)
            uvs.append(uv)
            nverts += len(v)
        # entities made while parsing (MeshInstance, Sphere, LightSphere) come before the meshes' instances
        first = sum(1 for e in root.find("Objects") if e.tag in ("MeshInstance", "Sphere", "LightSphere"))
        descs = []
        for mi, (base, count, uv_off) in enumerate(ranges):
            d = self.mesh_arrays(mi)[3]
            d.face_base, d.face_count, d.unique_entity_id = base, count, first + mi
            assert d.uv_offset == uv_off
            descs.append(d)
        return (np.concatenate(verts), np.concatenate(faces).astype(np.uint32), np.concatenate(uvs), descs)

    @property
    def soup_ptr(self):
        """An az_mesh_soup of soup() (kept alive with this object)."""
        if self._soup is None:
            v, f, uv, descs = self.soup()
            v, f, uv = (np.ascontiguousarray(x) for x in (v, f, uv))
            arr = (az.MeshDesc * len(descs))(*descs)
            soup = az.MeshSoup(v.ctypes.data, f.ctypes.data, uv.ctypes.data, C.addressof(arr), len(v), len(f),
                               len(uv), len(descs))
            self._soup = (v, f, uv, arr, soup)
        return C.addressof(self._soup[4])


def read_ply(path):
    """Vertices (x y z), triangles (quads split) and UVs of a PLY file as azimuth's loader reads it:
    eight floats per vertex (x y z nx ny nz u v), faces as a uchar count and int indices."""
    data = open(path, "rb").read()
    head, body = data.split(b"end_header\n", 1)
    words = head.decode().split()
    nv = int(words[words.index("vertex") + 1])
    nf = int(words[words.index("face") + 1])
    if "ascii" in words:
        tok = body.split()
        v8 = np.array(tok[:8 * nv], np.float32).reshape(nv, 8)
        pos, polys = 8 * nv, []
        for _ in range(nf):
            k = int(tok[pos])
            polys.append([int(t) for t in tok[pos + 1:pos + 1 + k]])
            pos += 1 + k
    else:
        v8 = np.frombuffer(body, "<f4", 8 * nv).reshape(nv, 8)
        pos, polys = 32 * nv, []
        for _ in range(nf):
            k = body[pos]
            polys.append(list(struct.unpack_from("<%di" % k, body, pos + 1)))
            pos += 1 + 4 * k
    tris = []
    for p in polys:
        tris += [p[:3]] if len(p) == 3 else [[p[0], p[1], p[2]], [p[0], p[2], p[3]]]
    return v8[:, :3].copy(), np.array(tris, np.int64), v8[:, 6:8].copy()


def check_mesh_results(scene, tris, attrs, areas):
    """The post-processed soup (face order) against azimuth's finished meshes, bit for bit."""
    _, _, _, descs = scene.soup()
    for mi, d in enumerate(descs):
        want_tris, ents, want_area, _ = scene.mesh_arrays(mi)
        b, n = d.face_base, d.face_count
        assert len(want_tris) == n
        assert np.array_equal(tris[b:b + n].view(np.uint32), want_tris.view(np.uint32))
        assert areas[mi].view(np.uint32) == want_area.view(np.uint32)
        # the entities sit in BVH order: find each by its corners
        index = {tris[b + i, :9].tobytes(): i for i in range(n)}
        assert len(index) == n
        for e in ents:
            i = index[e[:9].tobytes()]
            assert np.array_equal(attrs[b + i].view(np.uint32), e[9:].view(np.uint32))


@pytest.fixture(scope="module")
def box(tmp_path_factory):
    sc = ImportedScene(write_box_scene(str(tmp_path_factory.mktemp("box"))))
    assert sc.ok
    return sc


@pytest.fixture(scope="module")
def features(tmp_path_factory):
    sc = ImportedScene(write_features_scene(str(tmp_path_factory.mktemp("features"))))
    assert sc.ok
    return sc


@pytest.fixture(params=["box", "features"])
def imported(request):
    return request.getfixturevalue(request.param)


def test_importer_reads_the_scene(box):
    assert box.camera_count == 1
    assert box.resolution() == (48, 40) and box.sample_count() == 4
    # meshes 1-3, the light mesh, the PLY pyramid (4 triangles + a quad split in two), the PLY cube
    # (6 quads); one instance per mesh plus the explicit MeshInstance; lights: the point light and
    # the light mesh as an entity light
    assert box.summary() == {"meshes": 6, "materials": 4, "lights": 2, "triangles": 6 + 2 + 2 + 2 + 6 + 12,
                             "spheres": 2, "instances": 7, "emitters": 1, "path_trace": 1, "max_depth": 4}


def test_importer_reads_the_feature_scene(features):
    assert features.camera_count == 1 and features.resolution() == (40, 32)
    # lights: area, spot, directional, then the light sphere as an entity light (ambient is a
    # scene colour); one instance per mesh plus the explicit MeshInstance
    assert features.summary() == {"meshes": 5, "materials": 6, "lights": 4, "triangles": 10, "spheres": 3,
                                  "instances": 6, "emitters": 0, "path_trace": 1, "max_depth": 5}
    assert np.abs(features._grad).max() > 0     # the Perlin textures filled the gradient table


def test_restatement_renders_the_imported_scene_like_azimuth(imported):
    ref = ol.ref_film(imported, seed=5, threads=1)
    port = ol.port_film(imported, seed=5, threads=1)
    assert np.array_equal(ref.view(np.uint32), port.view(np.uint32))
    assert (ref[..., :3] > 0).mean() > 0.5     # the scene is lit


def test_mesh_restatement_matches_the_importer(imported):
    v, f, uv, descs = imported.soup()
    out = mo.postprocess(v, f, uv, [{"face_base": d.face_base, "face_count": d.face_count,
                                     "uv_offset": d.uv_offset} for d in descs])
    check_mesh_results(imported, out["triangles"], out["attrs"], out["total_area"])


@pytest.mark.parametrize("edit", [
    ("<Radius>0.3</Radius>", "<Radius>0.3</Radius><Bogus/>"),            # an element the importer does not know
    ("<Faces>1 4 8   1 8 5</Faces>", "<Faces>1 4 8   1 8 5</Mesh>"),      # mismatched end tag
    ('<Mesh id="1">', "<Mesh id=1>"),                                    # unquoted attribute value
    ("<Objects>", "<Objects><Radius>1</Radius>"),                        # an element out of place
])
def test_import_failures_are_reported(tmp_path, edit):
    text = open(os.path.join(SCENES, "box.xml")).read()
    assert edit[0] in text
    sc = ImportedScene(write_box_scene(str(tmp_path), text.replace(edit[0], edit[1], 1)))
    assert not sc.ok


@pytest.mark.gpu
def test_gpu_renders_the_imported_scene(gpu, imported):
    ref = ol.ref_film(imported, seed=9)
    film = az.produce_image(imported, seed=9)
    other = az.produce_image(imported, seed=10)
    ok, _, relmse = ol.film_compare(film, ref, 1e-4)
    _, _, noise = ol.film_compare(other, ref, 1e-4)
    assert np.allclose(film[..., 3], ref[..., 3], rtol=1e-5, atol=1e-6)
    assert ok >= 0.95 and relmse <= 0.05 * noise


@pytest.mark.gpu
def test_gpu_mesh_postprocess_matches_the_importer(gpu, imported):
    out = az.mesh_postprocess(imported)
    check_mesh_results(imported, out["triangles"], out["attrs"], out["total_area"])


@pytest.mark.gpu
def test_gpu_scene_from_the_importers_arrays(gpu, imported):
    # az_gpu_scene_create_from_meshes: the importer's arrays post-processed on the GPU, the rest of
    # the scene (materials, lights, spheres, the MeshInstance element) from azimuth's structs
    ref = ol.ref_film(imported, seed=9)
    w, h = imported.resolution()
    film, other = np.zeros((h, w, 4), np.float32), np.zeros((h, w, 4), np.float32)
    with az.GpuScene(imported, from_soup=True) as g:
        g.render_host(film, seed=9)
        g.render_host(other, seed=10)
    ok, _, relmse = ol.film_compare(film, ref, 1e-4)
    _, _, noise = ol.film_compare(other, ref, 1e-4)
    assert ok >= 0.95 and relmse <= 0.05 * noise


@pytest.mark.gpu
@pytest.mark.parametrize("from_soup", [False, True], ids=["structs", "soup"])
def test_gpu_hits_on_the_imported_scene(gpu, imported, from_soup):
    rng = np.random.default_rng(4)
    n = 1 << 14
    o = rng.uniform((-0.95, 0.05, -0.95), (0.95, 1.95, 0.95), (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = rng.uniform(0.0, 1.0, (n, 1)).astype(np.float32)
    rays = np.concatenate([o, d, t], axis=1)
    want = ol.closest_hit("ref", imported, rays)
    with az.GpuScene(imported, from_soup=from_soup) as g:
        got = g.closest_hit(rays)
    # the importer sets every triangle entity's ID to 0 (src/azimuth_xml.cpp:3695); a soup-built
    # scene reports the face's index within its mesh instead
    same = (got[0] == want[0]) & (got[1] == want[1]) & ((got[2] == want[2]) | from_soup)
    if from_soup:
        mesh_hit = want[2][same] != 0xFFFFFFFF
        assert np.array_equal(got[2][same] == 0xFFFFFFFF, ~mesh_hit) and (got[2][same][mesh_hit] < 12).all()
    assert want[0].mean() > 0.75                 # both boxes are open only at the front (+z)
    assert same.mean() >= 0.999
    assert np.array_equal(got[3][same].view(np.uint32), want[3][same].view(np.uint32))


def test_binary_vertex_and_face_files_import_like_inline(tmp_path, box):
    # the importer's binaryFile forms (src/azimuth_xml.cpp:2397-2430, 2653-2697): a u32 count, then
    # float xyz per vertex or u32 index triples per face
    text = open(os.path.join(SCENES, "box.xml")).read()
    v0, v1 = text.index("<VertexData>"), text.index("</VertexData>") + len("</VertexData>")
    verts = np.array(text[v0 + len("<VertexData>"):v1 - len("</VertexData>")].split(), np.float32)
    vpath = str(tmp_path / "verts.bin")
    with open(vpath, "wb") as f:
        f.write(struct.pack("<I", len(verts) // 3) + verts.tobytes())
    text = text[:v0] + '<VertexData binaryFile="%s"/>' % vpath + text[v1:]
    f0 = text.index("<Faces>")
    f1 = text.index("</Faces>", f0) + len("</Faces>")
    faces = np.array(text[f0 + len("<Faces>"):f1 - len("</Faces>")].split(), np.uint32)
    fpath = str(tmp_path / "faces.bin")
    with open(fpath, "wb") as f:
        f.write(struct.pack("<I", len(faces) // 3) + faces.tobytes())
    text = text[:f0] + '<Faces binaryFile="%s"/>' % fpath + text[f1:]
    sc = ImportedScene(write_box_scene(str(tmp_path), text))
    assert sc.ok
    assert sc.summary() == box.summary()
    for m in range(box.summary()["meshes"]):
        a, b = sc.mesh_arrays(m), box.mesh_arrays(m)
        assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
        assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
        assert a[2].view(np.uint32) == b[2].view(np.uint32)
