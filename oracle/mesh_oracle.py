"""CPU restatement of azimuth's mesh post-processing, for the tests only.

ImportXML's loop over the parsed meshes (src/azimuth_xml.cpp:3632-3750) in
numpy float32, with every operation rounded as azimuth's IEEE build rounds it
(no contraction; numpy applies each float32 operation separately):

  * per-vertex normals (:3632-3667): for every face in order, the unnormalised
    Cross(P1 - P0, P2 - P0) (src/azimuth_math.cpp:1325-1333) is added to the
    running sums of its three vertices (x, then y, then z corner), each sum
    starting at 0; then Normalize (src/azimuth_math.cpp:1299-1313: divide by
    sqrt(x*x + y*y + z*z) unless it is 0)
  * per mesh (:3669-3750): FaceNormalLen = Length(Cross(...)), TotalArea +=
    FaceNormalLen / 2 serially in face order, the unit face normal by three
    divisions, N0-N2 from the vertex normals, UVk = UVs[index_k + UVOffset]
    when 0 <= index_k + UVOffset < len(UVs), else 0.

Pinned two ways: against azimuth's own ImportXML, run through the
header-only reader of include/az_xmlreader.h on tests/scenes/box.xml (inline,
ASCII PLY and binary PLY meshes; tests/test_xml_import.py), bit for bit; and
against the library's host scene builder, whose finished azimuth structs are
what azimuth's own renderer consumes in the render parity tests.
"""
import numpy as np

F32 = np.float32


def _cross(a, b):
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                     a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1).astype(F32)


def _length(v):
    return np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]).astype(F32)


def face_normals(vertices, faces):
    """Unnormalised face normals (F, 3) and their lengths (F,)."""
    v = np.asarray(vertices, F32)
    f = np.asarray(faces, np.int64)
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    fn = _cross((p1 - p0).astype(F32), (p2 - p0).astype(F32))
    return fn, _length(fn)


def vertex_normals(vertices, faces):
    """Per-vertex normals (V, 3): each vertex's serial sum in face, then corner, order, normalised."""
    v = np.asarray(vertices, F32)
    f = np.asarray(faces, np.int64)
    fn, _ = face_normals(v, f)
    nv = v.shape[0]
    acc = np.zeros((nv, 3), F32)
    if f.shape[0]:
        inc_v = f.reshape(-1)                        # incidence 3*face + corner
        inc_f = np.repeat(np.arange(f.shape[0]), 3)
        order = np.argsort(inc_v, kind="stable")     # per vertex: face order, then corner order
        sv, sf = inc_v[order], inc_f[order]
        first = np.searchsorted(sv, sv, side="left")
        rank = np.arange(sv.size) - first            # position of the incidence within its vertex
        for k in range(int(rank.max()) + 1):         # k-th addition of every vertex, in order
            sel = rank == k
            acc[sv[sel]] = (acc[sv[sel]] + fn[sf[sel]]).astype(F32)
    L = _length(acc)
    out = np.zeros_like(acc)
    nz = L != 0
    out[nz] = (acc[nz] / L[nz, None]).astype(F32)
    return out


def postprocess(vertices, faces, uvs, meshes):
    """Everything az_gpu_mesh_postprocess returns: vertex_normals (V, 3), triangles (F, 12: P0, P1, P2, unit
    N), attrs (F, 15: N0, N1, N2, UV0, UV1, UV2; UVs 0 for faces outside every mesh), total_area (M,).
    `meshes`: dicts with face_base, face_count, uv_offset."""
    v = np.asarray(vertices, F32)
    f = np.asarray(faces, np.int64)
    uv = np.asarray(uvs, F32).reshape(-1, 2)
    fn, ln = face_normals(v, f)
    with np.errstate(divide="ignore", invalid="ignore"):
        unit = (fn / ln[:, None]).astype(F32)
    vn = vertex_normals(v, f)
    nf = f.shape[0]
    tris = np.concatenate([v[f[:, 0]], v[f[:, 1]], v[f[:, 2]], unit], axis=1) if nf else np.zeros((0, 12), F32)
    attrs = np.zeros((nf, 15), F32)
    if nf:
        attrs[:, 0:3], attrs[:, 3:6], attrs[:, 6:9] = vn[f[:, 0]], vn[f[:, 1]], vn[f[:, 2]]
    area = np.zeros(len(meshes), F32)
    half = (ln / F32(2.0)).astype(F32)
    for mi, m in enumerate(meshes):
        b, n = m["face_base"], m["face_count"]
        if n:
            area[mi] = np.cumsum(half[b:b + n], dtype=F32)[-1]   # numpy's cumsum adds serially
        for c in range(3):
            u = f[b:b + n, c] + m["uv_offset"]
            ok = (u >= 0) & (u < uv.shape[0])
            vals = np.zeros((n, 2), F32)
            vals[ok] = uv[u[ok]]
            attrs[b:b + n, 9 + 2 * c:11 + 2 * c] = vals
    return {"vertex_normals": vn, "triangles": tris.astype(F32), "attrs": attrs, "total_area": area}
