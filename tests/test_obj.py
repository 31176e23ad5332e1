"""OBJ / MTL import (pm_obj_load): against the reference's own loader
(loadOBJ, CPM/ObjLoader.cpp, compiled from its sources into
oracle/_ref/libref_host.so) on files it parses, and against hand-checked
answers where the reference's loader is undefined."""
import ctypes as C
import os

import numpy as np
import pytest

import photonmap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
# the reference's Cornell-sphere scene, where the reference is mounted
# ($PM_REFERENCE_ROOT, default /root/reference; the test skips without it)
REF_OBJ = os.path.join(os.environ.get("PM_REFERENCE_ROOT", "/root/reference"), "CudaPhotonMapping", "Models",
                       "cornell_box_sphere")

MTL = """# materials
newmtl white
    Kd 0.75 0.75 0.75
    Ks 0 0 0
    Ns 0
newmtl red
\tKd 0.75 0.25 0.25
\tKs 0 0 0
newmtl glass
    Kd 0.01 0.01 0.01
    Ks 0.9 0.9 0.9
    Tr 0.9
    Ni 1.5
newmtl lamp
    Kd 0.78 0.78 0.78
    Ke 10 10 10
    d 1.0
"""

# faces in the forms the reference parses (v/vt/vn, v//vn), a quad model, a
# triangle model with negative indices, a run split by an 's' line (the name
# repeats: the second copy becomes "wall1"), a material without Ks (specular
# stays Material()'s 1), an unknown material (all defaults).  Each model keeps
# one face form: the reference's build_vertices (ObjLoader.cpp:102-105) reads
# a texcoord index for every vertex once any face of the model had one, so a
# model mixing v/vt/vn and v//vn faces makes it read past its index vector
# (undefined behaviour, an occasional crash).
OBJ = """mtllib box.mtl
# floor: two quads
g floor
usemtl white
v -1 -1 -1
v 1 -1 -1
v 1 -1 1
v -1 -1 1
v -1 -1 3
v 1 -1 3
vn 0 1 0
vt 0 0
vt 1 0
vt 1 1
f 1/1/1 2/2/1 3/3/1 4/1/1
f 4/1/1 3/2/1 6/3/1 5/1/1

g wall
usemtl red
v -1 -1 -1
v -1 1 -1
v -1 1 1
vn 1 0 0
vn 0.6 0.8 0
f -3//-1 -2//-2 -1//-1
s 1
f -3//-2 -1//-1 -2//-1
g sphere
usemtl glass
v 0 0 0
v 0.5 0 0
v 0 0.5 0
v 0 0 0.5
vn 0 0 1
f 10//4 11//4 12//4
f 10//4 12//4 13//4
f 10//4 13//4 11//4
g light
usemtl lamp
v -0.25 0.99 -0.25
v 0.25 0.99 -0.25
v 0.25 0.99 0.25
v -0.25 0.99 0.25
vn 0 -1 0
f 14//5 15//5 16//5 17//5
g odd
usemtl nosuchmaterial
f 1//1 2//1 3//1
"""


def _write(tmp, obj=OBJ, mtl=MTL, name="box.obj", crlf=False):
    if crlf:
        obj = obj.replace("\n", "\r\n")
    (tmp / name).write_text(obj)
    (tmp / "box.mtl").write_text(mtl)
    return str(tmp / name)


def _lib():
    return photonmap.library()


def _ref():
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libref_host.so not built (the reference sources are absent)")
    L = C.CDLL(REF_LIB)
    L.ref_obj_load.restype = C.c_void_p
    L.ref_obj_load.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.ref_obj_model.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p,
                                C.c_char_p, C.c_int]
    L.ref_obj_vertices.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.ref_obj_free.argtypes = [C.c_void_p]
    return L


def _ref_scene(path):
    """The reference loader's models as a triangle soup in the reference's
    intersection order (a quad v0..v3 is (v0 v1 v3) then (v1 v2 v3))."""
    L = _ref()
    d, f = os.path.split(path)
    nm, nv = C.c_int(), C.c_int()
    h = L.ref_obj_load(d.encode(), f.encode(), C.byref(nm), C.byref(nv))
    assert h, "the reference loader threw"
    try:
        pos = np.zeros((nv.value, 3), np.float32)
        nrm = np.zeros((nv.value, 3), np.float32)
        L.ref_obj_vertices(h, pos.ctypes.data, nrm.ctypes.data)
        tp, tn, tm, mats, names = [], [], [], [], []
        at = 0
        for m in range(nm.value):
            ty, sz = C.c_int(), C.c_int()
            mat = np.zeros(12, np.float32)
            name = C.create_string_buffer(256)
            L.ref_obj_model(h, m, C.byref(ty), C.byref(sz), mat.ctypes.data, name, 256)
            corners = {0: [[0, 1, 2]], 1: [[0, 1, 3], [1, 2, 3]]}[ty.value]
            step = 3 if ty.value == 0 else 4
            for p0 in range(at, at + sz.value, step):
                for c in corners:
                    tp.append(pos[[p0 + i for i in c]])
                    tn.append(nrm[[p0 + i for i in c]])
                    tm.append(m)
            at += sz.value
            mats.append(mat)
            names.append(name.value.decode())
        return np.array(tp), np.array(tn), np.array(tm, np.int32), np.array(mats), tuple(names)
    finally:
        L.ref_obj_free(h)


def _compare(sc, ref):
    tp, tn, tm, mats, names = ref
    assert sc.names == names
    assert np.array_equal(sc.tri_model, tm)
    assert np.array_equal(sc.tri_pos, tp)
    assert np.array_equal(sc.tri_nrm, tn)
    assert np.array_equal(sc.materials, mats)


def test_loader_matches_reference_loader(tmp_path):
    path = _write(tmp_path)
    sc = photonmap.load_obj(path, default_ior=1.0)
    _compare(sc, _ref_scene(path))
    assert sc.names == ("floor", "wall", "wall1", "sphere", "light", "odd")
    assert sc.light_model == 4
    assert sc.ntri == 4 + 2 + 3 + 2 + 1
    # Material() defaults where the MTL is silent: specular 1 (lamp), everything (odd)
    assert np.array_equal(sc.materials[4, 3:6], [1, 1, 1])
    assert np.array_equal(sc.materials[5], np.array([1, 1, 1, 1, 1, 1, 0, 0, 0, 1, 1, 16], np.float32))
    assert np.isclose(sc.materials[3, 10], 0.1) and sc.materials[3, 9] == np.float32(1.5)


def test_crlf_line_ends_read_like_lf(tmp_path):
    # (the reference's face parser miscounts the last vertex before a '\r')
    a = photonmap.load_obj(_write(tmp_path, name="lf.obj"))
    b = photonmap.load_obj(_write(tmp_path, name="crlf.obj", crlf=True))
    assert a.names == b.names and a.light_model == b.light_model
    for x, y in ((a.tri_pos, b.tri_pos), (a.tri_nrm, b.tri_nrm), (a.tri_model, b.tri_model), (a.materials, b.materials)):
        assert np.array_equal(x, y)


def test_loader_matches_reference_on_its_cornell_scene():
    if not os.path.isdir(REF_OBJ):
        pytest.skip("reference sources absent")
    path = os.path.join(REF_OBJ, "CornellBox-Sphere.obj")
    sc = photonmap.load_obj(path)
    _compare(sc, _ref_scene(path))
    assert sc.ntri == 2188 and sc.names[sc.light_model] == "light"


def test_forms_the_reference_loader_gets_wrong(tmp_path):
    """Position-only faces, faces without normals (flat normal), a polygon
    (fan), mixed triangles and quads in one model."""
    obj = """mtllib box.mtl
g light
usemtl lamp
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v -1 0.5 0
f 1 2 3
f 1 2 3 4
f 1 2 3 4 5
"""
    sc = photonmap.load_obj(_write(tmp_path, obj=obj))
    assert sc.ntri == 1 + 2 + 3 and sc.nmodel == 1
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [-1, 0.5, 0]], np.float32)
    expect = [v[[0, 1, 2]], v[[0, 1, 3]], v[[1, 2, 3]], v[[0, 1, 2]], v[[0, 2, 3]], v[[0, 3, 4]]]
    assert np.array_equal(sc.tri_pos, np.array(expect))
    assert np.array_equal(sc.tri_nrm, np.broadcast_to(np.float32([0, 0, 1]), (6, 3, 3)))


def test_mixed_face_forms_in_one_model(tmp_path):
    """v/vt/vn and v//vn faces in one model (the reference's loader reads past
    its texture-index vector here): positions and normals as indexed."""
    obj = """mtllib box.mtl
g light
usemtl lamp
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
vt 0 0
vt 1 0
vn 0 0 1
vn 0 0.6 0.8
f 1/1/1 2/2/1 3/1/2
f 1//2 3//1 4//2
"""
    sc = photonmap.load_obj(_write(tmp_path, obj=obj))
    assert sc.ntri == 2 and sc.nmodel == 1
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    n = np.array([[0, 0, 1], [0, 0.6, 0.8]], np.float32)
    assert np.array_equal(sc.tri_pos, np.array([v[[0, 1, 2]], v[[0, 2, 3]]]))
    assert np.array_equal(sc.tri_nrm, np.array([n[[0, 0, 1]], n[[1, 0, 1]]]))


@pytest.mark.parametrize("obj, what", [
    ("g light\nf 1 2 3\n", "vertex index out of range"),
    ("v 0 0 0\nv 1 0 0\nf 1 2\n", "at least 3 vertices"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1//7 2//7 3//7\n", "normal index out of range"),
    ("v 0 0\n", "three numbers"),
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1/x 2 3\n", "bad face vertex"),
    ("mtllib missing.mtl\nusemtl a\n", "cannot open material file"),
])
def test_malformed_files_are_errors(tmp_path, obj, what):
    with pytest.raises(photonmap.PMError, match=what):
        photonmap.load_obj(_write(tmp_path, obj=obj))


def test_missing_file_and_missing_light(tmp_path):
    with pytest.raises(photonmap.PMError, match="PM_ERR_IO"):
        photonmap.load_obj(str(tmp_path / "nope.obj"))
    with pytest.raises(photonmap.PMError, match="no model named 'light'"):
        photonmap.load_obj(_write(tmp_path, obj="v 0 0 0\nv 1 0 0\nv 0 1 0\ng tri\nf 1 2 3\n"))


def _save_obj(sc, tmp, name="scene.obj"):
    """A photonmap Scene as OBJ + MTL (one group and material per model, one
    vertex and one normal per triangle corner, shortest round-trip floats)."""
    f = lambda x: repr(float(np.float32(x)))  # noqa: E731
    obj, mtl = ["mtllib scene.mtl"], []
    vi = 1
    for m in range(sc.nmodel):
        mat = sc.materials[m]
        mtl += [f"newmtl m{m}", "Kd " + " ".join(map(f, mat[0:3])), "Ks " + " ".join(map(f, mat[3:6])),
                "Ke " + " ".join(map(f, mat[6:9])), f"Ni {f(mat[9])}", f"d {f(mat[10])}", f"Ns {f(mat[11])}"]
        obj += [f"g {sc.names[m]}", f"usemtl m{m}"]
        tris = np.flatnonzero(sc.tri_model == m)
        for t in tris:
            for c in range(3):
                obj.append("v " + " ".join(map(f, sc.tri_pos[t, c])))
                obj.append("vn " + " ".join(map(f, sc.tri_nrm[t, c])))
        obj += [f"f {vi + 3 * i}//{vi + 3 * i} {vi + 3 * i + 1}//{vi + 3 * i + 1} {vi + 3 * i + 2}//{vi + 3 * i + 2}"
                for i in range(len(tris))]
        vi += 3 * len(tris)
    (tmp / name).write_text("\n".join(obj) + "\n")
    (tmp / "scene.mtl").write_text("\n".join(mtl) + "\n")
    return str(tmp / name)


def test_scene_round_trips_through_obj(tmp_path):
    from photonmap import scenes
    sc = scenes.cornell(sphere_level=2)
    back = photonmap.load_obj(_save_obj(sc, tmp_path), default_ior=sc.default_ior)
    assert back.names == sc.names and back.light_model == sc.light_model
    for a, b in ((back.tri_pos, sc.tri_pos), (back.tri_nrm, sc.tri_nrm), (back.tri_model, sc.tri_model),
                 (back.materials, sc.materials), (back.light_intensity, sc.light_intensity)):
        assert np.array_equal(a, np.asarray(b, a.dtype))


@pytest.mark.gpu
def test_obj_scene_renders_like_the_original(tmp_path):
    """The imported scene drives the photon pass and the frame exactly as the
    scene it was written from."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from photonmap import scenes
    sc = scenes.cornell(sphere_level=2)
    back = photonmap.load_obj(_save_obj(sc, tmp_path), default_ior=sc.default_ior)
    ctx = photonmap.Context(0)
    cam = photonmap.camera_setup((0, 0, 3.5), (0, 0, -1), (0, 1, 0), 45.0, 128, 96)
    out = []
    for s in (sc, back):
        ctx.set_scene(s)
        ctx.trace_photons(0, 8, 50_000, 5_000)
        ctx.build_grid(0)
        ctx.build_grid(1)
        rgb, rad = ctx.render(cam, 100, 0.1, 4, k_caustic=32, r_caustic=0.1)
        out.append((ctx.photons(0, sorted_=False)["list_pos"].cpu().numpy(), rgb.cpu().numpy(), rad.cpu().numpy()))
        assert ctx.status() == 0
    for a, b in zip(*out):
        assert np.array_equal(a, b)
