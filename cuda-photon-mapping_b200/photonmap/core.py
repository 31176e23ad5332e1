"""Python host side of the B200 photon-mapping core: ctypes over the C ABI.

Every method is one call into ``lib/libpm_b200.so`` (declared in
include/pm_api.h).  PyTorch supplies device memory (tensors are passed by
``data_ptr()``); no computation happens in Python.  The library must be built
(``make -C cuda-photon-mapping_b200/csrc``): there is no fallback path, and a
missing library or CUDA device raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libpm_b200.so")

PM_MAP_GLOBAL = 0
PM_MAP_CAUSTIC = 1

ERRORS = {-1: "PM_ERR_INVALID", -2: "PM_ERR_CUDA", -3: "PM_ERR_OOM", -4: "PM_ERR_TIMEOUT",
          -5: "PM_ERR_OVERFLOW", -6: "PM_ERR_IO"}


class PMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _DeviceOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("stream", C.c_void_p)]


class _SceneDesc(C.Structure):
    _fields_ = [("ntri", C.c_int32), ("tri_pos", C.c_void_p), ("tri_nrm", C.c_void_p), ("tri_model", C.c_void_p),
                ("tri_diffuse", C.c_void_p), ("nmodel", C.c_int32), ("materials", C.c_void_p),
                ("light_model", C.c_int32), ("light_intensity", C.c_float * 3), ("default_ior", C.c_float)]


class _TraceOpts(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("stream_tag", C.c_uint32), ("max_bounces", C.c_int32),
                ("global_capacity", C.c_int64), ("caustic_capacity", C.c_int64), ("max_paths", C.c_int64)]


class _GridOpts(C.Structure):
    _fields_ = [("desired_per_cell", C.c_int32), ("regrid_mult", C.c_int32), ("regrid_div", C.c_int32),
                ("sub_div", C.c_int32), ("k_hint", C.c_int32)]


class Camera(C.Structure):
    """The reference Camera's fields (CudaPhotonMapping/Camera.cuh:11-33)."""
    _fields_ = [("position", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
                ("up", C.c_float * 3), ("viewport_w", C.c_float), ("viewport_h", C.c_float), ("focal", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32)]

    def as_vector(self):
        return np.array(list(self.position) + list(self.forward) + list(self.right) + list(self.up) +
                        [self.viewport_w, self.viewport_h, self.focal], np.float32)


class _CacheOpts(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("eps", C.c_float), ("out_scale", C.c_float), ("aabb", C.c_float * 6), ("octave0", C.c_int32)]


CACHE_PARAMS = 5 * 64 * 64


class _RequestView(C.Structure):
    _fields_ = [("count", C.c_int64), ("pixels", C.c_int64), ("a", C.c_void_p), ("b", C.c_void_p),
                ("c", C.c_void_p), ("px_base", C.c_void_p), ("px_count", C.c_void_p), ("est_global", C.c_void_p)]


class _BatchInstance(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", Camera), ("seed", C.c_uint64), ("photons", C.c_int64),
                ("max_bounces", C.c_int32), ("k", C.c_int32), ("radius", C.c_float), ("max_depth", C.c_int32)]


class _BatchOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("autotune", C.c_int32), ("use_graph", C.c_int32)]


class _BatchInfo(C.Structure):
    _fields_ = [("instances", C.c_int32), ("paths", C.c_int64), ("photon_slots", C.c_int64), ("keys", C.c_int64),
                ("pixels", C.c_int64), ("request_capacity", C.c_int64), ("desired_per_cell", C.c_int32),
                ("gather_warps", C.c_int32), ("trace_refill", C.c_int32), ("graph", C.c_int32),
                ("launches_per_frame", C.c_int32), ("ms_last_frame", C.c_float), ("photons_last_frame", C.c_int64),
                ("requests_last_frame", C.c_int64), ("underfilled", C.c_int32), ("stage_ms", C.c_float * 5),
                ("gather_guess", C.c_float), ("subcell_khint", C.c_float)]


class _LearnedOpts(C.Structure):
    _fields_ = [("tile", C.c_int32), ("probes", C.c_int32), ("max_rel_err", C.c_float), ("noise_z", C.c_float)]


class _LearnedStats(C.Structure):
    _fields_ = [("tiles", C.c_int64), ("fallback_tiles", C.c_int64), ("requests", C.c_int64),
                ("fallback_requests", C.c_int64)]


class _RenderOpts(C.Structure):
    _fields_ = [("max_depth", C.c_int32), ("k_global", C.c_int32), ("r_global", C.c_float),
                ("k_caustic", C.c_int32), ("r_caustic", C.c_float), ("faithful_caustic", C.c_int32)]


class _PhotonView(C.Structure):
    _fields_ = [("count", C.c_int64), ("cells", C.c_int64), ("dims", C.c_int32 * 3), ("cell_size", C.c_float),
                ("aabb", C.c_float * 6), ("cell_starts", C.c_void_p), ("cell_sizes", C.c_void_p),
                ("sorted_pos", C.c_void_p), ("sorted_dir", C.c_void_p), ("sorted_power", C.c_void_p),
                ("list_pos", C.c_void_p), ("list_dir", C.c_void_p), ("list_power", C.c_void_p),
                ("sub_div", C.c_int32), ("key_starts", C.c_void_p)]


_LIB = None


def library():
    """Load libpm_b200.so (once).  Raises when it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `make -C cuda-photon-mapping_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, f32 = C.c_void_p, C.c_int32, C.c_int64, C.c_float
    sig = {
        "pm_create": ([C.POINTER(C.c_void_p), C.POINTER(_DeviceOpts)], C.c_int),
        "pm_destroy": ([vp], None),
        "pm_last_error": ([vp], C.c_char_p),
        "pm_sync": ([vp], C.c_int),
        "pm_set_scene": ([vp, C.POINTER(_SceneDesc)], C.c_int),
        "pm_scene_aabb": ([vp, vp], C.c_int),
        "pm_trace_photons": ([vp, C.POINTER(_TraceOpts), C.POINTER(C.c_int64)], C.c_int),
        "pm_trace_paths": ([vp, C.POINTER(_TraceOpts), i64, i64, i64, vp, vp, vp, vp, vp,
                            C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
        "pm_set_photons": ([vp, C.c_int, i64, vp, vp, vp], C.c_int),
        "pm_build_grid": ([vp, C.c_int, C.POINTER(_GridOpts), vp], C.c_int),
        "pm_get_photons": ([vp, C.c_int, C.POINTER(_PhotonView)], C.c_int),
        "pm_save_photons": ([vp, C.c_int, C.c_char_p], C.c_int),
        "pm_load_photons": ([vp, C.c_int, C.c_char_p], C.c_int),
        "pm_gather": ([vp, C.c_int, i64, vp, vp, C.c_int, f32, vp, vp, vp], C.c_int),
        "pm_camera_setup": ([vp, vp, vp, f32, i32, i32, C.POINTER(Camera)], C.c_int),
        "pm_render": ([vp, C.POINTER(Camera), C.POINTER(_RenderOpts), vp, vp], C.c_int),
        "pm_render_rows": ([vp, C.POINTER(Camera), C.POINTER(_RenderOpts), i32, i32, vp, vp], C.c_int),
        "pm_scan_u32": ([vp, vp, vp, i64, C.c_int], C.c_int),
        "pm_debug_scan_stall": ([vp, vp, vp, i64, i64, i32], C.c_int),
        "pm_trace_work": ([vp, vp, vp, vp], C.c_int),
        "pm_stage_times": ([vp, vp], C.c_int),
        "pm_status": ([vp, vp], C.c_int),
        "pm_launch_count": ([vp, C.POINTER(C.c_int64)], C.c_int),
        "pm_render_requests": ([vp, C.POINTER(C.c_int64)], C.c_int),
        "pm_cache_init": ([vp, C.POINTER(_CacheOpts)], C.c_int),
        "pm_cache_train_step": ([vp, vp, vp, vp, vp, i64, vp], C.c_int),
        "pm_cache_train_steps": ([vp, vp, vp, vp, vp, i64, i64, C.c_int, vp, vp], C.c_int),
        "pm_set_bvh_builder": ([vp, C.c_int], C.c_int),
        "pm_obj_load": ([C.c_char_p, C.c_char_p, vp, C.c_char_p, C.c_int], C.c_int),
        "pm_obj_desc": ([vp, C.c_float, vp], C.c_int),
        "pm_obj_model_count": ([vp], C.c_int32),
        "pm_obj_model_name": ([vp, C.c_int32], C.c_char_p),
        "pm_obj_light_model": ([vp], C.c_int32),
        "pm_obj_free": ([vp], None),
        "pm_bvh_info": ([vp, vp, vp, vp], C.c_int),
        "pm_write_ppm": ([C.c_char_p, vp, i32, i32], C.c_int),
        "pm_write_pfm": ([C.c_char_p, vp, i32, i32], C.c_int),
        "pm_cache_gradient": ([vp, vp, vp, vp, vp, i64, vp, vp], C.c_int),
        "pm_cache_infer": ([vp, vp, vp, i64, vp], C.c_int),
        "pm_cache_get_params": ([vp, vp], C.c_int),
        "pm_cache_set_params": ([vp, vp], C.c_int),
        "pm_cache_sample_points": ([vp, vp, i64, C.c_uint64, vp, vp, vp], C.c_int),
        "pm_render_learned": ([vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "pm_frame": ([vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "pm_learned_graph_create": ([vp, vp, vp, vp, vp, vp, vp, i64, i64, i32, i64, i32, vp, vp, vp], C.c_int),
        "pm_learned_graph_run": ([vp, vp], C.c_int),
        "pm_learned_graph_offset": ([vp, vp], C.c_int),
        "pm_learned_graph_destroy": ([vp], None),
        "pm_get_requests": ([vp, C.POINTER(_RequestView)], C.c_int),
        "pm_batch_create": ([C.POINTER(C.c_void_p), vp, C.c_int32, C.POINTER(_BatchOpts)], C.c_int),
        "pm_batch_destroy": ([vp], None),
        "pm_batch_last_error": ([vp], C.c_char_p),
        "pm_batch_frame": ([vp, C.c_uint64], C.c_int),
        "pm_batch_image": ([vp, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
        "pm_batch_get_info": ([vp, C.POINTER(_BatchInfo)], C.c_int),
        "pm_batch_photons": ([vp, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                              C.POINTER(C.c_int64)], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def load_obj(path, default_ior=1.0):
    """Scene of an OBJ file (and its mtllib) through the library's loader
    (pm_obj_load): a photonmap.scenes.Scene with the model names; the model
    named "light" emits (intensity 1)."""
    from . import scenes
    L = library()
    d, f = os.path.split(os.path.abspath(str(path)))
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    rc = L.pm_obj_load(d.encode(), f.encode(), C.byref(h), err, len(err))
    if rc:
        raise PMError(rc, f"pm_obj_load: {err.value.decode()}")
    try:
        names = tuple(L.pm_obj_model_name(h, m).decode() for m in range(L.pm_obj_model_count(h)))
        if L.pm_obj_light_model(h) < 0:
            raise PMError(-1, f"pm_obj_load: no model named 'light' in {path} (models: {names})")
        desc = _SceneDesc()
        rc = L.pm_obj_desc(h, float(default_ior), C.byref(desc))
        if rc:
            raise PMError(rc, "pm_obj_desc")
        T, M = desc.ntri, desc.nmodel

        def arr(ptr, n, ctype):
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,)).copy()
        return scenes.Scene(tri_pos=arr(desc.tri_pos, 9 * T, C.c_float).reshape(T, 3, 3),
                            tri_nrm=arr(desc.tri_nrm, 9 * T, C.c_float).reshape(T, 3, 3),
                            tri_model=arr(desc.tri_model, T, C.c_int32),
                            materials=arr(desc.materials, 12 * M, C.c_float).reshape(M, 12),
                            light_model=int(desc.light_model),
                            light_intensity=np.array(list(desc.light_intensity), np.float32),
                            default_ior=float(desc.default_ior), names=names)
    finally:
        L.pm_obj_free(h)


def _write_frame(fn, path, frame, itemsize, width, height):
    """Call fn (pm_write_ppm / pm_write_pfm) on a frame buffer: a torch tensor
    on any device, or a numpy array, of width * height * 3 contiguous items of
    itemsize bytes."""
    want = int(width) * int(height) * 3 * itemsize
    host = None
    if hasattr(frame, "data_ptr"):
        if not frame.is_contiguous() or frame.numel() * frame.element_size() != want:
            raise PMError(-1, f"{fn}: want {want} contiguous bytes")
        ptr = C.c_void_p(frame.data_ptr())
    else:
        host = np.ascontiguousarray(frame)   # kept alive across the call
        if host.nbytes != want:
            raise PMError(-1, f"{fn}: want {want} bytes")
        ptr = C.c_void_p(host.ctypes.data)
    rc = getattr(library(), fn)(os.fspath(path).encode(), ptr, int(width), int(height))
    if rc:
        raise PMError(rc, fn)


def write_ppm(path, rgb8, width, height):
    """pm_write_ppm: an 8-bit frame in pm_render's layout (row 0 = bottom; uint8
    tensor on the GPU or host, or numpy) as a binary PPM, top row first."""
    _write_frame("pm_write_ppm", path, rgb8, 1, width, height)


def write_pfm(path, radiance, width, height):
    """pm_write_pfm: a float32 radiance frame in pm_render's layout as a colour
    PFM (little-endian, rows bottom to top)."""
    _write_frame("pm_write_pfm", path, radiance, 4, width, height)


def camera_setup(position, direction, up, fov_deg, width, height) -> Camera:
    """Camera(position, direction, up, fov, W, H) as the reference constructs it."""
    L = library()
    cam = Camera()
    p = np.asarray(position, np.float32); d = np.asarray(direction, np.float32); u = np.asarray(up, np.float32)
    rc = L.pm_camera_setup(p.ctypes.data, d.ctypes.data, u.ctypes.data, float(fov_deg), int(width), int(height),
                           C.byref(cam))
    if rc:
        raise PMError(rc, "pm_camera_setup")
    return cam


def _scene_desc(sc):
    """pm_scene_desc of a photonmap.scenes.Scene and the arrays it points into (keep them alive)."""
    pos = np.ascontiguousarray(sc.tri_pos, np.float32)
    nrm = np.ascontiguousarray(sc.tri_nrm, np.float32)
    tm = np.ascontiguousarray(sc.tri_model, np.int32)
    mats = np.ascontiguousarray(sc.materials, np.float32)
    td = None if sc.tri_diffuse is None else np.ascontiguousarray(sc.tri_diffuse, np.float32)
    d = _SceneDesc(sc.ntri, pos.ctypes.data, nrm.ctypes.data, tm.ctypes.data,
                   None if td is None else td.ctypes.data, sc.nmodel, mats.ctypes.data, int(sc.light_model),
                   (C.c_float * 3)(*[float(x) for x in sc.light_intensity]), float(sc.default_ior))
    return d, (pos, nrm, tm, mats, td)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class Context:
    """One pm_ctx: a device, a stream, a scene, two photon maps."""

    def __init__(self, device: int = 0, stream=None):
        import torch
        self.torch = torch
        self.L = library()
        if not torch.cuda.is_available():
            raise RuntimeError("photonmap needs a CUDA device")
        self.device = torch.device("cuda", device)
        h = C.c_void_p()
        opts = _DeviceOpts(device, None if stream is None else C.c_void_p(stream.cuda_stream))
        rc = self.L.pm_create(C.byref(h), C.byref(opts))
        if rc:
            raise PMError(rc, "pm_create")
        self.h = h
        self._scene = None

    def close(self):
        if getattr(self, "h", None):
            self.L.pm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            raise PMError(rc, f"{what}: {self.L.pm_last_error(self.h).decode()}")

    # ------------------------------------------------------------ scene
    def set_bvh_builder(self, builder):
        """'host_sah' (default) or 'device_lbvh': the BVH builder of the next set_scene."""
        code = {"host_sah": 0, "device_lbvh": 1}[builder]
        self._check(self.L.pm_set_bvh_builder(self.h, code), "pm_set_bvh_builder")

    def bvh_info(self):
        b, n, ms = C.c_int32(), C.c_int64(), C.c_float()
        self._check(self.L.pm_bvh_info(self.h, C.byref(b), C.byref(n), C.byref(ms)), "pm_bvh_info")
        return dict(builder=("host_sah", "device_lbvh")[b.value], nodes=n.value, build_ms=ms.value)

    def set_scene(self, sc):
        d, _keep = _scene_desc(sc)
        self._check(self.L.pm_set_scene(self.h, C.byref(d)), "pm_set_scene")
        self._scene = sc

    @property
    def light_intensity(self):
        """The current scene's light intensity (3 floats)."""
        return np.asarray(self._scene.light_intensity, np.float32)

    def scene_aabb(self):
        out = np.empty(6, np.float32)
        self._check(self.L.pm_scene_aabb(self.h, out.ctypes.data), "pm_scene_aabb")
        return out

    # ----------------------------------------------------------- photons
    def trace_photons(self, seed, max_bounces, global_capacity, caustic_capacity=0, tag=0, max_paths=0):
        o = _TraceOpts(seed, tag, max_bounces, global_capacity, caustic_capacity, max_paths)
        paths = C.c_int64()
        self._check(self.L.pm_trace_photons(self.h, C.byref(o), C.byref(paths)), "pm_trace_photons")
        return paths.value

    def trace_work(self, seed, max_bounces, global_capacity, caustic_capacity=0, tag=0, max_paths=0):
        """trace_photons with the tracer's work counted: (paths, rays, BVH node visits, triangle tests)."""
        o = _TraceOpts(seed, tag, max_bounces, global_capacity, caustic_capacity, max_paths)
        paths = C.c_int64()
        w = (C.c_uint64 * 3)()
        self._check(self.L.pm_trace_work(self.h, C.byref(o), C.byref(paths), w), "pm_trace_work")
        return paths.value, int(w[0]), int(w[1]), int(w[2])

    def trace_paths(self, seed, max_bounces, power_capacity, p0, p1, tag=0):
        torch = self.torch
        n = p1 - p0
        cap = n * max_bounces
        gp = torch.empty((cap, 3), dtype=torch.float32, device=self.device)
        gd = torch.empty_like(gp); cp = torch.empty_like(gp); cd = torch.empty_like(gp)
        counts = torch.empty((n, 2), dtype=torch.int32, device=self.device)
        o = _TraceOpts(seed, tag, max_bounces, 0, 0, 0)
        ng, nc = C.c_int64(), C.c_int64()
        self._check(self.L.pm_trace_paths(self.h, C.byref(o), p0, p1, power_capacity, _ptr(gp), _ptr(gd), _ptr(cp),
                                          _ptr(cd), _ptr(counts), C.byref(ng), C.byref(nc)), "pm_trace_paths")
        return dict(counts=counts, g_pos=gp[:ng.value], g_dir=gd[:ng.value], c_pos=cp[:nc.value], c_dir=cd[:nc.value])

    def set_photons(self, map_id, pos, power, direction):
        """A map's photon list from host arrays or device tensors (3 floats per photon)."""
        torch = self.torch
        if all(isinstance(a, torch.Tensor) and a.is_cuda for a in (pos, power, direction)):
            arrs = [a.to(self.device, torch.float32).contiguous().reshape(-1, 3) for a in (pos, power, direction)]
            ptrs = [a.data_ptr() for a in arrs]
        else:
            arrs = [np.ascontiguousarray(a.cpu().numpy() if isinstance(a, torch.Tensor) else a, np.float32)
                    .reshape(-1, 3) for a in (pos, power, direction)]
            ptrs = [a.ctypes.data for a in arrs]
        self._check(self.L.pm_set_photons(self.h, map_id, arrs[0].shape[0], *ptrs), "pm_set_photons")

    def build_grid(self, map_id=PM_MAP_GLOBAL, desired=1000, regrid_mult=5, regrid_div=5, aabb=None, sub_div=0,
                   k_hint=0):
        o = _GridOpts(desired, regrid_mult, regrid_div, sub_div, k_hint)
        box = None if aabb is None else np.ascontiguousarray(aabb, np.float32)
        self._check(self.L.pm_build_grid(self.h, map_id, C.byref(o), None if box is None else box.ctypes.data),
                    "pm_build_grid")

    def view(self, map_id=PM_MAP_GLOBAL):
        v = _PhotonView()
        self._check(self.L.pm_get_photons(self.h, map_id, C.byref(v)), "pm_get_photons")
        return v

    def photons(self, map_id=PM_MAP_GLOBAL, sorted_=True):
        """Copies of a map's device arrays as torch tensors."""
        torch = self.torch
        v = self.view(map_id)
        n = v.count

        def dev(ptr, count, dtype, shape):
            if not count:
                return torch.empty(shape, dtype=dtype, device=self.device)
            return torch.as_tensor(_DeviceArray(ptr, shape, dtype), device=self.device).clone()

        out = dict(count=n, list_pos=dev(v.list_pos, n, torch.float32, (n, 3)),
                   list_dir=dev(v.list_dir, n, torch.float32, (n, 3)),
                   list_power=dev(v.list_power, n, torch.float32, (n, 3)))
        if sorted_ and v.cell_starts:
            cells = v.cells
            S = v.sub_div
            out.update(dims=tuple(v.dims), cell=v.cell_size, aabb=np.array(list(v.aabb), np.float32), cells=cells,
                       sub_div=S, key_starts=dev(v.key_starts, cells * S ** 3 + 1, torch.int32, (cells * S ** 3 + 1,)),
                       cell_starts=dev(v.cell_starts, cells, torch.int32, (cells,)),
                       cell_sizes=dev(v.cell_sizes, cells, torch.int32, (cells,)),
                       sorted_pos=dev(v.sorted_pos, n, torch.float32, (n, 4)),
                       sorted_dir=dev(v.sorted_dir, n, torch.float32, (n, 3)),
                       sorted_power=dev(v.sorted_power, n, torch.float32, (n, 3)))
        return out

    def save_photons(self, map_id, path):
        self._check(self.L.pm_save_photons(self.h, map_id, str(path).encode()), "pm_save_photons")

    def load_photons(self, map_id, path):
        self._check(self.L.pm_load_photons(self.h, map_id, str(path).encode()), "pm_load_photons")

    # ------------------------------------------------------------ gather
    def gather(self, qpos, qnrm, k, radius, map_id=PM_MAP_GLOBAL, want_ids=False):
        torch = self.torch
        qpos = qpos.to(self.device, torch.float32).contiguous()
        qnrm = qnrm.to(self.device, torch.float32).contiguous()
        n = qpos.shape[0]
        rad = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        ids = torch.empty((n, k), dtype=torch.int32, device=self.device) if want_ids else None
        cnt = torch.empty(n, dtype=torch.int32, device=self.device)
        self._check(self.L.pm_gather(self.h, map_id, n, _ptr(qpos), _ptr(qnrm), int(k), float(radius), _ptr(rad),
                                     _ptr(ids), _ptr(cnt)), "pm_gather")
        return rad, ids, cnt

    # ------------------------------------------------------------ learned radiance cache
    def cache_init(self, seed=0, lr=1e-3, beta1=0.9, beta2=0.99, eps=1e-8, out_scale=1.0, aabb=None, octave0=0):
        box = (C.c_float * 6)(*([0.0] * 6 if aabb is None else [float(x) for x in aabb]))
        o = _CacheOpts(int(seed), float(lr), float(beta1), float(beta2), float(eps), float(out_scale), box,
                       int(octave0))
        self._check(self.L.pm_cache_init(self.h, C.byref(o)), "pm_cache_init")

    def _samples(self, *arrays):
        torch = self.torch
        return [None if a is None else torch.as_tensor(a).to(self.device, torch.float32).contiguous() for a in arrays]

    def cache_train_step(self, pos, nrm, target, weight=None):
        """One Adam step; returns the step's mean squared error (network units, before the update)."""
        pos, nrm, target, weight = self._samples(pos, nrm, target, weight)
        loss = C.c_float()
        self._check(self.L.pm_cache_train_step(self.h, _ptr(pos), _ptr(nrm), _ptr(target), _ptr(weight),
                                               pos.shape[0], C.byref(loss)), "pm_cache_train_step")
        return loss.value

    def cache_train_steps(self, pos, nrm, target, steps, batch, offset=0, weight=None, want_loss=True):
        """`steps` Adam steps over consecutive `batch`-sample slices of the pool from
        `offset` (wrapping); returns (last step's loss, next offset).  With
        want_loss=False the steps are only queued (loss nan, no host wait)."""
        pos, nrm, target, weight = self._samples(pos, nrm, target, weight)
        loss = C.c_float(float("nan"))
        off = C.c_int64(int(offset))
        self._check(self.L.pm_cache_train_steps(self.h, _ptr(pos), _ptr(nrm), _ptr(target), _ptr(weight),
                                                pos.shape[0], int(batch), int(steps), C.byref(off),
                                                C.byref(loss) if want_loss else None), "pm_cache_train_steps")
        return loss.value, off.value

    def cache_gradient(self, pos, nrm, target, weight=None):
        pos, nrm, target, weight = self._samples(pos, nrm, target, weight)
        g = np.zeros(CACHE_PARAMS, np.float32)
        loss = C.c_float()
        self._check(self.L.pm_cache_gradient(self.h, _ptr(pos), _ptr(nrm), _ptr(target), _ptr(weight),
                                             pos.shape[0], g.ctypes.data, C.byref(loss)), "pm_cache_gradient")
        return g, loss.value

    def cache_infer(self, pos, nrm):
        pos, nrm = self._samples(pos, nrm)
        out = self.torch.empty((pos.shape[0], 3), dtype=self.torch.float32, device=self.device)
        self._check(self.L.pm_cache_infer(self.h, _ptr(pos), _ptr(nrm), pos.shape[0], _ptr(out)), "pm_cache_infer")
        return out

    def cache_params(self):
        w = np.zeros(CACHE_PARAMS, np.float32)
        self._check(self.L.pm_cache_get_params(self.h, w.ctypes.data), "pm_cache_get_params")
        return w

    def cache_set_params(self, w):
        w = np.ascontiguousarray(w, np.float32).reshape(-1)
        assert w.size == CACHE_PARAMS
        self._check(self.L.pm_cache_set_params(self.h, w.ctypes.data), "pm_cache_set_params")

    def cache_sample_points(self, cam, n, seed=0):
        """Training points: primary hits of n stratified jittered camera rays -> (pos, nrm, weight) device tensors."""
        torch = self.torch
        pos = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        nrm = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        w = torch.empty(n, dtype=torch.float32, device=self.device)
        self._check(self.L.pm_cache_sample_points(self.h, C.byref(cam), int(n), int(seed), _ptr(pos), _ptr(nrm),
                                                  _ptr(w)), "pm_cache_sample_points")
        return pos, nrm, w

    def render_learned(self, cam: Camera, k_global, r_global, max_depth=4, tile=16, probes=16, max_rel_err=0.05,
                       k_caustic=0, r_caustic=0.2, faithful_caustic=True, radiance=True, out_rgb8=None,
                       out_radiance=None, noise_z=0.0):
        torch = self.torch
        W, H = cam.width, cam.height
        rgb = out_rgb8 if out_rgb8 is not None else torch.empty((H * W * 3,), dtype=torch.uint8, device=self.device)
        rad = out_radiance
        if rad is None and radiance:
            rad = torch.empty((H * W, 3), dtype=torch.float32, device=self.device)
        o = _RenderOpts(max_depth, k_global, r_global, k_caustic, r_caustic, int(faithful_caustic))
        lo = _LearnedOpts(int(tile), int(probes), float(max_rel_err), float(noise_z))
        st = _LearnedStats()
        self._check(self.L.pm_render_learned(self.h, C.byref(cam), C.byref(o), C.byref(lo), _ptr(rgb), _ptr(rad),
                                             C.byref(st)), "pm_render_learned")
        return rgb, rad, dict(tiles=st.tiles, fallback_tiles=st.fallback_tiles, requests=st.requests,
                              fallback_requests=st.fallback_requests)

    def learned_graph(self, cam: Camera, k_global, r_global, max_depth=4, pool=None, steps=4, batch=65536, offset=0,
                      tile=16, probes=16, max_rel_err=0.05, noise_z=0.0, radiance=False, out_rgb8=None,
                      out_radiance=None, overlap_training=False):
        """The learned frame (`steps` Adam steps on the pool + render_learned) as one
        replayable CUDA graph (pm_learned_graph_create); `pool` a photonmap.learned.Pool
        (or None with steps=0).  overlap_training: the render reads the cache as the
        previous frames trained it while this frame's training runs beside it.
        Returns a LearnedGraph: .run(stats=False) -> (rgb, radiance, stats)."""
        torch = self.torch
        W, H = cam.width, cam.height
        rgb = out_rgb8 if out_rgb8 is not None else torch.empty((H * W * 3,), dtype=torch.uint8, device=self.device)
        rad = out_radiance
        if rad is None and radiance:
            rad = torch.empty((H * W, 3), dtype=torch.float32, device=self.device)
        o = _RenderOpts(max_depth, k_global, r_global, 0, 0.2, 1)
        lo = _LearnedOpts(int(tile), int(probes), float(max_rel_err), float(noise_z))
        if pool is not None:
            pos, nrm, tgt = self._samples(pool.pos, pool.nrm, pool.target)
            n = pos.shape[0]
        else:
            pos = nrm = tgt = None
            n = 0
        h = C.c_void_p()
        self._check(self.L.pm_learned_graph_create(self.h, C.byref(cam), C.byref(o), C.byref(lo), _ptr(pos), _ptr(nrm),
                                                   _ptr(tgt), int(n), int(batch), int(steps), int(offset),
                                                   int(bool(overlap_training)), _ptr(rgb), _ptr(rad), C.byref(h)),
                    "pm_learned_graph_create")
        return LearnedGraph(self, h, rgb, rad, (pos, nrm, tgt))

    def frame(self, seed, max_bounces, global_capacity, cam: Camera, k_global, r_global, max_depth=4,
              caustic_capacity=0, k_caustic=0, r_caustic=0.2, faithful_caustic=True, desired=1000, sub_div=0,
              radiance=True, out_rgb8=None, out_radiance=None):
        """Photon pass + grid build(s) + frame in one call (pm_frame; the eye pass
        runs beside the photon pass).  Returns (rgb8, radiance, paths traced)."""
        torch = self.torch
        W, H = cam.width, cam.height
        rgb = out_rgb8 if out_rgb8 is not None else torch.empty((H * W * 3,), dtype=torch.uint8, device=self.device)
        rad = out_radiance
        if rad is None and radiance:
            rad = torch.empty((H * W, 3), dtype=torch.float32, device=self.device)
        to = _TraceOpts(seed, 0, max_bounces, global_capacity, caustic_capacity, 0)
        go = _GridOpts(desired, 5, 5, sub_div, 0)
        ro = _RenderOpts(max_depth, k_global, r_global, k_caustic, r_caustic, int(faithful_caustic))
        paths = C.c_int64()
        self._check(self.L.pm_frame(self.h, C.byref(to), C.byref(go), C.byref(cam), C.byref(ro), _ptr(rgb), _ptr(rad),
                                    C.byref(paths)), "pm_frame")
        return rgb, rad, paths.value

    # ------------------------------------------------------------ render
    def render(self, cam: Camera, k_global, r_global, max_depth=4, k_caustic=0, r_caustic=0.2,
               faithful_caustic=True, radiance=True, out_rgb8=None, out_radiance=None):
        torch = self.torch
        W, H = cam.width, cam.height
        rgb = out_rgb8 if out_rgb8 is not None else torch.empty((H * W * 3,), dtype=torch.uint8, device=self.device)
        rad = out_radiance
        if rad is None and radiance:
            rad = torch.empty((H * W, 3), dtype=torch.float32, device=self.device)
        o = _RenderOpts(max_depth, k_global, r_global, k_caustic, r_caustic, int(faithful_caustic))
        self._check(self.L.pm_render(self.h, C.byref(cam), C.byref(o), _ptr(rgb), _ptr(rad)), "pm_render")
        return rgb, rad

    def render_rows(self, cam: Camera, k_global, r_global, max_depth, y0, y1, k_caustic=0, r_caustic=0.2,
                    faithful_caustic=True, radiance=True, out_rgb8=None, out_radiance=None):
        """Rows [y0, y1) of render()'s frame (pm_render_rows)."""
        torch = self.torch
        W, H = cam.width, cam.height
        rgb = out_rgb8 if out_rgb8 is not None else torch.empty((H * W * 3,), dtype=torch.uint8, device=self.device)
        rad = out_radiance
        if rad is None and radiance:
            rad = torch.empty((H * W, 3), dtype=torch.float32, device=self.device)
        o = _RenderOpts(max_depth, k_global, r_global, k_caustic, r_caustic, int(faithful_caustic))
        self._check(self.L.pm_render_rows(self.h, C.byref(cam), C.byref(o), int(y0), int(y1), _ptr(rgb), _ptr(rad)),
                    "pm_render_rows")
        return rgb, rad

    def scan_u32(self, x, inclusive):
        torch = self.torch
        x = x.to(self.device, torch.int32).contiguous()
        out = torch.empty_like(x)
        self._check(self.L.pm_scan_u32(self.h, _ptr(x), _ptr(out), x.numel(), int(inclusive)), "pm_scan_u32")
        return out

    def debug_scan_stall(self, x, spin_limit, silent_tile):
        """Test hook: the inclusive scan with each look-back wait limited to
        spin_limit polls and tile silent_tile publishing nothing (pm_debug_scan_stall)."""
        torch = self.torch
        x = x.to(self.device, torch.int32).contiguous()
        out = torch.empty_like(x)
        self._check(self.L.pm_debug_scan_stall(self.h, _ptr(x), _ptr(out), x.numel(), int(spin_limit),
                                               int(silent_tile)), "pm_debug_scan_stall")
        return out

    def stage_times(self):
        out = np.zeros(8, np.float32)
        self._check(self.L.pm_stage_times(self.h, out.ctypes.data), "pm_stage_times")
        return dict(trace_ms=float(out[0]), grid_ms=float(out[1]), eye_ms=float(out[2]), gather_ms=float(out[3]),
                    resolve_ms=float(out[4]), k_trace_ms=float(out[5]), k_gather_ms=float(out[6]))

    def requests(self):
        """Copies of the last render's gather requests (see pm_request_view) as torch tensors."""
        torch = self.torch
        v = _RequestView()
        self._check(self.L.pm_get_requests(self.h, C.byref(v)), "pm_get_requests")
        n, npx = v.count, v.pixels

        def dev(ptr, count, dtype, shape):
            if not count:
                return torch.empty(shape, dtype=dtype, device=self.device)
            return torch.as_tensor(_DeviceArray(ptr, shape, dtype), device=self.device).clone()

        return dict(a=dev(v.a, n, torch.float32, (n, 4)), b=dev(v.b, n, torch.float32, (n, 4)),
                    c=dev(v.c, n, torch.float32, (n, 4)), px_base=dev(v.px_base, npx, torch.int32, (npx,)),
                    px_count=dev(v.px_count, npx, torch.int32, (npx,)),
                    est_global=dev(v.est_global, n, torch.float32, (n, 3)))

    def render_requests(self):
        """kNN queries answered by the last render's global-map gather."""
        out = C.c_int64()
        self._check(self.L.pm_render_requests(self.h, C.byref(out)), "pm_render_requests")
        return out.value

    def launch_count(self):
        out = C.c_int64()
        self._check(self.L.pm_launch_count(self.h, C.byref(out)), "pm_launch_count")
        return out.value

    def status(self):
        out = np.zeros(1, np.uint32)
        self._check(self.L.pm_status(self.h, out.ctypes.data), "pm_status")
        return int(out[0])

    def sync(self):
        self._check(self.L.pm_sync(self.h), "pm_sync")


class _DeviceArray:
    """Zero-copy view of a library-owned device array (CUDA array interface)."""
    _TYPESTR = {"torch.float32": "<f4", "torch.int32": "<i4", "torch.uint8": "|u1"}

    def __init__(self, ptr, shape, dtype):
        self.__cuda_array_interface__ = {"shape": tuple(int(x) for x in shape), "typestr": self._TYPESTR[str(dtype)],
                                         "data": (int(ptr), False), "version": 3, "strides": None}


class LearnedGraph:
    """A captured learned frame (Context.learned_graph); keeps its pool and outputs alive."""

    def __init__(self, ctx, h, rgb, rad, keep):
        self.ctx, self.h, self.rgb, self.rad, self._keep = ctx, h, rgb, rad, keep

    def run(self, stats=False):
        st = _LearnedStats() if stats else None
        self.ctx._check(self.ctx.L.pm_learned_graph_run(self.h, C.byref(st) if stats else None), "pm_learned_graph_run")
        d = None if st is None else dict(tiles=st.tiles, fallback_tiles=st.fallback_tiles, requests=st.requests,
                                         fallback_requests=st.fallback_requests)
        return self.rgb, self.rad, d

    def offset(self):
        o = C.c_int64()
        self.ctx._check(self.ctx.L.pm_learned_graph_offset(self.h, C.byref(o)), "pm_learned_graph_offset")
        return o.value

    def close(self):
        if self.h:
            self.ctx.L.pm_learned_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many scene instances rendered per frame by one work queue per stage
    (pm_batch_* in the C ABI).  instances: dicts with scene (scenes.Scene),
    camera (Camera), seed, photons, max_bounces, k, radius, max_depth."""

    def __init__(self, instances, device=0, autotune=False, use_graph=True):
        import torch
        self.torch = torch
        self.L = library()
        self.device = torch.device("cuda", device)
        descs = [_scene_desc(i["scene"]) for i in instances]
        arr = (_BatchInstance * len(instances))()
        for j, (i, (d, _)) in enumerate(zip(instances, descs)):
            arr[j] = _BatchInstance(C.cast(C.pointer(d), C.c_void_p), i["camera"], int(i["seed"]), int(i["photons"]),
                                    int(i["max_bounces"]), int(i["k"]), float(i["radius"]), int(i["max_depth"]))
        self.h = C.c_void_p()
        o = _BatchOpts(device, int(bool(autotune)), int(bool(use_graph)))
        rc = self.L.pm_batch_create(C.byref(self.h), arr, len(instances), C.byref(o))
        if rc != 0:
            msg = self.L.pm_batch_last_error(self.h).decode() if self.h.value else "no batch"
            self.close()
            raise RuntimeError(f"pm_batch_create failed ({rc}): {msg}")
        self.n = len(instances)

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc}): {self.L.pm_batch_last_error(self.h).decode()}")

    def frame(self, frame=0):
        self._check(self.L.pm_batch_frame(self.h, int(frame)), "pm_batch_frame")

    def image(self, i):
        """Copy of instance i's last image as a (height, width, 3) uint8 tensor."""
        p, w, h = C.c_void_p(), C.c_int32(), C.c_int32()
        self._check(self.L.pm_batch_image(self.h, int(i), C.byref(p), C.byref(w), C.byref(h)), "pm_batch_image")
        return self.torch.as_tensor(_DeviceArray(p.value, (h.value, w.value, 3), self.torch.uint8),
                                    device=self.device).clone()

    def photons(self, i):
        """Copies of the photon list instance i stored in the last frame (canonical
        order): dict of (count, 3) float32 CUDA tensors pos, power, dir."""
        ptr = [C.c_void_p() for _ in range(3)]
        n = C.c_int64()
        self._check(self.L.pm_batch_photons(self.h, int(i), *(C.byref(x) for x in ptr), C.byref(n)),
                    "pm_batch_photons")
        return {k: self.torch.as_tensor(_DeviceArray(x.value, (n.value, 3), self.torch.float32),
                                        device=self.device).clone()
                for k, x in zip(("pos", "power", "dir"), ptr)}

    def info(self):
        o = _BatchInfo()
        self._check(self.L.pm_batch_get_info(self.h, C.byref(o)), "pm_batch_get_info")
        d = {k: getattr(o, k) for k, _ in _BatchInfo._fields_}
        d["stage_ms"] = dict(zip(("trace", "grid", "eye", "gather", "resolve"), [float(x) for x in o.stage_ms]))
        return d

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.pm_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
