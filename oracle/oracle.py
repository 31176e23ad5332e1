"""ctypes bindings for the parity checkers (test infrastructure only).

``Oracle``     -> oracle/_build/liboracle.so (CPU restatement, pm_oracle.cpp)
``RefHost``    -> oracle/_ref/libref_host.so (the reference's own host render code)
``RefTrace``   -> oracle/_ref/libref_trace.so (the reference's own photon tracer, as host code)

Only tests/, __graft_entry__.smoke() and bench.py's reference / cpu_baseline leg
import this module.  Build both libraries with ``make -C oracle``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_host.so")
REF_TRACE_SO = os.path.join(HERE, "_ref", "libref_trace.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class GridResult:
    aabb: np.ndarray      # (6,) float32
    dims: np.ndarray      # (3,) int32
    cell: float
    starts: np.ndarray    # (cells,) uint32
    sizes: np.ndarray     # (cells,) uint32
    order: np.ndarray     # (n,) uint32 sorted slot -> source index
    spos: np.ndarray      # (n, 3) float32 sorted
    sdir: np.ndarray
    spow: np.ndarray
    sid: np.ndarray       # (n,) uint32 source index per slot


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        L = C.CDLL(path)
        self.L = L
        L.orc_scene_create.restype = C.c_void_p
        L.orc_scene_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_void_p, C.c_int, C.c_void_p, C.c_float]
        L.orc_scene_destroy.argtypes = [C.c_void_p]
        L.orc_scene_aabb.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_scene_critical_angles.restype = C.c_int
        L.orc_scene_critical_angles.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.orc_philox_raw.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_philox_uniforms.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_int, C.c_void_p]
        L.orc_intersect.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 6
        L.orc_trace_photons.restype = C.c_int64
        L.orc_trace_photons.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_int64, C.c_int64,
                                        C.c_int64] + [C.c_void_p] * 12
        L.orc_trace_paths.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_int64, C.c_int64,
                                      C.c_int64] + [C.c_void_p] * 10
        L.orc_grid_build.restype = C.c_int64
        L.orc_grid_build.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
        L.orc_gather.argtypes = [C.c_void_p, C.c_void_p, C.c_float] + [C.c_void_p] * 6 + \
            [C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_int] + [C.c_void_p] * 4
        L.orc_camera.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_int, C.c_void_p]
        L.orc_render.restype = C.c_int
        L.orc_render.argtypes = ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_void_p, C.c_void_p, C.c_float] + [C.c_void_p] * 6 +
                                 [C.c_void_p, C.c_float] + [C.c_void_p] * 6 +
                                 [C.c_int, C.c_float, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int] +
                                 [C.c_void_p] * 4)
        L.orc_scan_u32.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int]
        L.orc_camera_rays.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_ray_ops.argtypes = [C.c_int] + [C.c_void_p] * 7
        L.orc_hdr.argtypes = [C.c_int, C.c_void_p, C.c_void_p]

    # ---------------------------------------------------------------- scene
    def scene(self, sc):
        keep = [_c(sc.tri_pos, np.float32), _c(sc.tri_nrm, np.float32), _c(sc.tri_model, np.int32),
                None if sc.tri_diffuse is None else _c(sc.tri_diffuse, np.float32),
                _c(sc.materials, np.float32), _c(sc.light_intensity, np.float32)]
        h = self.L.orc_scene_create(sc.ntri, _ptr(keep[0]), _ptr(keep[1]), _ptr(keep[2]), _ptr(keep[3]),
                                    sc.nmodel, _ptr(keep[4]), int(sc.light_model), _ptr(keep[5]),
                                    float(sc.default_ior))
        return OracleScene(self, h)

    def philox(self, seed, tag, path, n):
        out = np.empty(n, np.float32)
        self.L.orc_philox_uniforms(seed, tag, path, n, _ptr(out))
        return out

    def philox_raw(self, ctr, key):
        c = np.array(ctr, np.uint32)
        k = np.array(key, np.uint32)
        self.L.orc_philox_raw(_ptr(c), _ptr(k))
        return c

    def camera(self, cam):
        out = np.empty(15, np.float32)
        self.L.orc_camera(_ptr(_c(cam.position, np.float32)), _ptr(_c(cam.direction, np.float32)),
                          _ptr(_c(cam.up, np.float32)), float(cam.fov_deg), cam.width, cam.height, _ptr(out))
        return out

    def grid_build(self, pos, power, direction, aabb, desired=1000, sub_div=1):
        pos = _c(pos, np.float32).reshape(-1, 3)
        n = pos.shape[0]
        aabb = _c(aabb, np.float32)
        dims = np.zeros(3, np.int32)
        cell = np.zeros(1, np.float32)
        cap = 1 << 16
        while True:
            starts = np.empty(cap, np.uint32)
            sizes = np.empty(cap, np.uint32)
            order = np.empty(max(n, 1), np.uint32)
            sub = np.zeros(1, np.int32)
            cells = self.L.orc_grid_build(_ptr(pos), n, _ptr(aabb), desired, int(sub_div), _ptr(sub), _ptr(dims),
                                          _ptr(cell), _ptr(starts), _ptr(sizes), _ptr(order), cap)
            if cells >= 0:
                break
            cap = -cells
        order = order[:n]
        g = GridResult(aabb, dims.copy(), float(cell[0]), starts[:cells].copy(), sizes[:cells].copy(), order,
                       pos[order], _c(direction, np.float32).reshape(-1, 3)[order],
                       _c(power, np.float32).reshape(-1, 3)[order], order.copy())
        g.sub_div = int(sub[0])
        return g

    def gather(self, g: GridResult, qpos, qnrm, radius, k, heap_mode=False):
        qpos = _c(qpos, np.float32).reshape(-1, 3)
        qnrm = _c(qnrm, np.float32).reshape(-1, 3)
        nq = qpos.shape[0]
        ids = np.empty((nq, k), np.uint32)
        cnt = np.empty(nq, np.int32)
        rk = np.empty(nq, np.float32)
        rad = np.empty((nq, 3), np.float32)
        self.L.orc_gather(_ptr(g.aabb), _ptr(g.dims), g.cell, _ptr(g.starts), _ptr(g.sizes),
                          _ptr(_c(g.spos, np.float32)), _ptr(_c(g.sdir, np.float32)), _ptr(_c(g.spow, np.float32)),
                          _ptr(_c(g.sid, np.uint32)), nq, _ptr(qpos), _ptr(qnrm), float(radius), int(k),
                          int(heap_mode), _ptr(ids), _ptr(cnt), _ptr(rk), _ptr(rad))
        return ids, cnt, rk, rad

    def camera_rays(self, cam_vec, W, H, xs, ys):
        xs = _c(xs, np.int32); ys = _c(ys, np.int32)
        out = np.empty((xs.size, 3), np.float32)
        self.L.orc_camera_rays(_ptr(_c(cam_vec, np.float32)), W, H, xs.size, _ptr(xs), _ptr(ys), _ptr(out))
        return out

    def ray_ops(self, dirs, frm, nrm, etas):
        dirs = _c(dirs, np.float32).reshape(-1, 3); n = dirs.shape[0]
        a = np.empty((n, 6), np.float32); b = np.empty((n, 6), np.float32); ok = np.empty(n, np.int32)
        self.L.orc_ray_ops(n, _ptr(dirs), _ptr(_c(frm, np.float32)), _ptr(_c(nrm, np.float32)),
                           _ptr(_c(etas, np.float32)), _ptr(a), _ptr(b), _ptr(ok))
        return a, b, ok

    def hdr(self, rgb):
        rgb = _c(rgb, np.float32).reshape(-1, 3)
        out = np.empty_like(rgb)
        self.L.orc_hdr(rgb.shape[0], _ptr(rgb), _ptr(out))
        return out

    def scan_u32(self, a, inclusive):
        a = _c(a, np.uint32)
        out = np.empty_like(a)
        self.L.orc_scan_u32(_ptr(a), _ptr(out), a.size, int(inclusive))
        return out


class OracleScene:
    def __init__(self, orc: Oracle, h):
        self.orc = orc
        self.h = h

    def __del__(self):
        try:
            self.orc.L.orc_scene_destroy(self.h)
        except Exception:
            pass

    def aabb(self):
        out = np.empty(6, np.float32)
        self.orc.L.orc_scene_aabb(self.h, _ptr(out))
        return out

    def critical_angles(self):
        out = np.empty(3 * 256, np.float32)
        n = self.orc.L.orc_scene_critical_angles(self.h, _ptr(out), 256)
        return out[:3 * n].reshape(-1, 3)

    def intersect(self, orig, dirs):
        orig = _c(orig, np.float32).reshape(-1, 3)
        dirs = _c(dirs, np.float32).reshape(-1, 3)
        n = orig.shape[0]
        t = np.empty(n, np.float32)
        m = np.empty(n, np.int32)
        tri = np.empty(n, np.int32)
        nn = np.empty((n, 3), np.float32)
        self.orc.L.orc_intersect(self.h, n, _ptr(orig), _ptr(dirs), _ptr(t), _ptr(m), _ptr(tri), _ptr(nn))
        return t, m, tri, nn

    def trace_photons(self, seed, max_bounces, cap_g, cap_c=0, tag=0, max_paths=1 << 40):
        gp = np.empty((cap_g, 3), np.float32); gw = np.empty_like(gp); gd = np.empty_like(gp)
        gpath = np.empty(cap_g, np.int64); gb = np.empty(cap_g, np.int32)
        cc = max(cap_c, 1)
        cp = np.empty((cc, 3), np.float32); cw = np.empty_like(cp); cd = np.empty_like(cp)
        cpath = np.empty(cc, np.int64); cb = np.empty(cc, np.int32)
        ng = np.zeros(1, np.int64); nc = np.zeros(1, np.int64)
        paths = self.orc.L.orc_trace_photons(self.h, seed, tag, max_bounces, cap_g, cap_c, max_paths,
                                             _ptr(gp), _ptr(gw), _ptr(gd), _ptr(gpath), _ptr(gb),
                                             _ptr(cp), _ptr(cw), _ptr(cd), _ptr(cpath), _ptr(cb),
                                             _ptr(ng), _ptr(nc))
        return dict(paths=int(paths), g_pos=gp[:ng[0]], g_pow=gw[:ng[0]], g_dir=gd[:ng[0]],
                    g_path=gpath[:ng[0]], g_bounce=gb[:ng[0]],
                    c_pos=cp[:nc[0]], c_pow=cw[:nc[0]], c_dir=cd[:nc[0]], c_path=cpath[:nc[0]],
                    c_bounce=cb[:nc[0]])

    def trace_paths(self, seed, max_bounces, power_cap, p0, p1, tag=0):
        n = p1 - p0
        counts = np.empty((n, 2), np.int32)
        draws = np.empty(n, np.int32)
        cap = n * max_bounces
        gp = np.empty((cap, 3), np.float32); gd = np.empty_like(gp); gb = np.empty(cap, np.int32)
        cp = np.empty((cap, 3), np.float32); cd = np.empty_like(cp); cb = np.empty(cap, np.int32)
        ng = np.zeros(1, np.int64); nc = np.zeros(1, np.int64)
        self.orc.L.orc_trace_paths(self.h, seed, tag, max_bounces, power_cap, p0, p1, _ptr(counts), _ptr(draws),
                                   _ptr(gp), _ptr(gd), _ptr(gb), _ptr(cp), _ptr(cd), _ptr(cb), _ptr(ng), _ptr(nc))
        return dict(counts=counts, draws=draws, g_pos=gp[:ng[0]], g_dir=gd[:ng[0]], g_bounce=gb[:ng[0]],
                    c_pos=cp[:nc[0]], c_dir=cd[:nc[0]], c_bounce=cb[:nc[0]])

    def eye_hits(self, cam_vec, width, height, pixels, max_depth=4):
        """The eye paths of `pixels` (y * width + x) as the reference's render_trace
        walks them: dict of a, b, c (hits, 4 floats each; the product's request
        layout), counts per pixel."""
        px = _c(pixels, np.int64)
        counts = np.empty(px.size, np.int32)
        cap = int(px.size) * (2 ** max(max_depth, 1))
        a = np.empty((cap, 4), np.float32); b = np.empty_like(a); c = np.empty_like(a)
        self.orc.L.orc_eye_hits.restype = C.c_int64
        n = self.orc.L.orc_eye_hits(self.h, _ptr(_c(cam_vec, np.float32)), C.c_int(width), C.c_int(height),
                                    C.c_int64(px.size), _ptr(px), C.c_int(max_depth), _ptr(counts), _ptr(a), _ptr(b),
                                    _ptr(c), C.c_int64(cap))
        if n < 0:
            raise RuntimeError("orc_eye_hits: record capacity exceeded")
        return dict(a=a[:n], b=b[:n], c=c[:n], counts=counts)

    def render(self, cam_vec, width, height, g: GridResult, k, radius, max_depth=4, y0=0, y1=None,
               c: GridResult = None, k_c=0, r_c=0.2, heap_mode=False, faithful_caustic=True):
        y1 = height if y1 is None else y1
        npx = (y1 - y0) * width
        rad = np.empty((npx, 3), np.float32)
        ldr = np.empty((npx, 3), np.float32)
        rgb = np.empty((npx, 3), np.uint8)
        hits = np.empty(npx, np.int32)
        cargs = [None, 0.0, None, None, None, None, None, None] if c is None else \
            [_c(c.dims, np.int32), c.cell, c.starts, c.sizes, _c(c.spos, np.float32), _c(c.sdir, np.float32),
             _c(c.spow, np.float32), _c(c.sid, np.uint32)]
        ovf = self.orc.L.orc_render(
            self.h, _ptr(_c(cam_vec, np.float32)), width, height, y0, y1,
            _ptr(g.aabb), _ptr(g.dims), g.cell, _ptr(g.starts), _ptr(g.sizes), _ptr(_c(g.spos, np.float32)),
            _ptr(_c(g.sdir, np.float32)), _ptr(_c(g.spow, np.float32)), _ptr(_c(g.sid, np.uint32)),
            _ptr(cargs[0]), float(cargs[1]), *[_ptr(x) for x in cargs[2:]],
            int(max_depth), float(radius), int(k), float(r_c), int(k_c), int(heap_mode), int(faithful_caustic),
            _ptr(rad), _ptr(ldr), _ptr(rgb), _ptr(hits))
        return dict(radiance=rad, ldr=ldr, rgb8=rgb, hits=hits, overflow=int(ovf))


class RefHost:
    """The reference's own host-callable render code (CudaPhotonMapping, CPU mode)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference is mounted")
        L = C.CDLL(path)
        self.L = L
        L.ref_scene_create.restype = C.c_void_p
        L.ref_scene_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                       C.c_int, C.c_void_p]
        L.ref_scene_destroy.argtypes = [C.c_void_p]
        L.ref_camera.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_int, C.c_void_p]
        L.ref_camera_rays.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_int, C.c_int,
                                      C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_intersect.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 5
        L.ref_ray_ops.argtypes = [C.c_int] + [C.c_void_p] * 7
        L.ref_hdr.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.ref_gather.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_float] + [C.c_void_p] * 5 + \
            [C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_int] + [C.c_void_p] * 5
        L.ref_grid_sizing.restype = C.c_int
        L.ref_grid_sizing.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_render.argtypes = ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_int,
                                  C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_float] +
                                 [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_float] + [C.c_void_p] * 5 +
                                 [C.c_int, C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_void_p])

    def scene(self, sc):
        keep = [_c(sc.tri_pos, np.float32), _c(sc.tri_nrm, np.float32), _c(sc.tri_model, np.int32),
                _c(sc.materials, np.float32), _c(sc.light_intensity, np.float32)]
        h = self.L.ref_scene_create(sc.ntri, _ptr(keep[0]), _ptr(keep[1]), _ptr(keep[2]), sc.nmodel,
                                    _ptr(keep[3]), int(sc.light_model), _ptr(keep[4]))
        return _RefScene(self, h)

    def camera(self, cam):
        out = np.empty(15, np.float32)
        self.L.ref_camera(_ptr(_c(cam.position, np.float32)), _ptr(_c(cam.direction, np.float32)),
                          _ptr(_c(cam.up, np.float32)), float(cam.fov_deg), cam.width, cam.height, _ptr(out))
        return out

    def camera_rays(self, cam, xs, ys):
        xs = _c(xs, np.int32); ys = _c(ys, np.int32)
        out = np.empty((xs.size, 3), np.float32)
        self.L.ref_camera_rays(_ptr(_c(cam.position, np.float32)), _ptr(_c(cam.direction, np.float32)),
                               _ptr(_c(cam.up, np.float32)), float(cam.fov_deg), cam.width, cam.height, xs.size,
                               _ptr(xs), _ptr(ys), _ptr(out))
        return out

    def ray_ops(self, dirs, frm, nrm, etas):
        dirs = _c(dirs, np.float32).reshape(-1, 3); n = dirs.shape[0]
        a = np.empty((n, 6), np.float32); b = np.empty((n, 6), np.float32); ok = np.empty(n, np.int32)
        self.L.ref_ray_ops(n, _ptr(dirs), _ptr(_c(frm, np.float32)), _ptr(_c(nrm, np.float32)),
                           _ptr(_c(etas, np.float32)), _ptr(a), _ptr(b), _ptr(ok))
        return a, b, ok

    def hdr(self, rgb):
        rgb = _c(rgb, np.float32).reshape(-1, 3)
        out = np.empty_like(rgb)
        self.L.ref_hdr(rgb.shape[0], _ptr(rgb), _ptr(out))
        return out

    def grid_sizing(self, pos, aabb, desired=1000):
        """The reference's grid sizing + density re-grid for these photon positions:
        (dims, cell, regridded, largest cell count of the first grid)."""
        pos = _c(pos, np.float32).reshape(-1, 3)
        dims = np.empty(3, np.int32); cell = np.empty(1, np.float32); mx = np.empty(1, np.uint32)
        rg = self.L.ref_grid_sizing(pos.shape[0], _ptr(pos), _ptr(_c(aabb, np.float32)), int(desired), _ptr(dims),
                                    _ptr(cell), _ptr(mx))
        return dims, float(cell[0]), bool(rg), int(mx[0])

    def gather(self, g: GridResult, qpos, qnrm, radius, k):
        qpos = _c(qpos, np.float32).reshape(-1, 3); qnrm = _c(qnrm, np.float32).reshape(-1, 3)
        nq = qpos.shape[0]
        slots = np.empty((nq, k), np.uint32); dist = np.empty((nq, k), np.float32)
        cnt = np.empty(nq, np.int32); full = np.empty(nq, np.int32); rad = np.empty((nq, 3), np.float32)
        n = g.spos.shape[0]
        self.L.ref_gather(n, _ptr(g.aabb), _ptr(_c(g.dims, np.int32)), g.cell, _ptr(g.starts), _ptr(g.sizes),
                          _ptr(_c(g.spos, np.float32)), _ptr(_c(g.sdir, np.float32)), _ptr(_c(g.spow, np.float32)),
                          nq, _ptr(qpos), _ptr(qnrm), float(radius), int(k), _ptr(slots), _ptr(dist), _ptr(cnt),
                          _ptr(full), _ptr(rad))
        return slots, dist, cnt, full, rad


class _RefScene:
    def __init__(self, ref: RefHost, h):
        self.ref = ref
        self.h = h

    def __del__(self):
        try:
            self.ref.L.ref_scene_destroy(self.h)
        except Exception:
            pass

    def intersect(self, orig, dirs):
        orig = _c(orig, np.float32).reshape(-1, 3); dirs = _c(dirs, np.float32).reshape(-1, 3)
        n = orig.shape[0]
        p = np.empty((n, 3), np.float32); m = np.empty(n, np.int32); nn = np.empty((n, 3), np.float32)
        self.ref.L.ref_intersect(self.h, n, _ptr(orig), _ptr(dirs), _ptr(p), _ptr(m), _ptr(nn))
        return p, m, nn

    def render(self, cam, g: GridResult, k, radius, max_depth=4, y0=0, y1=None, def_ior=1.0,
               c: GridResult = None, k_c=0):
        y1 = cam.height if y1 is None else y1
        npx = (y1 - y0) * cam.width
        ldr = np.empty((npx, 3), np.float32)
        rgb = np.empty((npx, 3), np.uint8)
        ng = g.spos.shape[0]
        if c is None:
            cargs = [0, None, 0.0, None, None, None, None, None]
        else:
            cargs = [c.spos.shape[0], _c(c.dims, np.int32), c.cell, c.starts, c.sizes, _c(c.spos, np.float32),
                     _c(c.sdir, np.float32), _c(c.spow, np.float32)]
        self.ref.L.ref_render(
            self.h, _ptr(_c(cam.position, np.float32)), _ptr(_c(cam.direction, np.float32)),
            _ptr(_c(cam.up, np.float32)), float(cam.fov_deg), cam.width, cam.height, y0, y1, ng,
            _ptr(g.aabb), _ptr(_c(g.dims, np.int32)), g.cell, _ptr(g.starts), _ptr(g.sizes),
            _ptr(_c(g.spos, np.float32)), _ptr(_c(g.sdir, np.float32)), _ptr(_c(g.spow, np.float32)),
            int(cargs[0]), _ptr(cargs[1]), float(cargs[2]), *[_ptr(x) for x in cargs[3:]],
            int(max_depth), float(def_ior), int(k), int(k_c), _ptr(ldr), _ptr(rgb))
        return dict(ldr=ldr, rgb8=rgb)


class RefTrace:
    """The reference's own photon tracer (CudaPhotonMapping/PhotonTracing.cu and
    what it calls), compiled as host code and driven one path at a time by
    oracle/ref_host/ref_trace.cu.  Its bounce limit is the reference's fixed 10."""

    MAX_BOUNCES = 10

    def __init__(self, path: str = REF_TRACE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference is mounted")
        L = C.CDLL(path)
        self.L = L
        L.ref_trace_scene_create.restype = C.c_void_p
        L.ref_trace_scene_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                             C.c_int, C.c_void_p]
        L.ref_trace_scene_destroy.argtypes = [C.c_void_p]
        L.ref_trace_critical_angles.restype = C.c_int
        L.ref_trace_critical_angles.argtypes = [C.c_void_p, C.c_float, C.c_void_p, C.c_int]
        L.ref_trace_paths.argtypes = ([C.c_void_p, C.c_float, C.c_uint64, C.c_uint32, C.c_int64, C.c_int64,
                                       C.c_int64, C.c_int] + [C.c_void_p] * 12)
        L.ref_gpu_trace_paths.restype = C.c_int
        L.ref_gpu_trace_paths.argtypes = ([C.c_void_p, C.c_float, C.c_uint64, C.c_uint32, C.c_int64, C.c_int64,
                                           C.c_int64] + [C.c_void_p] * 10)

    def scene(self, sc):
        """A reference scene (one Model per model index).  The reference holds one
        material per model, so a per-triangle diffuse override is not representable."""
        if sc.tri_diffuse is not None:
            raise ValueError("the reference's Model has one material per model: no per-triangle diffuse")
        keep = [_c(sc.tri_pos, np.float32), _c(sc.tri_nrm, np.float32), _c(sc.tri_model, np.int32),
                _c(sc.materials, np.float32), _c(sc.light_intensity, np.float32)]
        h = self.L.ref_trace_scene_create(sc.ntri, _ptr(keep[0]), _ptr(keep[1]), _ptr(keep[2]), sc.nmodel,
                                          _ptr(keep[3]), int(sc.light_model), _ptr(keep[4]))
        return _RefTraceScene(self, h, float(sc.default_ior))


class _RefTraceScene:
    def __init__(self, ref: RefTrace, h, default_ior):
        self.ref = ref
        self.h = h
        self.default_ior = default_ior

    def __del__(self):
        try:
            self.ref.L.ref_trace_scene_destroy(self.h)
        except Exception:
            pass

    def critical_angles(self):
        """(n1, n2, cos) rows of the reference's critical-angle hash table, in slot order."""
        out = np.empty(3 * 1024, np.float32)
        n = self.ref.L.ref_trace_critical_angles(self.h, self.default_ior, _ptr(out), 1024)
        return out[:3 * min(n, 1024)].reshape(-1, 3)

    def trace_paths(self, seed, power_cap, p0, p1, tag=0, threads=None):
        n = p1 - p0
        cap = n * RefTrace.MAX_BOUNCES
        counts = np.empty((n, 2), np.int32)
        draws = np.empty(n, np.int32)
        gp = np.empty((cap, 3), np.float32); gw = np.empty_like(gp); gd = np.empty_like(gp)
        gb = np.empty(cap, np.int32)
        cp = np.empty((cap, 3), np.float32); cw = np.empty_like(cp); cd = np.empty_like(cp)
        cb = np.empty(cap, np.int32)
        ng = np.zeros(1, np.int64); nc = np.zeros(1, np.int64)
        threads = threads or max(1, os.cpu_count() or 1)
        self.ref.L.ref_trace_paths(self.h, self.default_ior, seed, tag, power_cap, p0, p1, int(threads),
                                   _ptr(counts), _ptr(draws), _ptr(gp), _ptr(gw), _ptr(gd), _ptr(gb),
                                   _ptr(cp), _ptr(cw), _ptr(cd), _ptr(cb), _ptr(ng), _ptr(nc))
        return dict(counts=counts, draws=draws, g_pos=gp[:ng[0]], g_pow=gw[:ng[0]], g_dir=gd[:ng[0]],
                    g_bounce=gb[:ng[0]], c_pos=cp[:nc[0]], c_pow=cw[:nc[0]], c_dir=cd[:nc[0]],
                    c_bounce=cb[:nc[0]])

    def gpu_trace_paths(self, seed, power_cap, p0, p1, tag=0):
        """The same paths through the reference's device build on the current GPU
        (its GPU numerics: vec3 rounded toward zero), one path per thread."""
        n = p1 - p0
        cap = n * RefTrace.MAX_BOUNCES
        counts = np.empty((n, 2), np.int32)
        draws = np.empty(n, np.int32)
        gp = np.empty((cap, 3), np.float32); gd = np.empty_like(gp); gb = np.empty(cap, np.int32)
        cp = np.empty((cap, 3), np.float32); cd = np.empty_like(cp); cb = np.empty(cap, np.int32)
        ng = np.zeros(1, np.int64); nc = np.zeros(1, np.int64)
        rc = self.ref.L.ref_gpu_trace_paths(self.h, self.default_ior, seed, tag, power_cap, p0, p1, _ptr(counts),
                                            _ptr(draws), _ptr(gp), _ptr(gd), _ptr(gb), _ptr(cp), _ptr(cd), _ptr(cb),
                                            _ptr(ng), _ptr(nc))
        if rc != 0:
            raise RuntimeError(f"ref_gpu_trace_paths: CUDA error {rc}")
        return dict(counts=counts, draws=draws, g_pos=gp[:ng[0]], g_dir=gd[:ng[0]], g_bounce=gb[:ng[0]],
                    c_pos=cp[:nc[0]], c_dir=cd[:nc[0]], c_bounce=cb[:nc[0]])
