"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container where the reference is mounted (it reads the reference's
100-photon dump and drives the reference's own host render code through
oracle/_ref/libref_host.so, which `make -C oracle ref` compiles from the
reference sources in place):

    make -C oracle all && python tests/golden/make_golden.py [fixture100] [cornell] [tracer] [grid]

(no argument: all four; `cornell` continues the random stream of `fixture100`,
so those two are written together).  The reference root is $PM_REFERENCE_ROOT (default
/root/reference).

Outputs (all small .npz files, committed):
  fixture100.npz  the reference's 100-photon map (CudaPhotonMapping/global_map_test.txt,
                  read as CudaPhotonMapping/Initializer.cu:102-141 does) and, on the grid the
                  oracle builds from it, PhotonGrid::find_nearests + get_color_from_photon_grid
                  results of the reference for 300 query points.
  cornell_ref.npz reference results on the small Cornell workload at reduced size:
                  Camera vectors, eye-ray directions, Raytracer::find_intersection for 4096
                  rays, Ray::reflect / refract, HDR, gathers for 512 points and the CPU-mode
                  render (Raytracer::render_trace per pixel) of an 80 x 60 frame over a
                  20k-photon map traced by the oracle (seed 0; its checksum is stored).
  tracer_ref.npz  the reference's own photon tracer (CudaPhotonMapping/PhotonTracing.cu and the
                  functions it calls, compiled as host code into oracle/_ref/libref_trace.so) on
                  the cases of tests/golden/ref_cases.py: per case the checksum of the whole
                  path range and, for its first paths, the per-path counts and draws and the
                  photon records.
  grid_sizing_ref.npz  the reference's grid sizing and density re-grid (PhotonGrid(n, aabb),
                  compute_grid_and_cell_size, analyze_density's rule; CudaPhotonMapping/PhotonGrid.cu:41-141)
                  on the seeded photon sets of tests/golden/ref_cases.py GRID_CASES.
"""
from __future__ import annotations

import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "cuda-photon-mapping_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from photonmap import scenes  # noqa: E402
from oracle import Oracle, RefHost, RefTrace  # noqa: E402
import ref_cases  # noqa: E402

REF_ROOT = os.environ.get("PM_REFERENCE_ROOT", "/root/reference")
REF_DUMP = os.path.join(REF_ROOT, "CudaPhotonMapping", "global_map_test.txt")
OUT = os.path.dirname(os.path.abspath(__file__))


def read_dump(path):
    raw = open(path, "rb").read()
    (n,) = struct.unpack_from("<Q", raw, 0)
    rec = np.frombuffer(raw, dtype="<f4", count=9 * n, offset=8).reshape(n, 9)
    return rec[:, 0:3].copy(), rec[:, 3:6].copy(), rec[:, 6:9].copy()


def photons_checksum(tr):
    h = np.concatenate([tr["g_pos"].ravel(), tr["g_dir"].ravel(), tr["g_pow"].ravel()]).view(np.uint32)
    return int(np.bitwise_xor.reduce(h * np.arange(1, h.size + 1, dtype=np.uint32)))


def main(parts):
    orc, ref = Oracle(), RefHost()
    rng = np.random.default_rng(7)
    if "fixture100" in parts:
        make_fixture100(orc, ref, rng)
    if "cornell" in parts:
        make_cornell(orc, ref, rng)
    if "tracer" in parts:
        make_tracer()
    if "grid" in parts:
        make_grid_sizing(ref)
    print("wrote", os.listdir(OUT))


def make_fixture100(orc, ref, rng):
    pos, powr, dirs = read_dump(REF_DUMP)
    lo = pos.min(0) - 0.05
    hi = pos.max(0) + 0.05
    aabb = np.concatenate([lo, hi]).astype(np.float32)
    g = orc.grid_build(pos, powr, dirs, aabb, desired=10)
    q = (pos[rng.integers(0, len(pos), 300)] + rng.normal(scale=0.1, size=(300, 3))).astype(np.float32)
    qn = rng.normal(size=(300, 3)).astype(np.float32)
    qn /= np.linalg.norm(qn, axis=1, keepdims=True)
    k, r = 8, 0.6
    slots, dist, cnt, full, rad = ref.gather(g, q, qn, r, k)
    ids = np.where(slots == 0xFFFFFFFF, 0xFFFFFFFF, g.sid[np.minimum(slots, len(g.sid) - 1)]).astype(np.uint32)
    np.savez_compressed(os.path.join(OUT, "fixture100.npz"), pos=pos, power=powr, dir=dirs, aabb=aabb, desired=10,
                        dims=g.dims, cell=np.float32(g.cell), starts=g.starts, sizes=g.sizes, q=q, qn=qn, k=k, r=r,
                        ref_ids=ids, ref_dist=dist, ref_cnt=cnt, ref_full=full, ref_rad=rad)


def make_cornell(orc, ref, rng):
    sc, _, _ = scenes.workload("cornell_small")
    cam = scenes.default_camera(80, 60)
    os_, rs = orc.scene(sc), ref.scene(sc)
    cams = [cam, scenes.CameraSpec((0.3, 0.2, 3.0), (-0.1, -0.05, -1.0), (0, 1, 0), 60.0, 64, 48),
            scenes.CameraSpec((0.0, 0.5, 2.5), (0.0, -0.3, -1.0), (0, 1, 0), 45.0, 1920, 1080)]
    cam_vecs = np.stack([ref.camera(c) for c in cams])
    xs = rng.integers(0, 1920, 1000); ys = rng.integers(0, 1080, 1000)
    eye_dirs = ref.camera_rays(cams[2], xs, ys)

    N = 4096
    orig = rng.uniform(-0.95, 0.95, (N, 3)).astype(np.float32)
    d = rng.normal(size=(N, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True); d = d.astype(np.float32)
    ipt, imodel, inrm = rs.intersect(orig, d)

    M = 2000
    rd = rng.normal(size=(M, 3)); rd /= np.linalg.norm(rd, axis=1, keepdims=True); rd = rd.astype(np.float32)
    rn = rng.normal(size=(M, 3)); rn /= np.linalg.norm(rn, axis=1, keepdims=True); rn = rn.astype(np.float32)
    rn[(rd * rn).sum(1) > 0] *= -1
    rf = rng.uniform(-1, 1, (M, 3)).astype(np.float32)
    etas = np.stack([rng.choice([1.0, 1.5], M), rng.choice([1.0, 1.5, 1.33], M)], 1).astype(np.float32)
    refl, refr, refr_ok = ref.ray_ops(rd, rf, rn, etas)

    hdr_in = np.abs(rng.normal(scale=0.7, size=(1000, 3))).astype(np.float32)
    hdr_out = ref.hdr(hdr_in)

    tr = os_.trace_photons(0, 8, 20000)
    gg = orc.grid_build(tr["g_pos"], tr["g_pow"], tr["g_dir"], os_.aabb())
    hit = imodel >= 0
    qp = ipt[hit][:512]
    qnn = inrm[hit][:512]
    gslots, gdist, gcnt, gfull, grad = ref.gather(gg, qp, qnn, 0.1, 100)
    gids = np.where(gslots == 0xFFFFFFFF, 0xFFFFFFFF, gg.sid[np.minimum(gslots, len(gg.sid) - 1)]).astype(np.uint32)
    ren = rs.render(cam, gg, 100, 0.1, 4)
    np.savez_compressed(os.path.join(OUT, "cornell_ref.npz"),
                        cam_vecs=cam_vecs, eye_xs=xs, eye_ys=ys, eye_dirs=eye_dirs,
                        ray_orig=orig, ray_dir=d, ref_point=ipt, ref_model=imodel, ref_normal=inrm,
                        op_dir=rd, op_nrm=rn, op_from=rf, op_etas=etas, ref_reflect=refl, ref_refract=refr,
                        ref_refract_ok=refr_ok, hdr_in=hdr_in, hdr_out=hdr_out,
                        photons=20000, seed=0, max_bounces=8, photons_checksum=photons_checksum(tr),
                        gather_q=qp, gather_n=qnn, ref_gather_ids=gids, ref_gather_dist=gdist,
                        ref_gather_cnt=gcnt, ref_gather_full=gfull, ref_gather_rad=grad,
                        render_w=80, render_h=60, render_k=100, render_r=0.1, render_depth=4,
                        ref_ldr=ren["ldr"], ref_rgb8=ren["rgb8"])


def make_tracer():
    rt = RefTrace()
    arrays = {}
    for name, (build, seed, cap, p0, p1, sub) in ref_cases.CASES.items():
        rsc = rt.scene(build())
        full = rsc.trace_paths(seed, cap, p0, p1)
        part = rsc.trace_paths(seed, cap, p0, sub)
        arrays[f"{name}__checksum"] = np.uint32(ref_cases.checksum(full))
        arrays[f"{name}__n"] = np.array([full["g_pos"].shape[0], full["c_pos"].shape[0]], np.int64)
        arrays[f"{name}__power"] = np.concatenate([full["g_pow"], full["c_pow"]])[:1]
        for f in ref_cases.FIELDS:
            arrays[f"{name}__{f}"] = part[f]
    np.savez_compressed(os.path.join(OUT, "tracer_ref.npz"), **arrays)


def make_grid_sizing(ref):
    arrays = {}
    for name, (build, desired) in ref_cases.GRID_CASES.items():
        pos, aabb = build()
        dims, cell, regrid, mx = ref.grid_sizing(pos, aabb, desired)
        arrays[f"{name}__dims"] = dims
        arrays[f"{name}__cell"] = np.float32(cell)
        arrays[f"{name}__regrid"] = np.int32(regrid)
        arrays[f"{name}__max"] = np.uint32(mx)
    np.savez_compressed(os.path.join(OUT, "grid_sizing_ref.npz"), **arrays)


if __name__ == "__main__":
    main(sys.argv[1:] or ["fixture100", "cornell", "tracer", "grid"])
