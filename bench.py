"""Benchmark: the plain photon-mapping frame at 10M photons, 1920x1080.

One step = one full frame of the plain method on the ``cornell_hf_1080p``
workload: trace 10M global photons (max 10 bounces), build the photon grid,
render 1920x1080 (kNN k = 64, r = 0.05, eye depth 4).  ``value`` is Mphotons/s
of the whole frame pipeline (photons / step time) summed over ranks;
``ms_per_step`` is ms/frame, from CUDA events on the stream the context
launches on.  Inputs (scene, photon maps ~0.5 GB) are larger than L2.
``e2e``: the same frames through the public API with every frame read back
to pinned host memory (6.2 MB at 1080p), the read-back of frame i on a copy
stream beside frame i + 1 (two frame buffers); host-to-device bytes are 0,
since a step's only input is its seed (the scene stays resident).
Multi-GPU: independent replicas (weak scaling, no collective on the data
path; the photon maps do not exchange).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cuda-photon-mapping_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "Mphotons/s + ms/frame @10M,1080p"
WORKLOAD = "cornell_hf_1080p"


def max_over_ranks(values, world):
    """Each value's maximum over the ranks (the slowest rank times the job);
    the tensor lives where the process group's backend works (CUDA for nccl)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def step_seed(seed, rank, step):
    """Photon-stream key of a rank's step: every rank traces its own
    independent photons (replicas, weak scaling), every step new ones."""
    return seed + (rank << 32) + step   # 64-bit stream keys: 2^32 steps per rank


def job_mphotons(world, photons_per_rank, ms):
    """Whole-job throughput: all ranks' photons over the (max-over-ranks) step time."""
    return world * photons_per_rank / (ms * 1e-3) / 1e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-cache frame comparison")
    ap.add_argument("--no-rmse", action="store_true", help="skip the learned frame's RMSE against the FP64 reference")
    ap.add_argument("--train-batch", type=int, default=LEARNED["batch"],
                    help="samples per Adam step of the learned frame's 2^20 training samples")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-instance batched workload")
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--bvh", default="host_sah", choices=["host_sah", "device_lbvh"],
                    help="BVH builder of the scene (same photons and image either way)")
    # size overrides (profiling captures run reduced cases of the same workload)
    ap.add_argument("--photons", type=int, default=0)
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event reasons sampled every 10 ms while running
    (read-only NVML queries of the device torch uses; nvidia-smi at 200 ms
    when NVML is unavailable)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.samples = []
        self.stop_evt = threading.Event()
        self.nv = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            self.nv, self.h = self._nvml_handle()
            self.max_mhz = float(self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _poll(self):
        nv, h = self.nv, self.h
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop_evt.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(get_reasons(h))))
            except Exception:
                pass
            self.stop_evt.wait(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nv is not None:
            self.stop_evt.set()
            self.t.join(timeout=2)
            if not self.samples:
                return None
            reasons = sorted(nm for nm, bit in self.BITS.items() if any(r & bit for _, r in self.samples))
            return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(self.samples), "source": "nvml 10 ms"}
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi 200 ms"}


# ----------------------------------------------------------------- CPU leg
def cpu_reference_estimate(sc, w, rows=8, trace_paths=16384, threads=None):
    """The reference's CPU path on the host cores, on a bounded sample, scaled
    to one full frame of the workload.

    * photon pass: the reference's tracer is device code (emit is __global__,
      trace / destiny __device__); its algorithm (brute-force closest hit) is
      timed as the oracle's restatement, which tests/test_tracer_pin.py pins
      bit for bit to the reference's own tracer compiled as host code,
      OpenMP over the host cores, on the exact path range [0, trace_paths);
      scaled by the paths the workload needs (its photon count over the
      sample's global photons per path);
    * grid: the oracle's grid build over a map of the workload's size (the
      traced sample replicated with a 1e-4 jitter);
    * frame: the reference's own Raytracer::render_trace (oracle/_ref, its CPU
      mode, single-threaded by design) on ``rows`` image rows spread over the
      frame, one process per host core, over that map; the mean row time is
      scaled to all rows and divided over the cores.
    Returns the scaled times and wall_s, the sample's own wall time.
    """
    import multiprocessing as mp
    import tempfile
    from oracle import Oracle
    w0 = time.perf_counter()
    orc = Oracle()
    s = orc.scene(sc)
    threads = threads or os.cpu_count() or 1
    n = w["photons"]
    t0 = time.perf_counter()
    tr = s.trace_paths(w["seed"], w["max_bounces"], n, 0, trace_paths)
    t_sample = time.perf_counter() - t0
    got = int(tr["g_pos"].shape[0])
    per_path = got / trace_paths
    paths_needed = n / max(per_path, 1e-9)
    t_trace = t_sample * paths_needed / trace_paths
    rep = int(np.ceil(n / max(got, 1)))
    rng = np.random.default_rng(1)
    pos = (np.tile(tr["g_pos"], (rep, 1))[:n] + rng.normal(scale=1e-4, size=(n, 3)).astype(np.float32)).astype(np.float32)
    dirs = np.tile(tr["g_dir"], (rep, 1))[:n]
    pw = np.tile(np.asarray(sc.light_intensity, np.float32) / np.float32(n), (n, 1))
    t0 = time.perf_counter()
    g = orc.grid_build(pos, pw, dirs, s.aabb())
    t_grid = time.perf_counter() - t0
    H = w["height"]
    ys = np.linspace(0, H - 1, rows).astype(int)
    with tempfile.TemporaryDirectory() as tmp:
        for name in ("spos", "sdir", "spow", "starts", "sizes", "dims", "aabb"):
            np.save(os.path.join(tmp, name + ".npy"), getattr(g, name))
        np.save(os.path.join(tmp, "cell.npy"), np.float32(g.cell))
        ctx = mp.get_context("spawn")
        args = [(w, tmp, int(y), sc) for y in ys]
        with ctx.Pool(min(threads, rows)) as pool:
            per_row = pool.map(_ref_row, args)
    t_row = float(np.mean(per_row))
    t_frame = t_row * H / threads
    total = t_trace + t_grid + t_frame
    return dict(step_s=total, trace_s=t_trace, grid_s=t_grid, frame_s=t_frame, row_s=t_row, cores=threads,
                sample=f"photon pass: paths [0, {trace_paths}) traced by the oracle's restatement of the "
                       f"reference's tracer ({got} global photons, scaled to the {paths_needed:.0f} paths of "
                       f"{n} photons); grid of {n} photons (sample replicated); {rows} of {H} rows rendered by "
                       f"the reference's own render_trace; {threads} threads / processes",
                wall_s=time.perf_counter() - w0)


def _ref_row(arg):
    w, tmp, y, sc = arg
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import GridResult, RefHost
    from photonmap import scenes
    ld = lambda nm: np.load(os.path.join(tmp, nm + ".npy"), mmap_mode="r")  # noqa: E731
    g = GridResult(np.array(ld("aabb")), np.array(ld("dims")), float(ld("cell")), np.array(ld("starts")),
                   np.array(ld("sizes")), None, np.array(ld("spos")), np.array(ld("sdir")), np.array(ld("spow")), None)
    rs = RefHost().scene(sc)
    cam = scenes.default_camera(w["width"], w["height"])
    t0 = time.perf_counter()
    rs.render(cam, g, w["k"], w["radius"], w["max_depth"], y0=y, y1=y + 1)
    return time.perf_counter() - t0


def override(w, cs, args):
    w = dict(w)
    if args.photons:
        w["photons"] = args.photons
    if args.width:
        w["width"] = args.width
    if args.height:
        w["height"] = args.height
    from photonmap import scenes
    cs = scenes.CameraSpec(cs.position, cs.direction, cs.up, cs.fov_deg, w["width"], w["height"])
    return w, cs


# ----------------------------------------------------------------- GPU arm
def batched_frames(args, rank):
    """The batched workload: seeded instances of the small room (light jitter,
    sphere radii, photon counts log-uniform in [10k, 2M], square images with
    edge log-uniform in [128, 1024], k in {32, 64, 128}), one frame of all of
    them per step through the batch (one work queue per stage, autotuned,
    replayed from a CUDA graph), against the same instances rendered one after
    another through the single-instance API (trace + grid + render each)."""
    import torch
    import photonmap
    from photonmap import scenes
    insts = []
    for d in scenes.batch_instances(n=args.batch_instances, seed=rank):
        cs = d.pop("camera_spec")
        d["camera"] = photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, cs.width, cs.height)
        insts.append(d)
    t0 = time.perf_counter()
    b = photonmap.Batch(insts, autotune=True, use_graph=True)
    t_create = time.perf_counter() - t0
    K = max(args.steps, 3)
    for f in range(2):
        b.frame(f)
    ms_dev = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for f in range(K):
        b.frame(2 + f)
        ms_dev.append(b.info()["ms_last_frame"])
    torch.cuda.synchronize()
    ms_wall = (time.perf_counter() - t0) * 1000 / K
    info = b.info()
    b.close()
    # the same instances one after another through the single-instance API
    ctxs = []
    for d in insts:
        c = photonmap.Context(torch.cuda.current_device())
        c.set_scene(d["scene"])
        ctxs.append(c)

    dev_ms = [0.0]

    def sequential(f):
        for c, d in zip(ctxs, insts):
            c.trace_photons(d["seed"] + f, d["max_bounces"], d["photons"])
            c.build_grid(photonmap.PM_MAP_GLOBAL)
            c.render(d["camera"], d["k"], d["radius"], d["max_depth"], radiance=False)
            st = c.stage_times()
            dev_ms[0] += st["trace_ms"] + st["grid_ms"] + st["eye_ms"] + st["gather_ms"] + st["resolve_ms"]
        for c in ctxs:
            c.sync()

    sequential(0)
    torch.cuda.synchronize()
    dev_ms[0] = 0.0
    t0 = time.perf_counter()
    for f in range(K):
        sequential(2 + f)
    ms_seq = (time.perf_counter() - t0) * 1000 / K
    ms_seq_dev = dev_ms[0] / K
    for c in ctxs:
        c.close()
    photons = sum(d["photons"] for d in insts)
    pixels = sum(d["camera"].width * d["camera"].height for d in insts)
    ms = float(np.median(ms_dev))
    return {"instances": len(insts), "photons_per_frame": photons, "pixels_per_frame": pixels,
            "ms_per_frame": ms, "mphotons_per_s": photons / (ms * 1e-3) / 1e6,
            "ms_per_frame_wall": ms_wall, "ms_per_frame_sequential_api": ms_seq,
            "speedup_vs_sequential": ms_seq / ms_wall,
            "ms_per_frame_sequential_device": ms_seq_dev, "speedup_vs_sequential_device": ms_seq_dev / ms,
            "sequential": "the instances one after another through the single-instance API, 64 contexts, host "
                          "clock (host-synchronous calls: depends on the host); _device: the sum of their stage "
                          "times (CUDA events), against the batch's device time",
            "launches_per_frame": info["launches_per_frame"],
            "graph": bool(info["graph"]), "autotuned": {"desired_per_cell": info["desired_per_cell"],
                                                        "gather_warps": info["gather_warps"],
                                                        "gather_guess": info["gather_guess"],
                                                        "subcell_khint": info["subcell_khint"],
                                                        "trace_refill": info["trace_refill"]},
            "underfilled_instances": info["underfilled"], "create_s": t_create,
            "stage_ms_eager": info["stage_ms"]}


LEARNED = dict(train_per_frame=1 << 20, batch=1 << 18, warm_steps=3000, pool_samples=2_200_000,
               rmse_pixels=65_536, rmse_maps=10)


def learned_frames(ctx, sc, cs, cam, w, rgb, args, world):
    """Frame time of the plain render against the learned render on the same
    photon map (the map stays resident, as in the reference's render loop).
    Learned frame = online training on 2^20 pooled samples (the learned-cache
    configuration: 1M seeded surface points per frame) + the cache-answered render with its
    per-tile exact-gather fallback.  The pool (stratified primary hits
    labelled by the kNN gather, at least 2^20 of them) is built once per map;
    the cache's first fit (warm_steps Adam steps) is a one-time cost reported
    beside the per-frame times.  The frames' images are then compared with an
    FP64 reference of 10x the photons (learned_rmse)."""
    import torch
    import torch.distributed as dist
    from photonmap import learned
    P = LEARNED
    TRAIN_PER_FRAME, BATCH, WARM_STEPS = P["train_per_frame"], args.train_batch, P["warm_steps"]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    pool = learned.training_pool(ctx, cam, w["k"], w["radius"], n=P["pool_samples"], seed=1)
    ev[1].record()
    ctx.cache_init(seed=0, lr=3e-3, out_scale=pool.scale)
    learned.cache_fit(ctx, pool, WARM_STEPS, batch=1 << 16)
    ev[2].record()
    torch.cuda.synchronize()
    pool_ms, warm_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    K = max(args.steps, 3)
    steps_per_frame = TRAIN_PER_FRAME // BATCH

    def plain():
        ctx.render(cam, w["k"], w["radius"], w["max_depth"], radiance=False, out_rgb8=rgb)

    off = [0]
    stats = {}

    def learned_frame():
        _, off[0] = learned.cache_fit(ctx, pool, steps_per_frame, batch=BATCH, offset=off[0], want_loss=False)
        _, _, st = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], radiance=False, out_rgb8=rgb,
                                      **learned.FRAME_SETTINGS)
        stats.update(st)

    def timed(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(K):
            fn()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / K
        return max_over_ranks([ms], world)[0]

    ms_plain = timed(plain)
    ms_learned = timed(learned_frame)
    # the same frame captured once and replayed as one CUDA graph per frame: the
    # training first, then the render with the trained cache (serial), or the
    # render with the cache the previous frames trained while this frame's
    # training runs beside it (overlapped; the timed learned form)
    gstats = {}
    ms_graphs = {}
    for overlap in (False, True):
        graph = ctx.learned_graph(cam, w["k"], w["radius"], w["max_depth"], pool=pool, steps=steps_per_frame,
                                  batch=BATCH, offset=off[0], out_rgb8=rgb, overlap_training=overlap,
                                  **learned.FRAME_SETTINGS)
        ms_graphs[overlap] = timed(graph.run)
        gstats[overlap] = graph.run(stats=True)[2]
        off[0] = graph.offset()
        graph.close()
    ms_graph = ms_graphs[True]
    # tensor-core throughput of the cache kernels (forward 32,640 flop per sample, backward ~2x)
    fwd = 2 * (60 * 64 + 3 * 64 * 64 + 64 * 3)
    n = min(pool.n, 1 << 20)

    def infer():
        ctx.cache_infer(pool.pos[:n], pool.nrm[:n])

    def train():
        learned.cache_fit(ctx, pool, 1, batch=min(1 << 20, pool.n))

    ms_inf = timed(infer)
    ms_tr = timed(train)
    peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"] \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 1590.0
    inf_tf = fwd * n / (ms_inf * 1e-3) / 1e12
    tr_tf = 3 * fwd * min(1 << 20, pool.n) / (ms_tr * 1e-3) / 1e12
    block = {"ms_per_frame_plain": ms_plain, "ms_per_frame_learned": ms_learned, "speedup": ms_plain / ms_learned,
             "ms_per_frame_learned_graph": ms_graph, "speedup_graph": ms_plain / ms_graph,
             "ms_per_frame_learned_graph_serial": ms_graphs[False],
             "speedup_graph_serial": ms_plain / ms_graphs[False],
             "graph_fallback_requests_frac": gstats[True]["fallback_requests"] / max(gstats[True]["requests"], 1),
             "frame": "eye pass + global estimate + resolve, photon map resident",
             "graph": "overlapped: the render reads the cache as the previous frames trained it (a copy at the "
                      "frame's start) while the frame's 2^20-sample training runs beside it; serial: training, "
                      "then the render",
             "train_samples_per_frame": TRAIN_PER_FRAME, "train_batch": BATCH, "adam_steps_per_frame": steps_per_frame,
             "pool": pool.n, "one_time": {"pool_labelling_ms": pool_ms, "warmup_steps": WARM_STEPS,
                                          "warmup_ms": warm_ms},
             "check": dict(learned.FRAME_SETTINGS), "fallback_tiles_frac": stats["fallback_tiles"] / max(stats["tiles"], 1),
             "fallback_requests_frac": stats["fallback_requests"] / max(stats["requests"], 1),
             "mlp": {"infer_tflops": inf_tf, "train_tflops": tr_tf, "peak_bf16_tflops": peak,
                     "infer_frac": inf_tf / peak, "train_frac": tr_tf / peak, "unit": "TFLOP/s",
                     "flop_per_sample_forward": fwd, "train_samples_per_launch": min(1 << 20, pool.n)}}
    if not args.no_rmse and world == 1:
        block["rmse"] = learned_rmse(ctx, sc, cs, cam, w)
    elif not args.no_rmse:
        block["rmse"] = {"skipped": "measured on one GPU (the frames are the same on every replica)"}
    return block


def learned_rmse(ctx, sc, cs, cam, w):
    """Relative RMSE of the timed plain and learned frames against an FP64
    reference, on a seeded sample of pixels of the same 10M-photon 1080p frame.

    * eye paths: the oracle's restatement of the reference's render_trace
      walks the sampled pixels on the host (its hits are also compared with the
      GPU eye pass's requests for those pixels);
    * reference radiance: per hit, the mean over 10 independent 10M-photon maps
      (photon streams 1..10: 10x the frame's photons) of the FP64 estimate over
      the oracle's kNN selection (k, r of the frame) on the oracle's grid of
      that map; resolved per pixel in FP64;
    * frames: the plain render and the learned render (frame settings, cache
      as trained by the timed frames) of the resident map, radiance before
      tone mapping.
    relative RMSE = sqrt(mean((x - ref)^2)) / sqrt(mean(ref^2)) over the
    sampled pixels' channels."""
    import torch
    import photonmap
    import render64
    from photonmap import learned
    from oracle import Oracle
    P = LEARNED
    W, H = cs.width, cs.height
    t0 = time.perf_counter()
    _, rad_plain = ctx.render(cam, w["k"], w["radius"], w["max_depth"])
    req = {k: v.cpu().numpy() for k, v in ctx.requests().items()}
    _, rad_learned, _ = ctx.render_learned(cam, w["k"], w["radius"], w["max_depth"], **learned.FRAME_SETTINGS)
    torch.cuda.synchronize()
    pixels = np.sort(np.random.default_rng(7).choice(W * H, P["rmse_pixels"], replace=False))
    orc = Oracle()
    s = orc.scene(sc)
    hits = s.eye_hits(orc.camera(cs), W, H, pixels, w["max_depth"])
    # the oracle's eye paths against the GPU eye pass's requests of the same
    # pixels: per pixel the same number of hits, and per hit the same point,
    # triangle, normal, global-estimate flag and path weight (bit for bit)
    cnt = req["px_count"][pixels].astype(np.int64)
    same_px = cnt == hits["counts"]
    q = np.repeat(req["px_base"][pixels].astype(np.int64), cnt) + \
        (np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt))
    hb = np.concatenate([[0], np.cumsum(hits["counts"])]).astype(np.int64)
    gb_ = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    ok_px = np.zeros(pixels.size, bool)
    fl = lambda x: (x[:, 3].view(np.uint32) & 1)  # noqa: E731
    for i in np.nonzero(same_px)[0]:
        o, g0 = slice(hb[i], hb[i + 1]), slice(gb_[i], gb_[i + 1])
        ga, gbb, gc = req["a"][q[g0]], req["b"][q[g0]], req["c"][q[g0]]
        ok_px[i] = (np.array_equal(ga, hits["a"][o]) and np.array_equal(gbb[:, :3], hits["b"][o, :3]) and
                    np.array_equal(fl(gbb), fl(hits["b"][o])) and np.array_equal(gc[:, :3], hits["c"][o, :3]))
    hits_equal = bool(ok_px.all())
    tables = render64.scene_tables(sc)
    g_mask = (hits["b"][:, 3].view(np.uint32) & 1) != 0
    qp, qn = hits["a"][g_mask, :3], hits["b"][g_mask, :3]
    maps = []
    for m in range(1, P["rmse_maps"] + 1):
        ctx.trace_photons(step_seed(w["seed"], 0, 1_000_000 + m), w["max_bounces"], w["photons"])
        ph = ctx.photons(0, sorted_=False)
        maps.append(tuple(ph[k].cpu().numpy() for k in ("list_pos", "list_dir", "list_power")))

    def fp64_estimate(mp):   # the oracle's calls release the GIL: maps in parallel host threads
        pos, dr, pw = mp
        g = orc.grid_build(pos, pw, dr, s.aabb())
        ids, c, _, _ = orc.gather(g, qp, qn, w["radius"], w["k"])
        return render64.estimate_ids(pos, dr, pw, qp, qn, ids, c)

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(maps), max(1, (os.cpu_count() or 2) // 2))) as ex:
        est = sum(ex.map(fp64_estimate, maps)) / len(maps)
    full = np.zeros((hits["a"].shape[0], 3))
    full[g_mask] = est
    ref = render64.resolve_hits(hits, tables, lambda idx: full[idx])
    rel = lambda x: float(np.sqrt(np.mean((x - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))  # noqa: E731
    plain = rad_plain.cpu().numpy().reshape(-1, 3)[pixels]
    learn = rad_learned.cpu().numpy().reshape(-1, 3)[pixels]
    return {"rmse_plain": rel(plain), "rmse_learned": rel(learn), "pixels": int(pixels.size),
            "reference": f"FP64 estimates over the oracle's kNN of {P['rmse_maps']} independent "
                         f"{w['photons'] // 1_000_000}M-photon maps ({P['rmse_maps']}x the frame's photons), "
                         f"eye paths walked by the oracle",
            "oracle_eye_hits": int(hits["a"].shape[0]), "oracle_eye_hits_equal_gpu_requests": hits_equal,
            "pixels_same_hit_count": float(same_px.mean()), "pixels_hits_bit_equal": float(ok_px.mean()),
            "seconds": time.perf_counter() - t0}


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# default workload's two large kernels: constants from one ncu capture of the
# timed step's launches (the line names the capture in "traffic_source")
DRAM_TRAFFIC = {"k_trace": 149_363_200 + 429_206_272, "k_gather": 333_646_592 + 13_331_456}
TRAFFIC_SOURCE = ("constant from one ncu capture of the default workload (the timed step's launches): ncu --metrics "
                  "gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum --clock-control none "
                  "-c 400 python bench.py --steps 1 --warmup 1 --no-cpu-baseline --no-learned --no-batched")
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # 148 SMs x 128 FP32 lanes x 2 flop (FMA) x 1965 MHz
FLOP_PER_BOX_TEST = 20      # one child-box slab test (6 FMA, 6 min/max, 4 min/max and compares)
FLOP_PER_TRI_TEST = 86      # the reference's count for its triangle test (CudaPhotonMapping/Model.cuh:65-67)
PHOTON_RECORD_BYTES = 28    # position f32x3 + power f32x3 + octahedral direction u16x2 (a photon's answer bytes)


def rooflines(w, sc, bvh, nreq, paths, k_trace_ms, k_gather_ms, work, hbm, src, default_workload):
    """Rooflines of the step's two large kernels, each timed alone with CUDA
    events on the context stream (k_trace summed over the photon pass's batches).

    k_trace: FP32 flops of its traversal work, counted by the tracer's
    work-counting launch (pm_trace_work, the same photons): 2 child-box tests
    x 20 flop per BVH node visited + 86 flop per triangle test, against the
    nominal FP32 peak (MEASURED_PEAKS.json holds no FP32 figure); rays / s
    beside it.  Its HBM view: the 32-byte stage record per stored photon, 8 B
    per-path counts and the scene once, against the measured copy bandwidth.
    k_gather: per kNN query k photons x 28 B (position and power f32x3, an
    octahedral u16x2 direction) + 12 B hit point + 12 B radiance out, against
    the measured copy bandwidth.
    """
    paths_w, rays, nodes, tris = work
    flop = 2 * FLOP_PER_BOX_TEST * nodes + FLOP_PER_TRI_TEST * tris
    scene_bytes = bvh["nodes"] * 64 + sc.ntri * (80 + 36)
    trace_bytes = w["photons"] * 32 + paths * 8 + scene_bytes
    out = {}
    tf = flop / (k_trace_ms * 1e-3) / 1e12 if k_trace_ms > 0 else 0.0
    out["k_trace"] = {
        "bound": "fp32", "achieved": tf, "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": tf / FP32_PEAK_TFLOPS,
        "peak_source": "nominal (148 SMs x 128 FP32 lanes x 2 flop x 1965 MHz); no measured FP32 peak",
        "traffic": DRAM_TRAFFIC["k_trace"] if default_workload else None,
        "traffic_source": TRAFFIC_SOURCE if default_workload else None,
        "flop_per_launch": int(flop), "ms_per_launch": k_trace_ms,
        "work": {"rays": rays, "bvh_node_visits": nodes, "box_tests": 2 * nodes, "triangle_tests": tris,
                 "flop_per_box_test": FLOP_PER_BOX_TEST, "flop_per_triangle_test": FLOP_PER_TRI_TEST,
                 "paths": paths_w},
        "mrays_per_s": rays / (k_trace_ms * 1e-3) / 1e6 if k_trace_ms > 0 else 0.0,
        "hbm_view": {"algorithmic_bytes_per_launch": int(trace_bytes),
                     "achieved_gbs": trace_bytes / (k_trace_ms * 1e-3) / 1e9 if k_trace_ms > 0 else 0.0,
                     "peak_gbs": hbm, "peak_source": src},
        "note": "BVH traversal: latency / issue bound", "paths_per_launch": paths,
        "photons_per_launch": w["photons"]}
    g_bytes = nreq * (w["k"] * PHOTON_RECORD_BYTES + 24)
    gb = g_bytes / (k_gather_ms * 1e-3) / 1e9 if k_gather_ms > 0 else 0.0
    out["k_gather"] = {
        "bound": "hbm", "achieved": gb, "peak": hbm, "unit": "GB/s", "frac": gb / hbm, "peak_source": src,
        "traffic": DRAM_TRAFFIC["k_gather"] if default_workload else None,
        "traffic_source": TRAFFIC_SOURCE if default_workload else None,
        "algorithmic_bytes_per_launch": int(g_bytes), "bytes_per_query": w["k"] * PHOTON_RECORD_BYTES + 24,
        "ms_per_launch": k_gather_ms, "note": "kNN walk: issue / L1-L2 latency bound", "queries_per_launch": nreq}
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    import photonmap
    from photonmap import scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    sc, cs, w = scenes.workload(args.workload)
    w, cs = override(w, cs, args)
    # the context launches on this stream, and the timing events below are
    # recorded on it (it is the thread's current torch stream from here on)
    ctx_st = torch.cuda.Stream()
    torch.cuda.set_stream(ctx_st)
    ctx = photonmap.Context(local, stream=ctx_st)
    ctx.set_bvh_builder(args.bvh)
    ctx.set_scene(sc)
    bvh = ctx.bvh_info()
    cam = photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, cs.width, cs.height)
    W, H = cs.width, cs.height
    rgb = torch.empty(W * H * 3, dtype=torch.uint8, device="cuda")
    # end to end: two frame buffers, each frame read back to pinned host memory
    # on a copy stream while the next frame (into the other buffer) runs
    rgbs = [rgb, torch.empty_like(rgb)]
    hosts = [torch.empty(W * H * 3, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
    copy_st = torch.cuda.Stream()
    copied = [None, None]

    paths = [0]

    def step(i, e2e=False):
        # pm_frame: photon pass, grid build and frame in one call (the eye pass
        # runs beside the photon pass); same photons and image as
        # trace_photons + build_grid + render
        b = i % 2 if e2e else 0
        if e2e and copied[b] is not None:
            copied[b].synchronize()   # the read-back of this buffer's previous frame has ended
        _, _, paths[0] = ctx.frame(step_seed(w["seed"], rank, i), w["max_bounces"], w["photons"], cam, w["k"],
                                   w["radius"], w["max_depth"], radiance=False, out_rgb8=rgbs[b])
        if e2e:
            copy_st.wait_stream(ctx_st)
            with torch.cuda.stream(copy_st):
                hosts[b].copy_(rgbs[b], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(copy_st)
            copied[b] = ev

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    stage_sum = np.zeros(7)
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ctx.launch_count()
    ev0.record()
    for i in range(args.steps):
        step(args.warmup + i)
        st = ctx.stage_times()
        stage_sum += np.array([st["trace_ms"], st["grid_ms"], st["eye_ms"], st["gather_ms"], st["resolve_ms"],
                               st["k_trace_ms"], st["k_gather_ms"]])
    paths_timed = paths[0]
    ev1.record()
    torch.cuda.synchronize()
    launches = ctx.launch_count() - launches0
    barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    # end to end through the public API with the frame read back to pinned host memory
    # (one untimed step first: new seeds, so the photon pass re-sizes its batches)
    step(9_999, e2e=True)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        step(10_000 + i, e2e=True)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1000 / args.steps
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], world)
    stages = stage_sum / args.steps
    # the tracer's work on one step's photon pass (untimed counting launch, same photons as a timed step)
    work = ctx.trace_work(step_seed(w["seed"], rank, args.warmup), w["max_bounces"], w["photons"])
    ctx.build_grid(photonmap.PM_MAP_GLOBAL)   # the resident map of the learned-frame comparison

    learned_block = None
    if not args.no_learned:
        learned_block = learned_frames(ctx, sc, cs, cam, w, rgb, args, world)
    batched_block = None
    if not args.no_batched:
        batched_block = batched_frames(args, rank)
    ph = ctx.photons(0, sorted_=False)  # noqa: F841  (map still resident)
    hbm, src = peaks()
    line = None
    if rank == 0:
        nreq = ctx.render_requests()   # kNN queries of the frame's gather
        kernels = rooflines(w, sc, bvh, nreq, paths_timed, stages[5], stages[6], work, hbm, src,
                            default_workload=(args.workload == WORKLOAD and not (args.photons or args.width
                                                                                  or args.height)))
        dominant = max(kernels, key=lambda k: kernels[k]["ms_per_launch"])
        cpu = None
        if not args.no_cpu_baseline:
            est = cpu_reference_estimate(sc, w)
            cpu = {"value": w["photons"] / est["step_s"] / 1e6, "unit": "Mphotons/s", "cores": est["cores"],
                   "kind": "reference", "sample": est["sample"],
                   "ms_per_frame": est["step_s"] * 1000, "stages_s": {k: est[k] for k in ("trace_s", "grid_s", "frame_s")}}
        line = {
            "metric": METRIC, "value": job_mphotons(world, w["photons"], ms), "unit": "Mphotons/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene, seeded Philox photon streams)",
            "config": {"workload": args.workload, "photons": w["photons"], "max_bounces": w["max_bounces"],
                       "image": f"{W}x{H}", "k": w["k"], "radius": w["radius"], "eye_depth": w["max_depth"],
                       "triangles": sc.ntri, "bvh": bvh, "api": "pm_frame (photon pass + grid + frame)",
                       "l2": f"inputs larger than L2 (grid records of the photon map "
                             f"~{w['photons'] * 40 / 1e9:.1f} GB)",
                       "parallelism": f"replicas{world}"},
            "stages_ms": {"trace": stages[0], "grid": stages[1], "eye": stages[2], "gather": stages[3],
                          "resolve": stages[4]},
            "roofline": dict(kernel=dominant, **kernels[dominant]),
            "roofline_kernels": kernels,
            "e2e": {"value": job_mphotons(world, w["photons"], e2e_ms), "unit": "Mphotons/s",
                    "ms_per_step": e2e_ms, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": W * H * 3},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "learned": learned_block,
            "batched": batched_block,
        }
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return line


def run_reference(args):
    """The reference arm: the reference's CPU path (cpu_reference_estimate) on
    a bounded sample per step; ms_per_step is the sample step's own wall
    time, value the workload's Mphotons/s scaled from it."""
    from photonmap import scenes
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    sc, cs, w = scenes.workload(args.workload)
    ests = []
    for i in range(args.warmup + args.steps):
        est = cpu_reference_estimate(sc, w)
        if i >= args.warmup:
            ests.append(est)
    step_s = float(np.mean([e["step_s"] for e in ests]))
    wall_ms = float(np.mean([e["wall_s"] for e in ests])) * 1000
    v = w["photons"] / step_s / 1e6
    return {"metric": METRIC, "value": v, "unit": "Mphotons/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "ms_per_frame_estimated": step_s * 1000,
            "config": {"workload": args.workload, "photons": w["photons"], "max_bounces": w["max_bounces"],
                       "image": f"{w['width']}x{w['height']}", "k": w["k"], "radius": w["radius"],
                       "eye_depth": w["max_depth"], "triangles": sc.ntri, "parallelism": "replicas1",
                       "api": "the reference's CPU mode (render_cpu) + the oracle's CPU photon pass and grid",
                       "step": "one bounded sample (cpu_baseline.sample) scaled to the workload; ms_per_step is "
                               "the sample's wall time, ms_per_frame_estimated the scaled full frame"},
            "cpu_baseline": {"value": v, "unit": "Mphotons/s", "cores": ests[-1]["cores"], "kind": "reference",
                             "sample": ests[-1]["sample"]},
            "e2e": {"value": v, "unit": "Mphotons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    line = run_reference(args) if args.impl == "reference" else run_ours(args)
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
