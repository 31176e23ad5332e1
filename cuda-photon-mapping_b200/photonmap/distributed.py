"""One frame split over ranks (one process per GPU, torch.distributed).

The reference renders on one GPU (CudaPhotonMapping/kernel.cu).  Its photon
paths are independent and its gather needs the whole photon map, so a frame
splits into:

  1. photon pass: rank r of W traces the paths [base + r C, base + (r + 1) C)
     of each round (pm_trace_paths: per-path photon counts and records, every
     path on its own random stream); the ranks' per-round photon counts are
     all-gathered, and rounds go on until the maps hold their capacities;
  2. exchange: the photon records of every rank are all-gathered, rank order
     within a round and round order being path order, and cut at the
     capacities: every rank then holds exactly the lists of the one-GPU photon
     pass (canonical order: path, then bounce);
  3. grid: every rank builds the full grid of the global map (and of the
     caustic map when it has one);
  4. frame: rank r renders the pixel rows of its band (pm_render_rows) and the
     bands are gathered into the frame.

Nothing but the photon records and the bands crosses ranks.  Photon power is
intensity / global capacity for every photon, as in the one-GPU pass.

The engine is the per-rank renderer with the methods below (photonmap.Context
on a GPU); the exchanges go through the process group's backend (NCCL with
CUDA tensors; gloo with host tensors).

    trace_paths(seed, max_bounces, power_capacity, p0, p1, tag=0)
        -> dict(counts (n, 2), g_pos, g_dir, c_pos, c_dir)
    set_photons(map_id, pos, power, direction); build_grid(map_id)
    render_rows(cam, k, r, max_depth, y0, y1, k_caustic=..., r_caustic=...) -> (rgb8, radiance)
    light_intensity: 3 floats
"""
from __future__ import annotations

import numpy as np


def band(height, rank, world):
    """Pixel rows [y0, y1) of a rank: equal shares, the first (height % world) ranks one row more."""
    q, r = divmod(height, world)
    y0 = rank * q + min(rank, r)
    return y0, y0 + q + (1 if rank < r else 0)


def _t(x, torch):
    return x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))


class SplitFrame:
    def __init__(self, engine, group=None, chunk=65536):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.engine = engine
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.chunk = int(chunk)
        self.nccl = dist.is_initialized() and dist.get_backend(group) == "nccl"

    # ------------------------------------------------------------ exchanges
    def _dev(self, t):
        return t.cuda() if self.nccl else t.cpu()

    def _all_gather(self, t):
        """Every rank's tensor t (same dtype, any first-axis length), in rank order."""
        torch, dist = self.torch, self.dist
        if self.world == 1:
            return [t]
        t = self._dev(t.contiguous())
        n = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
        ns = [torch.empty_like(n) for _ in range(self.world)]
        dist.all_gather(ns, n, group=self.group)
        ns = [int(x.item()) for x in ns]
        m = max(ns)
        pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
        pad[:t.shape[0]] = t
        outs = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(outs, pad, group=self.group)
        return [o[:k] for o, k in zip(outs, ns)]

    # ---------------------------------------------------------- photon pass
    def trace(self, seed, max_bounces, global_capacity, caustic_capacity=0, tag=0, max_paths=None):
        """Steps 1-3: the one-GPU photon lists on every rank, grids built.
        Returns the number of paths traced (all ranks)."""
        torch = self.torch
        gcap, ccap = int(global_capacity), int(caustic_capacity)
        max_paths = max_paths or 64 * max(gcap, ccap, 1)
        lists = {"g_pos": [], "g_dir": [], "c_pos": [], "c_dir": []}
        have_g = have_c = 0
        base = 0
        C = self.chunk
        while (have_g < gcap or have_c < ccap) and base < max_paths:
            p0 = base + self.rank * C
            p1 = min(p0 + C, max_paths)
            if p1 > p0:
                out = self.engine.trace_paths(seed, max_bounces, gcap, p0, p1, tag=tag)
            else:   # past max_paths: nothing to trace this round
                z = torch.zeros((0, 3), dtype=torch.float32)
                out = {"g_pos": z, "g_dir": z, "c_pos": z, "c_dir": z}
            for key in lists:
                parts = self._all_gather(_t(out[key], torch).float().reshape(-1, 3))
                lists[key].extend(p.cpu() for p in parts)
            have_g = sum(x.shape[0] for x in lists["g_pos"])
            have_c = sum(x.shape[0] for x in lists["c_pos"])
            base += self.world * C
        if have_g < gcap or have_c < ccap:
            raise RuntimeError("split photon pass: maps not filled within max_paths")
        inten = np.asarray(self.engine.light_intensity, np.float32)
        power = inten / np.float32(gcap)   # intensity / global capacity, in float32 (PhotonTracing.cu:369)
        maps = ((0, "g", gcap), (1, "c", ccap))
        for map_id, key, cap in maps:
            if cap == 0:
                continue
            pos = torch.cat(lists[f"{key}_pos"])[:cap]
            dr = torch.cat(lists[f"{key}_dir"])[:cap]
            pw = torch.from_numpy(np.tile(power, (pos.shape[0], 1)))
            self.engine.set_photons(map_id, pos, pw, dr)
            self.engine.build_grid(map_id)
        return min(base, max_paths)

    # ---------------------------------------------------------------- frame
    def render(self, cam, k_global, r_global, max_depth=4, k_caustic=0, r_caustic=0.2, gather_to=0):
        """Step 4: this rank's band, then the frame on rank gather_to (None:
        on every rank).  Returns host tensors: (rgb8 (H * W * 3,) uint8,
        radiance (H * W, 3)) on the ranks that hold the frame, else the band's."""
        torch = self.torch
        W, H = cam.width, cam.height
        y0, y1 = band(H, self.rank, self.world)
        rgb, rad = self.engine.render_rows(cam, k_global, r_global, max_depth, y0, y1, k_caustic=k_caustic,
                                           r_caustic=r_caustic)
        rgb = _t(rgb, torch).reshape(H, W * 3)[y0:y1]
        rad = _t(rad, torch).reshape(H, W * 3)[y0:y1]
        rgbs = self._all_gather(rgb)
        rads = self._all_gather(rad)
        if gather_to is not None and self.rank != gather_to:
            return rgb.reshape(-1).cpu(), rad.reshape(-1, 3).cpu()
        return (torch.cat([x.cpu() for x in rgbs]).reshape(-1), torch.cat([x.cpu() for x in rads]).reshape(-1, 3))
