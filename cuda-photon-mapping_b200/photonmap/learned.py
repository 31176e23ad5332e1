"""Training recipe of the learned radiance cache (host-side orchestration of
the library's entry points; all data stays on the device).

  pool = training_pool(ctx, cam, k, r, n)   # stratified primary hits, labelled by the kNN gather
  cache_fit(ctx, pool, steps, batch)        # Adam steps over shuffled batches of the pool

The pool's points are sampled in image order (coherent, so the labelling
gather is fast), the misses are dropped, and the pool is then shuffled once so
that every training batch covers the whole image.
"""
from __future__ import annotations

import dataclasses

# Settings of the learned frame that is timed and quality-checked: 16x16
# tiles, 8 exact probes per tile, a tile falls back to the exact gather when
# its cache bias exceeds 5 % of the probes' estimate by more than two standard
# errors of the probe differences (so the probes' own kNN noise does not
# flag it).  render_learned(**FRAME_SETTINGS, ...).
FRAME_SETTINGS = dict(tile=16, probes=8, max_rel_err=0.05, noise_z=2.0)


@dataclasses.dataclass
class Pool:
    pos: object      # (n, 3) float32 device tensor
    nrm: object
    target: object   # (n, 3) kNN estimates
    scale: float     # mean target: the network's output unit

    @property
    def n(self):
        return int(self.pos.shape[0])


def training_pool(ctx, cam, k, radius, n=1 << 20, seed=1, map_id=0) -> Pool:
    torch = ctx.torch
    pos, nrm, wt = ctx.cache_sample_points(cam, n, seed=seed)
    keep = wt > 0
    pos, nrm = pos[keep].contiguous(), nrm[keep].contiguous()
    target, _, _ = ctx.gather(pos, nrm, k, radius, map_id=map_id)
    gen = torch.Generator(device=pos.device)
    gen.manual_seed(int(seed))
    perm = torch.randperm(pos.shape[0], device=pos.device, generator=gen)
    pos, nrm, target = pos[perm].contiguous(), nrm[perm].contiguous(), target[perm].contiguous()
    scale = float(target.mean()) if pos.shape[0] else 1.0
    return Pool(pos, nrm, target, scale if scale > 0 else 1.0)


def cache_fit(ctx, pool: Pool, steps, batch=65536, offset=0, want_loss=True):
    """Runs `steps` Adam steps over consecutive batches of the (shuffled) pool,
    starting at `offset`; returns (last loss, next offset).  want_loss=False
    queues the steps without waiting for them (loss nan)."""
    if int(steps) <= 0:
        return float("nan"), offset
    return ctx.cache_train_steps(pool.pos, pool.nrm, pool.target, int(steps), int(batch), offset,
                                 want_loss=want_loss)
