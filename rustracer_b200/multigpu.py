"""Multi-GPU rendering of one frame: one process per GPU.

Path samples are independent, so a frame's samples are split into contiguous
per-rank ranges of sample indices (no exchange while rendering), and the
ranks' device accumulators are combined once at the end (the reference's
accumulate_sample, main.rs:603-643, keeps a per-pixel running sum, M2 and
count).

The combine is exact for sums and counts and uses the pooled-variance identity
for M2 — M2 = Σ_r (M2_r + S_r²/n_r) − S²/n — evaluated in float64, which is
what Welford's update over the concatenated sample sequence gives (the firefly
clamp, which depends on the running mean, is not shard-invariant: merge only
unclamped accumulations).

The caustic photon map is built once per frame across the ranks: each rank
traces a contiguous share of the emission order (RtPhotonParams.first_photon /
shard_photons, the reference parallelises the same photon loop over its
threads, photon.rs:78,112), the ranks all-gather what they stored (position,
power, normal, emission index; ≤ 2M × 40 B), and every rank builds the same
gather structure from the union, ordered by emission index: the map one
unsharded build gives.

The learned proposal trains on one rank and is then shared: the source
rank's frozen parameters (rt_guide_params, 16.8M float32) are broadcast and
written into every other rank's guide, so all ranks sample from the same
network for the rest of the frame.
"""
import torch


def shard(total_spp, world, rank):
    """Contiguous sample range of `rank`: (first sample index offset, count)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank / world size")
    base, rem = divmod(int(total_spp), int(world))
    start = rank * base + min(rank, rem)
    return start, base + (1 if rank < rem else 0)


def merge_accumulators(acc_sum, acc_m2, acc_count, group=None):
    """All-reduce the ranks' (sum (H,W,3), M2 (H,W,3), count (H,W)) into the
    frame's; every rank gets the merged tensors (float32 sum/M2, int32 count)."""
    import torch.distributed as dist
    s = acc_sum.to(torch.float64)
    n = acc_count.to(torch.float64).unsqueeze(-1)
    pos = n > 0
    t = acc_m2.to(torch.float64) + torch.where(pos, s * s / n.clamp(min=1.0), torch.zeros_like(s))
    for x in (s, t, n):
        dist.all_reduce(x, op=dist.ReduceOp.SUM, group=group)
    pos = n > 0
    m2 = torch.where(pos, t - s * s / n.clamp(min=1.0), torch.zeros_like(s))
    return s.to(torch.float32), m2.clamp(min=0.0).to(torch.float32), n.squeeze(-1).to(torch.int32)


def broadcast_guide(scene, src=0, group=None):
    """Copy global rank `src`'s guide parameters into every rank of `group`
    (each rank's scene must have called guide_init).  The broadcast is one float32 tensor
    of RT_GUIDE_PARAMS values; the receiving guides' Adam state is reset,
    as rt_guide_params does on a write."""
    import torch.distributed as dist
    # `src` is a global rank (dist.broadcast reads it that way), so compare it
    # with this process's global rank, also inside a subgroup
    rank = dist.get_rank()
    t = torch.from_numpy(scene.guide_get_params()) if rank == src else None
    if t is None:
        from . import abi
        t = torch.empty(abi.RT_GUIDE_PARAMS, dtype=torch.float32)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.broadcast(t, src, group=group)
    if rank != src:
        scene.guide_set_params(t.cpu().numpy())
    return t.numel()


def build_photon_map(scene, params, group=None):
    """Sharded caustic photon map: every rank of `group` traces its share of
    `params`' photons, the stored photons are all-gathered and each rank's
    scene receives the whole map (rt_photon_set with emission indices).
    Returns the number of stored photons in the map.  `scene` needs
    photon_build / photon_export / photon_set (a GpuScene)."""
    import numpy as np
    import torch.distributed as dist
    from . import photons
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    scene.photon_build(photons.shard_params(params, world, rank))
    pos, power, nor, idx = scene.photon_export()
    rec = np.concatenate([pos, power, nor, idx.view(np.float32)[:, None]], 1).astype(np.float32)   # n × 10
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    n = torch.tensor([len(rec)], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    m = max(max(counts), 1)
    mine = torch.zeros((m, 10), dtype=torch.float32, device=dev)
    if len(rec):
        mine[: len(rec)] = torch.from_numpy(rec).to(dev)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    allrec = np.concatenate([p[:c].cpu().numpy() for p, c in zip(parts, counts)], 0)
    order = np.argsort(allrec[:, 9].view(np.int32), kind="stable")
    allrec = allrec[order]
    scene.photon_set(allrec[:, 0:3], allrec[:, 3:6], allrec[:, 6:9], allrec[:, 9].view(np.int32).copy(),
                     radius=params.gather_radius, knn_k=params.knn_k)
    return len(allrec)
