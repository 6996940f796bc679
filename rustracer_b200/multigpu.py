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
    """Copy rank `src`'s guide parameters into every rank's guide (each rank's
    scene must have called guide_init).  The broadcast is one float32 tensor
    of RT_GUIDE_PARAMS values; the receiving guides' Adam state is reset,
    as rt_guide_params does on a write."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
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
