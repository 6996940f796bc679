"""Multi-rank frame rendering host logic on CPU (gloo, world size 2): sample
sharding and the accumulator merge, against one sequential Welford
accumulation (main.rs:603-643) of all samples."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from rustracer_b200.multigpu import merge_accumulators, shard


def test_shard_covers_every_sample_once():
    for total in (1, 7, 64, 257):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                s, n = shard(total, world, r)
                got.extend(range(s, s + n))
            assert got == list(range(total))


def welford(samples):
    """Sequential accumulate_sample without clamping: samples (N, P, 3)."""
    mean = np.zeros(samples.shape[1:], np.float64)
    m2 = np.zeros_like(mean)
    s = np.zeros_like(mean)
    for k, x in enumerate(samples.astype(np.float64), 1):
        s += x
        d = x - mean
        mean += d / k
        m2 += d * (x - mean)
    return s, m2, len(samples)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, samples, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        start, n = shard(len(samples), world, rank)
        s, m2, c = welford(samples[start:start + n])
        npix = samples.shape[1]
        ms, mm, mc = merge_accumulators(torch.tensor(s, dtype=torch.float32).reshape(1, npix, 3),
                                        torch.tensor(m2, dtype=torch.float32).reshape(1, npix, 3),
                                        torch.full((1, npix), c, dtype=torch.int32))
        out[rank] = (ms.numpy(), mm.numpy(), mc.numpy())
    finally:
        dist.destroy_process_group()


def test_merge_matches_sequential_welford():
    rng = np.random.default_rng(0)
    samples = rng.gamma(2.0, 1.5, size=(37, 50, 3)).astype(np.float32)
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, samples, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    s, m2, n = welford(samples)
    for r in range(2):
        ms, mm, mc = out[r]
        np.testing.assert_allclose(ms[0], s, rtol=1e-5)
        np.testing.assert_allclose(mm[0], m2, rtol=1e-4, atol=1e-4)
        assert (mc[0] == n).all()


class _GuideStandIn:
    """The two guide calls broadcast_guide makes, on host arrays."""

    def __init__(self, params):
        self.params = params

    def guide_get_params(self):
        return self.params.copy()

    def guide_set_params(self, p):
        self.params = np.array(p, np.float32)


def _guide_worker(rank, world, port, out):
    import torch.distributed as dist
    from rustracer_b200 import abi
    from rustracer_b200.multigpu import broadcast_guide
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(rank)
        g = _GuideStandIn(rng.standard_normal(abi.RT_GUIDE_PARAMS).astype(np.float32))
        n = broadcast_guide(g, src=0)
        out[rank] = (n, float(g.params[:1000].sum()), float(g.params[-1000:].sum()))
    finally:
        dist.destroy_process_group()


def test_broadcast_guide_shares_rank0_parameters():
    """The trained guide of rank 0 reaches every rank unchanged (gloo, 2 ranks)."""
    from rustracer_b200 import abi
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_guide_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    ref = np.random.default_rng(0).standard_normal(abi.RT_GUIDE_PARAMS).astype(np.float32)
    for r in range(2):
        n, a, b = out[r]
        assert n == abi.RT_GUIDE_PARAMS
        assert a == float(ref[:1000].sum()) and b == float(ref[-1000:].sum())


def _guide_subgroup_worker(rank, world, port, out):
    import torch.distributed as dist
    from rustracer_b200 import abi
    from rustracer_b200.multigpu import broadcast_guide
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grp = dist.new_group([1, 2])            # every rank takes part in creating it
        rng = np.random.default_rng(rank)
        g = _GuideStandIn(rng.standard_normal(abi.RT_GUIDE_PARAMS).astype(np.float32))
        if rank in (1, 2):
            broadcast_guide(g, src=2, group=grp)
        out[rank] = float(g.params[:1000].sum())
    finally:
        dist.destroy_process_group()


def test_broadcast_guide_in_a_subgroup_uses_the_global_source_rank():
    """In the subgroup {1, 2} the source is global rank 2: rank 1 receives
    rank 2's parameters and rank 0 keeps its own (gloo, 3 ranks)."""
    from rustracer_b200 import abi
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_guide_subgroup_worker, args=(r, 3, port, out)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    own = [float(np.random.default_rng(r).standard_normal(abi.RT_GUIDE_PARAMS).astype(np.float32)[:1000].sum())
           for r in range(3)]
    assert out[0] == own[0]
    assert out[1] == own[2] and out[2] == own[2]


def _photon_worker(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as O
    from rustracer_b200 import configs
    from rustracer_b200.multigpu import build_photon_map
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sb, st = configs.gem_scene(width=32, height=18, env_w=64, env_h=32)
        o = O.OracleScene(sb)                     # the CPU restatement stands in for a GPU scene
        n = build_photon_map(o, st["photon_params"](5, 60000))
        out[rank] = (n,) + tuple(o.photon_export())
    finally:
        dist.destroy_process_group()


def test_sharded_photon_map_equals_the_single_rank_map():
    """Two ranks each trace half of the emission order and exchange what they
    stored (gloo): both end with exactly the map of one unsharded build —
    the same photons, powers, normals and emission indices."""
    from oracle import oracle as O
    from rustracer_b200 import configs
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_photon_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    sb, st = configs.gem_scene(width=32, height=18, env_w=64, env_h=32)
    o = O.OracleScene(sb)
    n = o.photon_build(st["photon_params"](5, 60000))
    ref = o.photon_export()
    assert n > 1000
    for r in range(2):
        got = out[r]
        assert got[0] == n
        for a, b in zip(got[1:], ref):
            assert np.array_equal(a, b)
