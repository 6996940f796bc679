"""The launch autotuner's selection logic without a GPU: every candidate is
timed, the fastest is set on the scene and cached, and the probe render stays
within its sample budget."""
from rustracer_b200 import autotune
from rustracer_b200.renderer import pass_params


class FakeScene:
    def __init__(self):
        self.set = []

    def set_tuning(self, **t):
        self.set.append(t)


def test_candidates_cover_the_space():
    c = autotune.candidates({"max_paths": (1, 2), "trace_blocks_per_sm": (3,), "shade_blocks_per_sm": (4, 5, 6)})
    assert len(c) == 6
    assert {(t["max_paths"], t["shade_blocks_per_sm"]) for t in c} == {(a, b) for a in (1, 2) for b in (4, 5, 6)}


def test_autotune_picks_the_fastest_and_caches_it():
    autotune.clear_cache()
    g = FakeScene()
    calls = []

    def timer(t):
        calls.append(t)
        # fastest at 4M paths, 6 traversal blocks, 8 shading blocks, full nodes
        return abs(t["max_paths"] - (1 << 22)) / 1e6 + abs(t["trace_blocks_per_sm"] - 6) + \
            abs(t["shade_blocks_per_sm"] - 8) + t["node_format"] + 1.0
    best, table = autotune.autotune(g, None, pass_params(64, 64), key="k", timer=timer, repeats=2)
    assert best == {"max_paths": 1 << 22, "trace_blocks_per_sm": 6, "shade_blocks_per_sm": 8, "node_format": 0}
    assert len(table) == len(autotune.candidates()) and len(calls) == 2 * len(table)
    assert g.set[-1] == best
    g2 = FakeScene()
    best2, table2 = autotune.autotune(g2, None, pass_params(64, 64), key="k", timer=lambda t: 1 / 0)
    assert best2 == best and table2 is None and g2.set == [best]


def test_probe_stays_within_its_budget():
    p = autotune.probe_params(pass_params(1920, 1080, 0, 256))
    assert p.n_samples == 9 and p.width == 1920 and 1920 * 1080 * (p.n_samples - 1) < autotune.PROBE_SAMPLES
    assert autotune.probe_params(pass_params(128, 128, 0, 4)).n_samples == 4


def test_autotune_skips_layouts_the_scene_lacks():
    """A scene whose tree was built on the host has no 4-wide nodes:
    rt_set_tuning refuses RT_NODES_WIDE4 and the tuner passes those
    candidates over instead of failing."""
    from rustracer_b200 import abi
    from rustracer_b200.renderer import RtError

    autotune.clear_cache()
    g = FakeScene()

    def timer(t):
        if t["node_format"] == abi.RT_NODES_WIDE4:
            raise RtError(1, "4-wide nodes exist for trees built on the device only")
        g.set_tuning(**t)
        return 10.0 - t["node_format"] - t["shade_blocks_per_sm"] / 100.0
    best, table = autotune.autotune(g, None, pass_params(64, 64), timer=timer, repeats=1)
    assert best["node_format"] == abi.RT_NODES_QUANTISED and best["shade_blocks_per_sm"] == 16
    assert all(t["node_format"] != abi.RT_NODES_WIDE4 for _, t in table)
    assert len(table) == len(autotune.candidates()) * 2 // 3
