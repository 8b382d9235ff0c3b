"""Host-side parts of batched indexing and the synthetic phases (no GPU)."""

import json

import torch


def test_launch_tuner_picks_fastest_and_caches(tmp_path):
    from ebsdtorch_b200.batch import LAUNCH_SHAPES, LaunchTuner

    calls = []
    cost = {i: 5.0 - 0.5 * i for i in range(len(LAUNCH_SHAPES))}

    def time_shape(shape):
        i = [dict(s) for s in LAUNCH_SHAPES].index(shape)
        calls.append(i)
        return cost[i]

    path = tmp_path / "tune.json"
    t = LaunchTuner(cache_file=str(path), repeats=2)
    key = LaunchTuner.key(16384, 328720, "bf16", 32, True, 148)
    best = t.pick(key, time_shape)
    assert best == dict(LAUNCH_SHAPES[-1])
    assert len(calls) == 3 * len(LAUNCH_SHAPES)  # warm-up + 2 repeats each
    assert t.pick(key, time_shape) == best and len(calls) == 3 * len(LAUNCH_SHAPES)
    saved = json.loads(path.read_text())
    assert saved[key]["shape"] == best
    t2 = LaunchTuner(cache_file=str(path))

    def never(shape):
        raise AssertionError("re-timed a cached shape")

    assert t2.pick(key, never) == best
    assert LaunchTuner.key(3600, 36829, "fp8", 32, False, 148) != key


def test_synthetic_master_pattern_bands_are_closed_under_the_laue_group():
    """Every band normal of a non-cubic synthetic phase maps to a band normal
    (up to sign) under each rotation of its Laue group, so the pattern has
    the group's symmetry and FZ dictionaries index it correctly."""
    from ebsdtorch_b200 import synthetic

    for laue, order in ((5, 8), (9, 12), (7, 6), (3, 4)):
        rots = synthetic.laue_rotations(laue)
        assert rots.shape[0] == order
        g = torch.Generator().manual_seed(0)
        nv = torch.randn(3, generator=g, dtype=torch.float64)
        nv = nv / nv.norm()
        orbit = [synthetic._qrot(q, nv) for q in rots]
        for q in rots:
            for o in orbit:
                m = synthetic._qrot(q, o)
                assert max(abs(float(m @ x)) for x in orbit) > 1 - 1e-9
    img = synthetic.synthetic_master_pattern(33, seed=4, laue_group=9)
    assert img.shape == (33, 66) and torch.isfinite(img).all()


def test_planner_caps_query_chunks_for_streamed_patterns():
    """With a budget that fits everything, the planner takes all queries in one
    chunk. With max_query_chunk (set for patterns streamed from pinned host
    memory), the chunks are capped so that each chunk's copy can run under the
    previous chunk's match, while the dictionary stays in one chunk."""
    from ebsdtorch_b200.engine import Searcher, SearchConfig

    one = Searcher(328720, 262144, 16384, 8, SearchConfig(workspace_bytes=150 << 30), "cpu")
    assert one.query_chunk == 262144 and one.dict_chunk >= 328720
    capped = Searcher(328720, 262144, 16384, 8, SearchConfig(workspace_bytes=150 << 30, max_query_chunk=18944), "cpu")
    assert capped.query_chunk == 18944 and capped.dict_chunk == one.dict_chunk
    small = Searcher(328720, 5000, 16384, 8, SearchConfig(workspace_bytes=150 << 30, max_query_chunk=18944), "cpu")
    assert small.query_chunk == 5120  # the whole (padded) map when it is smaller than the cap


def test_match_traffic_model_reproduces_its_captures():
    import bench

    for rows, dram in bench.MATCH_DRAM_BYTES:
        assert abs(bench.match_traffic_estimate(rows) - dram) < 1.0
    # the 18-query-tile launches read each dictionary row about twice
    operands = (328960 + bench.MATCH_WAVE_QUERIES) * 16384 * 2
    assert 1.5 * operands < bench.match_traffic_estimate(328720) < 2.5 * operands


def test_wave_shape_rule():
    """One-wave query-tile counts on a 148-SM, 126 MB-L2 device: bf16 rows of
    128^2 px (32 KB) take 18 tiles, e4m3 rows (16 KB) 37, or 36 when the
    launch takes query tiles two at a time; unknown row sizes take 18."""
    from ebsdtorch_b200.engine import even_tiles, wave_tiles_for

    l2 = 126 << 20
    assert wave_tiles_for(148, l2, 32768) == 18
    assert wave_tiles_for(148, l2, 16384) == 37
    assert wave_tiles_for(148, l2, 16384, tile_pairs=True) == 36
    assert wave_tiles_for(148, l2, 32768, tile_pairs=True) == 18
    assert wave_tiles_for(148, l2) == 18
    assert even_tiles(1, True) == 1 and even_tiles(7, False) == 7 and even_tiles(7, True) == 6
