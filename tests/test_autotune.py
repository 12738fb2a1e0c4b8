"""The batch autotuner's search on a synthetic cost surface (no GPU)."""
from nebula_b200 import autotune


def test_coordinate_descent_finds_separable_minimum():
    calls = []

    def cost(cap, blk, thr, cells):
        calls.append((cap, blk, thr, cells))
        return (1.0 + abs(cap.bit_length() - 23) * 10 + abs(blk - 512) / 128 + abs(thr - 0.3) * 5
                + abs(cells - 2) * 3)

    best, table = autotune.tune_batch(None, None, [(0, 1, [0] * 10)], timer=cost)
    assert (best["capacity"], best["block"], best["threshold"], best["walk_cells"]) == (1 << 22, 512, 0.3, 2)
    # every point timed once (cache), within the documented ranges
    assert len(calls) == len(set(calls)) == len(table)
    assert all((1 << 18) <= c <= (1 << 24) and b in (128, 256, 512) and 0.1 <= t <= 1.0 and w in (1, 2, 4)
               for c, b, t, w in calls)


def test_sample_keeps_every_job():
    jobs = [(0, 1, list(range(1000))), (1, 2, list(range(7)))]
    s = autotune.sample_jobs(jobs, 0.1)
    assert [len(p) for _, _, p in s] == [100, 1]
    assert [(g, k) for g, k, _ in s] == [(0, 1), (1, 2)]
