"""Tuning of the fused RC pass: every valid tuning (class bounds, tile
shapes, the block/global-workspace boundary) gives the same outputs bit for
bit; the autotuner returns and applies a valid tuning; invalid tunings are
refused."""
import numpy as np
import pytest

import opentimer_b200 as otg
from opentimer_b200 import _lib

pytestmark = pytest.mark.gpu
OUT = ["node2bfs", "pid", "edges", "load", "delay", "ldelay", "impulse", "sink_slew"]
SHAPES = [(64, 4), (64, 8), (128, 4), (128, 8), (256, 2), (256, 4), (256, 8), (512, 2),
          (512, 4), (512, 8), (1024, 2), (1024, 4)]


@pytest.fixture
def restore_tuning():
    yield
    otg.set_tuning(None)


def forest(cuda, seed=31):
    import torch
    rng = np.random.default_rng(seed)
    sizes = np.concatenate([rng.integers(2, 33, 80), rng.integers(33, 300, 200),
                            rng.integers(300, 1500, 60), rng.integers(1500, 4800, 25),
                            [5200, 7000]])
    ns = np.zeros(len(sizes) + 1, np.int32)
    ns[1:] = np.cumsum(sizes)
    return otg.synth_forest(seed, torch.from_numpy(ns).to(cuda))


def run(g):
    import torch
    b = otg.RcBatch(g["nodes_start"], g["edges"].clone(), g["roots"], g["res"], g["cap"],
                    sinks_start=g["sinks_start"], sink_nodes=g["sink_nodes"],
                    driver_slew=g["driver_slew"])
    b.run()
    b.check()
    torch.cuda.synchronize()
    return b, {k: getattr(b, k).cpu().numpy() for k in OUT}


def random_tuning(rng, hi):
    """A random valid table; hi: the largest net the block path holds in
    shared memory (the default table's last bound)."""
    k = int(rng.integers(1, 7))
    bounds = np.sort(rng.choice(np.arange(40, hi + 1), k, replace=False))
    shapes = [SHAPES[int(i)] for i in rng.integers(0, len(SHAPES), k)]
    return {"class_max": [int(x) for x in bounds], "class_threads": [s[0] for s in shapes],
            "class_items": [s[1] for s in shapes]}


def test_every_tuning_gives_identical_outputs(cuda, restore_tuning):
    g = forest(cuda)
    otg.set_tuning(None)
    hi = otg.get_tuning()["class_max"][-1]
    _, ref = run(g)
    rng = np.random.default_rng(8)
    for _ in range(6):
        t = random_tuning(rng, hi)
        otg.set_tuning(t)
        assert otg.get_tuning() == t
        _, got = run(g)
        for k in OUT:
            assert np.array_equal(got[k], ref[k]), (k, t)


def test_autotune_applies_a_valid_tuning(cuda, restore_tuning):
    g = forest(cuda, seed=5)
    otg.set_tuning(None)
    b, ref = run(g)
    t = otg.autotune(b)
    assert otg.get_tuning() == t
    assert 1 <= len(t["class_max"]) <= 6
    assert t["class_max"] == sorted(t["class_max"]) and t["class_max"][0] > 32
    _, got = run(g)
    for k in OUT:
        assert np.array_equal(got[k], ref[k]), k


def test_invalid_tunings_are_refused(cuda, restore_tuning):
    before = otg.get_tuning()
    bad = [
        {"class_max": [100, 90], "class_threads": [64, 64], "class_items": [4, 4]},
        {"class_max": [100], "class_threads": [96], "class_items": [4]},
        {"class_max": [30], "class_threads": [64], "class_items": [4]},
        {"class_max": [9000], "class_threads": [256], "class_items": [4]},
    ]
    for t in bad:
        with pytest.raises(_lib.OtgError) as e:
            otg.set_tuning(t)
        assert e.value.code == 1
        assert otg.get_tuning() == before
