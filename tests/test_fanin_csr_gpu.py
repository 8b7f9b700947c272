"""Device build of the levelization input (otg_fanin_csr, the GPU form of
Timer::_build_prop_tasks_cuda steps 1-2, ot/timer/timer.cpp:996-1061)
against the same construction on the host: per pin its counted fanin arcs
in arc order (source pins, or arc indices), fanout counts, and the
candidates without fanout in candidate order.  Arcs count when they are
not loop breakers and both pins are candidates.  Exact equality."""
import numpy as np
import pytest

import opentimer_b200 as otg

pytestmark = pytest.mark.gpu


def host_csr(n, frm, to, skip, cand, cand_order, as_arcs):
    keep = ~skip & cand[frm] & cand[to]
    arcs = np.nonzero(keep)[0]
    order = arcs[np.argsort(to[arcs], kind="stable")]
    start = np.zeros(n + 1, np.int64)
    start[1:] = np.cumsum(np.bincount(to[arcs], minlength=n))
    out_deg = np.bincount(frm[arcs], minlength=n)
    fanin = order if as_arcs else frm[order]
    front = np.array([c for c in cand_order if out_deg[c] == 0], np.int64)
    return start, fanin, out_deg, front


@pytest.mark.parametrize("seed,n,A,as_arcs", [(1, 1, 0, False), (2, 50, 300, False),
                                              (3, 20000, 90000, True), (4, 300000, 1200000, False)])
def test_device_csr_matches_host(cuda, seed, n, A, as_arcs):
    import torch
    rng = np.random.default_rng(seed)
    frm = rng.integers(0, n, A)
    to = rng.integers(0, n, A)
    # a few hubs with long fanin lists
    if A > 100:
        to[rng.integers(0, A, A // 50)] = rng.integers(0, 4, A // 50)
    skip = rng.random(A) < 0.05
    cand = rng.random(n) < 0.9
    cand_order = rng.permutation(np.nonzero(cand)[0])
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).to(cuda)  # noqa: E731
    got = otg.fanin_csr(n, t(frm, np.int32), t(to, np.int32), t(skip, np.uint8),
                        t(cand, np.uint8), t(cand_order, np.int32), as_arcs=as_arcs)
    want = host_csr(n, frm, to, skip, cand, cand_order, as_arcs)
    for g, w in zip(got, want):
        assert np.array_equal(g.cpu().numpy().astype(np.int64), w)


def test_device_csr_levelizes_like_the_host_input(cuda):
    """Fed to otg_levelize, the device-built input gives the levels of the
    host-built one (a seeded 200-level pin DAG)."""
    import torch
    import rcgen
    fs, fi, od, f0 = rcgen.pin_dag(5, 20000, 50000, 200)
    n = len(od)
    to = np.repeat(np.arange(n), np.diff(fs))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.int32)).to(cuda)  # noqa: E731
    start, fanin, out_deg, front = otg.fanin_csr(n, t(fi), t(to))
    order_d, ends_d, _ = otg.levelize(start, fanin, out_deg, front)
    order_h, ends_h, _ = otg.levelize(t(fs), t(fi), t(od), t(f0))
    assert np.array_equal(ends_d, ends_h) and np.array_equal(order_d, order_h)
