"""Design server (otg_server_*): incremental re-timing of dirty nets must
leave every design bit-identical to a full pass over its updated inputs,
whatever the batching; admission refuses designs beyond the budget."""
import numpy as np
import pytest

import opentimer_b200 as otg
from opentimer_b200 import _lib
from opentimer_b200.serve import TimingServer, synth_design

pytestmark = pytest.mark.gpu
Q = ["node2bfs", "load", "delay", "ldelay", "impulse", "sink_slew"]


def design(seed, n_nets, lo=2, hi=512, big=()):
    ns = otg.net_sizes(seed, n_nets, lo, hi)
    if big:
        sizes = np.concatenate([np.diff(ns), np.array(big, np.int64)])
        ns = np.zeros(len(sizes) + 1, np.int32)
        ns[1:] = np.cumsum(sizes)
    return synth_design(seed, ns)


def full_pass(d):
    c = {k: v.copy() for k, v in d.items()}
    return otg.rc_timing_host(c["nodes_start"], c["edges"], c["roots"], c["res"], c["cap"],
                              c["sinks_start"], c["sink_nodes"], c["driver_slew"])


def random_request(rng, d, n_cap, n_slew):
    ns, ss, sn = d["nodes_start"], d["sinks_start"], d["sink_nodes"]
    N = len(ns) - 1
    cnet = rng.integers(0, N, n_cap).astype(np.int32)
    # a sink pin of the net (every synthetic net has at least one leaf)
    pick = ss[cnet] + (rng.integers(0, 1 << 30, n_cap) % np.maximum(ss[cnet + 1] - ss[cnet], 1))
    cnode = sn[pick].astype(np.int32)
    cval = rng.uniform(0.05, 5.0, (n_cap, 4)).astype(np.float32)
    snet = rng.integers(0, N, n_slew).astype(np.int32)
    sval = rng.uniform(5.0, 200.0, (n_slew, 4)).astype(np.float32)
    return (cnet, cnode, cval), (snet, sval)


def apply(d, cap, slew):
    ns = d["nodes_start"]
    for net, node, v in zip(*cap):
        d["cap"][ns[net] + node] = v
    for net, v in zip(*slew):
        d["driver_slew"][net] = v


def worst_over(out, d, nets):
    ss, sn, ns = d["sinks_start"], d["sink_nodes"], d["nodes_start"]
    ws = np.zeros(4, np.float32)
    wd = np.zeros(4, np.float32)
    for net in set(int(x) for x in nets):
        for s in range(ss[net], ss[net + 1]):
            ws = np.maximum(ws, np.abs(out["sink_slew"][s]))
            b = ns[net]
            slot = out["node2bfs"][b + sn[s]]
            wd = np.maximum(wd, np.abs(out["delay"][b + slot]))
    return ws, wd


def assert_same(a, b):
    for k in Q:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_initial_pass_equals_full_pass(cuda):
    d = design(11, 4000, big=(1500, 5000))
    with TimingServer() as srv:
        did, fp = srv.add_design(d)
        assert fp > 0
        assert_same(srv.read(did), full_pass(d))


def test_sync_updates_match_full_recompute_each_step(cuda):
    rng = np.random.default_rng(5)
    d = design(12, 1500)
    with TimingServer() as srv:
        did, _ = srv.add_design(d)
        for step in range(6):
            cap, slew = random_request(rng, d, 8, 3)
            r = srv.update_sync(did, cap=cap, slew=slew)
            apply(d, cap, slew)
            ref = full_pass(d)
            assert_same(srv.read(did), ref)
            ws, wd = worst_over(ref, d, np.concatenate([cap[0], slew[0]]))
            np.testing.assert_array_equal(r["worst_slew"], ws)
            np.testing.assert_array_equal(r["worst_delay"], wd)
            assert r["dirty_nets"] == len(set(np.concatenate([cap[0], slew[0]]).tolist()))


def test_batched_requests_equal_sync_requests(cuda):
    rng = np.random.default_rng(6)
    d = design(13, 3000, big=(2000,))
    reqs = [random_request(rng, d, int(rng.integers(1, 40)), int(rng.integers(0, 8)))
            for _ in range(40)]
    with TimingServer(slots=3, max_requests=8) as a, TimingServer() as b:
        da, _ = a.add_design(d)
        db, _ = b.add_design(d)
        tickets = [a.submit(da, cap=c, slew=s) for c, s in reqs]
        got = [a.wait(t, 20000) for t in tickets]
        want = [b.update_sync(db, cap=c, slew=s) for c, s in reqs]
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g["worst_slew"], w["worst_slew"])
            np.testing.assert_array_equal(g["worst_delay"], w["worst_delay"])
            assert g["dirty_nets"] == w["dirty_nets"]
        assert_same(a.read(da), b.read(db))
    for c, s in reqs:
        apply(d, c, s)
    with TimingServer() as c:
        dc, _ = c.add_design(d)
        assert_same(c.read(dc), full_pass(d))


def test_isolation_alone_vs_mixed(cuda):
    """A design's results do not depend on which other designs share its
    batches."""
    rng = np.random.default_rng(7)
    designs = [design(20 + i, 800 + 500 * i, hi=1024) for i in range(4)]
    reqs = {i: [random_request(rng, designs[i], int(rng.integers(1, 30)),
                               int(rng.integers(0, 5))) for _ in range(25)] for i in range(4)}
    with TimingServer(slots=2) as alone:
        d0, _ = alone.add_design(designs[0])
        solo = [alone.wait(alone.submit(d0, cap=c, slew=s), 20000) for c, s in reqs[0]]
        solo_state = alone.read(d0)
    with TimingServer(slots=4, max_requests=3) as mixed:
        ids = [mixed.add_design(x)[0] for x in designs]
        tickets = {i: [] for i in range(4)}
        for k in range(25):
            for i in (3, 0, 2, 1):
                c, s = reqs[i][k]
                tickets[i].append(mixed.submit(ids[i], cap=c, slew=s))
        res = {i: [mixed.wait(t, 20000) for t in tickets[i]] for i in range(4)}
        for g, w in zip(res[0], solo):
            np.testing.assert_array_equal(g["worst_slew"], w["worst_slew"])
            np.testing.assert_array_equal(g["worst_delay"], w["worst_delay"])
        assert_same(mixed.read(ids[0]), solo_state)
        for i in range(1, 4):
            x = {k: v.copy() for k, v in designs[i].items()}
            for c, s in reqs[i]:
                apply(x, c, s)
            assert_same(mixed.read(ids[i]), full_pass(x))


def test_admission_by_footprint(cuda):
    a = design(30, 2000)
    b = design(31, 2000)
    with TimingServer() as probe:
        _, fa = probe.add_design(a)
        _, fb = probe.add_design(b)
    with TimingServer(budget_bytes=fa + fb // 2) as srv:
        ia, _ = srv.add_design(a)
        with pytest.raises(_lib.OtgError) as e:
            srv.add_design(b)
        assert e.value.code == 9  # OTG_ERR_ADMISSION
        srv.remove_design(ia)
        ib, _ = srv.add_design(b)
        assert_same(srv.read(ib), full_pass(b))


def test_bad_update_is_reported_and_design_unchanged(cuda):
    d = design(40, 500)
    with TimingServer() as srv:
        did, _ = srv.add_design(d)
        before = srv.read(did)
        N = len(d["roots"])
        n0 = int(d["nodes_start"][1] - d["nodes_start"][0])
        bad = [dict(cap=(np.array([N + 5], np.int32), np.array([0], np.int32),
                         np.ones((1, 4), np.float32))),
               dict(cap=(np.array([0], np.int32), np.array([n0], np.int32),
                         np.ones((1, 4), np.float32))),
               dict(slew=(np.array([-1], np.int32), np.ones((1, 4), np.float32)))]
        for kw in bad:
            for call in (srv.submit, srv.update_sync):
                with pytest.raises(_lib.OtgError) as e:
                    call(did, **kw)
                assert e.value.code == 1  # OTG_ERR_INVALID
        assert_same(srv.read(did), before)
        # the server still serves the design
        r = srv.wait(srv.submit(did, slew=(np.array([3], np.int32),
                                           np.full((1, 4), 50.0, np.float32))), 20000)
        assert r["dirty_nets"] == 1
    with TimingServer(max_updates=4) as small:
        did, _ = small.add_design(d)
        with pytest.raises(_lib.OtgError) as e:  # more updates than a batch holds
            small.submit(did, slew=(np.zeros(5, np.int32), np.ones((5, 4), np.float32)))
        assert e.value.code == 1
