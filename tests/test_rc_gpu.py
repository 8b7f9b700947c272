"""GPU parity of the fused RC path (libotg, through the C ABI) against the
oracle and the reference fixtures.  BFS order / pid / directed edges are
bit-exact; Elmore values within RTOL=1e-5 relative with an absolute floor of
1e-6 x the net's max |value| (helpers.py), per quantity and corner."""
import ctypes
import os

import numpy as np
import pytest

import opentimer_b200 as otg
import oracle as O
import rcgen
from helpers import AFLOOR, RTOL, bfs_local, elmore_err, max_rel_vs_f64, net_max, worst_net

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
Q = ["load", "delay", "ldelay", "impulse"]


def dev_batch(f, cuda, sinks=None, slew=None):
    import torch
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    kw = {}
    if sinks is not None:
        kw = dict(sinks_start=t(sinks[0]), sink_nodes=t(sinks[1]), driver_slew=t(slew))
    return otg.RcBatch(t(f.nodes_start), t(f.edges.copy()), t(f.roots), t(f.res), t(f.cap), **kw)


def run(f, cuda, **kw):
    b = dev_batch(f, cuda, **kw)
    b.run()
    b.check()
    return b


def assert_parity(f, b, ref_local=None):
    st, e, n2b, pid, depth = O.bfs(f)
    assert st == 0
    got_n2b = b.node2bfs.cpu().numpy()
    assert np.array_equal(got_n2b, n2b)
    assert np.array_equal(b.pid.cpu().numpy(), pid)
    assert np.array_equal(b.edges.cpu().numpy(), e)
    if ref_local is None:
        st, ref_local = O.elmore_cpu_f32(f)
        assert st == 0
    errs = {}
    for q, r in zip(Q, ref_local):
        got = bfs_local(f.nodes_start, got_n2b, getattr(b, q).cpu().numpy())
        errs[q] = elmore_err(f.nodes_start, got, r)
        if errs[q] > 1.0:
            e, i = worst_net(f.nodes_start, got, r)
            n = int(f.nodes_start[i + 1] - f.nodes_start[i])
            raise AssertionError(f"{q}: err/tol {e:.3f} at net {i} ({n} nodes)")
    return errs


def test_every_size_class(cuda):
    sizes = [1, 2, 3, 5, 31, 32, 33, 34, 64, 127, 128, 129, 200, 255, 256, 257, 511, 512, 513,
             1000, 1024, 1025, 1500, 2048, 2300]
    kinds = []
    for n in sizes:
        kinds += ["rrt", "chain", "path", "star"]
    f = rcgen.forest(21, [n for n in sizes for _ in range(4)], kinds)
    assert_parity(f, run(f, cuda))


def test_random_heavy_tail(cuda):
    f = rcgen.random_forest(8, 400, 2, 4096)
    assert_parity(f, run(f, cuda))


def test_global_workspace_path(cuda):
    # nets beyond the shared-memory budget run in the workspace slices
    f = rcgen.forest(4, [3000, 5000, 9000, 6000, 17, 700],
                     ["chain", "rrt", "path", "star", "rrt", "chain"])
    assert_parity(f, run(f, cuda))


HUGE_SIZES = [5000, 20000, 12000, 7000, 30, 600, 16000, 9000, 20000, 5500]
HUGE_KINDS = ["chain", "rrt", "path", "star", "rrt", "chain", "chain", "rrt", "path", "rrt"]


@pytest.mark.parametrize("cl", ["8", "16", "2"])
def test_huge_nets_cluster_path(cuda, monkeypatch, cl):
    """Nets of 5k-20k nodes (random trees, chains with side branches, bare
    paths, stars) run on a thread-block cluster per net, the cluster's CTAs
    acting as one block over the net's workspace slice.  BFS slots, pid and
    directed edges are bit-exact with the oracle; load, delay and ldelay are
    within the tolerance of the reference's fp32 recursion; every quantity
    is at least as close to the FP64 oracle as that recursion (4x slack, as
    test_error_against_fp64).  Impulse is held to the FP64 bar only: on the
    12k-node bare path the fp32 recursion's own impulse (2 beta - delay^2,
    a difference of two ~1e10 terms) lies 1.4 tolerance units from FP64.
    Every output is bit-identical to the one-CTA-per-net path (the sums are
    exact, so the thread count changes no bit)."""
    f = rcgen.forest(31, HUGE_SIZES, HUGE_KINDS)
    ss, sn = rcgen.sinks_of(f)
    slew = np.random.default_rng(3).uniform(5, 200, (f.num_nets, 4)).astype(np.float32)
    slew[::3] *= -1
    monkeypatch.setenv("OTG_RC_HUGE_CLUSTER", "1")
    one = run(f, cuda, sinks=(ss, sn), slew=slew)
    monkeypatch.setenv("OTG_RC_HUGE_CLUSTER", cl)
    b = run(f, cuda, sinks=(ss, sn), slew=slew)
    for q in ["node2bfs", "pid", "edges", "sink_slew"] + Q:
        assert np.array_equal(getattr(b, q).cpu().numpy(), getattr(one, q).cpu().numpy()), q
    # the sink slews are the reference's formula on our own impulses, bit for bit
    imp = bfs_local(f.nodes_start, b.node2bfs.cpu().numpy(), b.impulse.cpu().numpy())
    want = O.sink_slew(f, ss, sn, slew, imp)
    assert np.array_equal(b.sink_slew.cpu().numpy().view(np.int32), want.view(np.int32))
    st, e, n2b, pid, depth = O.bfs(f)
    assert st == 0
    got_n2b = b.node2bfs.cpu().numpy()
    assert np.array_equal(got_n2b, n2b)
    assert np.array_equal(b.pid.cpu().numpy(), pid)
    assert np.array_equal(b.edges.cpu().numpy(), e)
    st, ex = O.elmore_f64(f)
    st2, ref = O.elmore_cpu_f32(f)
    for q, x, r in zip(Q, ex, ref):
        got = bfs_local(f.nodes_start, got_n2b, getattr(b, q).cpu().numpy())
        if q != "impulse":
            assert elmore_err(f.nodes_start, got, r) <= 1.0, q
        assert max_rel_vs_f64(f.nodes_start, got, x) <= 4 * max_rel_vs_f64(f.nodes_start, r, x) \
            + 1e-7, q


@pytest.mark.parametrize("name", ["rc_cpu_small.npz", "rc_cpu_c17.npz", "rc_cpu_s27.npz"])
def test_reference_cpu_fixtures(cuda, name):
    d = np.load(os.path.join(GOLD, name))
    f = O.Forest(d["nodes_start"], d["edges"], d["roots"], d["res"], d["cap"])
    assert_parity(f, run(f, cuda), [d[q] for q in Q])


def test_reference_gpu_fixture(cuda):
    path = os.path.join(GOLD, "rc_gpu_small.npz")
    if not os.path.exists(path):
        pytest.skip("reference-GPU fixture not generated")
    d = np.load(path)
    f = O.Forest(d["nodes_start"], d["edges"], d["roots"], d["res"], d["cap"])
    b = run(f, cuda)
    assert np.array_equal(b.node2bfs.cpu().numpy(), d["node2bfs"])
    assert np.array_equal(b.pid.cpu().numpy(), d["pid"])
    assert np.array_equal(b.edges.cpu().numpy(), d["directed_edges"])
    for q in Q:
        assert elmore_err(f.nodes_start, getattr(b, q).cpu().numpy(), d[q]) <= 1.0, q


def test_error_against_fp64(cuda):
    f = rcgen.random_forest(12, 200, 2, 4096)
    b = run(f, cuda)
    st, ex = O.elmore_f64(f)
    st2, ref = O.elmore_cpu_f32(f)
    n2b = b.node2bfs.cpu().numpy()
    for q, x, r in zip(Q, ex, ref):
        got = bfs_local(f.nodes_start, n2b, getattr(b, q).cpu().numpy())
        # ours is at least as close to exact as the reference's fp32 recursion (x4 slack)
        assert max_rel_vs_f64(f.nodes_start, got, x) <= 4 * max_rel_vs_f64(f.nodes_start, r, x) \
            + 1e-7, q


def test_sink_slew_epilogue(cuda):
    f = rcgen.random_forest(13, 120, 2, 3000)
    ss, sn = rcgen.sinks_of(f)
    rng = np.random.default_rng(1)
    slew = rng.uniform(5, 200, (f.num_nets, 4)).astype(np.float32)
    slew[::7] *= -1  # falling-edge sign convention
    b = run(f, cuda, sinks=(ss, sn), slew=slew)
    st, ref = O.elmore_cpu_f32(f)
    want = O.sink_slew(f, ss, sn, slew, ref[3])
    got = b.sink_slew.cpu().numpy()
    assert np.all(np.sign(got) == np.sign(want))
    # slew^2 = si^2 + impulse: the impulse tolerance (RTOL, AFLOOR) carries
    # over as d(slew) = d(impulse) / (2 |slew|), plus fp32 rounding of slew
    imp = ref[3][f.nodes_start[:-1].repeat(np.diff(ss)) + sn]
    imp_max = net_max(f.nodes_start, ref[3])[f.nodes_start[:-1].repeat(np.diff(ss)) + sn]
    tol = (RTOL * np.abs(imp) + AFLOOR * imp_max) / (2 * np.abs(want)) + 1e-6 * np.abs(want)
    assert np.max(np.abs(got - want) / tol) <= 1.0


def test_deterministic(cuda):
    f = rcgen.random_forest(14, 150, 2, 4096)
    b1 = run(f, cuda)
    b2 = run(f, cuda)
    for q in Q + ["node2bfs", "pid"]:
        x, y = getattr(b1, q).cpu().numpy(), getattr(b2, q).cpu().numpy()
        assert np.array_equal(x.view(np.int32), y.view(np.int32)), q


def test_bad_inputs_report_status_without_fault(cuda):
    good = rcgen.forest(2, [40, 10, 300], ["rrt", "rrt", "chain"])
    # out-of-range root
    f = good.copy()
    f.roots[1] = 99
    b = dev_batch(f, cuda)
    b.run()
    code, net = b.status()
    assert code == 1 and net == 1
    # not a tree: duplicate edge in a block-path net
    f = good.copy()
    e0 = int(f.nodes_start[2]) - 2
    f.edges[e0 + 5] = f.edges[e0 + 4]
    b = dev_batch(f, cuda)
    b.run()
    code, net = b.status()
    assert code == 4 and net == 2
    # the other nets are still exact
    st, e, n2b, pid, depth = O.bfs(good)
    got = b.node2bfs.cpu().numpy()
    assert np.array_equal(got[:50], n2b[:50])
    # edge id out of range in a warp-path net
    f = good.copy()
    f.edges[int(f.nodes_start[1]) - 1 + 2, 0] = 1000
    b = dev_batch(f, cuda)
    b.run()
    assert b.status()[0] == 1


def test_host_path_matches_device(cuda):
    f = rcgen.random_forest(15, 300, 2, 4096)
    ss, sn = rcgen.sinks_of(f)
    slew = np.random.default_rng(2).uniform(5, 200, (f.num_nets, 4)).astype(np.float32)
    b = run(f, cuda, sinks=(ss, sn), slew=slew)
    e = f.edges.copy()
    out = otg.rc_timing_host(f.nodes_start, e, f.roots, f.res, f.cap, ss, sn, slew)
    assert np.array_equal(e, b.edges.cpu().numpy())
    for q in Q + ["node2bfs", "pid", "sink_slew"]:
        x = out[q]
        y = getattr(b, q).cpu().numpy()
        assert np.array_equal(x.view(np.int32), y.view(np.int32)), q


def test_gpu_generator_matches_host(cuda):
    import torch
    ns = otg.net_sizes(3, 500, 2, 4096)
    g = otg.synth_forest(77, torch.from_numpy(ns).to(cuda))
    h = otg.synth_forest_host(77, ns)
    for k in ["edges", "roots", "res", "cap", "driver_slew"]:
        assert np.array_equal(g[k].cpu().numpy(), h[k]), k
    f = O.Forest(ns, h["edges"], h["roots"], h["res"], h["cap"])
    ss, sn = rcgen.sinks_of(f)
    assert np.array_equal(g["sinks_start"].cpu().numpy(), ss)
    assert np.array_equal(g["sink_nodes"].cpu().numpy(), sn)


class RctEdgeArrayCUDA(ctypes.Structure):
    _fields_ = [("num_nets", ctypes.c_int), ("total_num_nodes", ctypes.c_int),
                ("total_num_edges", ctypes.c_int)] + [
        (n, ctypes.c_void_p) for n in
        ["rct_nodes_start", "rct_edges", "rct_roots", "rct_edges_res", "rct_nodes_cap",
         "rct_distances", "rct_sort_counts", "pres", "cap", "rct_node2bfs_order", "rct_pid",
         "load", "delay", "ldelay", "impulse"]]


def test_reference_symbol_rct_bfs_and_compute_cuda(cuda):
    """The drop-in C++ symbol, called exactly as FlatRctStorage does."""
    f = rcgen.random_forest(16, 100, 2, 2000)
    L = otg.lib()
    fn = getattr(L, otg.CXX_SYMBOLS["rct_bfs_and_compute_cuda"])
    fn.argtypes = [RctEdgeArrayCUDA]
    fn.restype = None
    V = f.total_nodes
    e = f.edges.copy()
    n2b = np.zeros(V, np.int32)
    pid = np.zeros(V, np.int32)
    outs = [np.zeros((V, 4), np.float32) for _ in Q]
    a = RctEdgeArrayCUDA(f.num_nets, V, V - f.num_nets, f.nodes_start.ctypes.data, e.ctypes.data,
                         f.roots.ctypes.data, f.res.ctypes.data, f.cap.ctypes.data, None, None,
                         None, None, n2b.ctypes.data, pid.ctypes.data,
                         *[o.ctypes.data for o in outs])
    fn(a)
    st, e_ref, n2b_ref, pid_ref, _ = O.bfs(f)
    assert np.array_equal(n2b, n2b_ref) and np.array_equal(pid, pid_ref)
    assert np.array_equal(e, e_ref)
    st, ref = O.elmore_cpu_f32(f)
    for o, r in zip(outs, ref):
        assert elmore_err(f.nodes_start, bfs_local(f.nodes_start, n2b, o), r) <= 1.0


def test_against_reference_gpu_live(cuda):
    """The reference's own rct_bfs_and_compute_cuda (sm_100a build) on the
    same input: BFS bit-exact, floats within tolerance."""
    if not O.ref_available():
        pytest.skip("reference harness not built")
    f = rcgen.random_forest(17, 300, 2, 1500)
    e, n2b, pid, outs = O.ref_rct_gpu(f)
    b = run(f, cuda)
    pid[f.nodes_start[:-1]] = 0
    assert np.array_equal(b.node2bfs.cpu().numpy(), n2b)
    assert np.array_equal(b.pid.cpu().numpy(), pid)
    assert np.array_equal(b.edges.cpu().numpy(), e)
    for q, r in zip(Q, outs):
        assert elmore_err(f.nodes_start, getattr(b, q).cpu().numpy(), r) <= 1.0, q
