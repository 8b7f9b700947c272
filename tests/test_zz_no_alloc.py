"""otg_rc_timing_noalloc -- the fused RC pass with the workspace compiled into
libotg, for callers that may not allocate device memory (a host whose pool
allocator owns all device memory, a loop that cannot afford cudaMalloc's
device-wide synchronization) -- against the workspace entry point
otg_rc_timing, through the C ABI.  Both run the same kernels with exact
fixed-point sums, so their outputs must be identical bit for bit.

Collected last on purpose: a failure here leaves every other test already
run when pytest stops at the first failure."""
import ctypes

import numpy as np
import pytest

import opentimer_b200 as otg
import rcgen
from opentimer_b200 import _lib

pytestmark = pytest.mark.gpu
Q = ["load", "delay", "ldelay", "impulse"]


def noalloc_fn():
    fn = otg.lib().otg_rc_timing_noalloc
    fn.argtypes = [ctypes.POINTER(_lib.RcForest), ctypes.c_int32, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def device_inputs(f, cuda, sinks, slew):
    import torch
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    return dict(nodes_start=t(f.nodes_start), edges=t(f.edges.copy()), roots=t(f.roots),
                res=t(f.res), cap=t(f.cap), sinks_start=t(sinks[0]), sink_nodes=t(sinks[1]),
                driver_slew=t(slew))


def run_noalloc(f, cuda, sinks, slew, max_nodes):
    import torch
    d = device_inputs(f, cuda, sinks, slew)
    V, S = f.total_nodes, len(sinks[1])
    out = dict(node2bfs=torch.empty(V, dtype=torch.int32, device=cuda),
               pid=torch.empty(V, dtype=torch.int32, device=cuda),
               sink_slew=torch.empty(S, 4, dtype=torch.float32, device=cuda))
    for q in Q:
        out[q] = torch.empty(V, 4, dtype=torch.float32, device=cuda)
    P = lambda x: x.data_ptr()  # noqa: E731
    forest = _lib.RcForest(f.num_nets, V, P(d["nodes_start"]), P(d["edges"]), P(d["roots"]),
                           P(d["res"]), P(d["cap"]), P(out["node2bfs"]), P(out["pid"]),
                           *[P(out[q]) for q in Q], P(d["sinks_start"]), P(d["sink_nodes"]),
                           P(d["driver_slew"]), P(out["sink_slew"]))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    code = noalloc_fn()(ctypes.byref(forest), max_nodes, stream)
    out["edges"] = d["edges"]
    return code, out


def run_workspace(f, cuda, sinks, slew, max_nodes):
    d = device_inputs(f, cuda, sinks, slew)
    b = otg.RcBatch(max_net_nodes=max_nodes, **d)
    b.run()
    b.check()
    return b


def test_noalloc_matches_workspace_entry_on_two_calls_in_a_row(cuda):
    # two different batches back to back: the second call reuses the array
    # the first one left behind
    for seed, nets in ((41, 300), (42, 120)):
        f = rcgen.random_forest(seed, nets, 2, 4000)
        sinks = rcgen.sinks_of(f)
        slew = np.random.default_rng(seed).uniform(5, 200, (f.num_nets, 4)).astype(np.float32)
        code, got = run_noalloc(f, cuda, sinks, slew, 4000)
        assert code == 0, _lib.STATUS.get(code, code)
        ref = run_workspace(f, cuda, sinks, slew, 4000)
        for k in ["node2bfs", "pid", "edges"] + Q + ["sink_slew"]:
            g, r = got[k].cpu().numpy(), getattr(ref, k).cpu().numpy()
            assert np.array_equal(g.view(np.int32), r.view(np.int32)), k


def test_noalloc_empty_call_after_a_failed_batch(cuda):
    # a batch with an out-of-range root fails; an empty call right after it
    # must report its own (clean) status, not the failed batch's
    f = rcgen.forest(3, [40, 10, 300], ["rrt", "rrt", "chain"])
    f.roots[1] = 99
    sinks = rcgen.sinks_of(f)
    slew = np.full((f.num_nets, 4), 50.0, np.float32)
    code, _ = run_noalloc(f, cuda, sinks, slew, 300)
    assert code == 1  # OTG_ERR_INVALID from the kernel's own check
    import torch
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    empty = _lib.RcForest(0, 0, *([None] * 15))
    assert noalloc_fn()(ctypes.byref(empty), 1, stream) == 0
    # and a good batch after both is still exact
    f = rcgen.forest(4, [40, 10, 300], ["rrt", "rrt", "chain"])
    sinks = rcgen.sinks_of(f)
    code, got = run_noalloc(f, cuda, sinks, slew, 300)
    assert code == 0
    ref = run_workspace(f, cuda, sinks, slew, 300)
    for k in ["node2bfs", "pid", "edges"] + Q:
        g, r = got[k].cpu().numpy(), getattr(ref, k).cpu().numpy()
        assert np.array_equal(g.view(np.int32), r.view(np.int32)), k


def test_noalloc_rejects_batches_beyond_its_array(cuda):
    fn = noalloc_fn()
    import torch
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    too_many = _lib.RcForest(600_000, 1_200_000, *([None] * 15))
    assert fn(ctypes.byref(too_many), 2, stream) == 8   # OTG_ERR_WORKSPACE, nothing launched
    too_big = _lib.RcForest(10, 200_000, *([None] * 15))
    assert fn(ctypes.byref(too_big), 20_000, stream) == 8
