"""opentimer_b200 -- B200-native RC-net timing and timing-graph levelization
for OpenTimer.

The compute lives in libotg.so (hand-written sm_100a CUDA behind the C ABI of
include/otg.h).  This package binds it with ctypes; PyTorch only supplies
device memory and streams.  There is no CPU fallback: without the built
library, or without a GPU, the device entry points raise.

Device entry points take CUDA tensors; *_host entry points take numpy arrays
and do the host<->device copies inside the call (the end-to-end path a
reference caller sees through rct_bfs_and_compute_cuda).
"""
import ctypes

import numpy as np

from . import workloads  # noqa: F401
from ._lib import C_SYMBOLS, CXX_SYMBOLS, OtgError, RcForest, check, lib  # noqa: F401

__all__ = ["RcBatch", "rc_timing", "rc_timing_host", "levelize", "levelize_host", "fanin_csr",
           "synth_forest", "kernel_launches", "get_tuning", "set_tuning", "autotune",
           "OtgError", "lib"]

NC = 4  # corners: split*2 + tran


def _ptr(t):
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def _np_ptr(a):
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _tuning_dict(t):
    k = t.num_classes
    return {"class_max": list(t.class_max[:k]), "class_threads": list(t.class_threads[:k]),
            "class_items": list(t.class_items[:k])}


def get_tuning():
    """The current device's RC-pass tuning: per block size class its upper
    net size, CTA threads and scan items per thread."""
    from ._lib import RcTuning
    t = RcTuning()
    check("otg_rc_get_tuning", lib().otg_rc_get_tuning(ctypes.byref(t)))
    return _tuning_dict(t)


def set_tuning(tuning=None):
    """Applies a tuning (dict as from get_tuning; None: the default)."""
    from ._lib import RcTuning
    if tuning is None:
        check("otg_rc_set_tuning", lib().otg_rc_set_tuning(None))
        return
    t = RcTuning()
    t.num_classes = len(tuning["class_max"])
    for c in range(t.num_classes):
        t.class_max[c] = tuning["class_max"][c]
        t.class_threads[c] = tuning["class_threads"][c]
        t.class_items[c] = tuning["class_items"][c]
    check("otg_rc_set_tuning", lib().otg_rc_set_tuning(ctypes.byref(t)))


def autotune(batch, stream=None):
    """Runs the autotuner on an RcBatch (its outputs are overwritten),
    applies the fastest tuning and returns it."""
    from ._lib import RcTuning
    t = RcTuning()
    check("otg_rc_autotune", lib().otg_rc_autotune(
        ctypes.byref(batch._forest), batch.max_net_nodes, _stream(stream), ctypes.byref(t)))
    return _tuning_dict(t)


def kernel_launches():
    """Number of kernels libotg has launched in this process."""
    return int(lib().otg_kernel_launches())


class RcBatch:
    """A device-resident batch of RC nets plus its outputs and workspace.

    Inputs (CUDA tensors, int32 / float32):
      nodes_start [N+1], edges [E,2] (undirected, rewritten to parent->child
      by run()), roots [N], res [E], cap [V,4];
      optional sinks_start [N+1], sink_nodes [S], driver_slew [N,4].
    Outputs after run(): node2bfs [V], pid [V], load/delay/ldelay/impulse
      [V,4] in BFS order, sink_slew [S,4].
    """

    def __init__(self, nodes_start, edges, roots, res, cap, sinks_start=None, sink_nodes=None,
                 driver_slew=None, max_net_nodes=None):
        import torch
        self.nodes_start = nodes_start
        self.edges = edges
        self.roots = roots
        self.res = res
        self.cap = cap
        self.num_nets = int(roots.numel())
        self.total_nodes = int(cap.shape[0])
        dev = cap.device
        if max_net_nodes is None:
            max_net_nodes = int((nodes_start[1:] - nodes_start[:-1]).max().item()) \
                if self.num_nets else 1
        self.max_net_nodes = int(max(1, max_net_nodes))
        V = self.total_nodes
        self.node2bfs = torch.empty(V, dtype=torch.int32, device=dev)
        self.pid = torch.empty(V, dtype=torch.int32, device=dev)
        self.load = torch.empty(V, NC, dtype=torch.float32, device=dev)
        self.delay = torch.empty_like(self.load)
        self.ldelay = torch.empty_like(self.load)
        self.impulse = torch.empty_like(self.load)
        self.sinks_start = sinks_start
        self.sink_nodes = sink_nodes
        self.driver_slew = driver_slew
        self.sink_slew = None
        if sinks_start is not None:
            self.sink_slew = torch.empty(int(sink_nodes.numel()), NC, dtype=torch.float32,
                                         device=dev)
        sz = ctypes.c_size_t()
        check("otg_rc_workspace_size",
              lib().otg_rc_workspace_size(self.num_nets, self.max_net_nodes, ctypes.byref(sz)))
        self.workspace = torch.empty(max(sz.value, 256), dtype=torch.uint8, device=dev)
        self._forest = RcForest(
            self.num_nets, V, self.nodes_start.data_ptr(), self.edges.data_ptr(),
            self.roots.data_ptr(), self.res.data_ptr(), self.cap.data_ptr(),
            self.node2bfs.data_ptr(), self.pid.data_ptr(), self.load.data_ptr(),
            self.delay.data_ptr(), self.ldelay.data_ptr(), self.impulse.data_ptr(),
            sinks_start.data_ptr() if sinks_start is not None else None,
            sink_nodes.data_ptr() if sinks_start is not None else None,
            driver_slew.data_ptr() if sinks_start is not None else None,
            self.sink_slew.data_ptr() if sinks_start is not None else None)

    def run(self, stream=None):
        """Enqueue the fused BFS + Elmore pass on `stream` (asynchronous)."""
        check("otg_rc_timing",
              lib().otg_rc_timing(ctypes.byref(self._forest), self.max_net_nodes,
                                  _ptr(self.workspace), self.workspace.numel(), _stream(stream)))
        return self

    def status(self, stream=None):
        """Synchronize and return (status_code, bad_net)."""
        bad = ctypes.c_int32(-1)
        code = lib().otg_rc_status(_ptr(self.workspace), _stream(stream), ctypes.byref(bad))
        return int(code), int(bad.value)

    def check(self, stream=None):
        code, net = self.status(stream)
        if code != 0:
            raise OtgError(f"otg_rc_timing (net {net})", code)
        moved = getattr(self, "_move_status", None)
        if moved is not None and int(moved.item()) != 0:
            raise OtgError("otg_rc_move_nets", int(moved.item()))

    def replace_nets(self, nets, nodes_start, edges, roots, res, cap, stream=None):
        """Incremental SPEF ingestion: a new batch in which the forest nets
        `nets` (distinct indices) carry new RC trees, given as a forest of
        len(nets) nets in the constructor's layout (numpy arrays or CUDA
        tensors), while every other net keeps its tree AND its results,
        moved into the new layout on the device (otg_rc_move_nets).  Only
        the replaced nets are re-timed (otg_rc_timing_subset), so the
        result equals a full pass over the new forest.  This batch must
        have run; sink arrays are not carried over."""
        import torch
        assert self.sinks_start is None, "sink arrays are not carried over"
        dev = self.cap.device
        nets = np.asarray(nets, np.int64).reshape(-1)
        K, N = len(nets), self.num_nets
        assert len(np.unique(nets)) == K, "a net is replaced twice"
        assert K == 0 or (nets.min() >= 0 and nets.max() < N)

        def t(a, dt):
            if torch.is_tensor(a):
                return a.to(dev).contiguous()
            return torch.from_numpy(np.ascontiguousarray(a, dt)).to(dev)
        host = lambda a: a.cpu().numpy() if torch.is_tensor(a) else np.asarray(a)  # noqa: E731
        sub = [t(nodes_start, np.int32), t(edges, np.int32), t(roots, np.int32),
               t(res, np.float32), t(cap, np.float32)]
        sizes = host(self.nodes_start).astype(np.int64)
        sizes = sizes[1:] - sizes[:-1]
        sub_sizes = np.diff(host(nodes_start).astype(np.int64))
        assert len(sub_sizes) == K
        sizes[nets] = sub_sizes
        ns_new = np.zeros(N + 1, np.int64)
        np.cumsum(sizes, out=ns_new[1:])
        assert ns_new[-1] < 2 ** 31, "32-bit node offsets"
        V, E = int(ns_new[-1]), int(ns_new[-1]) - N
        new = RcBatch(t(ns_new, np.int32), torch.empty((E, 2), dtype=torch.int32, device=dev),
                      torch.empty(N, dtype=torch.int32, device=dev),
                      torch.empty(E, dtype=torch.float32, device=dev),
                      torch.empty((V, NC), dtype=torch.float32, device=dev),
                      max_net_nodes=int(sizes.max()) if N else 1)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        keep = np.arange(N, dtype=np.int32)
        keep[nets] = -1
        put = np.full(N, -1, np.int32)
        put[nets] = np.arange(K, dtype=np.int32)
        keep_d, put_d = t(keep, np.int32), t(put, np.int32)
        s = _stream(stream)
        check("otg_rc_move_nets", lib().otg_rc_move_nets(
            ctypes.byref(self._forest), ctypes.byref(new._forest), _ptr(keep_d), 1, _ptr(status), s))
        if K:
            staging = RcForest(K, int(host(nodes_start)[-1]), *[x.data_ptr() for x in sub],
                               *([None] * 10))
            check("otg_rc_move_nets", lib().otg_rc_move_nets(
                ctypes.byref(staging), ctypes.byref(new._forest), _ptr(put_d), 0, _ptr(status),
                s))
        net_list = t(nets, np.int32)
        num = torch.tensor([K], dtype=torch.int32, device=dev)
        if K:
            check("otg_rc_timing_subset", lib().otg_rc_timing_subset(
                ctypes.byref(new._forest), new.max_net_nodes, _ptr(net_list), _ptr(num), K,
                _ptr(new.workspace), new.workspace.numel(), s))
        else:  # nothing re-timed: clear the status word the moves leave alone
            new.workspace.zero_()
        # the staging tensors live until the stream has used them
        new._move_status, new._keep = status, (sub, keep_d, put_d, net_list, num)
        return new


def rc_timing(nodes_start, edges, roots, res, cap, **kw):
    """Run the fused pass on device tensors and return the RcBatch."""
    b = RcBatch(nodes_start, edges, roots, res, cap, **kw)
    b.run()
    b.check()
    return b


def rc_timing_host(nodes_start, edges, roots, res, cap, sinks_start=None, sink_nodes=None,
                   driver_slew=None):
    """End-to-end host path: numpy in, numpy out (BFS order).  `edges` is
    rewritten in place to parent->child, as the reference does."""
    V = int(cap.shape[0])
    out = {
        "node2bfs": np.empty(V, np.int32), "pid": np.empty(V, np.int32),
        "load": np.empty((V, NC), np.float32), "delay": np.empty((V, NC), np.float32),
        "ldelay": np.empty((V, NC), np.float32), "impulse": np.empty((V, NC), np.float32),
    }
    sink_slew = None
    if sinks_start is not None:
        sink_slew = np.empty((len(sink_nodes), NC), np.float32)
        out["sink_slew"] = sink_slew
    for a in (nodes_start, edges, roots, res, cap):
        assert a.flags.c_contiguous
    f = RcForest(len(roots), V, nodes_start.ctypes.data, edges.ctypes.data, roots.ctypes.data,
                 res.ctypes.data, cap.ctypes.data, out["node2bfs"].ctypes.data,
                 out["pid"].ctypes.data, out["load"].ctypes.data, out["delay"].ctypes.data,
                 out["ldelay"].ctypes.data, out["impulse"].ctypes.data,
                 sinks_start.ctypes.data if sinks_start is not None else None,
                 sink_nodes.ctypes.data if sinks_start is not None else None,
                 driver_slew.ctypes.data if sinks_start is not None else None,
                 sink_slew.ctypes.data if sinks_start is not None else None)
    check("otg_rc_timing_host", lib().otg_rc_timing_host(ctypes.byref(f)))
    return out


class LevelizeBatch:
    """Device-resident levelization problem (CUDA int32 tensors)."""

    def __init__(self, fanin_start, fanin, out_deg, frontier0):
        import torch
        self.n = int(out_deg.numel())
        self.num_edges = int(fanin.numel())
        self.fanin_start, self.fanin, self.out_deg, self.frontier0 = \
            fanin_start, fanin, out_deg, frontier0
        dev = out_deg.device
        self.order = torch.empty(max(self.n, 1), dtype=torch.int32, device=dev)
        self.level = torch.empty(max(self.n, 1), dtype=torch.int32, device=dev)
        self.level_ends = torch.empty(self.n + 2, dtype=torch.int32, device=dev)
        self.counts = torch.zeros(2, dtype=torch.int32, device=dev)
        sz = ctypes.c_size_t()
        check("otg_levelize_workspace_size",
              lib().otg_levelize_workspace_size(self.n, self.num_edges, ctypes.byref(sz)))
        self.workspace = torch.empty(max(sz.value, 256), dtype=torch.uint8, device=dev)

    def run(self, stream=None):
        check("otg_levelize", lib().otg_levelize(
            self.n, self.num_edges, _ptr(self.fanin_start), _ptr(self.fanin),
            _ptr(self.out_deg), _ptr(self.frontier0), int(self.frontier0.numel()),
            _ptr(self.order), _ptr(self.level), _ptr(self.level_ends), _ptr(self.counts),
            _ptr(self.workspace), self.workspace.numel(), _stream(stream)))
        return self

    def check(self, stream=None):
        code = lib().otg_levelize_status(_ptr(self.workspace), _stream(stream))
        if code != 0:
            raise OtgError("otg_levelize", code)

    def result(self):
        self.check()
        L, emitted = [int(x) for x in self.counts.tolist()]
        return (self.order[:emitted].cpu().numpy(), self.level_ends[:L + 1].cpu().numpy(),
                self.level[:self.n].cpu().numpy())


def fanin_csr(num_pins, arc_from, arc_to, arc_skip=None, pin_cand=None, cand_order=None,
              as_arcs=False, stream=None):
    """The levelization input built on the device (otg_fanin_csr): arcs
    (CUDA int32 tensors from, to; optional uint8 arc_skip) over num_pins
    pins, candidates pin_cand (uint8, optional) listed in cand_order (int32;
    default: all pins in index order).  Returns CUDA tensors (fanin_start,
    fanin, out_deg, frontier0) -- fanin as source pins, or arc indices with
    as_arcs -- ready for levelize / LevelizeBatch."""
    import torch
    dev = arc_from.device
    n, A = int(num_pins), int(arc_from.numel())
    if cand_order is None:
        cand_order = torch.arange(n, dtype=torch.int32, device=dev)
    C = int(cand_order.numel())
    ws = ctypes.c_size_t()
    check("otg_fanin_csr_workspace_size",
          lib().otg_fanin_csr_workspace_size(n, A, C, ctypes.byref(ws)))
    work = torch.empty(max(ws.value, 256), dtype=torch.uint8, device=dev)
    start = torch.empty(n + 1, dtype=torch.int32, device=dev)
    fanin = torch.empty(max(A, 1), dtype=torch.int32, device=dev)
    out_deg = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    front = torch.empty(max(C, 1), dtype=torch.int32, device=dev)
    counts = torch.zeros(2, dtype=torch.int32, device=dev)
    s = _stream(stream)
    check("otg_fanin_csr", lib().otg_fanin_csr(
        n, A, _ptr(arc_from), _ptr(arc_to), _ptr(arc_skip), _ptr(pin_cand), C, _ptr(cand_order),
        1 if as_arcs else 0, _ptr(start), _ptr(fanin), _ptr(out_deg), _ptr(front),
        _ptr(counts), _ptr(work), work.numel(), s))
    check("otg_fanin_csr_status", lib().otg_fanin_csr_status(_ptr(work), s))
    first, E = [int(x) for x in counts.tolist()]
    return start, fanin[:E], out_deg[:n], front[:first]


def levelize(fanin_start, fanin, out_deg, frontier0):
    """Device levelization; returns (order, level_ends, level) as numpy."""
    return LevelizeBatch(fanin_start, fanin, out_deg, frontier0).run().result()


def levelize_host(fanin_start, fanin, out_deg, frontier0):
    """Host path: numpy in, (order, level_ends, level) out."""
    n = len(out_deg)
    fanin_start = np.ascontiguousarray(fanin_start, np.int32)
    fanin = np.ascontiguousarray(fanin, np.int32)
    out_deg = np.ascontiguousarray(out_deg, np.int32)
    frontier0 = np.ascontiguousarray(frontier0, np.int32)
    order = np.empty(max(n, 1), np.int32)
    level = np.empty(max(n, 1), np.int32)
    ends = np.empty(n + 2, np.int32)
    counts = np.zeros(2, np.int32)
    check("otg_levelize_host", lib().otg_levelize_host(
        n, len(fanin), _np_ptr(fanin_start), _np_ptr(fanin), _np_ptr(out_deg),
        _np_ptr(frontier0), len(frontier0), _np_ptr(order), _np_ptr(level), _np_ptr(ends),
        _np_ptr(counts)))
    L, emitted = int(counts[0]), int(counts[1])
    return order[:emitted], ends[:L + 1], level[:n]


def synth_forest(seed, nodes_start, with_sinks=True, stream=None):
    """Generate the seeded synthetic forest for `nodes_start` (CUDA int32
    tensor) on the device.  Returns a dict of CUDA tensors."""
    import torch
    N = int(nodes_start.numel()) - 1
    V = int(nodes_start[-1].item())
    dev = nodes_start.device
    edges = torch.empty(max(V - N, 0), 2, dtype=torch.int32, device=dev)
    roots = torch.empty(N, dtype=torch.int32, device=dev)
    res = torch.empty(max(V - N, 0), dtype=torch.float32, device=dev)
    cap = torch.empty(V, NC, dtype=torch.float32, device=dev)
    slew = torch.empty(N, NC, dtype=torch.float32, device=dev)
    cnt = torch.empty(N, dtype=torch.int32, device=dev)
    scratch = torch.empty(max(V, 1), dtype=torch.int32, device=dev)
    check("otg_synth_rc_forest", lib().otg_synth_rc_forest(
        seed, N, _ptr(nodes_start), _ptr(edges), _ptr(roots), _ptr(res), _ptr(cap), _ptr(slew),
        _ptr(cnt), _ptr(scratch), _stream(stream)))
    out = dict(nodes_start=nodes_start, edges=edges, roots=roots, res=res, cap=cap,
               driver_slew=slew)
    if with_sinks:
        ss = torch.zeros(N + 1, dtype=torch.int32, device=dev)
        ss[1:] = torch.cumsum(cnt, 0, dtype=torch.int32)
        S = int(ss[-1].item())
        sn = torch.empty(max(S, 1), dtype=torch.int32, device=dev)
        check("otg_synth_rc_sinks", lib().otg_synth_rc_sinks(
            N, _ptr(nodes_start), _ptr(edges), _ptr(roots), _ptr(ss), _ptr(sn), _ptr(scratch),
            _stream(stream)))
        out["sinks_start"] = ss
        out["sink_nodes"] = sn[:S]
    del scratch
    return out


def synth_forest_host(seed, nodes_start):
    """The same generator on the host (numpy in/out, no GPU needed)."""
    ns = np.ascontiguousarray(nodes_start, np.int32)
    N = len(ns) - 1
    V = int(ns[-1])
    edges = np.zeros((max(V - N, 0), 2), np.int32)
    roots = np.zeros(N, np.int32)
    res = np.zeros(max(V - N, 0), np.float32)
    cap = np.zeros((V, NC), np.float32)
    slew = np.zeros((N, NC), np.float32)
    cnt = np.zeros(N, np.int32)
    check("otg_synth_rc_forest_host", lib().otg_synth_rc_forest_host(
        seed, N, _np_ptr(ns), _np_ptr(edges), _np_ptr(roots), _np_ptr(res), _np_ptr(cap),
        _np_ptr(slew), _np_ptr(cnt)))
    return dict(nodes_start=ns, edges=edges, roots=roots, res=res, cap=cap, driver_slew=slew,
                sink_count=cnt)


def net_sizes(seed, num_nets, lo=2, hi=4096):
    """Log-uniform net sizes in [lo, hi] (seeded), as nodes_start (numpy)."""
    rng = np.random.default_rng(seed)
    u = rng.random(num_nets)
    n = np.floor(np.exp(np.log(lo) + u * (np.log(hi + 1) - np.log(lo)))).astype(np.int64)
    n = np.clip(n, lo, hi)
    ns = np.zeros(num_nets + 1, np.int64)
    ns[1:] = np.cumsum(n)
    assert ns[-1] < 2 ** 31
    return ns.astype(np.int32)
