"""ctypes bindings for the CPU oracle (liboracle.so) and the reference-code
harness (oracle/_ref/libotref.so).  TEST INFRASTRUCTURE ONLY: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU legs, never by the
opentimer_b200 product path.

Array conventions match the flat RC layout of OpenTimer's FlatRctStorage
(ot/timer/net.hpp:149-166): nodes_start[N+1]; edges[E][2] (local ids, edge
order = SPEF *RES order); roots[N]; res[E]; cap[V][4]; per-node outputs
[V][4] with corner c = split*2 + tran.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libotref.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

_oracle = None
_ref = None


def build(ref=True):
    """Compile liboracle.so (and the reference harness when the reference
    tree is present).  Returns True when libotref.so is available."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    refdir = os.environ.get("OTG_REFERENCE_DIR", "/root/reference")
    if ref and os.path.isdir(os.path.join(refdir, "ot")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + refdir, "-j8"], check=True)
        # the whole reference Timer, linked with the reference CUDA module
        # and with libotg (needs opentimer_b200/libotg.so built first)
        if os.path.exists(os.path.join(HERE, "..", "opentimer_b200", "libotg.so")):
            subprocess.run(["make", "-s", "-C", HERE, "timer", "REF=" + refdir, "-j8"],
                           check=True)
    return os.path.exists(LIB_REF)


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(LIB_ORACLE):
            build(ref=False)
        lib = ctypes.CDLL(LIB_ORACLE)
        I, P, F, D = ctypes.c_int, _i32p, _f32p, _f64p
        lib.oracle_rc_bfs.argtypes = [I, P, P, P, P, P, ctypes.c_void_p]
        lib.oracle_rc_bfs.restype = I
        lib.oracle_rc_prepare.argtypes = [I, P, P, P, F, F, F, F]
        lib.oracle_rc_prepare.restype = None
        lib.oracle_rc_elmore_flat_f32.argtypes = [I, P, P, F, F, F, F, F, F]
        lib.oracle_rc_elmore_flat_f32.restype = None
        lib.oracle_rc_elmore_cpu_f32.argtypes = [I, P, P, P, F, F, F, F, F, F]
        lib.oracle_rc_elmore_cpu_f32.restype = I
        lib.oracle_rc_elmore_f64.argtypes = [I, P, P, P, F, F, D, D, D, D]
        lib.oracle_rc_elmore_f64.restype = I
        lib.oracle_sink_slew.argtypes = [I, P, P, P, F, F, F]
        lib.oracle_sink_slew.restype = None
        lib.oracle_levelize.argtypes = [I, P, P, P, P, I, P, P, P, P]
        lib.oracle_levelize.restype = I
        lib.oracle_synth_rc_forest.argtypes = [ctypes.c_uint64, I, I, P, P, P, F, F, F, P, I]
        lib.oracle_synth_rc_forest.restype = I
        _oracle = lib
    return _oracle


def ref_available():
    return os.path.exists(LIB_REF)


def ref_lib():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(LIB_REF)
        I, P, F = ctypes.c_int, _i32p, _f32p
        lib.otref_rct_update.argtypes = [I, P, P, P, F, F, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, I]
        lib.otref_rct_update.restype = I
        lib.otref_rct_bfs_and_compute_cuda.argtypes = [I, I, P, P, P, F, F, P, P, F, F, F, F]
        lib.otref_rct_bfs_and_compute_cuda.restype = None
        lib.otref_toposort_levels_cuda.argtypes = [I, I, I, P, P, P, P, P, I]
        lib.otref_toposort_levels_cuda.restype = I
        lib.otref_spef_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(I), ctypes.POINTER(I)]
        lib.otref_spef_load.restype = I
        lib.otref_spef_fetch.argtypes = [P, P, P, F, F]
        lib.otref_spef_fetch.restype = None
        lib.otref_launch_timing_begin.argtypes = []
        lib.otref_launch_timing_begin.restype = None
        lib.otref_launch_timing_end.argtypes = [ctypes.POINTER(ctypes.c_double)]
        lib.otref_launch_timing_end.restype = I
        _ref = lib
    return _ref


class Forest:
    """A flat RC forest (host arrays)."""

    def __init__(self, nodes_start, edges, roots, res, cap):
        self.nodes_start = np.ascontiguousarray(nodes_start, dtype=np.int32)
        self.edges = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 2)
        self.roots = np.ascontiguousarray(roots, dtype=np.int32)
        self.res = np.ascontiguousarray(res, dtype=np.float32)
        self.cap = np.ascontiguousarray(cap, dtype=np.float32).reshape(-1, 4)

    @property
    def num_nets(self):
        return len(self.roots)

    @property
    def total_nodes(self):
        return int(self.nodes_start[-1])

    def copy(self):
        return Forest(self.nodes_start.copy(), self.edges.copy(), self.roots.copy(),
                      self.res.copy(), self.cap.copy())


def bfs(f):
    """Reference BFS flattening rule.  Returns (status, directed_edges,
    node2bfs, pid, depth)."""
    lib = oracle_lib()
    e = f.edges.copy()
    V = f.total_nodes
    node2bfs = np.zeros(V, np.int32)
    pid = np.zeros(V, np.int32)
    depth = np.zeros(V, np.int32)
    st = lib.oracle_rc_bfs(f.num_nets, f.nodes_start, f.roots, e.reshape(-1), node2bfs, pid,
                           depth.ctypes.data)
    return st, e, node2bfs, pid, depth


def prepare(f, directed_edges, node2bfs):
    V = f.total_nodes
    pres = np.zeros(V, np.float32)
    capb = np.zeros((V, 4), np.float32)
    oracle_lib().oracle_rc_prepare(f.num_nets, f.nodes_start, directed_edges.reshape(-1),
                                   node2bfs, f.res, f.cap.reshape(-1), pres, capb.reshape(-1))
    return pres, capb


def elmore_flat_f32(f, pid, pres, cap_bfs):
    V = f.total_nodes
    outs = [np.zeros((V, 4), np.float32) for _ in range(4)]
    oracle_lib().oracle_rc_elmore_flat_f32(f.num_nets, f.nodes_start, pid, pres,
                                           cap_bfs.reshape(-1), *[o.reshape(-1) for o in outs])
    return outs


def elmore_cpu_f32(f):
    """Reference CPU summation order, fp32, outputs by local id."""
    V = f.total_nodes
    outs = [np.zeros((V, 4), np.float32) for _ in range(4)]
    st = oracle_lib().oracle_rc_elmore_cpu_f32(f.num_nets, f.nodes_start, f.edges.reshape(-1),
                                               f.roots, f.res, f.cap.reshape(-1),
                                               *[o.reshape(-1) for o in outs])
    return st, outs


def elmore_f64(f):
    V = f.total_nodes
    outs = [np.zeros((V, 4), np.float64) for _ in range(4)]
    st = oracle_lib().oracle_rc_elmore_f64(f.num_nets, f.nodes_start, f.edges.reshape(-1),
                                           f.roots, f.res, f.cap.reshape(-1),
                                           *[o.reshape(-1) for o in outs])
    return st, outs


def sink_slew(f, sinks_start, sink_nodes, driver_slew, impulse_local):
    out = np.zeros((len(sink_nodes), 4), np.float32)
    oracle_lib().oracle_sink_slew(f.num_nets, f.nodes_start,
                                  np.ascontiguousarray(sinks_start, np.int32),
                                  np.ascontiguousarray(sink_nodes, np.int32),
                                  np.ascontiguousarray(driver_slew, np.float32).reshape(-1),
                                  np.ascontiguousarray(impulse_local, np.float32).reshape(-1),
                                  out.reshape(-1))
    return out


def levelize(n, fanin_start, fanin, out_deg, frontier0):
    fanin_start = np.ascontiguousarray(fanin_start, np.int32)
    fanin = np.ascontiguousarray(fanin, np.int32)
    if fanin.size == 0:
        fanin = np.zeros(1, np.int32)
    out_deg = np.ascontiguousarray(out_deg, np.int32)
    frontier0 = np.ascontiguousarray(frontier0, np.int32)
    f0 = frontier0 if frontier0.size else np.zeros(1, np.int32)
    order = np.zeros(max(n, 1), np.int32)
    ends = np.zeros(n + 2, np.int32)
    nl = np.zeros(1, np.int32)
    level = np.zeros(max(n, 1), np.int32)
    cnt = oracle_lib().oracle_levelize(n, fanin_start, fanin, out_deg, f0, int(frontier0.size),
                                       order, ends, nl, level)
    L = int(nl[0])
    return order[:cnt], ends[:L + 1], level[:n]


def synth_forest(seed, nodes_start, first_net=0, threads=None):
    """Nets first_net.. of the seeded batched-Elmore workload, generated on
    the host (synth_host.c: bit-identical to the product library's
    generator).  nodes_start holds the slice's node offsets (any base).
    Returns (Forest, driver_slew [N][4], sink_count [N])."""
    ns = np.ascontiguousarray(nodes_start, np.int64)
    ns = (ns - ns[0]).astype(np.int32)
    N = len(ns) - 1
    V = int(ns[-1])
    e = np.zeros((max(V - N, 1), 2), np.int32)
    roots = np.zeros(max(N, 1), np.int32)
    res = np.zeros(max(V - N, 1), np.float32)
    cap = np.zeros((max(V, 1), 4), np.float32)
    slew = np.zeros((max(N, 1), 4), np.float32)
    cnt = np.zeros(max(N, 1), np.int32)
    st = oracle_lib().oracle_synth_rc_forest(seed, int(first_net), N, ns, e.reshape(-1), roots,
                                             res, cap.reshape(-1), slew.reshape(-1), cnt,
                                             int(threads or os.cpu_count() or 1))
    if st != 0:
        raise MemoryError("oracle_synth_rc_forest")
    f = Forest(ns, e[:V - N], roots[:N], res[:V - N], cap[:V])
    return f, slew[:N], cnt[:N]


def to_local(f, node2bfs, arr_bfs):
    """Permute a [V][4] BFS-ordered array to local-id order."""
    b = np.repeat(f.nodes_start[:-1], np.diff(f.nodes_start))
    return arr_bfs[b + node2bfs]


# ---------------------------------------------------------------- reference

def ref_rct_update(f, num_threads=0, readback=True):
    """The reference's own CPU path (ot::Rct).  Outputs by local id."""
    lib = ref_lib()
    V = f.total_nodes
    outs = [np.zeros((V, 4), np.float32) for _ in range(4)] if readback else None
    ptrs = [o.ctypes.data for o in outs] if readback else [None] * 4
    st = lib.otref_rct_update(f.num_nets, f.nodes_start, f.edges.reshape(-1), f.roots, f.res,
                              f.cap.reshape(-1), *ptrs, num_threads)
    return st, outs


def ref_rct_gpu(f, timing=None):
    """The reference's own GPU path (needs a GPU).  Returns directed edges,
    node2bfs, pid and the four outputs in BFS order.  With a dict `timing`,
    its kernels' device time is recorded into it (CUDA events around each
    of its launches: "kernel_ms", "launches") next to the whole call's wall
    time ("call_s", host arrays in and out, as the Timer calls it)."""
    import time
    lib = ref_lib()
    V = f.total_nodes
    ns = f.nodes_start.copy()
    e = f.edges.copy()
    roots = f.roots.copy()
    res = f.res.copy()
    cap = f.cap.copy()
    node2bfs = np.zeros(V, np.int32)
    pid = np.zeros(V, np.int32)
    outs = [np.zeros((V, 4), np.float32) for _ in range(4)]
    if timing is not None:
        lib.otref_launch_timing_begin()
    t0 = time.perf_counter()
    lib.otref_rct_bfs_and_compute_cuda(f.num_nets, V, ns, e.reshape(-1), roots, res,
                                       cap.reshape(-1), node2bfs, pid,
                                       *[o.reshape(-1) for o in outs])
    if timing is not None:
        timing["call_s"] = time.perf_counter() - t0
        ms = ctypes.c_double()
        timing["launches"] = lib.otref_launch_timing_end(ctypes.byref(ms))
        timing["kernel_ms"] = ms.value
    return e, node2bfs, pid, outs


def ref_toposort_gpu(n, fanin_start, fanin, out_deg, frontier0):
    """Levels from the reference's own toposort_advance kernel (needs a GPU)."""
    lib = ref_lib()
    fs = np.ascontiguousarray(fanin_start, np.int32).copy()
    fi = np.ascontiguousarray(fanin, np.int32).copy()
    if fi.size == 0:
        fi = np.zeros(1, np.int32)
    out = np.ascontiguousarray(out_deg, np.int32).copy()
    fr = np.zeros(max(n, 1), np.int32)
    fr[:len(frontier0)] = frontier0
    ends = np.zeros(n + 2, np.int32)
    k = lib.otref_toposort_levels_cuda(n, int(len(fanin)), int(len(frontier0)), fs, fi, out, fr,
                                       ends, n + 2)
    if k < 0:
        raise RuntimeError("reference toposort_advance run failed")
    return fr, ends[:k]


def ref_spef_forest(path):
    lib = ref_lib()
    nn = ctypes.c_int()
    nv = ctypes.c_int()
    st = lib.otref_spef_load(path.encode(), ctypes.byref(nn), ctypes.byref(nv))
    if st != 0:
        raise RuntimeError(f"otref_spef_load({path}) failed: {st}")
    N, V = nn.value, nv.value
    ns = np.zeros(N + 1, np.int32)
    e = np.zeros((V - N, 2), np.int32)
    roots = np.zeros(N, np.int32)
    res = np.zeros(V - N, np.float32)
    cap = np.zeros((V, 4), np.float32)
    lib.otref_spef_fetch(ns, e.reshape(-1), roots, res, cap.reshape(-1))
    return Forest(ns, e, roots, res, cap)
