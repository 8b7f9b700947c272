"""GPU timing propagation (otg_propagate) on the small synthetic design,
fed only by this library: the SPEF reader, the fused RC pass and the
propagation kernels, over the timing graph the reference Timer builds
(exported by oracle/_ref/ot_run_ref: pins, arcs, Liberty timing records and
look-up tables, timing tests, assertions).  Every pin's arrival time, slew,
required time and slack, four corners, must match the reference Timer's own
update_timing, on its CUDA path and on its CPU path, within
|ours - ref| <= 1e-5 s + 1e-5 (ns), s = |ref| for arrival time and slew;
required time and slack are differences of path-length quantities, so
their rounding scales with the arrival time: s = max(|ref|, |ref at|).
What the reference leaves empty must be empty here (NaN)."""
import os
import subprocess

import numpy as np
import pytest

from opentimer_b200 import designgen
import opentimer_b200 as otg

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE_REF = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")
RTOL, ATOL = 1e-5, 1e-5


def ref_run(d, mode, graph=None):
    out = os.path.join(d, f"ref_{mode}.txt")
    cmd = [EXE_REF, d, mode, out] + ([graph] if graph else [])
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    pins, pin_cap = {}, {}
    with open(out) as f:
        for line in f:
            t = line.split()
            if t[0] == "P":
                pins[t[1]] = np.array([float(x) for x in t[2:]], np.float64).reshape(4, 4)
            elif t[0] == "K":
                pin_cap[t[1]] = np.array([float(x) for x in t[2:]], np.float32)
    return pins, pin_cap


def parse_graph(path):
    g = {"pins": [], "arcs": [], "tests": [], "timing": [], "luts": [], "period": np.nan}
    with open(path) as f:
        for line in f:
            t = line.split()
            if t[0] == "p":
                v = [float(x) for x in t[4:]]
                g["pins"].append((int(t[1]), t[2], t[3], v[0:4], v[4:8], v[8:12]))
            elif t[0] == "a":
                g["arcs"].append((int(t[1]), int(t[2]), int(t[3]), int(t[4]), t[5], t[6],
                                  int(t[7]), int(t[8])))
            elif t[0] == "s":
                g["tests"].append(int(t[1]))
            elif t[0] == "t":
                g["timing"].append([int(x) for x in t[2:11]])
            elif t[0] == "l":
                var, n1, n2 = int(t[2]), int(t[3]), int(t[4])
                g["luts"].append((var, n1, n2, np.array([float(x) for x in t[5:]], np.float32)))
            elif t[0] == "c":
                g["period"] = float(t[1])
    return g


@pytest.fixture(scope="module")
def design(tmp_path_factory, cuda):
    if not os.path.exists(EXE_REF):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    d = str(tmp_path_factory.mktemp("prop"))
    designgen.write_design(d, seed=2024, gates=2000)
    graph = os.path.join(d, "graph.txt")
    ref_gpu, pin_cap = ref_run(d, "cuda", graph)
    ref_cpu, _ = ref_run(d, "cpu")
    return d, parse_graph(graph), pin_cap, ref_gpu, ref_cpu


def our_timing(d, G, pin_cap):
    import torch
    from opentimer_b200.prop import TimingGraph
    from opentimer_b200.spef import read_spef
    # RC: SPEF -> flat layout (+ library pin caps on non-root pins) -> RC pass
    f = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    ns, ps = f["nodes_start"], f["pins_start"]
    net_idx = {n: i for i, n in enumerate(f["net_names"])}
    node_of = {}
    cap = f["cap"].copy()
    for i in range(len(ns) - 1):
        for q in range(ps[i], ps[i + 1]):
            node = int(f["pin_node"][q])
            name = f["pin_names"][q]
            node_of[(i, name)] = node  # local id in the net
            if node != f["roots"][i]:
                cap[int(ns[i]) + node] += pin_cap[name]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    batch = otg.RcBatch(t(ns), t(f["edges"].copy()), t(f["roots"]), t(f["res"]), t(cap))
    batch.run()
    batch.check()
    # the timing graph
    P = len(G["pins"])
    name = [None] * P
    pin_net = [None] * P
    pi_at, pi_slew, po_rat = (np.full((P, 4), np.nan, np.float32) for _ in range(3))
    for idx, nm, net, a, s, r in G["pins"]:
        name[idx], pin_net[idx] = nm, net
        pi_at[idx], pi_slew[idx], po_rat[idx] = a, s, r
    A = len(G["arcs"])
    arr = {k: np.full(A, -1, np.int32) for k in ("arc_from", "arc_to", "arc_kind", "arc_net",
                                                  "arc_node")}
    arc_timing = np.full((A, 2), -1, np.int32)
    for k, fr, to, state, kind, net, tmin, tmax in G["arcs"]:
        assert state == 0  # no loop breakers in a DAG
        arr["arc_from"][k], arr["arc_to"][k] = fr, to
        if kind == "net":
            arr["arc_kind"][k] = 0
            i = net_idx[net]
            arr["arc_net"][k] = i
            arr["arc_node"][k] = node_of.get((i, name[to]), -1)
        else:
            arr["arc_kind"][k] = 1
            arc_timing[k] = (tmin, tmax)
            arr["arc_net"][k] = net_idx.get(pin_net[to], -1)
    meta, data, off = [], [], 0
    for var, n1, n2, vals in G["luts"]:
        meta.append((n1, n2, off, var))
        data.append(vals)
        off += len(vals)
    graph = TimingGraph(dict(arr, num_pins=P, arc_timing=arc_timing,
                             test_arc=np.array(G["tests"], np.int32), pi_at=pi_at,
                             pi_slew=pi_slew, po_rat=po_rat,
                             timing=np.array(G["timing"], np.int32),
                             lut_meta=np.array(meta, np.int32), lut_data=np.concatenate(data),
                             period=G["period"]))
    out = graph.propagate(batch).result()
    # report_rat answers only where the pin has an arrival time (timer.cpp:1657-1663)
    out["rat"] = np.where(np.isnan(out["at"]), np.nan, out["rat"])
    return name, out, graph.num_levels


def compare(name, out, ref):
    worst = {}
    for q, k in enumerate(("at", "slew", "rat", "slack")):
        w = 0.0
        for i, nm in enumerate(name):
            r, g = ref[nm][q], out[k][i].astype(np.float64)
            assert np.array_equal(np.isnan(r), np.isnan(g)), (nm, k, r, g)
            m = ~np.isnan(r)
            scale = np.abs(r)
            if q >= 2:
                scale = np.maximum(scale, np.nan_to_num(np.abs(ref[nm][0])))
            if m.any():
                w = max(w, float(np.max(np.abs(g[m] - r[m]) / (RTOL * scale[m] + ATOL))))
        worst[k] = w
    return worst


def test_propagation_matches_reference_timer(design):
    d, G, pin_cap, ref_gpu, ref_cpu = design
    name, out, levels = our_timing(d, G, pin_cap)
    w_gpu = compare(name, out, ref_gpu)
    w_cpu = compare(name, out, ref_cpu)
    print(f"propagation over {len(name)} pins, {levels} levels: err/tol vs reference GPU path "
          f"{w_gpu}, vs CPU path {w_cpu}")
    assert max(w_gpu.values()) <= 1.0 and max(w_cpu.values()) <= 1.0
    assert np.isfinite(out["slack"]).sum() > 10000


def test_own_graph_matches_reference_timer(design, tmp_path):
    """The same check with nothing from the reference on the input side:
    the design's timing graph as the generator builds it by the Timer's
    construction rules (designgen.timing_graph), the library pin caps from
    the generator, the SPEF reader, the RC pass and the propagation."""
    import torch
    from opentimer_b200 import designgen
    from opentimer_b200.prop import TimingGraph, attach_nets, rc_inputs
    from opentimer_b200.spef import read_spef
    _, _, _, ref_gpu, ref_cpu = design
    keep = {}
    d = str(tmp_path)
    designgen.write_design(d, seed=2024, gates=2000, keep=keep)
    arrays, names, nets = designgen.timing_graph(keep)
    f = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    cap, node_of = rc_inputs(f, designgen.pin_caps(keep))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    batch = otg.RcBatch(t(f["nodes_start"]), t(f["edges"].copy()), t(f["roots"]), t(f["res"]),
                        t(cap))
    batch.run()
    batch.check()
    g = TimingGraph(attach_nets(arrays, names, nets, f, node_of))
    out = g.propagate(batch).result()
    out["rat"] = np.where(np.isnan(out["at"]), np.nan, out["rat"])
    w_gpu = compare(names, out, ref_gpu)
    w_cpu = compare(names, out, ref_cpu)
    print(f"own graph: err/tol vs reference GPU path {w_gpu}, vs CPU path {w_cpu}")
    assert max(w_gpu.values()) <= 1.0 and max(w_cpu.values()) <= 1.0


def _chain_graph(cyclic):
    """Two pins joined by net arcs without RC nodes: 0 -> 1, plus 1 -> 0
    when cyclic.  Pin 0 carries PI assertions."""
    arcs = [(0, 1), (1, 0)] if cyclic else [(0, 1)]
    A = len(arcs)
    nan4 = np.full((2, 4), np.nan, np.float32)
    pi_at, pi_slew = nan4.copy(), nan4.copy()
    pi_at[0], pi_slew[0] = 1.0, 2.0
    return dict(num_pins=2, arc_from=np.array([f for f, _ in arcs], np.int32),
                arc_to=np.array([t for _, t in arcs], np.int32), arc_kind=np.zeros(A, np.int32),
                arc_timing=np.full((A, 2), -1, np.int32), arc_net=np.full(A, -1, np.int32),
                arc_node=np.full(A, -1, np.int32), test_arc=np.zeros(0, np.int32),
                pi_at=pi_at, pi_slew=pi_slew, po_rat=nan4.copy(),
                timing=np.zeros((0, 9), np.int32), lut_meta=np.zeros((0, 4), np.int32),
                lut_data=np.zeros(0, np.float32), period=np.nan)


def test_bounded_wait_gives_up_on_a_cycle(cuda):
    """A pin order that breaks the dataflow rule (here a two-pin cycle, so
    each pin waits on the other) ends every wait after the 2 s limit with
    OTG_ERR_TIMEOUT; the context stays usable for the next propagation."""
    import time
    import torch
    from opentimer_b200.prop import TimingGraph
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    batch = otg.RcBatch(t(np.array([0, 2], np.int32)), t(np.array([[0, 1]], np.int32)),
                        t(np.zeros(1, np.int32)), t(np.ones(1, np.float32)),
                        t(np.ones((2, 4), np.float32)))
    batch.run()
    batch.check()
    g = TimingGraph(_chain_graph(True), order=np.array([1, 0], np.int32))
    t0 = time.time()
    g.propagate(batch)
    with pytest.raises(otg.OtgError) as e:
        g.check()
    assert e.value.code == 6  # OTG_ERR_TIMEOUT
    assert time.time() - t0 < 30
    out = TimingGraph(_chain_graph(False)).propagate(batch).result()
    assert np.all(out["at"][0] == 1.0) and np.all(out["slew"][0] == 2.0)
    assert np.all(np.isnan(out["at"][1]))  # a net arc without an RC node carries nothing


def test_forward_order_from_sources_is_identical(design, tmp_path):
    """The forward pass may take its pins by distance from the sources
    (fwd_order, a second levelization) instead of the backward order
    reversed: every pin's results are the same bits."""
    import torch
    from opentimer_b200 import designgen
    from opentimer_b200.prop import TimingGraph, attach_nets, rc_inputs
    from opentimer_b200.spef import read_spef
    keep = {}
    d = str(tmp_path)
    designgen.write_design(d, seed=2024, gates=2000, keep=keep)
    arrays, names, nets = designgen.timing_graph(keep)
    f = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    cap, node_of = rc_inputs(f, designgen.pin_caps(keep))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    batch = otg.RcBatch(t(f["nodes_start"]), t(f["edges"].copy()), t(f["roots"]), t(f["res"]),
                        t(cap))
    batch.run()
    batch.check()
    att = attach_nets(arrays, names, nets, f, node_of)
    a = TimingGraph(att, forward="sinks").propagate(batch).result()
    gs = TimingGraph(att, forward="sources")
    assert gs.fwd_order is not None
    b = gs.propagate(batch).result()
    for k in ("at", "slew", "rat", "slack"):
        assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k
