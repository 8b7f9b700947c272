"""Incremental SPEF ingestion (a TAU15-style change SPEF) on the device.

The reference re-attaches the parasitics of every net the change file
names (Timer::_read_spef, ot/timer/spef.cpp:40-53) and re-times on the next
update_timing.  Here RcBatch.replace_nets moves the unchanged nets, with
their results, into a new layout (otg_rc_move_nets), moves the changed
nets' new trees in, and re-times only those (otg_rc_timing_subset).

* The result equals a full pass over the final forest, bit for bit.
* RC values at every pin node and every pin's AT/slew/RAT/slack match the
  reference Timer after read_spef(change) + update_timing, in two runs: one
  whose first full update took its CPU path and one whose first full update
  took its CUDA path (RC: 1e-5 relative with a 1e-6 x net-max floor; pins:
  the propagation tolerance of test_prop_gpu).  The incremental update
  itself takes the Timer's CPU path in both runs: the Timer clears all its
  state bits, CUDA_ENABLED among them, at the end of every update
  (_remove_state() in Timer::_update_timing, ot/timer/timer.cpp), and the
  reference's CUDA kernels are not run on the zeroed clean nets that a
  second CUDA update would hand them.
"""
import os
import subprocess

import numpy as np
import pytest

import opentimer_b200 as otg
from opentimer_b200 import designgen

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE_REF = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")


def ref_run(d, mode, change):
    out = os.path.join(d, f"ref_{mode}.txt")
    p = subprocess.run([EXE_REF, d, mode, out, f"change={change}"], capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "incremental_update_timing_s" in p.stdout
    pins, rc = {}, {}
    with open(out) as f:
        for line in f:
            t = line.split()
            if t[0] == "P":
                pins[t[1]] = np.array([float(x) for x in t[2:]], np.float64).reshape(4, 4)
            elif t[0] == "R":
                rc[(t[1], t[2])] = np.array([float(x) for x in t[3:]], np.float64).reshape(4, 4)
    return pins, rc


@pytest.fixture(scope="module")
def design(tmp_path_factory, cuda):
    if not os.path.exists(EXE_REF):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    d = str(tmp_path_factory.mktemp("incr"))
    keep = {}
    designgen.write_design(d, seed=2024, gates=2000, keep=keep)
    change = os.path.join(d, "change.spef")
    names = designgen.change_spef(keep, change, frac=0.05, seed=7)
    return d, keep, change, names, ref_run(d, "cpu", change), ref_run(d, "cuda", change)


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ours(d, keep, change):
    from opentimer_b200.prop import change_nets, rc_inputs
    from opentimer_b200.spef import read_spef
    caps = designgen.pin_caps(keep)
    f0 = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    cap0, node_of0 = rc_inputs(f0, caps)
    b0 = otg.RcBatch(_t(f0["nodes_start"]), _t(f0["edges"].copy()), _t(f0["roots"]),
                     _t(f0["res"]), _t(cap0))
    b0.run()
    b0.check()
    index = {n: i for i, n in enumerate(f0["net_names"])}
    fc = read_spef(change, r_scale=np.float32(1e-3))
    nets, forest, node_of_c = change_nets(fc, index, caps)
    b1 = b0.replace_nets(nets, *forest)
    b1.check()
    return f0, cap0, node_of0, b0, nets, forest, node_of_c, b1


def test_replace_nets_equals_a_full_pass(design):
    d, keep, change, names, _, _ = design
    f0, cap0, _, _, nets, forest, _, b1 = _ours(d, keep, change)
    assert len(nets) == len(names) > 50
    # the final forest on the host, from the original (undirected) inputs
    ns0 = f0["nodes_start"]
    sub_ns, sub_e, sub_roots, sub_res, sub_cap = forest
    where = {int(n): k for k, n in enumerate(nets)}
    parts = {k: [] for k in ("e", "res", "cap", "root", "size")}
    for i in range(len(ns0) - 1):
        if i in where:
            k = where[i]
            a, b = int(sub_ns[k]), int(sub_ns[k + 1])
            parts["e"].append(sub_e[a - k:b - k - 1])
            parts["res"].append(sub_res[a - k:b - k - 1])
            parts["cap"].append(sub_cap[a:b])
            parts["root"].append(sub_roots[k])
            parts["size"].append(b - a)
        else:
            a, b = int(ns0[i]), int(ns0[i + 1])
            parts["e"].append(f0["edges"][a - i:b - i - 1])
            parts["res"].append(f0["res"][a - i:b - i - 1])
            parts["cap"].append(cap0[a:b])
            parts["root"].append(f0["roots"][i])
            parts["size"].append(b - a)
    ns = np.zeros(len(parts["size"]) + 1, np.int32)
    ns[1:] = np.cumsum(parts["size"])
    full = otg.RcBatch(_t(ns), _t(np.concatenate(parts["e"])), _t(np.array(parts["root"], np.int32)),
                       _t(np.concatenate(parts["res"])), _t(np.concatenate(parts["cap"])))
    full.run()
    full.check()
    assert np.array_equal(b1.nodes_start.cpu().numpy(), ns)
    for k in ("node2bfs", "edges", "load", "delay", "ldelay", "impulse"):
        assert np.array_equal(getattr(b1, k).cpu().numpy(), getattr(full, k).cpu().numpy()), k
    # pid is defined on non-root slots (the root's entry is 0 on both sides)
    assert np.array_equal(b1.pid.cpu().numpy(), full.pid.cpu().numpy())


def test_incremental_update_matches_reference_timer(design):
    from opentimer_b200.prop import TimingGraph, attach_nets
    d, keep, change, names, (ref_cpu, rc_cpu), (ref_cuda, rc_cuda) = design
    f0, _, node_of0, b0, nets, _, node_of_c, b1 = _ours(d, keep, change)
    arrays, pin_names, pin_nets = designgen.timing_graph(keep)
    g = TimingGraph(attach_nets(arrays, pin_names, pin_nets, f0, node_of0))
    g.propagate(b0)
    g.check()
    # arcs into the changed nets point at their sinks' new local ids
    changed = set(int(n) for n in nets)
    arcs, nodes = [], []
    index = {n: j for j, n in enumerate(f0["net_names"])}
    for k in range(len(arrays["arc_from"])):
        if arrays["arc_kind"][k] != 0:
            continue
        i = index[arrays["arc_net_name"][k]]
        if i in changed:
            arcs.append(k)
            nodes.append(node_of_c.get((i, pin_names[int(arrays["arc_to"][k])]), -1))
    assert arcs
    # the graph's own mapping (what a caller uses) agrees and applies it
    got_arcs, got_nodes = g.change_nets(nets, node_of_c, pin_names)
    assert got_arcs.tolist() == arcs and got_nodes == nodes
    out = g.propagate(b1).result()
    out["rat"] = np.where(np.isnan(out["at"]), np.nan, out["rat"])
    # RC at every pin node, all nets (changed and moved)
    ns = b1.nodes_start.cpu().numpy()
    n2b = b1.node2bfs.cpu().numpy()
    q = np.stack([getattr(b1, k).cpu().numpy() for k in ("load", "delay", "ldelay", "impulse")],
                 axis=1)
    node_of = dict(node_of0)
    for (i, pin), node in list(node_of.items()):
        if i in changed:
            del node_of[(i, pin)]
    node_of.update(node_of_c)
    for rc_ref in (rc_cpu, rc_cuda):
        worst, by_net = 0.0, {}
        for (i, pin), node in node_of.items():
            r = rc_ref[(f0["net_names"][i], pin)]
            got = q[ns[i] + n2b[ns[i] + node]].astype(np.float64)
            by_net.setdefault(i, []).append((got, r))
        for i, rows in by_net.items():
            gs, rs = np.stack([x for x, _ in rows]), np.stack([y for _, y in rows])
            tol = 1e-5 * np.abs(rs) + 1e-6 * np.abs(rs).max(axis=0, keepdims=True)
            e = np.abs(gs - rs)
            worst = max(worst, float(np.max(np.where(tol > 0, e / np.maximum(tol, 1e-30),
                                                     e * 1e30))))
        assert worst <= 1.0, worst
    # every pin, against both reference paths
    for ref in (ref_cpu, ref_cuda):
        worst = 0.0
        for idx, nm in enumerate(pin_names):
            r = ref[nm]
            gq = np.stack([out[k][idx] for k in ("at", "slew", "rat", "slack")]).astype(np.float64)
            assert np.array_equal(np.isnan(r), np.isnan(gq)), nm
            scale = np.abs(r)
            scale[2:] = np.maximum(scale[2:], np.nan_to_num(np.abs(r[0])))
            m = ~np.isnan(r)
            if m.any():
                worst = max(worst, float(np.max(np.abs(gq[m] - r[m]) / (1e-5 * scale[m] + 1e-5))))
        assert worst <= 1.0, worst


def test_empty_change_and_bad_move(cuda):
    """Replacing no net keeps every result bit for bit; a move whose source
    net index is out of range is skipped and reported (OTG_ERR_INVALID),
    never read."""
    import ctypes
    import torch
    from opentimer_b200 import synth_forest, workloads
    from opentimer_b200._lib import lib
    ns = torch.from_numpy(workloads.net_sizes(9, 300, 2, 300)).cuda()
    g = synth_forest(9, ns, with_sinks=False)
    b0 = otg.RcBatch(ns, g["edges"], g["roots"], g["res"], g["cap"])
    b0.run()
    b0.check()
    empty = (np.zeros(1, np.int32), np.zeros((0, 2), np.int32), np.zeros(0, np.int32),
             np.zeros(0, np.float32), np.zeros((0, 4), np.float32))
    b1 = b0.replace_nets([], *empty)
    b1.check()
    for k in ("nodes_start", "edges", "node2bfs", "pid", "load", "delay", "ldelay", "impulse"):
        assert torch.equal(getattr(b0, k), getattr(b1, k)), k
    # a source index past the source forest: skipped and flagged
    bad = torch.full((b0.num_nets,), -1, dtype=torch.int32, device="cuda")
    bad[0] = b0.num_nets + 5
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    before = b1.load.clone()
    code = lib().otg_rc_move_nets(ctypes.byref(b0._forest), ctypes.byref(b1._forest),
                                  ctypes.c_void_p(bad.data_ptr()), 1,
                                  ctypes.c_void_p(status.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert code == 0 and int(status.item()) == 1  # OTG_ERR_INVALID
    assert torch.equal(before, b1.load)
