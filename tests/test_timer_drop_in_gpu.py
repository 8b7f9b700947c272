"""Full update_timing on a small synthetic design: the reference OpenTimer
Timer, unchanged, with libotg linked in place of its CUDA module, against
the same Timer with the reference's own CUDA kernels and against its CPU
path.  This is the drop-in: Timer::update_timing (ot/timer/timer.cpp:1239)
calls rct_bfs_and_compute_cuda and toposort_compute_cuda, which resolve to
libotg in oracle/_ref/ot_run_otg.

* BFS slot and pid of every RC node: bit-exact with the reference kernels.
* load/delay/ldelay/impulse of every RC node, 4 corners: within the RC
  tolerance (1e-5 relative, floor 1e-6 x the net's max |value|).
* arrival time, slew, required time and slack of every pin, 4 corners:
  |ours - ref| <= 1e-5 s + 1e-5 (library time unit: ns), NaN where the
  reference has none; s = |ref| for arrival time and slew, max(|ref|,
  |ref at|) for required time and slack, which are differences of
  path-length quantities.  Each of the design's thousands of timing arcs
  turns the RC values into delays through the same NLDM tables, so the
  RC differences carry over at the same relative size.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from opentimer_b200 import designgen

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE_REF = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")
EXE_OTG = os.path.join(ROOT, "oracle", "_ref", "ot_run_otg")
PIN_RTOL, PIN_ATOL = 1e-5, 1e-5


def run(exe, d, mode):
    out = os.path.join(d, f"{os.path.basename(exe)}_{mode}.txt")
    p = subprocess.run([exe, d, mode, out], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "cannot" not in p.stderr and " E " not in p.stderr, p.stderr[-2000:]
    P, R, B, S = {}, {}, {}, {"pin_cap": {}, "root": {}, "edges": {}, "cap": {}}
    with open(out) as f:
        for line in f:
            t = line.split()
            if t[0] == "P":
                P[t[1]] = np.array([float(x) for x in t[2:]], np.float64)
            elif t[0] == "R":
                R[(t[1], t[2])] = np.array([float(x) for x in t[3:]], np.float64)
            elif t[0] == "B":
                B[(t[1], t[2])] = (int(t[3]), int(t[4]))
            elif t[0] == "K":
                S["pin_cap"][t[1]] = np.array([float(x) for x in t[2:]], np.float32)
            elif t[0] == "S":
                S["root"][t[1]] = int(t[3])
                S["edges"][t[1]] = []
                S["cap"][t[1]] = []
            elif t[0] == "E":
                S["edges"][t[1]].append((int(t[3]), int(t[4]), np.float32(float(t[5]))))
            elif t[0] == "C":
                S["cap"][t[1]].append(np.array([float(x) for x in t[3:]], np.float32))
    return P, R, B, S


def rc_ok(got, ref):
    """Worst err/tol over all nodes and quantities (<= 1 passes)."""
    nets = {}
    for (net, node), v in ref.items():
        nets.setdefault(net, []).append(node)
    worst = 0.0
    for net, nodes in nets.items():
        r = np.stack([ref[(net, n)] for n in nodes]).reshape(len(nodes), 4, 4)
        g = np.stack([got[(net, n)] for n in nodes]).reshape(len(nodes), 4, 4)
        floor = 1e-6 * np.abs(r).max(axis=0, keepdims=True)
        tol = 1e-5 * np.abs(r) + floor
        e = np.abs(g - r)
        worst = max(worst, float(np.max(np.where(tol > 0, e / np.maximum(tol, 1e-30), e * 1e30))))
    return worst


def pins_ok(got, ref):
    worst = 0.0
    assert set(got) == set(ref)
    for k, r in ref.items():
        g = got[k]
        assert np.array_equal(np.isnan(g), np.isnan(r)), k
        m = ~np.isnan(r)
        # [at x4, slew x4, rat x4, slack x4]
        scale = np.abs(r)
        scale[8:] = np.maximum(scale[8:], np.tile(np.nan_to_num(np.abs(r[:4])), 2))
        if m.any():
            tol = PIN_RTOL * scale[m] + PIN_ATOL
            worst = max(worst, float(np.max(np.abs(g[m] - r[m]) / tol)))
    return worst


@pytest.fixture(scope="module")
def runs(tmp_path_factory, cuda):
    if not (os.path.exists(EXE_REF) and os.path.exists(EXE_OTG)):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    d = str(tmp_path_factory.mktemp("design2k"))
    info = designgen.write_design(d, seed=2024, gates=2000)
    return (dict(info, dir=d), run(EXE_REF, d, "cuda"), run(EXE_OTG, d, "cuda"),
            run(EXE_REF, d, "cpu"))


def test_bfs_order_bit_exact(runs):
    _, ref, ours, _ = runs
    assert len(ref[2]) > 10000
    assert ours[2] == ref[2]


def test_rc_nodes_within_tolerance(runs):
    info, ref, ours, cpu = runs
    assert set(ours[1]) == set(ref[1]) == set(cpu[1])
    w_gpu = rc_ok(ours[1], ref[1])
    w_cpu = rc_ok(ours[1], cpu[1])
    print(f"2k-gate design ({info}): RC err/tol vs reference GPU {w_gpu:.3g}, vs CPU {w_cpu:.3g}")
    assert w_gpu <= 1.0 and w_cpu <= 1.0


def test_pin_timing_within_tolerance(runs):
    _, ref, ours, cpu = runs
    w_gpu = pins_ok(ours[0], ref[0])
    w_cpu = pins_ok(ours[0], cpu[0])
    w_ref = pins_ok(ref[0], cpu[0])
    print(f"pins: err/tol vs reference GPU {w_gpu:.3g}, vs CPU {w_cpu:.3g}; "
          f"reference GPU vs its CPU {w_ref:.3g}")
    assert w_gpu <= 1.0 and w_cpu <= 1.0
    slack = np.array([v[12:] for v in ours[0].values()])
    assert np.isfinite(slack).sum() > 1000 and not math.isnan(float(np.nanmin(slack)))


def test_spef_reader_matches_timer_storage(runs):
    """otg_spef_read on the design's SPEF gives the flat storage the
    reference Timer builds (read_spef + Net::_make_flat_rct): the same ids,
    edges, res and root for every net, and the same caps once each non-root
    pin's library cap is added in float, as the flat path does
    (ot/timer/net.cpp:433-446).  The Timer rebases the file's ohms to its
    kilo-ohm library unit, so the reader gets r_scale = 1e-3."""
    from opentimer_b200.spef import read_spef
    info, ref, _, _ = runs
    S = ref[3]
    f = read_spef(os.path.join(info["dir"], "design.spef"), r_scale=np.float32(1e-3))
    ns, ps = f["nodes_start"], f["pins_start"]
    assert len(f["net_names"]) == len(S["root"])
    k = 0
    for i, name in enumerate(f["net_names"]):
        b, e = int(ns[i]), int(ns[i + 1])
        eb = b - i
        assert f["roots"][i] == S["root"][name], name
        ref_edges = S["edges"][name]
        assert len(ref_edges) == e - b - 1
        for j, (s_, t_, r_) in enumerate(ref_edges):
            # the reference's edges are directed by its BFS by now
            assert {s_, t_} == {int(f["edges"][eb + j, 0]), int(f["edges"][eb + j, 1])}, name
            assert f["res"][eb + j] == r_, name
        cap = f["cap"][b:e].copy()
        for q in range(ps[i], ps[i + 1]):
            node = int(f["pin_node"][q])
            if node != f["roots"][i]:
                cap[node] = cap[node] + S["pin_cap"][f["pin_names"][q]]
        assert np.array_equal(cap, np.stack(S["cap"][name])), name
        k += e - b
    assert k == int(ns[-1]) > 10000


def test_second_cuda_update_after_repower(tmp_path, cuda):
    """The unchanged Timer's second update_timing in CUDA mode, after
    repower_gate.  Its CUDA path rebuilds the flat storage for every net but
    re-flattens only the dirty ones (ot/timer/timer.cpp:929-970,
    ot/timer/net.cpp:499-514): the clean nets reach rct_bfs_and_compute_cuda
    with zeroed edges and roots.  libotg checks every net, reports them
    (OTG_ERR_NOT_TREE, printed as "rct_bfs_and_compute_cuda: RC net is not
    a spanning tree") without reading out of range, and still
    times every re-flattened net: those nets' RC values must match the
    reference's CPU path after the same resizes."""
    if not (os.path.exists(EXE_REF) and os.path.exists(EXE_OTG)):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    from opentimer_b200.sizing import resize_trace, write_ops
    d = str(tmp_path)
    keep = {}
    designgen.write_design(d, seed=2025, gates=1500, keep=keep)
    steps = resize_trace(keep, seed=3, steps=1, per_step=30)
    ops = os.path.join(d, "ops.txt")
    write_ops(ops, steps)
    outs = {}
    for exe, mode in ((EXE_OTG, "cuda"), (EXE_REF, "cpu")):
        out = os.path.join(d, f"{os.path.basename(exe)}_{mode}_repower.txt")
        p = subprocess.run([exe, d, mode, out, f"repower={ops}"], capture_output=True, text=True,
                           timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        outs[mode] = (p.stderr, out)
    assert "rct_bfs_and_compute_cuda: RC net is not a spanning tree" in outs["cuda"][0]
    conn = {g: c for g, _, c in keep["gates"]}
    dirty = {n for g, _ in steps[0] for n in conn[g].values()}
    R = {}
    for mode in ("cuda", "cpu"):
        R[mode] = {}
        with open(outs[mode][1]) as f:
            for line in f:
                t = line.split()
                if t[0] == "R" and t[1] in dirty:
                    R[mode][(t[1], t[2])] = np.array([float(x) for x in t[3:]], np.float64)
    assert set(R["cuda"]) == set(R["cpu"]) and len(R["cpu"]) > 50
    assert rc_ok(R["cuda"], R["cpu"]) <= 1.0
