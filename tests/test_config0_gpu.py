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
  |ours - ref| <= 1e-5 |ref| + 1e-5 (library time unit: ns), NaN where
  the reference has none.  Each of the design's thousands of timing arcs
  turns the RC values into delays through the same NLDM tables, so the
  RC differences carry over at the same relative size.
"""
import math
import os
import subprocess

import numpy as np
import pytest

import config0_design

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
    P, R, B = {}, {}, {}
    with open(out) as f:
        for line in f:
            t = line.split()
            if t[0] == "P":
                P[t[1]] = np.array([float(x) for x in t[2:]], np.float64)
            elif t[0] == "R":
                R[(t[1], t[2])] = np.array([float(x) for x in t[3:]], np.float64)
            elif t[0] == "B":
                B[(t[1], t[2])] = (int(t[3]), int(t[4]))
    return P, R, B


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
        if m.any():
            tol = PIN_RTOL * np.abs(r[m]) + PIN_ATOL
            worst = max(worst, float(np.max(np.abs(g[m] - r[m]) / tol)))
    return worst


@pytest.fixture(scope="module")
def runs(tmp_path_factory, cuda):
    if not (os.path.exists(EXE_REF) and os.path.exists(EXE_OTG)):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    d = str(tmp_path_factory.mktemp("config0"))
    info = config0_design.write_design(d, seed=2024, gates=2000)
    return info, run(EXE_REF, d, "cuda"), run(EXE_OTG, d, "cuda"), run(EXE_REF, d, "cpu")


def test_bfs_order_bit_exact(runs):
    _, ref, ours, _ = runs
    assert len(ref[2]) > 10000
    assert ours[2] == ref[2]


def test_rc_nodes_within_tolerance(runs):
    info, ref, ours, cpu = runs
    assert set(ours[1]) == set(ref[1]) == set(cpu[1])
    w_gpu = rc_ok(ours[1], ref[1])
    w_cpu = rc_ok(ours[1], cpu[1])
    print(f"config 0 ({info}): RC err/tol vs reference GPU {w_gpu:.3g}, vs CPU {w_cpu:.3g}")
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
