"""Served incremental timing of gate-level designs (opentimer_b200.gateserve):
three designs on one device as a union, requests that resize gates and
ask for the design's worst slack.  Each request's result must be the same
served alone (one request at a time) and in a mix (continuous batching
across designs), bit for bit; and each design's pins after its requests,
and the worst slack after each request, must match the reference Timer
running the same repower_gate + update_timing sequence (CPU path), within
the pin tolerance of tests/helpers.pin_err."""
import os
import subprocess

import numpy as np
import pytest

from helpers import pin_err, read_ref_pins
from opentimer_b200 import designgen

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE_REF = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")
GATES = (1500, 2500, 4000)


@pytest.fixture(scope="module")
def designs(tmp_path_factory, cuda):
    out = []
    for i, g in enumerate(GATES):
        d = str(tmp_path_factory.mktemp(f"gs{i}"))
        keep = {}
        designgen.write_design(d, seed=300 + i, gates=g, keep=keep, lib_seed=77)
        out.append((d, keep))
    return out


def serve(designs, trace, plain):
    from opentimer_b200.gateserve import DesignSet, GateServer, build_design
    ds = DesignSet([build_design(d, keep) for d, keep in designs])
    srv = GateServer(ds)
    lat, span, res = srv.replay(trace, plain=plain)
    return ds, res


def test_alone_and_in_the_mix_and_against_the_reference(designs):
    from opentimer_b200.gateserve import request_trace
    from opentimer_b200.sizing import write_ops
    trace = request_trace([k for _, k in designs], seed=5, num=30, rate=None, lo=1, hi=24,
                          at_zero=True)
    ds_b, res_b = serve(designs, trace, plain=False)
    ds_p, res_p = serve(designs, trace, plain=True)
    assert np.array_equal(res_b.view(np.int32), res_p.view(np.int32))
    if not os.path.exists(EXE_REF):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    worst = {}
    for di, (d, _) in enumerate(designs):
        mine = [k for k in range(len(trace["design"])) if trace["design"][k] == di]
        if not mine:
            continue
        ops = os.path.join(d, "serve_ops.txt")
        write_ops(ops, [trace["resizes"][k] for k in mine])
        out = os.path.join(d, "serve_ref.txt")
        p = subprocess.run([EXE_REF, d, "cpu", out, f"repower={ops}", "dump_every=1"],
                           capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        for step, k in enumerate(mine, start=1):
            ref = read_ref_pins(f"{out}.step{step}")
            want = np.nanmin(np.array([v[3] for v in ref.values()]), axis=0)
            scale = 1e-5 * np.nanmax(np.abs(np.array([v[0] for v in ref.values()])))
            assert np.all(np.abs(res_b[k] - want) <= 1e-5 * np.abs(want) + 1e-5 + scale), \
                (di, step, res_b[k], want)
        worst[di] = pin_err(ds_b.pins(di), read_ref_pins(f"{out}.step{len(mine)}"))
    print(f"served designs: pins err/tol vs the reference after their requests: {worst}")
    assert max(worst.values()) <= 1.0


def test_propagate_items(designs):
    """otg_propagate_items over one design's slice of the union's order
    writes exactly that design's pins, with the bits of a full propagation;
    every other pin keeps its values; an item out of range is reported."""
    import torch
    from opentimer_b200._lib import OtgError
    from opentimer_b200.gateserve import DesignSet, build_design
    ds = DesignSet([build_design(d, keep) for d, keep in designs])
    g = ds.graph
    full = g.propagate(ds.batch).result()
    for v in g.out.values():
        v.fill_(7.0)
    d = 1
    a0, a1 = int(ds.seg[d]), int(ds.seg[d + 1])
    part = g.propagate_items(ds.batch, ds.dorder[a0:a1]).result()
    mine = np.zeros(ds.P, bool)
    mine[ds.dorder[a0:a1].cpu().numpy()] = True
    assert mine[int(ds.p_off[d]):int(ds.p_off[d + 1])].sum() == a1 - a0
    for k in full:
        assert np.array_equal(part[k][mine].view(np.int32), full[k][mine].view(np.int32)), k
        assert np.all(part[k][~mine] == 7.0), k
    bad = torch.tensor([0, ds.P + 5], dtype=torch.int32, device="cuda")
    with pytest.raises(OtgError):
        g.propagate_items(ds.batch, bad).check()
