"""Incremental gate sizing on the device (opentimer_b200.sizing: the GPU form
of Timer::repower_gate + update_timing) against the reference Timer running
the same resizes (oracle/_ref/ot_run_ref: repower_gate per gate, then
update_timing per step, CPU path -- the reference's CUDA path is valid for a
first full update only).  After every second step, every pin's arrival
time, slew, required time and slack, four corners, must match within
|ours - ref| <= 1e-5 s + 1e-5 (ns), s = |ref| for arrival time and slew and
max(|ref|, |ref at|) for required time and slack (tests/helpers.pin_err)."""
import os
import subprocess

import numpy as np
import pytest

from helpers import pin_err, read_ref_pins
from opentimer_b200 import designgen

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE_REF = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")
STEPS, PER_STEP, DUMP_EVERY = 6, 40, 2


@pytest.fixture(scope="module")
def sized(tmp_path_factory, cuda):
    if not os.path.exists(EXE_REF):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    from opentimer_b200.sizing import resize_trace, write_ops
    d = str(tmp_path_factory.mktemp("sizing"))
    keep = {}
    designgen.write_design(d, seed=2031, gates=2000, keep=keep)
    steps = resize_trace(keep, seed=7, steps=STEPS, per_step=PER_STEP)
    ops = os.path.join(d, "ops.txt")
    write_ops(ops, steps)
    out = os.path.join(d, "ref.txt")
    p = subprocess.run([EXE_REF, d, "cpu", out, f"repower={ops}", f"dump_every={DUMP_EVERY}"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    ref = {k: read_ref_pins(f"{out}.step{k}") for k in range(DUMP_EVERY, STEPS + 1, DUMP_EVERY)}
    return d, keep, steps, ref


def test_resizes_match_reference_repower_gate(sized):
    from opentimer_b200.sizing import SizingDesign
    d, keep, steps, ref = sized
    sd = SizingDesign(d, keep)
    worst = {}
    for k, step in enumerate(steps, start=1):
        sd.resize(step)
        if k in ref:
            worst[k] = pin_err(sd.pins(), ref[k])
            # the worst slack is the minimum over the pins' slacks
            wns = sd.worst_slack()
            r = np.array([[v[3][c] for v in ref[k].values()] for c in range(4)])
            want = np.nanmin(r, axis=1)
            assert np.allclose(wns, want, rtol=1e-5, atol=1e-5 + 1e-5 * np.abs(want).max()), \
                (wns, want)
    print(f"sizing: err/tol after steps {sorted(worst)}: {worst}")
    assert max(worst.values()) <= 1.0


def test_prepared_batches_give_the_same_state(sized):
    """The same resizes queued back to back from device arrays (the timed
    loop's path) end in the same pins, and each batch's worst slack is the
    one the step-by-step path reports."""
    from opentimer_b200.sizing import SizingDesign
    d, keep, steps, ref = sized
    a = SizingDesign(d, keep)
    seen = []
    for step in steps:
        a.resize(step)
        seen.append(a.worst_slack())
    b = SizingDesign(d, keep)
    prep = b.prepare(steps)
    b.run_prepared(prep)
    b.check()
    assert np.array_equal(prep["wns"].cpu().numpy(), np.array(seen))
    pa, pb = a.pins(), b.pins()
    assert all(np.array_equal(pa[n], pb[n], equal_nan=True) for n in pa)
    assert pin_err(pb, ref[STEPS]) <= 1.0
