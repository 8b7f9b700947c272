"""Host side of incremental gate sizing (opentimer_b200.sizing.ResizeTable):
resizing every combinational gate must leave the RC node caps and the cell
arcs' timing records exactly as if the design had been built with the new
cells from the start (rc_inputs over the new cells' pin caps, and
designgen.timing_graph over the new netlist)."""
import os

import numpy as np

from opentimer_b200 import designgen
from opentimer_b200.prop import rc_inputs
from opentimer_b200.sizing import ResizeTable, cell_family, resize_trace
from opentimer_b200.spef import read_spef


def test_resize_all_gates_equals_a_design_built_with_the_new_cells(tmp_path):
    d = str(tmp_path)
    keep = {}
    designgen.write_design(d, seed=11, gates=400, keep=keep)
    arrays, names, _ = designgen.timing_graph(keep)
    f = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    cap, node_of = rc_inputs(f, designgen.pin_caps(keep))
    table = ResizeTable(keep, arrays, f, node_of)
    new_cell = {g: (c if cell_family(c) == "DFF" else cell_family(c) + "_X4")
                for g, c, _ in keep["gates"]}
    cap_row, cap_val, arc_slot, arc_rec, nets = table.updates(
        [(g, c) for g, c in new_cell.items() if c.endswith("_X4")])
    cap2 = cap.copy()
    cap2[cap_row] = cap_val
    timing2 = arrays["arc_timing"].copy().reshape(-1)
    timing2[arc_slot] = arc_rec
    # the same design with the new cells from the start
    keep4 = dict(keep)
    keep4["gates"] = [(g, new_cell[g], conn) for g, _, conn in keep["gates"]]
    arrays4, names4, _ = designgen.timing_graph(keep4)
    want_cap, _ = rc_inputs(f, designgen.pin_caps(keep4))
    assert np.array_equal(cap2.view(np.int32), want_cap.view(np.int32))
    assert names4 == names
    # record ids differ between the two graphs (registration order); the
    # records' contents must agree arc by arc and split by split
    ids1 = timing2.reshape(-1, 2)[arrays["arc_kind"] == 1].reshape(-1)
    ids2 = arrays4["arc_timing"][arrays4["arc_kind"] == 1].reshape(-1)
    assert np.array_equal(ids1 >= 0, ids2 >= 0)

    def lut(a, i):
        if i < 0:
            return None
        n1, n2, off, _ = a["lut_meta"][i]
        return a["lut_data"][off:off + n1 + n2 + n1 * n2]
    for i1, i2 in zip(ids1[ids1 >= 0], ids2[ids2 >= 0]):
        r1, r2 = arrays["timing"][i1], arrays4["timing"][i2]
        assert np.array_equal(r1[:3], r2[:3])
        for l1, l2 in zip(r1[3:], r2[3:]):
            a1, a2 = lut(arrays, l1), lut(arrays4, l2)
            assert (a1 is None) == (a2 is None)
            if a1 is not None:
                assert np.array_equal(a1, a2)
    # the nets of the resized gates' input pins are dirty, and only those
    resized = [i for i, (g, c, _) in enumerate(keep["gates"]) if cell_family(c) != "DFF"]
    want = {n for i in resized for _, _, n in table.gate_inputs[i]}
    assert set(nets.tolist()) == want


def test_resize_trace_keeps_functions_and_changes_drive():
    keep = {}
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        designgen.write_design(d, seed=12, gates=300, keep=keep)
    steps = resize_trace(keep, seed=3, steps=4, per_step=25)
    cur = {g: c for g, c, _ in keep["gates"]}
    for step in steps:
        assert len({g for g, _ in step}) == len(step) == 25
        for g, c in step:
            assert cell_family(c) == cell_family(cur[g]) and c != cur[g]
            cur[g] = c
