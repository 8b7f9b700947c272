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


def test_relayout_after_change_spef_equals_a_table_built_on_the_new_trees(tmp_path):
    """A change SPEF replaces some nets' trees (new node counts, new pin
    nodes): ResizeTable.relayout must leave the table exactly as one built
    from the start on the spliced parasitics, and a resize batch after it
    must write the caps rc_inputs gives for the spliced trees."""
    from opentimer_b200.prop import change_nets
    d = str(tmp_path)
    keep = {}
    designgen.write_design(d, seed=13, gates=400, keep=keep)
    arrays, _, _ = designgen.timing_graph(keep)
    f = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    _, node_of = rc_inputs(f, designgen.pin_caps(keep))
    table = ResizeTable(keep, arrays, f, node_of)
    steps = resize_trace(keep, seed=4, steps=2, per_step=30)
    table.updates(steps[0])  # resizes before the change: its pin caps follow them
    path = os.path.join(d, "change.spef")
    designgen.change_spef(keep, path, frac=0.1, seed=9)
    fc = read_spef(path, r_scale=np.float32(1e-3))
    net_index = {n: i for i, n in enumerate(f["net_names"])}
    nets, forest, node_of_c, ground = change_nets(
        fc, net_index, table.current_pin_caps(keep), with_ground=True)
    assert len(nets) > 10
    ns_old = np.asarray(f["nodes_start"], np.int64)
    sizes = np.diff(ns_old)
    sizes[nets] = np.diff(forest[0].astype(np.int64))
    ns_new = np.zeros(len(sizes) + 1, np.int64)
    np.cumsum(sizes, out=ns_new[1:])
    table.relayout(ns_old, ns_new, nets, ground, node_of_c)
    # the spliced parasitics: changed nets' ground caps from the change file
    sub = np.asarray(forest[0], np.int64)
    slot = {int(n): k for k, n in enumerate(nets.tolist())}
    gcap = np.concatenate([ground[sub[slot[i]]:sub[slot[i] + 1]] if i in slot
                           else f["cap"][ns_old[i]:ns_old[i + 1]] for i in range(len(sizes))])
    spliced = {"cap": gcap, "nodes_start": ns_new, "net_names": f["net_names"]}
    node_of2 = {k: v for k, v in node_of.items() if k[0] not in slot}
    node_of2.update(node_of_c)
    fresh = ResizeTable(keep, arrays, spliced, node_of2)
    assert np.array_equal(table.gcap.view(np.int32), fresh.gcap.view(np.int32))
    assert table.gate_inputs == fresh.gate_inputs
    # a resize after the change writes what a cap build on the new trees gives
    cap_row, cap_val, _, _, _ = table.updates(steps[1])
    cells = {g: c for g, c, _ in keep["gates"]}
    cells.update(dict(steps[0]))
    cells.update(dict(steps[1]))
    keep2 = dict(keep, gates=[(g, cells[g], conn) for g, _, conn in keep["gates"]])
    pin_caps = designgen.pin_caps(keep2)
    want = gcap.copy()
    written = set(cap_row.tolist())
    for (i, pin), node in node_of2.items():
        c = pin_caps.get(pin)
        if c is not None and ns_new[i] + node in written:
            want[ns_new[i] + node] += np.float32(c)
    assert np.array_equal(cap_val.view(np.int32), want[cap_row].view(np.int32))
