"""Host side of incremental SPEF ingestion (no GPU): the change file's nets
are mapped to the design's forest nets by name, unknown names are skipped
as Timer::_read_spef skips them (ot/timer/spef.cpp:40-53), the staged
forest holds exactly the named nets' trees with their pin caps, and the
net arcs into the replaced nets get their sinks' new local ids."""
import os

import numpy as np

from opentimer_b200 import designgen
from opentimer_b200.prop import (attach_nets, change_arcs, change_nets, net_arc_index,
                                  rc_inputs)
from opentimer_b200.spef import read_spef


def test_change_nets_maps_names_and_skips_unknown(tmp_path):
    d = str(tmp_path)
    keep = {}
    designgen.write_design(d, seed=11, gates=300, keep=keep)
    change = os.path.join(d, "change.spef")
    names = designgen.change_spef(keep, change, frac=0.1, seed=3)
    assert names == designgen.change_spef(keep, change, frac=0.1, seed=3)  # seeded
    caps = designgen.pin_caps(keep)
    f0 = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    fc = read_spef(change, r_scale=np.float32(1e-3))
    index = {n: i for i, n in enumerate(f0["net_names"])}
    # drop one name from the design's index: that net must be skipped
    gone = names[0]
    partial = {n: i for n, i in index.items() if n != gone}
    nets, forest, node_of = change_nets(fc, partial, caps)
    assert len(nets) == len(names) - 1
    assert index[gone] not in set(nets.tolist())
    sub_ns, edges, roots, res, cap = forest
    assert sub_ns[0] == 0 and sub_ns[-1] == len(cap) and len(edges) == len(res)
    assert len(edges) == sub_ns[-1] - len(nets) and len(roots) == len(nets)
    # each staged net is the change file's tree, pin caps added on non-root pins
    capc, _ = rc_inputs(fc, caps)
    ns_c = fc["nodes_start"]
    k = 0
    for i, name in enumerate(fc["net_names"]):
        if name == gone:
            continue
        a, b = int(ns_c[i]), int(ns_c[i + 1])
        assert np.array_equal(cap[sub_ns[k]:sub_ns[k + 1]], capc[a:b]), name
        assert roots[k] == fc["roots"][i]
        k += 1
    assert all(i in set(nets.tolist()) for (i, _) in node_of)


def test_change_arcs_and_node_of_match_a_direct_restatement(tmp_path):
    d = str(tmp_path)
    keep = {}
    designgen.write_design(d, seed=12, gates=400, keep=keep)
    change = os.path.join(d, "change.spef")
    designgen.change_spef(keep, change, frac=0.2, seed=5)
    caps = designgen.pin_caps(keep)
    arrays, pin_names, pin_nets = designgen.timing_graph(keep)
    f0 = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    fc = read_spef(change, r_scale=np.float32(1e-3))
    _, node_of0 = rc_inputs(f0, caps)
    arc_net = attach_nets(arrays, pin_names, pin_nets, f0, node_of0)["arc_net"]
    index = {n: i for i, n in enumerate(f0["net_names"])}
    nets, _, node_of = change_nets(fc, index, caps)
    # node_of: the change file's pins keyed by forest net, as a re-keyed dict
    _, local = rc_inputs(fc, caps)
    to_forest = {i: index[n] for i, n in enumerate(fc["net_names"]) if n in index}
    assert node_of == {(to_forest[i], p): v for (i, p), v in local.items() if i in to_forest}
    # change_arcs: every net arc whose net was replaced, ascending, and the
    # sink's new local id (-1 when the sink is not in the new tree)
    arcs, nodes = change_arcs(net_arc_index(arrays["arc_kind"], arc_net),
                              np.asarray(arrays["arc_to"]), pin_names, nets, node_of)
    changed = set(nets.tolist())
    want = [k for k in range(len(arc_net))
            if arrays["arc_kind"][k] == 0 and int(arc_net[k]) in changed]
    assert arcs.tolist() == want and len(want) > 10
    assert nodes == [node_of.get((int(arc_net[k]), pin_names[int(arrays["arc_to"][k])]), -1)
                     for k in want]
    assert all(v >= 0 for v in nodes)
    empty_arcs, empty_nodes = change_arcs(net_arc_index(arrays["arc_kind"], arc_net),
                                          np.asarray(arrays["arc_to"]), pin_names,
                                          np.zeros(0, np.int64), node_of)
    assert empty_arcs.size == 0 and empty_nodes == []
