"""Host side of incremental SPEF ingestion (no GPU): the change file's nets
are mapped to the design's forest nets by name, unknown names are skipped
as Timer::_read_spef skips them (ot/timer/spef.cpp:40-53), and the staged
forest holds exactly the named nets' trees with their pin caps."""
import os

import numpy as np

from opentimer_b200 import designgen
from opentimer_b200.prop import change_nets, rc_inputs
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
