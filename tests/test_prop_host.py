"""Host helpers of the propagation path (no GPU): the CSR builder, the range
gather of change_nets, and the net/node attachment of a timing graph."""
import numpy as np

from opentimer_b200.prop import _csr, _ranges, attach_nets


def test_csr_groups_items_by_key_stably():
    keys = np.array([2, 0, 2, 1, 0, 2], np.int32)
    start, items = _csr(keys, 4)
    assert start.tolist() == [0, 2, 3, 6, 6]
    assert items.tolist() == [1, 4, 3, 0, 2, 5]


def test_ranges_concatenates_aranges():
    got = _ranges(np.array([5, 0, 9]), np.array([2, 0, 3]))
    assert got.tolist() == [5, 6, 9, 10, 11]
    assert _ranges(np.zeros(0, np.int64), np.zeros(0, np.int64)).size == 0


def test_attach_nets_points_net_arcs_at_local_nodes():
    # pins: 0 drives net "a" with sinks 1 and 2; cell arc 1 -> 3 drives net "b"
    arrays = {"arc_from": np.array([0, 0, 1]), "arc_to": np.array([1, 2, 3]),
              "arc_kind": np.array([0, 0, 1]), "arc_net_name": ["a", "a", None]}
    spef = {"net_names": ["b", "a"]}
    node_of = {(1, "p1"): 3, (1, "p2"): 1}
    out = attach_nets(arrays, ["p0", "p1", "p2", "p3"], [None, "a", "a", "b"], spef, node_of)
    assert out["arc_net"].tolist() == [1, 1, 0]
    assert out["arc_node"].tolist() == [3, 1, -1]
