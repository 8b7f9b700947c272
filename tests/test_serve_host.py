"""Host side of the design server: the synthetic design's sinks are the
leaves of each net (checked against the test generator's definition)."""
import types

import numpy as np

import opentimer_b200 as otg
from opentimer_b200.serve import synth_design

import rcgen


def test_synth_design_sinks_are_the_leaves():
    ns = otg.net_sizes(3, 400, 2, 300)
    d = synth_design(3, ns)
    f = types.SimpleNamespace(num_nets=len(ns) - 1, nodes_start=ns, edges=d["edges"],
                              roots=d["roots"])
    ss, sn = rcgen.sinks_of(f)
    np.testing.assert_array_equal(d["sinks_start"], ss)
    np.testing.assert_array_equal(d["sink_nodes"], sn)
    np.testing.assert_array_equal(np.diff(ss), d["sink_count"])
