"""Host side of the gate-level server: the union of designs that share a
library keeps every arc's timing record content (remapped to the shared
record table), offsets pins/arcs/nets per design, and the request trace
keeps each gate's function while changing its drive strength."""
import numpy as np

from opentimer_b200 import designgen
from opentimer_b200.gateserve import build_design, request_trace, union_arrays
from opentimer_b200.sizing import cell_family


def test_union_keeps_records_and_offsets(tmp_path):
    ds, keeps = [], []
    for i, g in enumerate((300, 500)):
        d = str(tmp_path / f"d{i}")
        keep = {}
        designgen.write_design(d, seed=40 + i, gates=g, keep=keep, lib_seed=9)
        ds.append(build_design(d, keep))
        keeps.append(keep)
    u, P, p_off, a_off, n_off, v_off, rec_map = union_arrays(ds)
    assert u["num_pins"] == sum(P)
    for i, d in enumerate(ds):
        a = d["arrays"]
        sl = slice(int(a_off[i]), int(a_off[i + 1]))
        assert np.array_equal(u["arc_from"][sl], a["arc_from"] + p_off[i])
        t_own, t_u = a["arc_timing"].reshape(-1), u["arc_timing"][sl].reshape(-1)
        assert np.array_equal(t_own >= 0, t_u >= 0)
        # same record content: the timing row and its tables
        for r1, r2 in zip(t_own[t_own >= 0], t_u[t_u >= 0]):
            assert np.array_equal(a["timing"][r1][:3], u["timing"][r2][:3])
            for l1, l2 in zip(a["timing"][r1][3:], u["timing"][r2][3:]):
                assert (l1 < 0) == (l2 < 0)
                if l1 >= 0:
                    m1, m2 = a["lut_meta"][l1], u["lut_meta"][l2]
                    n = m1[0] + m1[1] + m1[0] * m1[1]
                    assert np.array_equal(a["lut_data"][m1[2]:m1[2] + n],
                                          u["lut_data"][m2[2]:m2[2] + n])
    tr = request_trace(keeps, seed=1, num=40, rate=1000.0, lo=2, hi=9)
    assert np.all(np.diff(tr["arrival"]) >= 0) and len(tr["resizes"]) == 40
    cur = [{g: c for g, c, _ in k["gates"]} for k in keeps]
    for d, step in zip(tr["design"], tr["resizes"]):
        assert 2 <= len(step) <= 9
        for g, c in step:
            assert cell_family(c) == cell_family(cur[d][g]) and c != cur[d][g]
            cur[d][g] = c
