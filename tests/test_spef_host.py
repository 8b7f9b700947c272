"""SPEF ingestion (otg_spef_*): the flat RC arrays equal those the
reference's own SPEF parser and the flat path's rules give (oracle/_ref,
otref_spef_load), bit for bit, on a generated design, on a file with name
maps and coupling caps, and on the reference's bundled c17/s27 SPEFs when
the reference tree is present."""
import ctypes
import os

import numpy as np
import pytest

from opentimer_b200 import designgen
import oracle as O
from opentimer_b200.spef import read_spef

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


def ref_flat(path):
    L = O.ref_lib()
    n, v = ctypes.c_int(), ctypes.c_int()
    assert L.otref_spef_load(str(path).encode(), ctypes.byref(n), ctypes.byref(v)) == 0
    N, V = n.value, v.value
    ns = np.empty(N + 1, np.int32)
    e = np.empty(2 * (V - N), np.int32)
    r = np.empty(N, np.int32)
    res = np.empty(V - N, np.float32)
    cap = np.empty(4 * V, np.float32)
    L.otref_spef_fetch(ns, e, r, res, cap)
    return {"nodes_start": ns, "edges": e.reshape(-1, 2), "roots": r, "res": res,
            "cap": cap.reshape(-1, 4)}


def assert_same(path, **kw):
    got = read_spef(path, **kw)
    ref = ref_flat(path)
    for k in ref:
        assert np.array_equal(got[k], ref[k]), k
    assert not got["net_flags"].any()
    return got


def test_generated_design(tmp_path):
    designgen.write_design(str(tmp_path), seed=7, gates=800)
    f = assert_same(tmp_path / "design.spef", threads=3)
    assert len(f["net_names"]) > 800
    # every pin of every net is a tree node; the root is one of them
    ps = f["pins_start"]
    assert (f["pin_node"] >= 0).all()
    for i in range(len(f["roots"])):
        assert f["roots"][i] in f["pin_node"][ps[i]:ps[i + 1]]


SPEF_NAME_MAP = """*SPEF "IEEE 1481-1998"
*DESIGN "t"
*DIVIDER /
*DELIMITER :
*BUS_DELIMITER [ ]
*T_UNIT 1 NS
*C_UNIT 1 PF
*R_UNIT 1 KOHM
*L_UNIT 1 HENRY

*NAME_MAP
*1 net_a
*2 inst_0
*3 inst_1
*12 inst_22

*D_NET *1 0.123
*CONN
*I *2:ZN O *C 1.0 2.0 *L 0.0 *D INV
*I *3:A I *L 0.002
*I *12:B I
*CAP
1 *2:ZN 0.0011
2 *1:1 0.00215
3 *3:A 0.0033
4 *1:1 *9:2 0.0001
5 *12:B 4.5e-4
*RES
1 *1:1 *2:ZN 1.25
2 *3:A *1:1 0.75e-1
3 *1:2 *1:1 2
4 *1:2 *12:B 3.5
*END

*D_NET lonely 0.001
*CONN
*I inst_9:ZN O
*CAP
1 inst_9:ZN 0.001
*END
"""


def test_name_map_coupling_units(tmp_path):
    p = tmp_path / "nm.spef"
    p.write_text(SPEF_NAME_MAP)
    f = assert_same(p)
    # unit rebasing: every value times the scale, in float (as a Timer does)
    g = read_spef(p, r_scale=1000.0, c_scale=1000.0)
    assert np.array_equal(g["res"], f["res"] * np.float32(1000.0))
    assert np.array_equal(g["cap"], f["cap"] * np.float32(1000.0))
    assert f["net_names"] == ["net_a"]      # the net without *RES is left out
    assert f["units"]["ohm"] == 1e3 and abs(f["units"]["farad"] - 1e-12) < 1e-24
    # first appearance over the RES lines: net_a:1, inst_0:ZN, inst_1:A, net_a:2, inst_22:B
    assert f["edges"].tolist() == [[0, 1], [2, 0], [3, 0], [3, 4]]
    assert f["roots"].tolist() == [1]
    # the coupling line overwrote node net_a:1 with its value
    assert f["cap"][0, 0] == np.float32(0.0001)


@pytest.mark.parametrize("name", ["c17", "s27"])
def test_bundled_reference_spef(name):
    path = f"/root/reference/benchmark/{name}/{name}.spef"
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    assert_same(path)
