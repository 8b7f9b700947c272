"""Seeded synthetic small design for the full update_timing parity check
(test infrastructure).

    write_design(dirpath, seed=2024, gates=2000)

writes into `dirpath`:
  early.lib / late.lib  a 4-cell Liberty library (INV_X1, NAND2_X1, NOR2_X1,
                        DFF_X1), 7x7 NLDM delay and transition tables indexed
                        by input slew 0.01..1 ns and load 1..100 fF, values
                        growing with both plus +-10% noise; the flop has
                        setup/hold tables.  The early library is the late one
                        scaled by 0.9, so the MIN and MAX corners differ.
  design.v              a random gate DAG: 64 primary inputs and outputs,
                        fanin 1..2, sources drawn with a geometric bias
                        towards recent signals (a skewed fanout; the mean
                        look-back is max(50, gates/100)), 5% flops on
                        one clock port; outputs left without a sink are
                        gathered by extra NAND2 gates until 64 remain.
  design.spef           one RC tree per net: the net's pins plus internal
                        nodes up to 2..16 nodes, a random recursive tree
                        rooted at the driver, R ~ U(0.5, 20) ohm, ground
                        C ~ U(0.1, 3) fF, RES lines shuffled with random
                        orientation.
  design.timing         TAU15 assertions: a 1 ns clock (arriving at 0 rising,
                        0.5 falling), input arrival times and slews, output
                        loads and required times.

The formats are the ones the reference's parsers read (Liberty, structural
Verilog, SPEF, the TAU 2015 .timing file); every number is drawn here.
"""
import os

import numpy as np

SLEW_IDX = [0.01, 0.02, 0.05, 0.1, 0.2, 0.5, 1.0]   # ns
LOAD_IDX = [1.0, 2.0, 5.0, 10.0, 20.0, 50.0, 100.0]   # fF


def f32(x):
    """Values as the parsers will hold them: float32, written with 9
    significant digits (which read back as the same float32)."""
    return np.asarray(x, np.float64).astype(np.float32)


def _fmt_row(r):
    return ", ".join(f"{float(x):.9g}" for x in f32(r))


def _table(rng, a, b, c, scale):
    s = np.array(SLEW_IDX)[:, None]
    ld = np.array(LOAD_IDX)[None, :]
    base = (a + b * s + c * ld) * scale
    return f32(base * (1.0 + rng.uniform(-0.1, 0.1, base.shape)))


def _lut(name, tmpl, vals, groups=None):
    if groups is not None:
        groups[name] = vals
    rows = ", \\\n          ".join(f'"{_fmt_row(r)}"' for r in vals)
    return (f"      {name}({tmpl}) {{\n"
            f'        index_1 ("{_fmt_row(SLEW_IDX)}");\n'
            f'        index_2 ("{_fmt_row(LOAD_IDX)}");\n'
            f"        values ( \\\n          {rows});\n"
            f"      }}\n")


def _arc(rng, related, sense, scale, kind=None, groups=None):
    # delay ~ a + b*slew + c*load (ns, fF), transition likewise
    a, b, c = rng.uniform(0.01, 0.03), rng.uniform(0.1, 0.3), rng.uniform(0.002, 0.006)
    ta, tb, tc = rng.uniform(0.005, 0.02), rng.uniform(0.05, 0.2), rng.uniform(0.004, 0.01)
    g = {"related": related, "sense": sense, "type": kind} if groups is not None else None
    out = "    timing() {\n"
    out += f'      related_pin : "{related}";\n'
    out += f"      timing_sense : {sense};\n"
    if kind:
        out += f"      timing_type : {kind};\n"
    out += _lut("cell_rise", "tbl7x7", _table(rng, a, b, c, scale), g)
    out += _lut("cell_fall", "tbl7x7", _table(rng, a * 0.9, b, c * 1.1, scale), g)
    out += _lut("rise_transition", "tbl7x7", _table(rng, ta, tb, tc, scale), g)
    out += _lut("fall_transition", "tbl7x7", _table(rng, ta * 1.1, tb, tc, scale), g)
    out += "    }\n"
    if groups is not None:
        groups.append(g)
    return out


def _constraint(rng, kind, scale, groups=None):
    a = rng.uniform(0.02, 0.05) if kind == "setup_rising" else rng.uniform(0.005, 0.015)
    g = {"related": "CK", "sense": None, "type": kind}
    out = "    timing() {\n"
    out += '      related_pin : "CK";\n'
    out += f"      timing_type : {kind};\n"
    for name in ("rise_constraint", "fall_constraint"):
        vals = _table(rng, a, 0.05, 0.0, scale)
        g[name] = vals
        rows = ", \\\n          ".join(f'"{_fmt_row(r)}"' for r in vals)
        out += (f"      {name}(cons7x7) {{\n"
                f'        index_1 ("{_fmt_row(SLEW_IDX)}");\n'
                f'        index_2 ("{_fmt_row(SLEW_IDX)}");\n'
                f"        values ( \\\n          {rows});\n      }}\n")
    out += "    }\n"
    if groups is not None:
        groups.append(g)
    return out


def _pin_in(name, cap, clock=False):
    s = f"  pin({name}) {{\n    direction : input;\n    capacitance : {float(cap):.9g};\n"
    if clock:
        s += "    clock : true;\n"
    return s


def liberty(seed, scale, name, cells=None):
    """Liberty text; with `cells` (a dict), also fills cells[cell] = {
    "caps": {pin: cap}, "timings": {output pin: [timing groups]}}."""
    rng = np.random.default_rng(seed)  # same seed for both corners: same shapes
    caps = f32(rng.uniform(1.0, 3.0, 16))
    if cells is None:
        cells = {}
    out = [f"library({name}) {{",
           "  delay_model : table_lookup;",
           '  time_unit : "1ns";',
           '  voltage_unit : "1V";',
           '  current_unit : "1mA";',
           '  pulling_resistance_unit : "1kohm";',
           '  leakage_power_unit : "1nW";',
           "  capacitive_load_unit (1,ff);",
           "  slew_upper_threshold_pct_rise : 80;",
           "  slew_lower_threshold_pct_rise : 20;",
           "  slew_upper_threshold_pct_fall : 80;",
           "  slew_lower_threshold_pct_fall : 20;",
           "  input_threshold_pct_rise : 50;",
           "  input_threshold_pct_fall : 50;",
           "  output_threshold_pct_rise : 50;",
           "  output_threshold_pct_fall : 50;",
           "  lu_table_template(tbl7x7) {",
           "    variable_1 : input_net_transition;",
           "    variable_2 : total_output_net_capacitance;",
           f'    index_1 ("{_fmt_row(SLEW_IDX)}");',
           f'    index_2 ("{_fmt_row(LOAD_IDX)}");',
           "  }",
           "  lu_table_template(cons7x7) {",
           "    variable_1 : related_pin_transition;",
           "    variable_2 : constrained_pin_transition;",
           f'    index_1 ("{_fmt_row(SLEW_IDX)}");',
           f'    index_2 ("{_fmt_row(SLEW_IDX)}");',
           "  }"]
    text = "\n".join(out) + "\n"
    # INV_X1
    inv = cells["INV_X1"] = {"caps": {"A": caps[0]}, "timings": {"ZN": []}}
    text += "cell(INV_X1) {\n  area : 1;\n" + _pin_in("A", caps[0]) + "  }\n"
    text += '  pin(ZN) {\n    direction : output;\n    function : "(!A)";\n'
    text += _arc(rng, "A", "negative_unate", scale, groups=inv["timings"]["ZN"]) + "  }\n}\n"
    # NAND2_X1, NOR2_X1
    for k, (cell, fn) in enumerate([("NAND2_X1", "(!(A1 A2))"), ("NOR2_X1", "(!(A1+A2))")]):
        c = cells[cell] = {"caps": {"A1": caps[1 + 2 * k], "A2": caps[2 + 2 * k]},
                           "timings": {"ZN": []}}
        text += f"cell({cell}) {{\n  area : 2;\n"
        text += _pin_in("A1", caps[1 + 2 * k]) + "  }\n" + _pin_in("A2", caps[2 + 2 * k]) + "  }\n"
        text += f'  pin(ZN) {{\n    direction : output;\n    function : "{fn}";\n'
        text += _arc(rng, "A1", "negative_unate", scale, groups=c["timings"]["ZN"])
        text += _arc(rng, "A2", "negative_unate", scale, groups=c["timings"]["ZN"])
        text += "  }\n}\n"
    # DFF_X1
    ff = cells["DFF_X1"] = {"caps": {"CK": caps[5], "D": caps[6]}, "timings": {"D": [], "Q": []},
                            "clock": ("CK",)}
    text += "cell(DFF_X1) {\n  area : 5;\n"
    text += '  ff(IQ, IQN) {\n    next_state : "D";\n    clocked_on : "CK";\n  }\n'
    text += _pin_in("CK", caps[5], clock=True) + "  }\n"
    text += _pin_in("D", caps[6]) + _constraint(rng, "setup_rising", scale, ff["timings"]["D"])
    text += _constraint(rng, "hold_rising", scale, ff["timings"]["D"]) + "  }\n"
    text += '  pin(Q) {\n    direction : output;\n    function : "IQ";\n'
    text += _arc(rng, "CK", "non_unate", scale, kind="rising_edge",
                 groups=ff["timings"]["Q"]) + "  }\n}\n"
    text += _drive_variants(seed, scale, caps, cells)
    text += "}\n"
    return text


# Drive strengths of the combinational cells: input capacitance grows with
# the drive, the load-dependent part of the delay and transition tables
# shrinks with it, and the intrinsic part grows a little.  The variants are
# drawn from their own stream (the X1 cells above are unchanged by them).
DRIVES = (2, 4)


def _drive_arc(rng, related, sense, scale, drive, groups):
    a, b, c = rng.uniform(0.01, 0.03), rng.uniform(0.1, 0.3), rng.uniform(0.002, 0.006)
    ta, tb, tc = rng.uniform(0.005, 0.02), rng.uniform(0.05, 0.2), rng.uniform(0.004, 0.01)
    k = 1.0 + 0.15 * np.log2(drive)  # intrinsic delay of the bigger stack
    g = {"related": related, "sense": sense, "type": None}
    out = "    timing() {\n"
    out += f'      related_pin : "{related}";\n'
    out += f"      timing_sense : {sense};\n"
    out += _lut("cell_rise", "tbl7x7", _table(rng, a * k, b, c / drive, scale), g)
    out += _lut("cell_fall", "tbl7x7", _table(rng, a * 0.9 * k, b, c * 1.1 / drive, scale), g)
    out += _lut("rise_transition", "tbl7x7", _table(rng, ta * k, tb, tc / drive, scale), g)
    out += _lut("fall_transition", "tbl7x7", _table(rng, ta * 1.1 * k, tb, tc / drive, scale), g)
    out += "    }\n"
    groups.append(g)
    return out


def _drive_variants(seed, scale, caps, cells):
    rng = np.random.default_rng(seed + 7919)
    text = ""
    for drive in DRIVES:
        cg = drive ** 0.8  # input capacitance factor
        name = f"INV_X{drive}"
        c = cells[name] = {"caps": {"A": f32(caps[0] * cg)}, "timings": {"ZN": []}}
        text += f"cell({name}) {{\n  area : {drive};\n" + _pin_in("A", c["caps"]["A"]) + "  }\n"
        text += '  pin(ZN) {\n    direction : output;\n    function : "(!A)";\n'
        text += _drive_arc(rng, "A", "negative_unate", scale, drive, c["timings"]["ZN"])
        text += "  }\n}\n"
        for k, (base, fn) in enumerate([("NAND2", "(!(A1 A2))"), ("NOR2", "(!(A1+A2))")]):
            name = f"{base}_X{drive}"
            c = cells[name] = {"caps": {"A1": f32(caps[1 + 2 * k] * cg),
                                        "A2": f32(caps[2 + 2 * k] * cg)},
                               "timings": {"ZN": []}}
            text += f"cell({name}) {{\n  area : {2 * drive};\n"
            text += _pin_in("A1", c["caps"]["A1"]) + "  }\n" + _pin_in("A2", c["caps"]["A2"])
            text += "  }\n"
            text += f'  pin(ZN) {{\n    direction : output;\n    function : "{fn}";\n'
            text += _drive_arc(rng, "A1", "negative_unate", scale, drive, c["timings"]["ZN"])
            text += _drive_arc(rng, "A2", "negative_unate", scale, drive, c["timings"]["ZN"])
            text += "  }\n}\n"
    return text


def netlist(rng, gates, n_pi=64, n_po=64, dff_frac=0.05):
    """Returns (gate list [(inst, cell, {pin: net})], inputs, outputs).
    Signals are net names; 'clk' is the clock port."""
    signals = [f"in{i}" for i in range(n_pi)]
    fanout = {s: 0 for s in signals}
    glist = []

    # geometric bias towards recent signals (a skewed fanout); the mean
    # look-back grows with the design, so the logic depth stays in the
    # hundreds of levels instead of growing with the gate count
    p_back = min(0.02, 100.0 / max(gates, 1))

    def pick():
        back = min(int(rng.geometric(p_back)), len(signals))
        s = signals[-back]
        fanout[s] += 1
        return s

    for g in range(gates):
        out = f"n{g}"
        r = rng.random()
        if r < dff_frac:
            glist.append((f"u{g}", "DFF_X1", {"D": pick(), "CK": "clk", "Q": out}))
        elif r < dff_frac + 0.3:
            glist.append((f"u{g}", "INV_X1", {"A": pick(), "ZN": out}))
        else:
            cell = "NAND2_X1" if rng.random() < 0.5 else "NOR2_X1"
            a1 = pick()
            a2 = pick()
            glist.append((f"u{g}", cell, {"A1": a1, "A2": a2, "ZN": out}))
        signals.append(out)
        fanout[out] = 0
    # gather dangling gate outputs until at most n_po remain
    dangling = [s for s in signals[n_pi:] if fanout[s] == 0]
    k = gates
    while len(dangling) > n_po:
        a1, a2 = dangling.pop(0), dangling.pop(0)
        fanout[a1] += 1
        fanout[a2] += 1
        out = f"n{k}"
        glist.append((f"u{k}", "NAND2_X1", {"A1": a1, "A2": a2, "ZN": out}))
        fanout[out] = 0
        dangling.append(out)
        k += 1
    # outputs: the dangling ones first, then the most recent other signals
    outs = list(dangling)
    for s in reversed(signals):
        if len(outs) >= n_po:
            break
        if s not in outs and not s.startswith("in"):
            outs.append(s)
    return glist, [f"in{i}" for i in range(n_pi)], outs


def verilog(glist, ins, outs):
    po = [f"out{i}" for i in range(len(outs))]
    ports = ins + ["clk"] + po
    lines = ["module top (" + ", ".join(ports) + ");"]
    lines += [f"input {p};" for p in ins + ["clk"]]
    lines += [f"output {p};" for p in po]
    wires = sorted({n for _, _, pins in glist for n in pins.values()} - set(ins) - {"clk"})
    wires += [f"pon{i}" for i in range(len(outs))]
    lines += [f"wire {w};" for w in wires]
    for inst, cell, pins in glist:
        conn = ", ".join(f".{p}({n})" for p, n in pins.items())
        lines.append(f"{cell} {inst} ( {conn} );")
    # primary outputs are driven through buffers of inverter pairs
    for i, s in enumerate(outs):
        lines.append(f"INV_X1 po{i}a ( .A({s}), .ZN(pon{i}) );")
        lines.append(f"INV_X1 po{i}b ( .A(pon{i}), .ZN(out{i}) );")
    lines.append("endmodule")
    return "\n".join(lines) + "\n", [(f"po{i}a", s, f"pon{i}", f"po{i}b", f"out{i}")
                                      for i, s in enumerate(outs)]


def spef(path, rng, nets, rc_nodes=(2, 16), rc_log=False):
    """Writes the SPEF of `nets` ({name: (driver_pin, driver_is_port,
    [(sink_pin, sink_is_port)])}) to `path`: per net (sorted by name) an RC
    tree of its pins plus internal nodes <net>:<k>, rc_nodes[0]..rc_nodes[1]
    nodes (uniform, or log-uniform with rc_log) but never fewer than its
    pins, a random recursive tree rooted at the driver, R ~ U(0.5, 20) ohm,
    ground C ~ U(0.1, 3) fF (times 16/n on trees of n > 16 nodes, so that a
    net's load stays within the tables' range), RES lines shuffled with
    random orientation.
    The random draws are made here; the text is formatted by
    otg_spef_write (the library's SPEF writer)."""
    import ctypes
    from . import lib
    names = sorted(nets)
    N = len(names)
    # names: the nets, then every net's pins (driver first); a pin belongs to
    # one net, so every name is stored once
    pins = [(nets[nm][0], nets[nm][1], nets[nm][2]) for nm in names]
    npins = np.fromiter((1 + len(sk) for _, _, sk in pins), np.int64, N)
    blob = list(names)
    pin_port = []
    for drv, drv_port, sinks in pins:
        blob.append(drv)
        pin_port.append(1 if drv_port else 0)
        for sp, is_port in sinks:
            blob.append(sp)
            pin_port.append(1 if is_port else 0)
    net_name = np.arange(N, dtype=np.int32)
    pins_start = np.zeros(N + 1, np.int64)
    np.cumsum(npins, out=pins_start[1:])
    pin_name = (N + np.arange(int(pins_start[-1]))).astype(np.int32)
    lo, hi = rc_nodes
    if rc_log:
        size = np.minimum(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), N)).astype(np.int64), hi)
    else:
        size = rng.integers(lo, hi + 1, N)
    n = np.maximum(npins, size)
    nodes_start = np.zeros(N + 1, np.int64)
    np.cumsum(n, out=nodes_start[1:])
    V = int(nodes_start[-1])
    net_of = np.repeat(np.arange(N), n)
    local = np.arange(V) - nodes_start[:-1][net_of]
    # node order: the driver first, then the other pins and the internal nodes
    # <net>:<k> shuffled; code >= 0 is a pin of the net, -k internal node k
    npn = npins[net_of]
    code0 = np.where(local < npn, local, -(local - npn + 1))
    key = np.where(local == 0, -1.0, rng.random(V))
    order = np.lexsort((key, net_of))
    codes = code0[order]
    # ground caps U(0.1, 3) fF per node on trees of up to 16 nodes; larger
    # trees share out the same total per net (cap x 16/n), so a net's load
    # stays in the range of the library's tables (1..100 fF)
    caps = rng.uniform(0.1, 3.0, V) * np.minimum(1.0, 16.0 / n)[net_of]
    # random recursive tree over the positions: parent of position i in [0, i)
    E = V - N
    child = np.nonzero(local > 0)[0]
    enet = net_of[child]
    li = local[child]
    par = (rng.random(E) * li).astype(np.int64)
    r = rng.uniform(0.5, 20.0, E)
    perm = np.lexsort((rng.random(E), enet))  # RES lines shuffled within each net
    flip = rng.random(E) < 0.5
    a, b = par[perm], li[perm]
    edges = np.stack([np.where(flip, b, a), np.where(flip, a, b)], 1)
    res = r[perm]
    enc = [x.encode() + b"\0" for x in blob]
    off = np.zeros(len(enc) + 1, np.int64)
    np.cumsum([len(x) for x in enc], out=off[1:])
    buf = b"".join(enc)
    arr = lambda x, dt: np.ascontiguousarray(np.asarray(x, dt))  # noqa: E731
    net_name, pins_start = arr(net_name, np.int32), arr(pins_start, np.int32)
    pin_name, pin_port = arr(pin_name, np.int32), arr(pin_port, np.int8)
    nodes_start = arr(nodes_start, np.int32)
    codes, caps = arr(codes, np.int32), arr(caps, np.float32)
    edges, res = arr(edges.reshape(-1, 2), np.int32), arr(res, np.float32)
    P = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    L = lib()
    st = L.otg_spef_write(path.encode(), N, buf, P(off), P(net_name), P(pins_start),
                          P(pin_name), P(pin_port), P(nodes_start), P(codes), P(caps), P(edges),
                          P(res), 0)
    if st != 0:
        raise OSError(f"otg_spef_write({path}) failed: {st}")


def change_spef(design, path, frac=0.01, seed=0):
    """Writes a TAU15-style change SPEF: new random RC trees (same pins,
    new internal nodes, topology, R and C) for a seeded fraction of the
    design's nets (`design` as filled by write_design's keep).  Returns the
    changed net names, in file order."""
    rng = np.random.default_rng(seed)
    names = sorted(design["nets"])
    k = max(1, int(round(frac * len(names))))
    chosen = sorted(rng.choice(len(names), size=k, replace=False).tolist())
    nets = {names[i]: design["nets"][names[i]] for i in chosen}
    spef(path, rng, nets, **design.get("rc", {}))
    return [names[i] for i in chosen]


def write_design(dirpath, seed=2024, gates=2000, keep=None, rc_nodes=(2, 16), rc_log=False,
                 lib_seed=None):
    """Writes the design files; returns a summary.  With `keep` (a dict), it
    also receives the in-memory design for timing_graph/pin_caps.
    rc_nodes / rc_log: the RC tree sizes of the nets (see spef).  lib_seed:
    the seed of the cell library (default: seed), so that several designs
    can share one library."""
    rng = np.random.default_rng(seed)
    os.makedirs(dirpath, exist_ok=True)
    libs = {"early": {}, "late": {}}
    ls = (seed if lib_seed is None else lib_seed) + 1
    with open(os.path.join(dirpath, "late.lib"), "w") as f:
        f.write(liberty(ls, 1.0, "late", libs["late"]))
    with open(os.path.join(dirpath, "early.lib"), "w") as f:
        f.write(liberty(ls, 0.9, "early", libs["early"]))
    glist, ins, outs = netlist(rng, gates)
    vtext, po_chain = verilog(glist, ins, outs)
    with open(os.path.join(dirpath, "design.v"), "w") as f:
        f.write(vtext)
    # connectivity: net -> driver and sinks
    outpin = {"INV_X1": "ZN", "NAND2_X1": "ZN", "NOR2_X1": "ZN", "DFF_X1": "Q"}
    drivers, sinks = {}, {}
    for p in ins + ["clk"]:
        drivers[p] = (p, True)
    for inst, cell, pins in glist:
        for pin, net in pins.items():
            if pin == outpin[cell]:
                drivers[net] = (f"{inst}:{pin}", False)
            else:
                sinks.setdefault(net, []).append((f"{inst}:{pin}", False))
    for a, s, mid, b, po in po_chain:
        sinks.setdefault(s, []).append((f"{a}:A", False))
        drivers[mid] = (f"{a}:ZN", False)
        sinks.setdefault(mid, []).append((f"{b}:A", False))
        drivers[po] = (f"{b}:ZN", False)
        sinks.setdefault(po, []).append((po, True))
    # every driven net gets a tree, even one without sinks: the reference's
    # flat (CUDA) path expects SPEF data for every net (net.cpp:500-507)
    nets = {n: (drivers[n][0], drivers[n][1], sinks.get(n, [])) for n in drivers}
    spef(os.path.join(dirpath, "design.spef"), rng, nets, rc_nodes, rc_log)
    period = 1.0
    assert_at, assert_slew, assert_rat, assert_load = {}, {}, {}, {}
    assert_at["clk"] = f32([0.0, 0.5, 0.0, 0.5])  # rise at 0, fall at half a period
    for p in ins:
        assert_at[p] = f32([rng.uniform(0.0, 0.05)] * 4)
        assert_slew[p] = f32([rng.uniform(0.01, 0.1)] * 4)
    assert_slew["clk"] = f32([0.02] * 4)
    for i in range(len(outs)):
        assert_load[f"out{i}"] = f32([4.0] * 4)
        assert_rat[f"out{i}"] = f32([0.0, 0.0, 1.0, 1.0])
    v = lambda x: " ".join(f"{float(t):.9g}" for t in x)  # noqa: E731
    lines = [f"clock clk {period}"]
    for p, x in assert_at.items():
        lines.append(f"at {p} {v(x)}")
    for p, x in assert_slew.items():
        lines.append(f"slew {p} {v(x)}")
    for p in assert_load:
        lines.append(f"load {p} {v(assert_load[p][:1])}")
        lines.append(f"rat {p} {v(assert_rat[p])}")
    with open(os.path.join(dirpath, "design.timing"), "w") as f:
        f.write("\n".join(lines) + "\n")
    if keep is not None:
        gates_all = list(glist) + [(a, "INV_X1", {"A": s, "ZN": mid}) for a, s, mid, _, _ in po_chain]
        gates_all += [(b, "INV_X1", {"A": mid, "ZN": po}) for _, _, mid, b, po in po_chain]
        keep.update(libs=libs, gates=gates_all, ports_in=ins + ["clk"],
                    ports_out=[f"out{i}" for i in range(len(outs))], nets=nets,
                    at=assert_at, slew=assert_slew, rat=assert_rat, load=assert_load,
                    period=period, rc={"rc_nodes": tuple(rc_nodes), "rc_log": rc_log})
    return {"gates": len(glist) + 2 * len(outs), "nets": len(nets)}


_SENSE = {"positive_unate": 0, "negative_unate": 1}
_MIN_CONSTRAINT = {"hold_rising", "hold_falling"}
_MAX_CONSTRAINT = {"setup_rising", "setup_falling"}
_LUTS = ["cell_rise", "cell_fall", "rise_transition", "fall_transition", "rise_constraint",
         "fall_constraint"]


def timing_graph(design):
    """The timing graph of a kept design in the otg_prop_graph layout, by
    the Timer's construction rules: a net arc from each net's driver to
    each of its other pins; per split (early library for MIN, late for
    MAX) one cell arc per timing group of each gate's cell, leaving out
    setup checks on MIN and hold checks on MAX, and a timing test on every
    constraint arc (ot/timer/timer.cpp:240-268, ot/timer/celllib.cpp:6-23).
    Returns (arrays, pin_names, pin_net_names); net arcs carry the net's
    name in `arc_net_name` and their sink pin in `arc_to`, for the caller
    to resolve against its RC forest."""
    pins, index = [], {}

    def pin(name):
        if name not in index:
            index[name] = len(pins)
            pins.append(name)
        return index[name]

    pin_net = {}
    for p in design["ports_in"] + design["ports_out"]:
        pin(p)
    for inst, cell, conn in design["gates"]:
        for cp, net in conn.items():
            pin_net[pin(f"{inst}:{cp}")] = net
    for p in design["ports_in"] + design["ports_out"]:
        pin_net[index[p]] = p
    arc_from, arc_to, arc_kind, arc_timing, arc_net_name, tests = [], [], [], [], [], []
    for name, (drv, _, sinks) in sorted(design["nets"].items()):
        for s, _ in sinks:
            arc_from.append(index[drv])
            arc_to.append(index[s])
            arc_kind.append(0)
            arc_timing.append((-1, -1))
            arc_net_name.append(name)
    # timing records and look-up tables, per library and group
    timing, lut_meta, lut_data, off = [], [], [], 0
    rec = {}

    def lut_id(vals, cons):
        nonlocal off
        v = f32(vals)
        idx1 = f32(SLEW_IDX)
        idx2 = f32(SLEW_IDX) if cons else f32(LOAD_IDX)
        lut_meta.append((len(idx1), len(idx2), off, 0))  # variable_1: input / related slew
        lut_data.extend([idx1, idx2, v.reshape(-1)])
        off += len(idx1) + len(idx2) + v.size
        return len(lut_meta) - 1

    def record(lib, cell, cp, k, g):
        key = (lib, cell, cp, k)
        if key not in rec:
            t = g["type"] or ""
            edge = 1 if t.endswith("rising") or t == "rising_edge" else (
                2 if t.endswith("falling") or t == "falling_edge" else 0)
            cons = t in _MIN_CONSTRAINT or t in _MAX_CONSTRAINT
            luts = [lut_id(g[n], cons) if n in g else -1 for n in _LUTS]
            timing.append([_SENSE.get(g["sense"], 2), edge, int(cons)] + luts)
            rec[key] = len(timing) - 1
        return rec[key]

    gate_arcs = [[] for _ in design["gates"]]  # per gate: (arc, split, cell pin, group)
    for el, lib in ((0, "early"), (1, "late")):
        cells = design["libs"][lib]
        for gi, (inst, cell, conn) in enumerate(design["gates"]):
            for cp, groups in cells[cell]["timings"].items():
                for k, g in enumerate(groups):
                    t = g["type"] or ""
                    if (el == 0 and t in _MAX_CONSTRAINT) or (el == 1 and t in _MIN_CONSTRAINT):
                        continue
                    tm = [-1, -1]
                    tm[el] = record(lib, cell, cp, k, g)
                    gate_arcs[gi].append((len(arc_from), el, cp, k))
                    arc_from.append(index[f"{inst}:{g['related']}"])
                    arc_to.append(index[f"{inst}:{cp}"])
                    arc_kind.append(1)
                    arc_timing.append(tuple(tm))
                    arc_net_name.append(None)
                    if t in _MIN_CONSTRAINT or t in _MAX_CONSTRAINT:
                        tests.append(len(arc_from) - 1)
    # the timing records of every cell of the libraries, used or not, so that
    # a resize (Timer::repower_gate) only re-points a gate's arcs
    for el, lib in ((0, "early"), (1, "late")):
        cells = design["libs"][lib]
        for cell in sorted(cells):
            for cp, groups in cells[cell]["timings"].items():
                for k, g in enumerate(groups):
                    t = g["type"] or ""
                    if (el == 0 and t in _MAX_CONSTRAINT) or (el == 1 and t in _MIN_CONSTRAINT):
                        continue
                    record(lib, cell, cp, k, g)
    P = len(pins)
    nan4 = lambda: np.full((P, 4), np.nan, np.float32)  # noqa: E731
    pi_at, pi_slew, po_rat = nan4(), nan4(), nan4()
    for p, x in design["at"].items():
        pi_at[index[p]] = x
    for p, x in design["slew"].items():
        pi_slew[index[p]] = x
    for p, x in design["rat"].items():
        po_rat[index[p]] = x
    arrays = {"num_pins": P, "arc_from": np.array(arc_from, np.int32),
              "arc_to": np.array(arc_to, np.int32), "arc_kind": np.array(arc_kind, np.int32),
              "arc_timing": np.array(arc_timing, np.int32).reshape(-1, 2),
              "test_arc": np.array(tests, np.int32), "pi_at": pi_at, "pi_slew": pi_slew,
              "po_rat": po_rat, "timing": np.array(timing, np.int32),
              "lut_meta": np.array(lut_meta, np.int32),
              "lut_data": np.concatenate(lut_data).astype(np.float32),
              "period": design["period"], "arc_net_name": arc_net_name,
              "gate_arcs": gate_arcs,
              "records": {(cell, el, cp, k): r for (lib, cell, cp, k), r in rec.items()
                          for el in ((0,) if lib == "early" else (1,))}}
    return arrays, pins, [pin_net.get(i) for i in range(P)]


def pin_caps(design):
    """Per pin name, the capacitance the flat RC path adds at its node
    (Pin::cap, ot/timer/pin.cpp:286-305): a primary output's load, an
    instance pin's library capacitance (the same in both libraries here),
    0 for a primary input."""
    caps = {p: f32([0.0] * 4) for p in design["ports_in"]}
    for p, x in design["load"].items():
        caps[p] = x
    cells = design["libs"]["late"]
    for inst, cell, conn in design["gates"]:
        for cp in conn:
            c = cells[cell]["caps"].get(cp)
            caps[f"{inst}:{cp}"] = f32([c if c is not None else 0.0] * 4)
    return caps
