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
                        towards recent signals (a skewed fanout), 5% flops on
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


def _fmt_row(r):
    return ", ".join(f"{x:.6f}" for x in r)


def _table(rng, a, b, c, scale):
    s = np.array(SLEW_IDX)[:, None]
    ld = np.array(LOAD_IDX)[None, :]
    base = (a + b * s + c * ld) * scale
    return base * (1.0 + rng.uniform(-0.1, 0.1, base.shape))


def _lut(name, tmpl, vals):
    rows = ", \\\n          ".join(f'"{_fmt_row(r)}"' for r in vals)
    return (f"      {name}({tmpl}) {{\n"
            f'        index_1 ("{_fmt_row(SLEW_IDX)}");\n'
            f'        index_2 ("{_fmt_row(LOAD_IDX)}");\n'
            f"        values ( \\\n          {rows});\n"
            f"      }}\n")


def _arc(rng, related, sense, scale, kind=None):
    # delay ~ a + b*slew + c*load (ns, fF), transition likewise
    a, b, c = rng.uniform(0.01, 0.03), rng.uniform(0.1, 0.3), rng.uniform(0.002, 0.006)
    ta, tb, tc = rng.uniform(0.005, 0.02), rng.uniform(0.05, 0.2), rng.uniform(0.004, 0.01)
    out = "    timing() {\n"
    out += f'      related_pin : "{related}";\n'
    out += f"      timing_sense : {sense};\n"
    if kind:
        out += f"      timing_type : {kind};\n"
    out += _lut("cell_rise", "tbl7x7", _table(rng, a, b, c, scale))
    out += _lut("cell_fall", "tbl7x7", _table(rng, a * 0.9, b, c * 1.1, scale))
    out += _lut("rise_transition", "tbl7x7", _table(rng, ta, tb, tc, scale))
    out += _lut("fall_transition", "tbl7x7", _table(rng, ta * 1.1, tb, tc, scale))
    out += "    }\n"
    return out


def _constraint(rng, kind, scale):
    a = rng.uniform(0.02, 0.05) if kind == "setup_rising" else rng.uniform(0.005, 0.015)
    out = "    timing() {\n"
    out += '      related_pin : "CK";\n'
    out += f"      timing_type : {kind};\n"
    for name in ("rise_constraint", "fall_constraint"):
        vals = _table(rng, a, 0.05, 0.0, scale)
        rows = ", \\\n          ".join(f'"{_fmt_row(r)}"' for r in vals)
        out += (f"      {name}(cons7x7) {{\n"
                f'        index_1 ("{_fmt_row(SLEW_IDX)}");\n'
                f'        index_2 ("{_fmt_row(SLEW_IDX)}");\n'
                f"        values ( \\\n          {rows});\n      }}\n")
    out += "    }\n"
    return out


def _pin_in(name, cap, clock=False):
    s = f"  pin({name}) {{\n    direction : input;\n    capacitance : {cap:.6f};\n"
    if clock:
        s += "    clock : true;\n"
    return s


def liberty(seed, scale, name):
    rng = np.random.default_rng(seed)  # same seed for both corners: same shapes
    caps = rng.uniform(1.0, 3.0, 16)
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
    text += "cell(INV_X1) {\n  area : 1;\n" + _pin_in("A", caps[0]) + "  }\n"
    text += '  pin(ZN) {\n    direction : output;\n    function : "(!A)";\n'
    text += _arc(rng, "A", "negative_unate", scale) + "  }\n}\n"
    # NAND2_X1, NOR2_X1
    for k, (cell, fn) in enumerate([("NAND2_X1", "(!(A1 A2))"), ("NOR2_X1", "(!(A1+A2))")]):
        text += f"cell({cell}) {{\n  area : 2;\n"
        text += _pin_in("A1", caps[1 + 2 * k]) + "  }\n" + _pin_in("A2", caps[2 + 2 * k]) + "  }\n"
        text += f'  pin(ZN) {{\n    direction : output;\n    function : "{fn}";\n'
        text += _arc(rng, "A1", "negative_unate", scale) + _arc(rng, "A2", "negative_unate", scale)
        text += "  }\n}\n"
    # DFF_X1
    text += "cell(DFF_X1) {\n  area : 5;\n"
    text += '  ff(IQ, IQN) {\n    next_state : "D";\n    clocked_on : "CK";\n  }\n'
    text += _pin_in("CK", caps[5], clock=True) + "  }\n"
    text += _pin_in("D", caps[6]) + _constraint(rng, "setup_rising", scale)
    text += _constraint(rng, "hold_rising", scale) + "  }\n"
    text += '  pin(Q) {\n    direction : output;\n    function : "IQ";\n'
    text += _arc(rng, "CK", "non_unate", scale, kind="rising_edge") + "  }\n}\n"
    text += "}\n"
    return text


def netlist(rng, gates, n_pi=64, n_po=64, dff_frac=0.05):
    """Returns (gate list [(inst, cell, {pin: net})], inputs, outputs).
    Signals are net names; 'clk' is the clock port."""
    signals = [f"in{i}" for i in range(n_pi)]
    fanout = {s: 0 for s in signals}
    glist = []

    def pick():
        # geometric bias towards recent signals: a skewed fanout
        back = min(int(rng.geometric(0.02)), len(signals))
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


def spef(rng, nets):
    """nets: {name: (driver_pin, driver_is_port, [(sink_pin, sink_is_port)])}"""
    out = ['*SPEF "IEEE 1481-1998"', '*DESIGN "top"', '*DATE "0"', '*VENDOR "otg"',
           '*PROGRAM "config0_design"', '*VERSION "0"', '*DESIGN_FLOW "NETLIST_TYPE_VERILOG"',
           "*DIVIDER /", "*DELIMITER :", "*BUS_DELIMITER [ ]", "*T_UNIT 1 NS", "*C_UNIT 1 FF",
           "*R_UNIT 1 OHM", "*L_UNIT 1 HENRY", ""]
    for name in sorted(nets):
        drv, drv_port, sinks = nets[name]
        pins = [drv] + [s for s, _ in sinks]
        n = max(len(pins), int(rng.integers(2, 17)))
        internal = [f"{name}:{i + 1}" for i in range(n - len(pins))]
        order = [drv] + list(rng.permutation(pins[1:] + internal))
        caps = rng.uniform(0.1, 3.0, n)
        edges = [(order[int(rng.integers(0, i))], order[i]) for i in range(1, n)]
        res = rng.uniform(0.5, 20.0, n - 1)
        perm = rng.permutation(n - 1)
        out.append(f"*D_NET {name} {caps.sum():.4f}")
        out.append("*CONN")
        out.append(f"*P {drv} I" if drv_port else f"*I {drv} O")
        for s, is_port in sinks:
            out.append(f"*P {s} O" if is_port else f"*I {s} I")
        out.append("*CAP")
        for i, (node, c) in enumerate(zip(order, caps)):
            out.append(f"{i + 1} {node} {c:.4f}")
        out.append("*RES")
        for i, j in enumerate(perm):
            a, b = edges[j]
            if rng.random() < 0.5:
                a, b = b, a
            out.append(f"{i + 1} {a} {b} {res[j]:.4f}")
        out.append("*END")
        out.append("")
    return "\n".join(out) + "\n"


def write_design(dirpath, seed=2024, gates=2000):
    rng = np.random.default_rng(seed)
    os.makedirs(dirpath, exist_ok=True)
    with open(os.path.join(dirpath, "late.lib"), "w") as f:
        f.write(liberty(seed + 1, 1.0, "late"))
    with open(os.path.join(dirpath, "early.lib"), "w") as f:
        f.write(liberty(seed + 1, 0.9, "early"))
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
    with open(os.path.join(dirpath, "design.spef"), "w") as f:
        f.write(spef(rng, nets))
    lines = ["clock clk 1.0", "at clk 0.0 0.5 0.0 0.5"]  # rise at 0, fall at half a period
    for p in ins:
        a = rng.uniform(0.0, 0.05)
        lines.append(f"at {p} {a:.4f} {a:.4f} {a:.4f} {a:.4f}")
        s = rng.uniform(0.01, 0.1)
        lines.append(f"slew {p} {s:.4f} {s:.4f} {s:.4f} {s:.4f}")
    lines.append("slew clk 0.02 0.02 0.02 0.02")
    for i in range(len(outs)):
        lines.append(f"load out{i} 4.0")
        lines.append(f"rat out{i} 0.0 0.0 1.0 1.0")
    with open(os.path.join(dirpath, "design.timing"), "w") as f:
        f.write("\n".join(lines) + "\n")
    return {"gates": len(glist) + 2 * len(outs), "nets": len(nets)}
