"""The reference Timer's update and query names over a design resident on the
device (ot/timer/timer.hpp:41-140, timer.cpp).

    t = Timer(dirpath, keep)             # designgen.write_design's files + keep
    t.report_at("u12:ZN", MAX, RISE)     # arrival time, or None
    t.repower_gate("u12", "NAND2_X4")    # queued, as the Timer queues it
    t.read_spef("change.spef")           # queued: new parasitics of the nets it names
    t.update_timing()                    # applies the queued operations, re-times
    t.report_wns(), t.report_tns(MAX)    # over the endpoints, as the Timer
    t.report_load("n42", MAX, FALL)      # the net's load (its RC root)
    t.rc_node("n42", "u7:A")             # load/delay/ldelay/impulse [2][2]
    t.rc_slew("n42", "u7:A", MAX, RISE, 30.0)  # the node's slew for a root slew
    t.report_timing(10)                  # the 10 worst paths (paths.Path)

Split and Tran are the reference's indices (MIN=0, MAX=1; RISE=0, FALL=1),
corner c = split * 2 + tran.  A value the reference reports as an empty
std::optional is None here.  Every query first applies the pending operations, as
the reference's report_* first runs update_timing (timer.cpp:1705); the
results come from the device (one read per update, kept until the next).

Endpoints follow Timer::_update_endpoints (timer.cpp:1388-1450): the
primary outputs and the constrained pins of the timing tests, for each
corner those whose slack is defined.  WNS is their minimum slack; TNS the
sum of their negative slacks; a report over several corners combines the
corners' values the same way (report_wns / report_tns, timer.cpp:1456-
1520).
"""
import numpy as np

from .paths import PathGraph
from .sizing import SizingDesign, cell_family

MIN, MAX = 0, 1
RISE, FALL = 0, 1
NC = 4


class Timer:
    def __init__(self, dirpath, keep, device="cuda"):
        self._d = SizingDesign(dirpath, keep, device=device)
        self._pin = {n: i for i, n in enumerate(self._d.names)}
        self._net = {n: i for i, n in enumerate(self._d.net_names)}
        self._gate_cell = {g: c for g, c, _ in keep["gates"]}
        self._pending = []  # queued operations, in order: ("resize", (gate, cell)) | ("spef", path)
        self._res = None  # host copy of the last update's pin results
        self._rc = None   # host copy of the RC outputs, read on demand
        self._pg = None   # the path search's view of the graph (paths.PathGraph)
        self._pg_fresh = False

    # ------------------------------------------------------------- updates
    def repower_gate(self, gate, cell):
        """Queues a resize of `gate` to `cell` of the same function
        (Timer::repower_gate, timer.cpp:57-118); unknown gates and cells of
        another function are refused here, where the reference logs them."""
        if gate not in self._gate_cell:
            raise KeyError(f"gate {gate} not found")
        if cell_family(cell) != cell_family(self._gate_cell[gate]):
            raise ValueError(f"{gate}: {self._gate_cell[gate]} -> {cell} changes the function")
        self._gate_cell[gate] = cell
        self._pending.append(("resize", (gate, cell)))
        return self

    def read_spef(self, path):
        """Queues a change SPEF (Timer::read_spef, ot/timer/spef.cpp:40-53):
        at the next update the nets it names get their new trees (unknown
        names are skipped, as the reference does) and only they are re-timed
        in the RC pass."""
        self._pending.append(("spef", path))
        return self

    def update_timing(self):
        """Applies the queued operations in order -- each run of resizes as
        one batch (new pin caps and cell-arc timing on the device, the dirty
        nets re-timed, propagation), each change SPEF by itself -- and drops
        the host copies of older results."""
        if not self._pending:
            return self
        run = []
        for kind, arg in self._pending + [("end", None)]:
            if kind == "resize":
                run.append(arg)
                continue
            if run:
                self._d.resize(run)
                run = []
            if kind == "spef":
                self._d.change_spef(arg)
        self._pending = []
        self._res = self._rc = None
        self._pg_fresh = False
        return self

    def _results(self):
        self.update_timing()
        if self._res is None:
            r = self._d.result()
            r["rat"] = np.where(np.isnan(r["at"]), np.nan, r["rat"])
            self._res = r
        return self._res

    def _rc_results(self):
        self.update_timing()
        if self._rc is None:
            self._d.check()
            b = self._d.batch
            self._rc = {k: getattr(b, k).cpu().numpy() for k in
                        ("node2bfs", "load", "delay", "ldelay", "impulse")}
        return self._rc

    # ------------------------------------------------------------- queries
    def _pin_value(self, key, name, el, rf):
        i = self._pin.get(name)
        if i is None:
            return None
        v = float(self._results()[key][i][el * 2 + rf])
        return None if np.isnan(v) else v

    def report_at(self, pin, el, rf):
        return self._pin_value("at", pin, el, rf)

    def report_slew(self, pin, el, rf):
        return self._pin_value("slew", pin, el, rf)

    def report_rat(self, pin, el, rf):
        return self._pin_value("rat", pin, el, rf)

    def report_slack(self, pin, el, rf):
        return self._pin_value("slack", pin, el, rf)

    def report_load(self, net, el, rf):
        """The net's load: its RC root's (BFS slot 0) load, pin caps
        included (Net::_load, net.cpp:626-636)."""
        i = self._net.get(net)
        if i is None:
            return None
        b = int(self._d.nodes_start[i])
        return float(self._rc_results()["load"][b][el * 2 + rf])

    def rc_node(self, net, pin):
        """load, delay, ldelay, impulse [split][tran] of a pin's node in its
        net's RC tree (RctNode, net.hpp:20-52), or None."""
        i = self._net.get(net)
        if i is None:
            return None
        node = self._d.node_of.get((i, pin))
        if node is None:
            return None
        rc = self._rc_results()
        b = int(self._d.nodes_start[i])
        slot = b + int(rc["node2bfs"][b + node])
        return {k: rc[k][slot].reshape(2, 2).copy() for k in ("load", "delay", "ldelay",
                                                               "impulse")}

    def rc_slew(self, net, pin, el, rf, si):
        """The slew at a pin's RC node for input slew si at the net's root
        (RctNode::slew, ot/timer/net.cpp:30-32): sign(si) * sqrt(si^2 +
        impulse), in float32; None if the pin has no node."""
        v = self.rc_node(net, pin)
        if v is None:
            return None
        si = np.float32(si)
        r = np.sqrt(np.float32(si * si + v["impulse"][el][rf]), dtype=np.float32)
        return float(-r if si < 0 else r)

    def _endpoint_slacks(self, el, rf):
        s = self._results()["slack"][self._d.endpoints, el * 2 + rf]
        return s[~np.isnan(s)]

    def _corners(self, el, rf):
        els = [el] if el is not None else [MIN, MAX]
        rfs = [rf] if rf is not None else [RISE, FALL]
        return [(a, b) for a in els for b in rfs]

    def report_wns(self, el=None, rf=None):
        vals = [float(s.min()) for a, b in self._corners(el, rf)
                if len(s := self._endpoint_slacks(a, b))]
        return min(vals) if vals else None

    def report_tns(self, el=None, rf=None):
        vals = []
        for a, b in self._corners(el, rf):
            s = self._endpoint_slacks(a, b)
            if len(s):
                vals.append(float(np.sum(s[s < 0.0], dtype=np.float32)))
        return float(np.sum(np.asarray(vals, np.float32), dtype=np.float32)) if vals else None

    # --------------------------------------------------------------- paths
    def _path_graph(self):
        if self._pg is None:
            d, keep = self._d, self._d.keep
            g = d.graph
            frm = g.dev["arc_from"][:g.A].cpu().numpy()
            to = g.dev["arc_to"][:g.A].cpu().numpy()
            tests = g.dev["test_arc"][:g.T].cpu().numpy()
            # data-path sources (Pin::is_datapath_source, ot/timer/pin.cpp:
            # 170-190): pins without fanin, clock pins of cells, primary inputs
            source = np.bincount(to, minlength=d.P) == 0
            lib = keep["libs"]["late"]
            for inst, cell, _ in keep["gates"]:
                for cp in lib[cell].get("clock", ()):
                    i = self._pin.get(f"{inst}:{cp}")
                    if i is not None:
                        source[i] = True
            for p in keep.get("ports_in", ()):
                if p in self._pin:
                    source[self._pin[p]] = True
            self._pg = PathGraph(d.names, frm, to, tests, source, d.endpoints)
        if not self._pg_fresh:
            r = self._results()
            self._pg.values(self._d.graph.arc_delays(), r["at"], r["rat"], r["slack"])
            self._pg_fresh = True
        return self._pg

    def report_timing(self, K, el=None, rf=None):
        """The K worst paths (Timer::report_timing(K[, el][, rf]),
        ot/timer/path.cpp:365-420), by ascending slack: paths.Path(slack,
        endpoint (pin, split, transition), points [(pin, transition,
        arrival)]).  K = 1 gives the worst endpoint's path with the
        endpoint's slack; larger K the paths of negative slack only, as the
        reference's prefix-tree search does.  The search runs on the host
        over the device's arrival times and arc delays (paths.py)."""
        self.update_timing()
        return self._path_graph().report_timing(int(K), el, rf)
