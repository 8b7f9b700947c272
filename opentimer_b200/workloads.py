"""Seeded synthetic workloads (numpy, host side).

net_sizes      log-uniform RC net sizes -> nodes_start (the batched-Elmore
               workload: 1M nets of 2..4096 nodes, heavy tail)
pin_dag        levelled timing pin DAG in the fanin-CSR layout of
               Timer::_build_prop_tasks_cuda (ot/timer/timer.cpp:996-1061):
               pins spread over `levels` logic levels, fanin 1..4 uniform,
               sources drawn with a geometric-like skew so fanout has mean
               edges/pins, plus a fraction of high-fanout drivers with
               500..5000 sinks.
"""
import numpy as np


def net_sizes(seed, num_nets, lo=2, hi=4096):
    rng = np.random.default_rng(seed)
    u = rng.random(num_nets)
    n = np.floor(np.exp(np.log(lo) + u * (np.log(hi + 1) - np.log(lo)))).astype(np.int64)
    n = np.clip(n, lo, hi)
    ns = np.zeros(num_nets + 1, np.int64)
    ns[1:] = np.cumsum(n)
    if ns[-1] >= 2 ** 31:
        raise ValueError("more than 2^31-1 nodes")
    return ns.astype(np.int32)


def pin_dag(seed, n_pins, n_edges, levels, hf_frac=0.02, hf_lo=500, hf_hi=5000):
    """Returns (fanin_start, fanin, out_deg, frontier0), int32.

    Every level k >= 1 pin gets one fanin from level k-1 (so the DAG has
    exactly `levels` levels), the remaining fanins come from any earlier
    level.  A `hf_frac` share of the non-sink levels' pins become
    high-fanout drivers: each is the fanin of hf_lo..hf_hi later pins."""
    rng = np.random.default_rng(seed)
    lvl = np.sort(rng.integers(0, levels, n_pins))
    lvl[:levels] = np.arange(levels)
    lvl = np.sort(lvl)
    perm = rng.permutation(n_pins)  # pin index -> shuffled position
    level_of = np.empty(n_pins, np.int64)
    level_of[perm] = lvl
    starts = np.searchsorted(lvl, np.arange(levels + 1))
    by_pos = perm  # position i (sorted by level) holds pin perm[i]

    def pick_from_levels(lo_pos_end, count):
        # uniform among pins at sorted positions [0, lo_pos_end)
        return by_pos[(rng.random(count) * lo_pos_end).astype(np.int64)]

    dst_list, src_list = [], []
    # chain edge: each pin of level k>=1 takes one fanin from level k-1
    for k in range(1, levels):
        a, b = starts[k - 1], starts[k]
        cur = by_pos[starts[k]:starts[k + 1]]
        src_list.append(by_pos[a + (rng.random(len(cur)) * (b - a)).astype(np.int64)])
        dst_list.append(cur)
    base_edges = sum(len(d) for d in dst_list)
    # high-fanout drivers
    n_hf = int(hf_frac * n_pins / 100) if hf_frac > 0 else 0
    hf_edges = 0
    if n_hf:
        drv_pos = (rng.random(n_hf) * starts[levels // 2]).astype(np.int64)
        for p in drv_pos:
            k = int(np.searchsorted(starts, p, side="right") - 1)
            lo = starts[k + 1]
            if lo >= n_pins:
                continue
            cnt = int(rng.integers(hf_lo, hf_hi + 1))
            sinks = by_pos[lo + (rng.random(cnt) * (n_pins - lo)).astype(np.int64)]
            src_list.append(np.full(cnt, by_pos[p]))
            dst_list.append(sinks)
            hf_edges += cnt
    # remaining fanins: uniform among earlier levels, 0..3 extra per pin
    extra = max(0, n_edges - base_edges - hf_edges)
    if extra:
        dst_pos = starts[1] + (rng.random(extra) * (n_pins - starts[1])).astype(np.int64)
        dst = by_pos[dst_pos]
        k = np.searchsorted(starts, dst_pos, side="right") - 1
        src = by_pos[(rng.random(extra) * starts[k]).astype(np.int64)]
        src_list.append(src)
        dst_list.append(dst)
    src = np.concatenate(src_list).astype(np.int64)
    dst = np.concatenate(dst_list).astype(np.int64)
    key = np.unique(dst * n_pins + src)  # dedupe, sorted by (dst, src)
    dst, src = key // n_pins, key % n_pins
    fanin_start = np.zeros(n_pins + 1, np.int64)
    np.add.at(fanin_start, dst + 1, 1)
    fanin_start = np.cumsum(fanin_start)
    out_deg = np.bincount(src, minlength=n_pins)
    frontier0 = np.nonzero(out_deg == 0)[0]
    return (fanin_start.astype(np.int32), src.astype(np.int32), out_deg.astype(np.int32),
            frontier0.astype(np.int32))


# ------------------------------------------------------------ gate designs
# A gate-level view of a synthetic RC forest, for the incremental and
# serving workloads: gate g drives net g (its output pin is the net's root)
# and has 1..2 input pins, each a distinct sink node of another net.
# Resizing a gate changes its drive (the driver slew of net g) and its
# input pin caps (the cap of those sink nodes), which dirties 1..3 nets.

def uniform_sizes(seed, num_nets, lo=2, hi=16):
    """Net sizes uniform in [lo, hi] (the small-design RC trees)."""
    rng = np.random.default_rng(seed)
    ns = np.zeros(num_nets + 1, np.int64)
    ns[1:] = np.cumsum(rng.integers(lo, hi + 1, num_nets))
    return ns.astype(np.int32)


def gate_map(seed, design):
    """Input pins of each gate: (in_start[G+1], in_net, in_node), gate g
    driving net g.  Sinks are drawn without replacement; a gate whose draw
    would land on its own net keeps one input fewer."""
    rng = np.random.default_rng(seed)
    ss = design["sinks_start"]
    G = len(ss) - 1
    S = int(ss[-1])
    k = rng.integers(1, 3, G)
    total = int(k.sum())
    if total > S:
        raise ValueError("fewer sinks than gate inputs")
    pick = rng.choice(S, total, replace=False)
    net_of_sink = np.repeat(np.arange(G), np.diff(ss))
    gate = np.repeat(np.arange(G), k)
    keep = net_of_sink[pick] != gate
    gate, pick = gate[keep], pick[keep]
    in_start = np.zeros(G + 1, np.int64)
    in_start[1:] = np.cumsum(np.bincount(gate, minlength=G))
    return {"in_start": in_start.astype(np.int32),
            "in_net": net_of_sink[pick].astype(np.int32),
            "in_node": design["sink_nodes"][pick].astype(np.int32)}


def resize(rng, gmap, gates):
    """Updates of resizing `gates` (int array): ((cap_net, cap_node,
    cap[k,4]), (slew_net, slew[k,4])) with new values drawn from the
    generator's ranges (pin cap 0.05..5 fF, driver slew 5..200 ps)."""
    st = gmap["in_start"]
    cnt = st[gates + 1] - st[gates]
    idx = np.repeat(st[gates] - np.cumsum(cnt) + cnt, cnt) + np.arange(int(cnt.sum()))
    cap = (gmap["in_net"][idx], gmap["in_node"][idx],
           rng.uniform(0.05, 5.0, (len(idx), 4)).astype(np.float32))
    slew = (gates.astype(np.int32), rng.uniform(5.0, 200.0, (len(gates), 4)).astype(np.float32))
    return cap, slew


def request_trace(seed, gmaps, num_req, rate, lo=1, hi=64, design_of=None, arrival=None):
    """A request stream over several designs: request r resizes lo..hi
    distinct random gates of design design_of[r] (uniform over designs when
    not given).  Arrivals are Poisson at `rate` req/s unless `arrival`
    (ns) is given.  Returns the flat arrays otg_server_replay reads, plus
    the resized gates (gates, gate_start) for per_gate_trace."""
    rng = np.random.default_rng(seed)
    D = len(gmaps)
    if design_of is None:
        design_of = rng.integers(0, D, num_req)
    if arrival is None:
        arrival = np.cumsum(rng.exponential(1e9 / rate, num_req)).astype(np.int64)
    caps, slews, gl = [], [], []
    for r in range(num_req):
        g = gmaps[design_of[r]]
        G = len(g["in_start"]) - 1
        n = min(int(rng.integers(lo, hi + 1)), G)
        gates = rng.choice(G, n, replace=False) if n < G // 4 else rng.permutation(G)[:n]
        c, s = resize(rng, g, gates)
        caps.append(c)
        slews.append(s)
        gl.append(gates)
    return _flat(arrival, design_of, caps, slews, gl)


def _flat(arrival, design_of, caps, slews, gl):
    num_req = len(caps)
    cap_start = np.zeros(num_req + 1, np.int64)
    cap_start[1:] = np.cumsum([len(c[0]) for c in caps])
    slew_start = np.zeros(num_req + 1, np.int64)
    slew_start[1:] = np.cumsum([len(s[0]) for s in slews])
    gate_start = np.zeros(num_req + 1, np.int64)
    gate_start[1:] = np.cumsum([len(g) for g in gl])
    cat = lambda xs, dt, shape: (np.concatenate(xs).astype(dt) if xs else np.zeros(shape, dt))  # noqa: E731
    return {
        "arrival_ns": np.asarray(arrival, np.int64),
        "design": np.asarray(design_of, np.int32),
        "cap_start": cap_start.astype(np.int32),
        "cap_net": cat([c[0] for c in caps], np.int32, 0),
        "cap_node": cat([c[1] for c in caps], np.int32, 0),
        "cap_val": cat([c[2] for c in caps], np.float32, (0, 4)),
        "slew_start": slew_start.astype(np.int32),
        "slew_net": cat([s[0] for s in slews], np.int32, 0),
        "slew_val": cat([s[1] for s in slews], np.float32, (0, 4)),
        "gate_start": gate_start.astype(np.int32),
        "gates": cat(gl, np.int32, 0),
    }


def per_gate_trace(trace, gmaps, num_req=None, arrival=None):
    """The same updates as `trace` (its first num_req requests), split into
    one request per resized gate, in order -- the per-update workload."""
    R = len(trace["design"]) if num_req is None else num_req
    caps, slews, gl, des = [], [], [], []
    for r in range(R):
        g = gmaps[trace["design"][r]]
        st = g["in_start"]
        c0 = trace["cap_start"][r]
        s0 = trace["slew_start"][r]
        for i, gate in enumerate(trace["gates"][trace["gate_start"][r]:trace["gate_start"][r + 1]]):
            k = int(st[gate + 1] - st[gate])
            sl = slice(c0, c0 + k)
            caps.append((trace["cap_net"][sl], trace["cap_node"][sl], trace["cap_val"][sl]))
            slews.append((trace["slew_net"][s0 + i:s0 + i + 1], trace["slew_val"][s0 + i:s0 + i + 1]))
            gl.append(np.array([gate]))
            des.append(trace["design"][r])
            c0 += k
    if arrival is None:
        arrival = np.zeros(len(des), np.int64)
    return _flat(arrival, des, caps, slews, gl)


def apply_trace(design, trace, num_req=None):
    """Applies a trace's updates to a host design dict in place (later
    updates of the same node or net win)."""
    R = len(trace["design"]) if num_req is None else num_req
    ns = design["nodes_start"]
    c1 = trace["cap_start"][R]
    s1 = trace["slew_start"][R]
    idx = ns[trace["cap_net"][:c1]].astype(np.int64) + trace["cap_node"][:c1]
    last = len(idx) - 1 - np.unique(idx[::-1], return_index=True)[1]
    design["cap"][idx[last]] = trace["cap_val"][:c1][last]
    net = trace["slew_net"][:s1]
    last = len(net) - 1 - np.unique(net[::-1], return_index=True)[1]
    design["driver_slew"][net[last]] = trace["slew_val"][:s1][last]


def write_spef(path, forest, seed=0):
    """Writes a flat RC forest (host dict as from synth_forest_host, with
    sink_count) as SPEF text: one *D_NET per net, the root named as the
    driver pin D<i>:Z, leaves as sink pins S<i>_<k>:A, other nodes
    n<i>:<k>; *RES lines in edge order (so the flat ids come back as the
    forest's own ids), ground caps from corner 0, units ohm / fF / ns.
    Returns the number of nodes written."""
    ns = forest["nodes_start"]
    edges, roots, res, cap = forest["edges"], forest["roots"], forest["res"], forest["cap"]
    N = len(ns) - 1
    out = ['*SPEF "IEEE 1481-1998"', '*DESIGN "synth"', "*DIVIDER /", "*DELIMITER :",
           "*T_UNIT 1 NS", "*C_UNIT 1 FF", "*R_UNIT 1 OHM", "*L_UNIT 1 HENRY", ""]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
        for i in range(N):
            b, e = int(ns[i]), int(ns[i + 1])
            n = e - b
            eb = b - i
            deg = np.zeros(n, np.int64)
            ed = edges[eb:eb + n - 1]
            np.add.at(deg, ed.reshape(-1), 1)
            r = int(roots[i])
            names = [f"n{i}:{k}" for k in range(n)]
            names[r] = f"D{i}:Z"
            sinks = [k for k in range(n) if k != r and deg[k] == 1]
            for k in sinks:
                names[k] = f"S{i}_{k}:A"
            lines = [f"*D_NET N{i} {float(cap[b:e, 0].sum()):.6g}", "*CONN", f"*I D{i}:Z O"]
            lines += [f"*I {names[k]} I" for k in sinks]
            lines.append("*CAP")
            lines += [f"{k + 1} {names[k]} {float(cap[b + k, 0]):.7g}" for k in range(n)]
            lines.append("*RES")
            lines += [f"{j + 1} {names[int(ed[j, 0])]} {names[int(ed[j, 1])]} "
                      f"{float(res[eb + j]):.7g}" for j in range(n - 1)]
            lines.append("*END\n")
            f.write("\n".join(lines) + "\n")
    return int(ns[-1])
