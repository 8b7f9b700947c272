"""Shared checks for the parity tests."""
import numpy as np

# Elmore tolerance: per node |got - ref| <= RTOL*|ref| + AFLOOR*max_net|ref|,
# per quantity and corner (max over the node's net).
RTOL = 1e-5
AFLOOR = 1e-6


def net_max(nodes_start, x):
    """Per-node broadcast of max |x| over the node's net; x is [V,4]."""
    ax = np.abs(x)
    sizes = np.diff(nodes_start)
    m = np.maximum.reduceat(ax, nodes_start[:-1], axis=0) if len(sizes) else ax
    return np.repeat(m, sizes, axis=0)


def elmore_err(nodes_start, got, ref):
    """Max of |got-ref| / (RTOL*|ref| + AFLOOR*netmax|ref|); <= 1 passes."""
    tol = RTOL * np.abs(ref) + AFLOOR * net_max(nodes_start, ref)
    tol = np.maximum(tol, np.finfo(np.float32).tiny)
    return float(np.max(np.abs(got.astype(np.float64) - ref.astype(np.float64)) / tol)) \
        if ref.size else 0.0


def worst_net(nodes_start, got, ref):
    """(err/tol, net index) of the worst net -- for failure messages."""
    tol = RTOL * np.abs(ref) + AFLOOR * net_max(nodes_start, ref)
    e = np.abs(got.astype(np.float64) - ref) / np.maximum(tol, np.finfo(np.float32).tiny)
    per = np.maximum.reduceat(e.max(1), nodes_start[:-1])
    i = int(np.argmax(per))
    return float(per[i]), i


def max_rel_vs_f64(nodes_start, got, exact):
    """Largest error relative to max(|exact|, netmax|exact|*1e-1...) reported
    as plain max |got-exact| / netmax|exact| (a size-independent figure)."""
    nm = np.maximum(net_max(nodes_start, exact), 1e-30)
    return float(np.max(np.abs(got.astype(np.float64) - exact) / nm)) if exact.size else 0.0


def bfs_local(nodes_start, node2bfs, arr_bfs):
    b = np.repeat(nodes_start[:-1], np.diff(nodes_start))
    return arr_bfs[b + node2bfs]


def levels_as_sets(order, ends):
    return [sorted(order[ends[k]:ends[k + 1]].tolist()) for k in range(len(ends) - 1)]


def pin_err(got, ref, rtol=1e-5, atol=1e-5):
    """Worst |got - ref| / (rtol s + atol) over pins and quantities, for
    {pin: [4,4]} (at, slew, rat, slack by corner): s = |ref| for at and slew
    and max(|ref|, |ref at|) for rat and slack (their rounding follows the
    arrival time).  inf where one side has a value the other lacks."""
    worst = 0.0
    for name, r in ref.items():
        g = got[name]
        m = ~np.isnan(r)
        if not np.array_equal(m, ~np.isnan(g)):
            return float("inf")
        scale = np.abs(r)
        scale[2:] = np.maximum(scale[2:], np.nan_to_num(np.abs(r[0])))
        if m.any():
            worst = max(worst, float(np.max(np.abs(g[m] - r[m]) / (rtol * scale[m] + atol))))
    return worst


def read_ref_pins(path):
    """P lines of oracle/ot_run.cpp's output: {pin: [4,4]}."""
    pins = {}
    with open(path) as f:
        for line in f:
            if line.startswith("P "):
                t = line.split()
                pins[t[1]] = np.array([float(x) for x in t[2:]], np.float64).reshape(4, 4)
    return pins
