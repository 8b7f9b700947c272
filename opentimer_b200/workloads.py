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
