"""Generate the committed golden fixtures from the OpenTimer reference itself.

    python tests/golden/make_golden.py            # CPU fixtures (needs the
                                                  # reference tree to build
                                                  # oracle/_ref/libotref.so)
    python tests/golden/make_golden.py --gpu      # adds the fixtures of the
                                                  # reference's own CUDA path
                                                  # (run on a machine with a B200)

CPU fixtures: Rct::update_rc_timing (ot/timer/net.cpp:101-193) on
  * a seeded synthetic forest with random recursive trees, chains, stars,
    paths and the 1- and 2-node edge cases,
  * the RC nets of the bundled c17 and s27 SPEF files, read with the
    reference's own SPEF parser.
GPU fixtures: rct_bfs_and_compute_cuda (ot/cuda/rct.cu:361-397) on the
synthetic forest -- BFS order, pid, directed edges and float outputs -- and
toposort_compute_cuda (ot/cuda/toposort.cu:25-72) on a seeded pin DAG.
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import oracle as O  # noqa: E402
import rcgen  # noqa: E402

REF = os.environ.get("OTG_REFERENCE_DIR", "/root/reference")


def small_forest():
    rng = np.random.default_rng(11)
    sizes = list(rcgen.net_sizes(rng, 90, 2, 300))
    kinds = [None] * len(sizes)
    extra = [(1, "rrt"), (2, "rrt"), (3, "path"), (31, "path"), (32, "chain"), (33, "path"),
             (40, "star"), (64, "chain"), (129, "path"), (257, "star"), (300, "chain")]
    for n, k in extra:
        sizes.append(n)
        kinds.append(k)
    kinds = [k if k else ("chain" if rng.random() < 0.3 else "rrt") for k in kinds]
    return rcgen.forest(11, sizes, kinds)


OUT = HERE


def save(name, **arrs):
    os.makedirs(OUT, exist_ok=True)
    path = os.path.join(OUT, name)
    np.savez_compressed(path, **arrs)
    print("wrote", path, os.path.getsize(path), "bytes")


def forest_arrays(f):
    return dict(nodes_start=f.nodes_start, edges=f.edges, roots=f.roots, res=f.res, cap=f.cap)


def cpu_fixtures():
    f = small_forest()
    st, (load, delay, ldelay, impulse) = O.ref_rct_update(f, 1)
    assert st == 0
    save("rc_cpu_small.npz", **forest_arrays(f), load=load, delay=delay, ldelay=ldelay,
         impulse=impulse)
    for d in ("c17", "s27"):
        g = O.ref_spef_forest(os.path.join(REF, "benchmark", d, d + ".spef"))
        st, (load, delay, ldelay, impulse) = O.ref_rct_update(g, 1)
        assert st == 0
        save(f"rc_cpu_{d}.npz", **forest_arrays(g), load=load, delay=delay, ldelay=ldelay,
             impulse=impulse)


def gpu_fixtures():
    f = small_forest()
    e, node2bfs, pid, (load, delay, ldelay, impulse) = O.ref_rct_gpu(f)
    # the reference never writes the root's pid; normalise it to 0
    b = f.nodes_start[:-1]
    pid[b] = 0
    save("rc_gpu_small.npz", **forest_arrays(f), directed_edges=e, node2bfs=node2bfs, pid=pid,
         load=load, delay=delay, ldelay=ldelay, impulse=impulse)
    fs, fi, od, f0 = rcgen.pin_dag(5, 3000, 7000, 40)
    fr, ends = O.ref_toposort_gpu(len(od), fs, fi, od, f0)
    save("levelize_gpu_small.npz", fanin_start=fs, fanin=fi, out_deg=od, frontier0=f0,
         frontiers=fr[:ends[-1]], frontiers_ends=ends)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--cpu-only", action="store_true")
    ap.add_argument("--out", default=HERE, help="directory for the .npz files")
    a = ap.parse_args()
    OUT = a.out
    if not O.ref_available():
        O.build(ref=True)
    if not a.gpu or not a.cpu_only:
        if not a.gpu:
            cpu_fixtures()
    if a.gpu:
        gpu_fixtures()
