/*
 * otg_oracle.c -- CPU restatement of OpenTimer's RC-net timing and
 * timing-graph levelization.  TEST INFRASTRUCTURE ONLY.
 *
 * The CUDA product path is tested against this file.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
 * product library never links, loads or calls it.
 *
 * Parity pins: the restatement is checked against
 *   - the reference itself, built from its own sources into oracle/_ref/
 *     (Rct::update_rc_timing on the CPU; rct_bfs_and_compute_cuda and
 *     toposort_compute_cuda on a B200), and
 *   - the committed fixtures under tests/golden/ made from those runs.
 *
 * Every function cites the reference lines it restates (paths relative to
 * the OpenTimer source tree).  Build flags: -O2 -ffp-contract=off (no FMA
 * contraction, like the reference's x86-64 -O2 build).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NC 4 /* MAX_SPLIT_TRAN: corner c = el*2 + rf (ot/headerdef.hpp:172-177) */

enum {
  ORC_OK = 0,
  ORC_BAD_INPUT = 1, /* endpoint / root out of range                      */
  ORC_NOT_TREE = 4,  /* some node unreachable from the root (cycle/forest)  */
};

/* Undirected adjacency of one net in edge (RES line) order.
 * adj_start[n+1], adj_edge[2m]: the incident edges of node v, in increasing
 * edge index -- the order Rct::insert_segment appends them to each node's
 * _fanout list (ot/timer/net.cpp:84-98, 336-338). */
static void build_adj(int n, int m, const int* es, int* adj_start, int* adj_edge,
                      int* cursor) {
  memset(adj_start, 0, sizeof(int) * (size_t)(n + 1));
  for (int e = 0; e < m; ++e) {
    adj_start[es[2 * e] + 1]++;
    adj_start[es[2 * e + 1] + 1]++;
  }
  for (int v = 0; v < n; ++v) adj_start[v + 1] += adj_start[v];
  memcpy(cursor, adj_start, sizeof(int) * (size_t)n);
  for (int e = 0; e < m; ++e) {
    adj_edge[cursor[es[2 * e]]++] = e;
    adj_edge[cursor[es[2 * e + 1]]++] = e;
  }
}

/* DFS preorder from the root following each node's incident edges in edge
 * order, skipping the edge back to the parent -- the visit order of the
 * recursive Rct::_update_* passes (ot/timer/net.cpp:127-193).
 * Returns the number of nodes reached.  par_edge[v] = edge to the parent. */
static int dfs_preorder(int n, const int* es, int root, const int* adj_start,
                        const int* adj_edge, int* order, int* parent,
                        int* par_edge, int* stack_node, int* stack_it) {
  for (int v = 0; v < n; ++v) parent[v] = -2;
  int cnt = 0, sp = 0;
  parent[root] = -1;
  par_edge[root] = -1;
  order[cnt++] = root;
  stack_node[sp] = root;
  stack_it[sp] = adj_start[root];
  sp++;
  while (sp) {
    int v = stack_node[sp - 1];
    int it = stack_it[sp - 1];
    if (it == adj_start[v + 1]) {
      sp--;
      continue;
    }
    stack_it[sp - 1] = it + 1;
    int e = adj_edge[it];
    int w = es[2 * e] == v ? es[2 * e + 1] : es[2 * e];
    if (e == par_edge[v]) continue; /* the edge back to the parent */
    if (parent[w] != -2) continue;  /* not a tree: ignore revisits   */
    parent[w] = v;
    par_edge[w] = e;
    order[cnt++] = w;
    stack_node[sp] = w;
    stack_it[sp] = adj_start[w];
    sp++;
  }
  return cnt;
}

typedef struct {
  int *adj_start, *adj_edge, *cursor, *order, *parent, *par_edge, *sn, *si, *dist, *cnt;
} scratch_t;

static int scratch_alloc(scratch_t* s, int n) {
  size_t b = sizeof(int) * (size_t)(n + 2);
  s->adj_start = malloc(b);
  s->adj_edge = malloc(2 * b);
  s->cursor = malloc(b);
  s->order = malloc(b);
  s->parent = malloc(b);
  s->par_edge = malloc(b);
  s->sn = malloc(b);
  s->si = malloc(b);
  s->dist = malloc(b);
  s->cnt = malloc(b);
  return s->adj_start && s->adj_edge && s->cursor && s->order && s->parent && s->par_edge &&
         s->sn && s->si && s->dist && s->cnt;
}
static void scratch_free(scratch_t* s) {
  free(s->adj_start); free(s->adj_edge); free(s->cursor); free(s->order); free(s->parent);
  free(s->par_edge); free(s->sn); free(s->si); free(s->dist); free(s->cnt);
}

static int max_net_nodes(int num_nets, const int* nodes_start) {
  int mx = 1;
  for (int i = 0; i < num_nets; ++i) {
    int n = nodes_start[i + 1] - nodes_start[i];
    if (n > mx) mx = n;
  }
  return mx;
}

/*
 * oracle_rc_bfs -- the flat-RC BFS of compute_net_bfs (ot/cuda/rct.cu:120-245)
 * with its counting-sort placement (ot/cuda/sort.cuh:63-142).
 *
 *   dist   = hop distance from the root over the undirected tree (rct.cu:168-226)
 *   slot   = rank under (dist ascending, local id DEScending): after the
 *            inclusive scan of per-distance counts, ids are visited in
 *            ascending order and take --counts[dist] (sort.cuh:102-121), so
 *            the smallest id of a distance gets the last slot of its range.
 *   edges  = rewritten in place as (parent, child) (rct.cu:184-198)
 *   pid    = pid[slot(child)] = slot(child) - slot(parent) (rct.cu:234-243);
 *            the root's entry, which the reference never writes, is set to 0.
 *
 * edges: [2*E] ints (s,t pairs), E = V - num_nets; net i owns edges
 * [nodes_start[i]-i, nodes_start[i+1]-i-1).  depth (optional, [V]) gets
 * dist by local id.  Returns ORC_OK or the first error code.
 */
int oracle_rc_bfs(int num_nets, const int* nodes_start, const int* roots, int* edges,
                  int* node2bfs, int* pid, int* depth) {
  scratch_t s;
  int mx = max_net_nodes(num_nets, nodes_start);
  if (!scratch_alloc(&s, mx)) { scratch_free(&s); return -1; }
  int status = ORC_OK;
  for (int net = 0; net < num_nets; ++net) {
    int b = nodes_start[net], n = nodes_start[net + 1] - b, m = n - 1;
    int* es = edges + 2 * (size_t)(b - net);
    int root = roots[net];
    int bad = root < 0 || root >= n;
    for (int k = 0; k < 2 * m && !bad; ++k) bad = es[k] < 0 || es[k] >= n;
    if (bad) { if (!status) status = ORC_BAD_INPUT; continue; }
    build_adj(n, m, es, s.adj_start, s.adj_edge, s.cursor);
    /* BFS distances: unique in a tree, any visit order gives the same. */
    for (int v = 0; v < n; ++v) s.dist[v] = -1;
    int head = 0, tail = 0;
    s.order[tail++] = root;
    s.dist[root] = 0;
    while (head < tail) {
      int v = s.order[head++];
      for (int it = s.adj_start[v]; it < s.adj_start[v + 1]; ++it) {
        int e = s.adj_edge[it];
        int w = es[2 * e] == v ? es[2 * e + 1] : es[2 * e];
        if (s.dist[w] < 0) { s.dist[w] = s.dist[v] + 1; s.order[tail++] = w; }
      }
    }
    if (tail != n) { if (!status) status = ORC_NOT_TREE; continue; }
    /* counting sort: ranges per distance, ids in descending order fill them */
    memset(s.cnt, 0, sizeof(int) * (size_t)(n + 1));
    for (int v = 0; v < n; ++v) s.cnt[s.dist[v] + 1]++;
    for (int d = 0; d < n; ++d) s.cnt[d + 1] += s.cnt[d];
    for (int v = n - 1; v >= 0; --v) node2bfs[b + v] = s.cnt[s.dist[v]]++;
    if (depth) for (int v = 0; v < n; ++v) depth[b + v] = s.dist[v];
    pid[b + node2bfs[b + root]] = 0;
    for (int e = 0; e < m; ++e) {
      int u = es[2 * e], w = es[2 * e + 1];
      if (s.dist[u] > s.dist[w]) { es[2 * e] = w; es[2 * e + 1] = u; int t = u; u = w; w = t; }
      int ou = node2bfs[b + u], ow = node2bfs[b + w];
      pid[b + ow] = ow - ou;
    }
  }
  scratch_free(&s);
  return status;
}

/*
 * oracle_rc_prepare -- prepare_res_cap (ot/cuda/rct.cu:314-359): scatter edge
 * resistance to its child's BFS slot (root slot 0 stays 0, rct.cu:378-379) and
 * node capacitance [V][4] to BFS order.  edges must already be directed.
 */
void oracle_rc_prepare(int num_nets, const int* nodes_start, const int* edges,
                       const int* node2bfs, const float* res, const float* cap,
                       float* pres_bfs, float* cap_bfs) {
  for (int net = 0; net < num_nets; ++net) {
    int b = nodes_start[net], n = nodes_start[net + 1] - b, eb = b - net;
    for (int k = 0; k < n; ++k) pres_bfs[b + k] = 0.0f;
    for (int e = 0; e < n - 1; ++e)
      pres_bfs[b + node2bfs[b + edges[2 * (eb + e) + 1]]] = res[eb + e];
    for (int u = 0; u < n; ++u)
      for (int c = 0; c < NC; ++c)
        cap_bfs[(size_t)(b + node2bfs[b + u]) * NC + c] = cap[(size_t)(b + u) * NC + c];
  }
}

/*
 * oracle_rc_elmore_flat_f32 -- compute_net_timing (ot/cuda/rct.cu:11-59): the
 * four sweeps over a net's BFS-ordered nodes, parent = i - pid[i], fp32,
 * outputs [V][4] in BFS order.  Plain fp32 without contraction; the GPU
 * build may fuse multiply-adds, so compare with a tolerance.
 */
void oracle_rc_elmore_flat_f32(int num_nets, const int* nodes_start, const int* pid,
                               const float* pres, const float* cap, float* load,
                               float* delay, float* ldelay, float* impulse) {
  for (int net = 0; net < num_nets; ++net) {
    int st = nodes_start[net], ed = nodes_start[net + 1];
    for (int c = 0; c < NC; ++c) {
#define A(x, i) x[(size_t)(i) * NC + c]
      for (int i = st; i < ed; ++i) {
        A(load, i) = A(cap, i);
        A(delay, i) = A(ldelay, i) = A(impulse, i) = 0.0f;
      }
      for (int i = ed - 1; i > st; --i) A(load, i - pid[i]) += A(load, i);
      for (int i = st + 1; i < ed; ++i) A(delay, i) += A(delay, i - pid[i]) + A(load, i) * pres[i];
      for (int i = ed - 1; i > st; --i) {
        A(ldelay, i) += A(cap, i) * A(delay, i);
        A(ldelay, i - pid[i]) += A(ldelay, i);
      }
      A(ldelay, st) += A(cap, st) * A(delay, st);
      for (int i = st + 1; i < ed; ++i)
        A(impulse, i) += A(impulse, i - pid[i]) + A(ldelay, i) * pres[i];
      for (int i = st; i < ed; ++i) {
        float t = A(delay, i);
        A(impulse, i) = 2 * A(impulse, i) - t * t;
      }
#undef A
    }
  }
}

/*
 * oracle_rc_elmore_cpu_f32 -- Rct::update_rc_timing and its four recursive
 * passes (ot/timer/net.cpp:101-193), fp32, in the reference CPU's exact
 * summation order:
 *   load   (post-order) = ((0 + load(child_1)) + load(child_2) ...) + cap
 *   delay  (pre-order)  = delay(parent) + res * load
 *   ldelay (post-order) = ((0 + ldelay(child_1)) + ...) + cap * delay
 *   beta   (pre-order)  = beta(parent) + res * ldelay
 *   impulse             = (float)((double)(2.0f*beta) - pow((double)delay, 2))
 * with children visited in edge order.  `cap` already holds node + pin
 * capacitance per corner (RctNode::cap, net.cpp:25-27; the root has no pin).
 * Inputs are the UNDIRECTED edges in local ids; outputs [V][4] by local id.
 */
int oracle_rc_elmore_cpu_f32(int num_nets, const int* nodes_start, const int* edges,
                             const int* roots, const float* res, const float* cap,
                             float* load, float* delay, float* ldelay, float* impulse) {
  scratch_t s;
  int mx = max_net_nodes(num_nets, nodes_start);
  if (!scratch_alloc(&s, mx)) { scratch_free(&s); return -1; }
  int status = ORC_OK;
  for (int net = 0; net < num_nets; ++net) {
    int b = nodes_start[net], n = nodes_start[net + 1] - b, m = n - 1, eb = b - net;
    const int* es = edges + 2 * (size_t)eb;
    int root = roots[net];
    int bad = root < 0 || root >= n;
    for (int k = 0; k < 2 * m && !bad; ++k) bad = es[k] < 0 || es[k] >= n;
    if (bad) { if (!status) status = ORC_BAD_INPUT; continue; }
    build_adj(n, m, es, s.adj_start, s.adj_edge, s.cursor);
    int cnt = dfs_preorder(n, es, root, s.adj_start, s.adj_edge, s.order, s.parent, s.par_edge,
                           s.sn, s.si);
    if (cnt != n) { if (!status) status = ORC_NOT_TREE; continue; }
    for (int c = 0; c < NC; ++c) {
#define A(x, v) x[(size_t)(b + (v)) * NC + c]
      /* load: reverse preorder visits every child before its parent; the
         children of v are then summed in edge order. */
      for (int k = n - 1; k >= 0; --k) {
        int v = s.order[k];
        float acc = 0.0f;
        for (int it = s.adj_start[v]; it < s.adj_start[v + 1]; ++it) {
          int e = s.adj_edge[it];
          if (e == s.par_edge[v]) continue;
          int w = es[2 * e] == v ? es[2 * e + 1] : es[2 * e];
          acc += A(load, w);
        }
        acc += A(cap, v);
        A(load, v) = acc;
      }
      for (int k = 0; k < n; ++k) {
        int v = s.order[k];
        if (v == root) { A(delay, v) = 0.0f; continue; }
        float t = res[eb + s.par_edge[v]] * A(load, v);
        A(delay, v) = A(delay, s.parent[v]) + t;
      }
      for (int k = n - 1; k >= 0; --k) {
        int v = s.order[k];
        float acc = 0.0f;
        for (int it = s.adj_start[v]; it < s.adj_start[v + 1]; ++it) {
          int e = s.adj_edge[it];
          if (e == s.par_edge[v]) continue;
          int w = es[2 * e] == v ? es[2 * e + 1] : es[2 * e];
          acc += A(ldelay, w);
        }
        float t = A(cap, v) * A(delay, v);
        acc += t;
        A(ldelay, v) = acc;
      }
      /* beta is kept in `impulse` until the node is final */
      for (int k = 0; k < n; ++k) {
        int v = s.order[k];
        if (v == root) { A(impulse, v) = 0.0f; continue; }
        float t = res[eb + s.par_edge[v]] * A(ldelay, v);
        A(impulse, v) = A(impulse, s.parent[v]) + t;
      }
      for (int k = 0; k < n; ++k) {
        int v = s.order[k];
        float twob = 2.0f * A(impulse, v);
        double d = (double)A(delay, v);
        A(impulse, v) = (float)((double)twob - d * d);
      }
#undef A
    }
  }
  scratch_free(&s);
  return status;
}

/*
 * oracle_rc_elmore_f64 -- the same four passes in double precision (the
 * exact-arithmetic stand-in used to state each implementation's error).
 * Outputs [V][4] doubles by local id.
 */
int oracle_rc_elmore_f64(int num_nets, const int* nodes_start, const int* edges,
                         const int* roots, const float* res, const float* cap, double* load,
                         double* delay, double* ldelay, double* impulse) {
  scratch_t s;
  int mx = max_net_nodes(num_nets, nodes_start);
  if (!scratch_alloc(&s, mx)) { scratch_free(&s); return -1; }
  int status = ORC_OK;
  for (int net = 0; net < num_nets; ++net) {
    int b = nodes_start[net], n = nodes_start[net + 1] - b, m = n - 1, eb = b - net;
    const int* es = edges + 2 * (size_t)eb;
    int root = roots[net];
    int bad = root < 0 || root >= n;
    for (int k = 0; k < 2 * m && !bad; ++k) bad = es[k] < 0 || es[k] >= n;
    if (bad) { if (!status) status = ORC_BAD_INPUT; continue; }
    build_adj(n, m, es, s.adj_start, s.adj_edge, s.cursor);
    int cnt = dfs_preorder(n, es, root, s.adj_start, s.adj_edge, s.order, s.parent, s.par_edge,
                           s.sn, s.si);
    if (cnt != n) { if (!status) status = ORC_NOT_TREE; continue; }
    for (int c = 0; c < NC; ++c) {
#define A(x, v) x[(size_t)(b + (v)) * NC + c]
#define C(v) ((double)cap[(size_t)(b + (v)) * NC + c])
      for (int k = n - 1; k >= 0; --k) {
        int v = s.order[k];
        double acc = 0.0;
        for (int it = s.adj_start[v]; it < s.adj_start[v + 1]; ++it) {
          int e = s.adj_edge[it];
          if (e == s.par_edge[v]) continue;
          acc += A(load, es[2 * e] == v ? es[2 * e + 1] : es[2 * e]);
        }
        A(load, v) = acc + C(v);
      }
      for (int k = 0; k < n; ++k) {
        int v = s.order[k];
        A(delay, v) = v == root ? 0.0
                                : A(delay, s.parent[v]) + (double)res[eb + s.par_edge[v]] * A(load, v);
      }
      for (int k = n - 1; k >= 0; --k) {
        int v = s.order[k];
        double acc = 0.0;
        for (int it = s.adj_start[v]; it < s.adj_start[v + 1]; ++it) {
          int e = s.adj_edge[it];
          if (e == s.par_edge[v]) continue;
          acc += A(ldelay, es[2 * e] == v ? es[2 * e + 1] : es[2 * e]);
        }
        A(ldelay, v) = acc + C(v) * A(delay, v);
      }
      for (int k = 0; k < n; ++k) {
        int v = s.order[k];
        A(impulse, v) = v == root ? 0.0
                                  : A(impulse, s.parent[v]) + (double)res[eb + s.par_edge[v]] * A(ldelay, v);
      }
      for (int k = 0; k < n; ++k) {
        int v = s.order[k];
        A(impulse, v) = 2.0 * A(impulse, v) - A(delay, v) * A(delay, v);
      }
#undef C
#undef A
    }
  }
  scratch_free(&s);
  return status;
}

/*
 * oracle_sink_slew -- RctNode::slew / FlatRct::slew (ot/timer/net.cpp:30-32,
 * 280-283): slew = sign(si) * sqrt(si^2 + impulse) at each sink node.
 * impulse is [V][4] by LOCAL id here; sink_nodes are local ids.
 */
void oracle_sink_slew(int num_nets, const int* nodes_start, const int* sinks_start,
                      const int* sink_nodes, const float* driver_slew,
                      const float* impulse_local, float* sink_slew) {
  for (int net = 0; net < num_nets; ++net) {
    int b = nodes_start[net];
    for (int k = sinks_start[net]; k < sinks_start[net + 1]; ++k) {
      int v = sink_nodes[k];
      for (int c = 0; c < NC; ++c) {
        float si = driver_slew[(size_t)net * NC + c];
        float imp = impulse_local[(size_t)(b + v) * NC + c];
        float r = sqrtf(si * si + imp);
        sink_slew[(size_t)k * NC + c] = si < 0.0f ? -r : r;
      }
    }
  }
}

static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/*
 * oracle_levelize -- the frontier Kahn levelization of toposort_advance /
 * toposort_compute_cuda (ot/cuda/toposort.cu:4-72) over the fanin CSR built
 * by Timer::_build_prop_tasks_cuda (ot/timer/timer.cpp:996-1071).
 *
 * Frontier 0 is the caller's seed (pins with no candidate fanout).  A pin
 * joins frontier k+1 when the last of its fanouts leaves frontier k, so
 * level(v) = 1 + max level over its candidate fanouts (longest path to a
 * sink).  The reference's order inside a level depends on atomics; this
 * oracle keeps frontier 0 in seed order and sorts every later level by
 * ascending pin index -- the deterministic order the CUDA path promises.
 *
 * out_deg is copied, not consumed.  order[] gets the concatenated levels,
 * level_ends[0..L] the boundaries (level_ends[0] = 0), level[v] the level
 * or -1.  Returns the number of pins emitted.
 */
int oracle_levelize(int n, const int* fanin_start, const int* fanin, const int* out_deg,
                    const int* frontier0, int first_size, int* order, int* level_ends,
                    int* num_levels, int* level) {
  int* out = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  memcpy(out, out_deg, sizeof(int) * (size_t)n);
  for (int v = 0; v < n; ++v) level[v] = -1;
  int total = 0, L = 0;
  level_ends[0] = 0;
  for (int k = 0; k < first_size; ++k) {
    order[total++] = frontier0[k];
    level[frontier0[k]] = 0;
  }
  if (first_size > 0) { L = 1; level_ends[1] = total; }
  int lo = 0, hi = total;
  while (hi > lo) {
    int nxt = hi;
    for (int k = lo; k < hi; ++k) {
      int u = order[k];
      for (int i = fanin_start[u]; i < fanin_start[u + 1]; ++i) {
        int v = fanin[i];
        if (--out[v] == 0) { order[nxt++] = v; level[v] = L; }
      }
    }
    if (nxt == hi) break;
    qsort(order + hi, (size_t)(nxt - hi), sizeof(int), cmp_int);
    lo = hi;
    hi = nxt;
    level_ends[++L] = hi;
  }
  *num_levels = L;
  free(out);
  return hi;
}
