/*
 * synth_host.c -- the seeded batched-Elmore workload (RC forests) generated
 * on the host, for the reference arm of bench.py.  TEST / BENCHMARK
 * INFRASTRUCTURE ONLY: it lets the reference's own CPU path be timed on
 * exactly the nets the GPU arm times without loading the product library.
 *
 * It restates, bit for bit, the generator of the product library
 * (otg_synth_rc_forest / otg_synth_rc_forest_host): a splitmix64 stream per
 * net, 24-bit uniforms (exact in fp32) and correctly rounded fmaf only, so
 * the host and device results are identical.  tests/test_oracle.py checks
 * the two against each other.
 *
 * Per net (node count from nodes_start):
 *   - 30% chains with side branches (a spine of 80% of the nodes, the rest
 *     hung on uniformly chosen spine nodes), 70% random recursive trees;
 *   - the edge list shuffled (Fisher-Yates) and each edge randomly
 *     oriented, then local ids by first appearance over the edges -- the id
 *     rule of Net::_make_flat_rct (ot/timer/net.cpp:392-410); the root is
 *     canonical node 0;
 *   - R ~ U(0.1, 50) per edge, ground C ~ U(0.05, 5) per node, plus a
 *     per-corner pin cap U(0.5, 2) on every leaf; driver slew U(5, 200).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct {
  uint64_t s;
} rng_t;

static uint64_t rng_next(rng_t* g) {
  g->s += 0x9E3779B97F4A7C15ull;
  uint64_t z = g->s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static float rng_unif(rng_t* g) { return (float)(rng_next(g) >> 40) * (1.0f / 16777216.0f); }
static float rng_range(rng_t* g, float lo, float hi) { return fmaf(rng_unif(g), hi - lo, lo); }
static uint32_t rng_below(rng_t* g, uint32_t k) {
  return (uint32_t)(((rng_next(g) >> 32) * (uint64_t)k) >> 32);
}

#define LEAF_BIT (1 << 30)

static void synth_one(uint64_t seed, int first_net, int net, const int* nodes_start, int* edges,
                      int* roots, float* res, float* cap, float* slew, int* sink_count, int* S) {
  const int b = nodes_start[net];
  const int n = nodes_start[net + 1] - b;
  const int m = n - 1;
  const int eb = b - net;
  int* E = edges + 2 * (size_t)eb;
  rng_t g = {seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(first_net + net + 1))};
  const int chain = rng_unif(&g) < 0.3f;
  const int spine = (n * 4) / 5 > 0 ? (n * 4) / 5 : 1;
  for (int v = 0; v < n; ++v) S[v] = 0;
  for (int i = 1; i < n; ++i) {
    int p;
    if (chain) p = (i < spine) ? i - 1 : (int)rng_below(&g, (uint32_t)spine);
    else p = (int)rng_below(&g, (uint32_t)i);
    E[2 * (i - 1)] = p;
    E[2 * (i - 1) + 1] = i;
    S[p] += 1;
  }
  int leaves = 0;
  for (int v = 0; v < n; ++v) {
    const int leaf = v != 0 && S[v] == 0;
    S[v] = leaf ? LEAF_BIT : 0;
    leaves += leaf;
  }
  for (int i = m - 1; i > 0; --i) {
    const int j = (int)rng_below(&g, (uint32_t)(i + 1));
    const int tx = E[2 * i], ty = E[2 * i + 1];
    E[2 * i] = E[2 * j];
    E[2 * i + 1] = E[2 * j + 1];
    E[2 * j] = tx;
    E[2 * j + 1] = ty;
  }
  for (int i = 0; i < m; ++i)
    if (rng_next(&g) & 1ull) {
      const int t = E[2 * i];
      E[2 * i] = E[2 * i + 1];
      E[2 * i + 1] = t;
    }
  int cnt = 0;
  for (int i = 0; i < m; ++i) {
    const int x = E[2 * i], y = E[2 * i + 1];
    if ((S[x] & (LEAF_BIT - 1)) == 0) S[x] |= ++cnt;
    if ((S[y] & (LEAF_BIT - 1)) == 0) S[y] |= ++cnt;
    E[2 * i] = (S[x] & (LEAF_BIT - 1)) - 1;
    E[2 * i + 1] = (S[y] & (LEAF_BIT - 1)) - 1;
  }
  if (n == 1) S[0] |= ++cnt;
  roots[net] = (S[0] & (LEAF_BIT - 1)) - 1;
  for (int i = 0; i < m; ++i) res[eb + i] = rng_range(&g, 0.1f, 50.0f);
  for (int v = 0; v < n; ++v) {
    const int l = (S[v] & (LEAF_BIT - 1)) - 1;
    const float c = rng_range(&g, 0.05f, 5.0f);
    float* o = cap + 4 * (size_t)(b + l);
    o[0] = o[1] = o[2] = o[3] = c;
    if (S[v] & LEAF_BIT) {
      o[0] += rng_range(&g, 0.5f, 2.0f);
      o[1] += rng_range(&g, 0.5f, 2.0f);
      o[2] += rng_range(&g, 0.5f, 2.0f);
      o[3] += rng_range(&g, 0.5f, 2.0f);
    }
  }
  float* sl = slew + 4 * (size_t)net;
  sl[0] = rng_range(&g, 5.0f, 200.0f);
  sl[1] = rng_range(&g, 5.0f, 200.0f);
  sl[2] = rng_range(&g, 5.0f, 200.0f);
  sl[3] = rng_range(&g, 5.0f, 200.0f);
  sink_count[net] = leaves;
}

typedef struct {
  uint64_t seed;
  int first_net, net0, net1;
  const int* nodes_start;
  int *edges, *roots, *sink_count, *scratch;
  float *res, *cap, *slew;
} job_t;

static void* synth_range(void* p) {
  const job_t* j = (const job_t*)p;
  for (int net = j->net0; net < j->net1; ++net)
    synth_one(j->seed, j->first_net, net, j->nodes_start, j->edges, j->roots, j->res, j->cap, j->slew,
              j->sink_count, j->scratch + j->nodes_start[net]);
  return NULL;
}

/* Nets first_net .. first_net+num_nets-1 of the workload with the given
 * seed: edges [V-N][2], roots [N], res [V-N], cap [V][4], slew [N][4],
 * sink_count [N] (leaves per net).  nodes_start[num_nets+1] holds the
 * slice's node offsets from 0 (net k of the output is net first_net+k of
 * the workload).  Nets are split over `threads` host threads.  Returns 0,
 * or -1 when out of memory. */
int oracle_synth_rc_forest(uint64_t seed, int first_net, int num_nets, const int* nodes_start,
                           int* edges, int* roots, float* res, float* cap, float* slew,
                           int* sink_count, int threads) {
  if (num_nets <= 0) return 0;
  int* scratch = (int*)malloc(sizeof(int) * (size_t)(nodes_start[num_nets] > 0
                                                          ? nodes_start[num_nets] : 1));
  if (!scratch) return -1;
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  if (threads > num_nets) threads = num_nets;
  pthread_t tid[256];
  job_t job[256];
  /* split by nodes so the threads get similar work */
  const long long V = nodes_start[num_nets] - nodes_start[0];
  int net = 0;
  for (int t = 0; t < threads; ++t) {
    const long long goal = nodes_start[0] + (V * (t + 1)) / threads;
    int end = net;
    while (end < num_nets && (t == threads - 1 || nodes_start[end] < goal)) ++end;
    job[t] = (job_t){seed, first_net, net, end, nodes_start, edges, roots, sink_count, scratch, res, cap,
                     slew};
    net = end;
  }
  int joined[256];
  for (int t = 0; t < threads; ++t) {
    joined[t] = pthread_create(&tid[t], NULL, synth_range, &job[t]) == 0;
    if (!joined[t]) synth_range(&job[t]);
  }
  for (int t = 0; t < threads; ++t)
    if (joined[t]) pthread_join(tid[t], NULL);
  free(scratch);
  return 0;
}
