/*
 * otg.h -- C ABI of the B200-native RC-net timing and levelization library
 * (libotg.so).  Plain pointers and sizes only; every device entry point is
 * asynchronous on the caller's stream and allocates nothing -- the caller
 * passes a workspace whose size comes from the matching *_workspace_size
 * query (the cuBLAS/cuDNN workspace pattern).
 *
 * Layout conventions follow OpenTimer's flat RC storage (FlatRctStorage,
 * ot/timer/net.hpp:149-166, and RctEdgeArrayCUDA, ot/cuda/rct.cuh:20-42):
 *   corner c = split*2 + tran  (MIN=0,MAX=1; RISE=0,FALL=1;
 *                               ot/headerdef.hpp:79-91,172-177)
 *   nodes_start[N+1]  node offsets; net i owns nodes [ns[i], ns[i+1])
 *   edges[E]          E = V - N; net i owns edges [ns[i]-i, ns[i+1]-i-1),
 *                     local node ids, SPEF *RES order
 *   per-node arrays   [V][4] floats, corner-interleaved (16 B per node)
 */
#ifndef OTG_H_
#define OTG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* otg_stream_t; /* == cudaStream_t */

typedef enum otg_status {
  OTG_OK = 0,
  OTG_ERR_INVALID = 1,     /* bad argument, or an edge/root id out of range   */
  OTG_ERR_CUDA = 2,        /* a CUDA runtime call failed                      */
  OTG_ERR_OOM = 3,         /* device or host allocation failed                */
  OTG_ERR_NOT_TREE = 4,    /* an RC net is not a tree spanning its nodes      */
  OTG_ERR_CYCLE = 5,       /* levelization left pins unemitted (a cycle)      */
  OTG_ERR_TIMEOUT = 6,     /* a bounded device wait gave up                   */
  OTG_ERR_TOO_LARGE = 7,   /* a net exceeds the size the workspace was sized for */
  OTG_ERR_WORKSPACE = 8,   /* workspace smaller than the query returned       */
  OTG_ERR_ADMISSION = 9,   /* a request does not fit the device memory budget */
} otg_status;

/* One RC edge; same layout as RctEdgeCUDA {int s; int t;} (ot/cuda/rct.cuh:15-18). */
typedef struct otg_rc_edge {
  int32_t s;
  int32_t t;
} otg_rc_edge;

/*
 * A batch of RC nets on the DEVICE (all pointers are device pointers).
 * Replaces the device half of RctEdgeArrayCUDA (ot/cuda/rct.cuh:20-42).
 *
 * inputs : nodes_start, edges (undirected), roots (local id of the driver),
 *          edges_res [E], nodes_cap [V][4] (original order, pin caps of
 *          non-root pins already added as in Net::_make_flat_rct,
 *          ot/timer/net.cpp:425-446)
 * outputs: edges rewritten in place to (parent, child)
 *          node2bfs[V]  BFS slot of each local id (net-relative)
 *          pid[V]       BFS order; parent of slot i is i - pid[i]; root 0
 *          load/delay/ldelay/impulse [V][4] in BFS order
 * optional sink-slew epilogue (all four NULL to skip):
 *          sinks_start[N+1], sink_nodes[S] (local ids),
 *          driver_slew[N][4] in, sink_slew[S][4] out:
 *          slew = sign(si) * sqrt(si^2 + impulse)  (ot/timer/net.cpp:30-32)
 * BFS order is the reference's: distance from the root ascending, ties by
 * local id DESCENDING (ot/cuda/rct.cu:120-245, ot/cuda/sort.cuh:102-121).
 */
typedef struct otg_rc_forest {
  int32_t num_nets;
  int32_t total_nodes;
  const int32_t* nodes_start;
  otg_rc_edge* edges;
  const int32_t* roots;
  const float* edges_res;
  const float* nodes_cap;
  int32_t* node2bfs;
  int32_t* pid;
  float* load;
  float* delay;
  float* ldelay;
  float* impulse;
  const int32_t* sinks_start;
  const int32_t* sink_nodes;
  const float* driver_slew;
  float* sink_slew;
} otg_rc_forest;

/* Workspace bytes for otg_rc_timing over num_nets nets none of which has
 * more than max_net_nodes nodes. */
otg_status otg_rc_workspace_size(int32_t num_nets, int32_t max_net_nodes, size_t* bytes);

/*
 * otg_rc_timing -- RC-tree BFS flattening + Elmore load/delay/ldelay/impulse
 * for 2 splits x 2 transitions, fused in one pass over HBM.  Replaces
 * compute_net_bfs + prepare_res_cap + compute_net_timing
 * (ot/cuda/rct.cu:11-59,120-245,314-359) and the CPU Rct::update_rc_timing
 * (ot/timer/net.cpp:101-193).  Asynchronous on `stream`; device-detected
 * errors (bad ids, non-tree nets, oversize nets) are recorded in the
 * workspace and returned by otg_rc_status().
 */
otg_status otg_rc_timing(const otg_rc_forest* forest, int32_t max_net_nodes, void* workspace,
                         size_t workspace_bytes, otg_stream_t stream);

/*
 * otg_rc_timing_subset -- the same pass over only the nets listed in
 * net_list[0 .. *num_listed) (device memory, at most max_listed entries):
 * the incremental update of dirty nets.  The list and its length are read
 * on the device, so a CUDA graph captured once serves every update.  The
 * workspace is sized with otg_rc_workspace_size(max_listed, ...).
 */
otg_status otg_rc_timing_subset(const otg_rc_forest* forest, int32_t max_net_nodes,
                                const int32_t* net_list, const int32_t* num_listed,
                                int32_t max_listed, void* workspace, size_t workspace_bytes,
                                otg_stream_t stream);

/*
 * otg_rc_move_nets -- copies whole nets from forest src into forest dst on
 * the device: every net i of dst with src_net[i] >= 0 receives net
 * src_net[i] of src (root, edges, res and cap; with copy_outputs also
 * node2bfs, pid, load, delay, ldelay and impulse).  Nets with src_net[i] < 0
 * are left alone.  A size mismatch or an out-of-range src_net entry skips
 * that net and sets *status (device memory, caller-zeroed) to
 * OTG_ERR_INVALID.  Asynchronous; src_net is device memory [dst nets].
 *
 * The relayout step of incremental SPEF ingestion.  The reference
 * re-attaches each changed net's parasitics (Timer::_read_spef,
 * ot/timer/spef.cpp:40-53) and re-times on the next update_timing; here
 * the unchanged nets move into the new layout with their results, the
 * changed nets' inputs move in from a staging forest, and
 * otg_rc_timing_subset re-times only those.  No reference counterpart as
 * one call.
 */
otg_status otg_rc_move_nets(const otg_rc_forest* src, const otg_rc_forest* dst,
                            const int32_t* src_net, int32_t copy_outputs, int32_t* status,
                            otg_stream_t stream);

/* Synchronizes `stream` and returns the first device-side error recorded in
 * `workspace` by the last otg_rc_timing call (OTG_OK if none); *bad_net (if
 * non-NULL) gets the offending net index or -1. */
otg_status otg_rc_status(const void* workspace, otg_stream_t stream, int32_t* bad_net);

/*
 * Levelization of the timing graph -- replaces toposort_advance /
 * toposort_compute_cuda (ot/cuda/toposort.cu:4-72).  Device pointers.
 *   fanin_start[n+1], fanin[E]: fanin CSR over pins (LOOP_BREAKER arcs and
 *   non-candidates already excluded, ot/timer/timer.cpp:1005-1048)
 *   out_deg[n]: candidate fanout count per pin (read only; copied)
 *   frontier0[first_size]: the seed level (candidates with no fanout)
 * Outputs:
 *   order[n]        pins concatenated level by level (level 0 = seed order,
 *                   every later level in ascending pin index)
 *   level[n]        level of each pin, -1 if never emitted
 *   level_ends[n+2] level_ends[0]=0, level_ends[k+1] = end of level k
 *   counts[2]       counts[0] = number of levels, counts[1] = pins emitted
 * level(v) = 1 + max over candidate fanouts (longest path to a sink).  All
 * levels run inside one launch (no host round trip per level): a single
 * thread-block cluster for graphs of up to about a million pins, a
 * cooperative grid otherwise, whose grid
 * barrier is bounded and reports OTG_ERR_TIMEOUT instead of hanging.  Both
 * give identical outputs.
 */
otg_status otg_levelize_workspace_size(int32_t n, int32_t num_edges, size_t* bytes);
otg_status otg_levelize(int32_t n, int32_t num_edges, const int32_t* fanin_start,
                        const int32_t* fanin, const int32_t* out_deg, const int32_t* frontier0,
                        int32_t first_size, int32_t* order, int32_t* level, int32_t* level_ends,
                        int32_t* counts, void* workspace, size_t workspace_bytes,
                        otg_stream_t stream);
/* Synchronizes and returns the levelization status (OTG_ERR_TIMEOUT if the
 * bounded grid barrier gave up). */
otg_status otg_levelize_status(const void* workspace, otg_stream_t stream);

/*
 * Host-buffer entry points (end-to-end: host->device copies, compute,
 * device->host copies inside the call).  They keep a per-device context
 * with cached device buffers (grown, never shrunk) and pinned staging, and
 * stream large batches in chunks so transfers overlap compute.  Blocking.
 * Arrays as in otg_rc_forest but host pointers.
 */
otg_status otg_rc_timing_host(const otg_rc_forest* host_forest);
otg_status otg_levelize_host(int32_t n, int32_t num_edges, const int32_t* fanin_start,
                             const int32_t* fanin, const int32_t* out_deg,
                             const int32_t* frontier0, int32_t first_size, int32_t* order,
                             int32_t* level, int32_t* level_ends, int32_t* counts);
/* Frees the host-path context of the current device. */
void otg_release_host_context(void);

/*
 * otg_rc_timing_noalloc -- the fused pass of otg_rc_timing for callers that
 * may not allocate device memory when they run RC timing (a host whose pool
 * allocator owns all device memory, a loop that cannot afford cudaMalloc's
 * device-wide synchronization).  This entry point has no counterpart in the
 * reference.  Its workspace is a 16 MiB array compiled into libotg, held on
 * every GPU that loads it until the process exits; the caller passes only
 * inputs and outputs (device pointers, as for otg_rc_timing).  The first
 * call on a device loads the array (the CUDA runtime loads device code
 * lazily) and looks up its address: make it before a pool allocator takes
 * the device's memory and before any stream capture; a call with an empty
 * forest does only that set-up.  Calls share the array: calls that overlap
 * on the GPU race, so serialize them.  Blocks until `stream` finishes and
 * returns the device-side status of the call.  Limit: at most 524,284 nets
 * per call and no net beyond the shared-memory classes of the device's
 * tuning (4,265 nodes on a B200 with the default tuning); larger batches
 * return OTG_ERR_WORKSPACE without launching.  Allocates nothing.
 */
otg_status otg_rc_timing_noalloc(const otg_rc_forest* forest, int32_t max_net_nodes,
                                 otg_stream_t stream);

/*
 * ---- Device-resident designs and the incremental timing server ----------
 * (no counterpart in the reference, whose Timer recomputes dirty nets on the
 * CPU and whose CUDA path flattens and re-times every net of the design on
 * each update; ot/timer/timer.cpp:929-966).
 *
 * A server owns designs whose RC state stays on the device.  A request is
 * an incremental change to one design -- node capacitance updates (a gate
 * resize changes the pin caps of its inputs) and driver-slew updates (its
 * drive strength) -- whose dirty nets are re-timed.  The dispatcher thread
 * batches the pending requests of all idle designs (continuous batching:
 * requests that arrive while batches run are taken as soon as a slot and
 * their design are free), applies the updates, re-times every dirty net of
 * the batch in one fused pass over all designs, and reduces per request the
 * worst |sink slew| and worst sink delay over its dirty nets.  Each slot
 * replays a CUDA graph captured once; request data reach the device through
 * pinned, mapped host buffers.  Designs are admitted against a device-memory
 * budget (OTG_ERR_ADMISSION when one does not fit).
 */
typedef struct otg_server otg_server;

typedef struct otg_result {
  float worst_slew[4];   /* max |sink slew| over the request's dirty nets, per corner */
  float worst_delay[4];  /* max sink Elmore delay over the same nets, per corner       */
  int32_t status;        /* OTG_OK or the first device-side error of its design       */
  int32_t dirty_nets;    /* distinct nets the request dirtied                         */
  int64_t t_submit_ns;   /* steady-clock times of submission and completion           */
  int64_t t_done_ns;
} otg_result;

/* budget_bytes: device memory designs may hold (0 = no limit); slots:
 * batches in flight (>= 1); max_requests / max_updates: capacity of one
 * batch (requests, and cap + slew updates). */
otg_status otg_server_create(size_t budget_bytes, int32_t slots, int32_t max_requests,
                             int32_t max_updates, otg_server** out);
void otg_server_destroy(otg_server* s);
/* Uploads a design (host arrays of an otg_rc_forest with sinks), times it
 * fully once, and returns its id; OTG_ERR_ADMISSION if it does not fit. */
otg_status otg_server_add_design(otg_server* s, const otg_rc_forest* host_forest,
                                 int32_t* design_id, size_t* footprint_bytes);
otg_status otg_server_remove_design(otg_server* s, int32_t design_id);
/* Queues one request; cap_val is [num_cap][4], slew_val [num_slew][4].
 * OTG_ERR_INVALID (nothing queued) for an unknown design, a net or node
 * outside it, or more updates than a batch holds. */
otg_status otg_server_submit(otg_server* s, int32_t design_id, int32_t num_cap,
                             const int32_t* cap_net, const int32_t* cap_node, const float* cap_val,
                             int32_t num_slew, const int32_t* slew_net, const float* slew_val,
                             int64_t* ticket);
/* Blocks until `ticket` completes (timeout_ms < 0: no limit) and returns
 * its result; OTG_ERR_TIMEOUT if the limit passed first. */
otg_status otg_server_wait(otg_server* s, int64_t ticket, int32_t timeout_ms, otg_result* out);
/* The same request without batching: applied and timed by itself, one set
 * of launches and a stream synchronization per request (the per-update
 * path the batched server is measured against).  Blocking. */
otg_status otg_server_update_sync(otg_server* s, int32_t design_id, int32_t num_cap,
                                  const int32_t* cap_net, const int32_t* cap_node,
                                  const float* cap_val, int32_t num_slew, const int32_t* slew_net,
                                  const float* slew_val, otg_result* out);
/* Open-loop replay of a request trace (the load generator of the serving
 * measurement).  Request r goes to design[r] at t0 + arrival_ns[r] (t0 =
 * the call's start) with the cap updates [cap_start[r], cap_start[r+1])
 * and slew updates [slew_start[r], slew_start[r+1]) of the update arrays.
 * plain == 0: submitted to the batching server by a submitter thread;
 * plain != 0: applied with otg_server_update_sync, one request at a time in
 * arrival order (the per-update path).  latency_ns[r] = completion minus
 * scheduled arrival (queueing included); *makespan_ns = last completion
 * minus t0.  Blocks until every request is done. */
otg_status otg_server_replay(otg_server* s, int32_t num_req, const int64_t* arrival_ns,
                             const int32_t* design, const int32_t* cap_start,
                             const int32_t* cap_net, const int32_t* cap_node,
                             const float* cap_val, const int32_t* slew_start,
                             const int32_t* slew_net, const float* slew_val, int32_t plain,
                             int64_t* latency_ns, int64_t* makespan_ns);
/* Batches launched by the dispatcher and the requests they carried. */
otg_status otg_server_stats(otg_server* s, int64_t* batches, int64_t* requests);
/* Copies a design's per-node outputs (BFS order, as otg_rc_forest) and
 * sink slews back to host arrays (any may be NULL). */
otg_status otg_server_read(otg_server* s, int32_t design_id, int32_t* node2bfs, float* load,
                           float* delay, float* ldelay, float* impulse, float* sink_slew);

/*
 * Tuning of the fused RC pass (per device; applies to later launches; no
 * counterpart in the reference, whose kernels have fixed launch shapes).
 * Nets of <= 32 nodes always take the warp path.  Block class c takes the
 * nets with class_max[c-1] < n <= class_max[c] (class_max[-1] = 32), one
 * CTA of class_threads[c] threads with class_items[c] scan items per
 * thread, in shared memory; nets above the last class_max take the
 * global-workspace path.  Shapes must be among the compiled ones
 * (threads x items: 64x4, 64x8, 128x4, 128x8, 256x2, 256x4, 256x8, 512x2,
 * 512x4, 512x8, 1024x2, 1024x4) and each class must fit shared memory.
 * Every valid tuning gives identical outputs; only the speed differs.
 * otg_rc_workspace_size depends on the tuning (the global-workspace
 * slices): size workspaces after setting it.
 */
typedef struct otg_rc_tuning {
  int32_t num_classes; /* 1..6 */
  int32_t class_max[6];
  int32_t class_threads[6];
  int32_t class_items[6];
} otg_rc_tuning;
otg_status otg_rc_get_tuning(otg_rc_tuning* tuning);
/* NULL restores the default; OTG_ERR_INVALID for a tuning that does not
 * validate (nothing changes). */
otg_status otg_rc_set_tuning(const otg_rc_tuning* tuning);
/* Autotuner: times candidate tunings on a sample forest (device pointers;
 * its outputs are overwritten) and applies the fastest; returns it in
 * *tuning (may be NULL).  Allocates a temporary workspace.  Blocks. */
otg_status otg_rc_autotune(const otg_rc_forest* sample, int32_t max_net_nodes,
                           otg_stream_t stream, otg_rc_tuning* tuning);

/*
 * SPEF to the flat RC layout (host side, parallel over nets).  Replaces the
 * reference's read_spef + Net::_make_flat_rct pair for this layout
 * (ot/parser-spef/parser-spef.hpp, ot/timer/net.cpp:370-461): ids by first
 * appearance over each net's *RES lines, edges and res in *RES order, the
 * root at the net's driver (*I ... O or *P ... I), cap[id][*] = the node's
 * *CAP value (a coupling line counts for its first node), *NAME_MAP
 * references expanded, values rounded to float and multiplied by r_scale /
 * c_scale (a Timer's unit rebasing).  Pin caps are not added: they need the
 * cell library; otg_spef_pins gives each net's pins with their local ids.
 * Nets without *RES lines are left out.  threads <= 0: all host threads.
 */
typedef struct otg_spef otg_spef;
otg_status otg_spef_read(const char* path, int32_t threads, float r_scale, float c_scale,
                         otg_spef** out);
/* units: ohm, farad and second per unit of the file (*R_UNIT, *C_UNIT,
 * *T_UNIT); any output may be NULL. */
otg_status otg_spef_sizes(const otg_spef* spef, int32_t* num_nets, int32_t* total_nodes,
                          int32_t* total_pins, double* units);
/* Host arrays in the otg_rc_forest layout: nodes_start[N+1], edges[V-N],
 * roots[N], res[V-N], cap[V][4]; net_flags[N] (may be NULL): bit 0 no
 * driver pin in the tree, bit 1 ids != |RES|+1 (not a tree), bit 2 a *CAP
 * node outside the tree, bit 3 a malformed *CAP or *RES line. */
otg_status otg_spef_fill(const otg_spef* spef, int32_t* nodes_start, otg_rc_edge* edges,
                         int32_t* roots, float* res, float* cap, uint8_t* net_flags);
/* Per net, its *CONN pins: pins_start[N+1], local id (-1: not in the tree),
 * direction (0 I, 1 O, 2 B) and port flag (1 for *P). */
otg_status otg_spef_pins(const otg_spef* spef, int32_t* pins_start, int32_t* pin_node,
                         int8_t* pin_dir, int8_t* pin_port);
const char* otg_spef_net_name(const otg_spef* spef, int32_t net);
const char* otg_spef_pin_name(const otg_spef* spef, int32_t net, int32_t k);
/* Every net name, then every pin name (net order, *CONN order), each
 * NUL-terminated, into buf (*bytes: its size in, the size used out).  With
 * buf NULL it only sets *bytes.  OTG_ERR_WORKSPACE if buf is too small. */
otg_status otg_spef_names(const otg_spef* spef, char* buf, size_t* bytes);
/* The other direction (no single reference counterpart; the inverse of
 * spef::Spef::read for the subset above): writes nets as SPEF text with
 * units ns / fF / ohm.  names_blob holds '\0'-terminated names, name k at
 * name_off[k] (name_off has one more entry than there are names).  Net i:
 * name net_name[i]; pins pins_start[i]..pins_start[i+1]-1 (name pin_name[p],
 * pin_port[p] 1 for a port, the first pin is the driver); nodes
 * nodes_start[i]..nodes_start[i+1]-1 in *CAP order, node_code >= 0 the
 * net's pin of that index, < 0 the internal node "<net>:<-code>", ground
 * cap node_cap; edges [V-N][2] (node indices within the net) and res in
 * *RES order.  threads <= 0: all hardware threads. */
otg_status otg_spef_write(const char* path, int32_t num_nets, const char* names_blob,
                          const int64_t* name_off, const int32_t* net_name,
                          const int32_t* pins_start, const int32_t* pin_name,
                          const int8_t* pin_port, const int32_t* nodes_start,
                          const int32_t* node_code, const float* node_cap, const int32_t* edges,
                          const float* res, int32_t threads);
void otg_spef_free(otg_spef* spef);

/*
 * Levelized timing propagation (the consumer of the RC pass): slew, arc
 * delay, arrival time and timing-test required time forward; required time
 * and slack backward; corner c = split*2 + tran.  It restates the reference
 * Timer's per-pin tasks (ot/timer/timer.cpp:733-832, arc.cpp:82-205,
 * pin.cpp:324-380, test.cpp:88-135) and its NLDM look-ups
 * (ot/liberty/timing.cpp:198-628, lut.cpp:166-245) over a flat graph; the
 * Timer has no GPU counterpart for it.  All arrays are device pointers;
 * "none" (an empty value in the reference) is NaN.
 */
typedef struct otg_prop_graph {
  int32_t num_pins, num_arcs, num_tests;
  const int32_t* arc_from;     /* [A] */
  const int32_t* arc_to;       /* [A] */
  const int32_t* arc_kind;     /* [A] 0 net arc, 1 cell arc */
  const int32_t* arc_timing;   /* [A][2] cell arcs: timing record per split (-1 none) */
  const int32_t* arc_net;      /* [A] net arcs: the forest net; cell arcs: the net the
                                  arc drives (its load), -1 none (load 0) */
  const int32_t* arc_node;     /* [A] net arcs: the sink's local RC node id in its net
                                  (unchanged when nets move, otg_rc_move_nets), -1 not
                                  in the tree */
  const int32_t* fanin_start;  /* [P+1] CSR of the arcs into each pin */
  const int32_t* fanin;
  const int32_t* fanout_start; /* [P+1] CSR of the arcs out of each pin */
  const int32_t* fanout;
  const int32_t* test_arc;     /* [T] the constraint arc (related -> constrained pin) */
  const int32_t* test_start;   /* [P+1] CSR of the tests constrained at each pin */
  const int32_t* test_of_pin;
  const float* pi_at;          /* [P][4] primary-input assertions (NaN none) */
  const float* pi_slew;        /* [P][4] */
  const float* po_rat;         /* [P][4] primary-output assertions */
  const int32_t* timing;       /* [R][9] sense (0 positive, 1 negative, 2 other unate),
                                  edge (0 none, 1 rising, 2 falling), constraint flag,
                                  LUT ids of cell_rise, cell_fall, rise_transition,
                                  fall_transition, rise_constraint, fall_constraint */
  const int32_t* lut_meta;     /* [L][4] n1, n2, offset in lut_data, variable order
                                  (0: slew or related-pin slew first; 1: load or
                                  constrained-pin slew first; -1: no template) */
  const float* lut_data;       /* per LUT: index_1[n1], index_2[n2], values[n1*n2] */
  float period;                /* clock period of the timing tests (NaN: no clock) */
  int32_t num_lut_data;        /* floats in lut_data (0: unknown; the tables are then
                                  read from global memory, not staged on chip) */
} otg_prop_graph;

typedef struct otg_prop_rc {   /* outputs of otg_rc_timing for the design's nets */
  const int32_t* nodes_start;
  const int32_t* node2bfs;
  const float* load;
  const float* delay;
  const float* impulse;
} otg_prop_rc;

otg_status otg_prop_workspace_size(int32_t num_pins, int32_t num_arcs, int32_t num_tests,
                                   size_t* bytes);
/* order (device, num_pins entries) is otg_levelize's output over the
 * graph's fanin CSR: every pin after all of its fanout pins; the backward
 * pass takes it as is.  fwd_order (device, may be NULL) is the forward
 * pass's order, every pin after all of its fanin pins (otg_levelize over
 * the fanout CSR: by distance from the sources); NULL takes order
 * reversed.  Any such orders give the same results.  Writes at,
 * slew, rat, slack [P][4].  lut_meta and the four outputs must be 16-byte
 * aligned, the workspace 256-byte aligned.  A fill launch, then one
 * cooperative launch, dataflow-scheduled (a pin polls the values it reads
 * from its fanins, bounded waits); asynchronous.  otg_prop_status
 * synchronizes the stream and returns OTG_ERR_TIMEOUT if a wait gave up. */
otg_status otg_propagate(const otg_prop_graph* graph, const otg_prop_rc* rc,
                         const int32_t* order, const int32_t* fwd_order, float* at, float* slew,
                         float* rat, float* slack, void* workspace, size_t workspace_bytes,
                         otg_stream_t stream);
otg_status otg_prop_status(const void* workspace, otg_stream_t stream);
/* The arc delays the last propagation computed, as the Timer keeps them in
 * Arc::_delay[el][frf][trf] (ot/timer/arc.hpp): *arc_delay is set to a
 * device array [num_arcs][8] inside the workspace, entry
 * (el << 2) | (frf << 1) | trf, NaN where the reference's value is empty
 * (a net arc between different transitions, a transition the cell arc's
 * timing sense does not have, a constraint arc, no input slew).  Valid
 * until the next propagation on the same workspace.  The reference's path
 * reports (Timer::report_timing, ot/timer/path.cpp:365-420) walk these. */
otg_status otg_prop_arc_delays(const void* workspace, size_t workspace_bytes, int32_t num_arcs,
                               const float** arc_delay);

/* ---- path reports (host) -------------------------------------------------
 * A propagated timing graph for the path search, all HOST arrays: the arcs
 * (constraint arcs flagged: they carry no delay), the data-path sources
 * (Pin::is_datapath_source: no fanin, a cell's clock pin, a primary
 * input), the endpoints (primary outputs and the tests' constrained pins),
 * every arc's delay [num_arcs][8] by (split << 2 | from tran << 1 | to
 * tran), NaN where empty (otg_prop_arc_delays, copied to the host), and
 * at / rat / slack [num_pins][4] (corner = split * 2 + tran). */
typedef struct otg_path_graph {
  int32_t num_pins, num_arcs, num_endpoints;
  const int32_t* arc_from;
  const int32_t* arc_to;
  const uint8_t* arc_is_test;
  const uint8_t* pin_is_source;
  const int32_t* endpoints;
  const float* arc_delay;
  const float* at;
  const float* rat;
  const float* slack;
} otg_path_graph;

/* Timer::report_timing(K[, split][, tran]) (ot/timer/path.cpp:365-537):
 * the K worst data paths, ascending by slack.  split / tran: -1 for any.
 * K = 1 gives the worst endpoint's path with the endpoint's slack; larger
 * K the paths of negative slack only (the reference's prefix-tree
 * search).  Writes num_paths (<= K), path_slack [K], path_endpoint [K][3]
 * (pin, split, tran), path_start [K + 1] (offsets into the points) and,
 * up to max_points, point_pin / point_tran / point_at; points_needed gets
 * the total, and a result that does not fit returns OTG_ERR_WORKSPACE
 * (call again with a larger max_points).  float32 arithmetic in the
 * reference's order: on the reference's own graph values the paths are
 * the reference's, bit for bit. */
otg_status otg_report_paths(const otg_path_graph* graph, int32_t K, int32_t split, int32_t tran,
                            int32_t* num_paths, float* path_slack, int32_t* path_endpoint,
                            int32_t* path_start, int32_t max_points, int32_t* point_pin,
                            int32_t* point_tran, float* point_at, int32_t* points_needed);
/* The same over a graph that is the union of independent designs (no arc
 * between two of them): pin_group [P] gives each pin its design, and only
 * the pins whose group_active[design] is nonzero are propagated (and
 * marked pending); every other pin keeps its values.  order / fwd_order
 * cover all pins, as for otg_propagate (a levelization of the union).  An
 * incremental update of some designs then re-times only those. */
otg_status otg_propagate_groups(const otg_prop_graph* graph, const otg_prop_rc* rc,
                                const int32_t* order, const int32_t* fwd_order,
                                const int32_t* pin_group, const uint8_t* group_active,
                                float* at, float* slew, float* rat, float* slack,
                                void* workspace, size_t workspace_bytes, otg_stream_t stream);
/* The same over a list of pins only: items[num_items] (device) are the pins
 * to propagate, in a backward order as `order` above (every pin after all
 * of its fanout pins; the forward pass takes it reversed).  The list must
 * hold, with each pin, every pin it reads that is not final: for a union
 * of independent designs, the pins of whole designs, e.g. the union's
 * order regrouped design by design (a stable regrouping keeps each
 * design's pins in level order).  Only the listed pins are marked pending
 * and written; the work is in proportion to the list, not to the graph. */
otg_status otg_propagate_items(const otg_prop_graph* graph, const otg_prop_rc* rc,
                               const int32_t* items, int32_t num_items, float* at, float* slew,
                               float* rat, float* slack, void* workspace, size_t workspace_bytes,
                               otg_stream_t stream);

/*
 * ---- Incremental gate resizing (the device side of Timer::repower_gate,
 * ot/timer/timer.cpp:57-118, with Pin::_remap_cellpin, ot/timer/pin.cpp:
 * 382-399) ---------------------------------------------------------------
 * A resize remaps a gate's pins to another cell: each input pin's node in
 * its net's RC tree gets the new cell pin's capacitance (ground cap plus
 * pin cap, written whole), and each cell arc of the gate gets the new
 * cell's timing record for its split.  otg_apply_updates writes both kinds
 * of update in one launch (device arrays): cap_row[u] is a flat node index
 * (nodes_start[net] + local id) into nodes_cap [V][4], cap_val[u] its [4]
 * values; arc_slot[k] = arc * 2 + split into arc_timing [A][2], arc_rec[k]
 * the record.  Out-of-range indices are skipped and set *status (device,
 * caller-zeroed) to OTG_ERR_INVALID.  The caller re-times the nets of the
 * changed nodes (otg_rc_timing_subset) and propagates (otg_propagate), as
 * update_timing does for the dirty nets and the affected cone
 * (ot/timer/timer.cpp:888-923, 1245-1334).  Asynchronous.
 */
otg_status otg_apply_updates(int32_t num_cap, const int32_t* cap_row, const float* cap_val,
                             float* nodes_cap, int32_t total_nodes, int32_t num_arc,
                             const int32_t* arc_slot, const int32_t* arc_rec,
                             int32_t* arc_timing, int32_t num_arcs, int32_t* status,
                             otg_stream_t stream);
/*
 * otg_fanin_csr -- the levelization input of a timing update, built on the
 * device (replaces Timer::_build_prop_tasks_cuda steps 1-2,
 * ot/timer/timer.cpp:996-1061, which build it on the host with taskflow
 * and a serial prefix sum).  An arc counts when arc_skip[a] is 0 (a loop
 * breaker otherwise; arc_skip may be NULL) and both its pins are
 * candidates (pin_cand[p] != 0; NULL: every pin).  Outputs (device):
 * fanin_start[n+1] and fanin[]: per pin its counted fanin arcs in arc
 * order, as source pins (or, with fanin_as_arcs, as arc indices);
 * out_deg[n]: counted fanout arcs; frontier0: the candidates of
 * cand_order[num_cands] without counted fanout, in that order (the first
 * frontier); counts[0] = their number, counts[1] = the arcs counted.  These
 * are exactly otg_levelize's inputs.  Asynchronous; otg_fanin_csr_status
 * synchronizes and reports OTG_ERR_INVALID for an out-of-range pin. */
otg_status otg_fanin_csr_workspace_size(int32_t num_pins, int32_t num_arcs, int32_t num_cands,
                                        size_t* bytes);
otg_status otg_fanin_csr(int32_t num_pins, int32_t num_arcs, const int32_t* from,
                         const int32_t* to, const uint8_t* arc_skip, const uint8_t* pin_cand,
                         int32_t num_cands, const int32_t* cand_order, int32_t fanin_as_arcs,
                         int32_t* fanin_start, int32_t* fanin, int32_t* out_deg,
                         int32_t* frontier0, int32_t* counts, void* workspace,
                         size_t workspace_bytes, otg_stream_t stream);
otg_status otg_fanin_csr_status(const void* workspace, otg_stream_t stream);

/* Worst (minimum) finite slack per corner over slack [P][4] (device) into
 * out4 [4] (device; NaN where no pin has one), the per-corner worst slack
 * of Timer::report_wns over the propagated pins.  scratch4: 4 uint32 of
 * device scratch.  Asynchronous. */
otg_status otg_worst_slack(const float* slack, int32_t num_pins, uint32_t* scratch4,
                           float* out4, otg_stream_t stream);
/* Per group (the pin_group / group_active of otg_propagate_groups): the
 * worst finite slack per corner of the active groups' pins into
 * out [num_groups][4] (NaN for inactive groups and groups without slack).
 * scratch: 4 * num_groups uint32 of device scratch.  Asynchronous. */
otg_status otg_worst_slack_groups(const float* slack, int32_t num_pins, const int32_t* pin_group,
                                  const uint8_t* group_active, int32_t num_groups,
                                  uint32_t* scratch, float* out, otg_stream_t stream);

/* Human-readable name of a status code. */
const char* otg_status_string(otg_status s);

/* Number of kernel launches issued by this library since load (a counter
 * for measurement harnesses). */
uint64_t otg_kernel_launches(void);

/*
 * Seeded synthetic RC forest (the batched-Elmore workload): net sizes are
 * given (nodes_start), 70% random recursive trees / 30% chains with side
 * branches, shuffled edges with random orientation, local ids by first
 * appearance over the edges, R ~ U(0.1,50), C ~ U(0.05,5) plus a per-corner
 * pin cap on leaves, driver slews U(5,200).  Device pointers; writes edges,
 * roots, res, cap, driver_slew and sink_count[N] (leaves per net).  The
 * sinks themselves come from otg_synth_rc_sinks once sinks_start (the
 * exclusive scan of sink_count) is known.  scratch: V int32 (device).
 */
otg_status otg_synth_rc_forest(uint64_t seed, int32_t num_nets, const int32_t* nodes_start,
                               otg_rc_edge* edges, int32_t* roots, float* res, float* cap,
                               float* driver_slew, int32_t* sink_count, int32_t* scratch,
                               otg_stream_t stream);
otg_status otg_synth_rc_sinks(int32_t num_nets, const int32_t* nodes_start,
                              const otg_rc_edge* edges, const int32_t* roots,
                              const int32_t* sinks_start, int32_t* sink_nodes, int32_t* scratch,
                              otg_stream_t stream);
/* The same generator on the host (no GPU needed); host pointers. */
otg_status otg_synth_rc_forest_host(uint64_t seed, int32_t num_nets, const int32_t* nodes_start,
                                    otg_rc_edge* edges, int32_t* roots, float* res, float* cap,
                                    float* driver_slew, int32_t* sink_count);

#ifdef __cplusplus
}
#endif

#endif /* OTG_H_ */
