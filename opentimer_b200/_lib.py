"""ctypes binding of libotg.so (the C ABI declared in include/otg.h).

The library must be built in-tree (opentimer_b200/libotg.so); importing
without it raises -- there is no fallback path.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libotg.so")

OK = 0
STATUS = {
    0: "OTG_OK", 1: "OTG_ERR_INVALID", 2: "OTG_ERR_CUDA", 3: "OTG_ERR_OOM",
    4: "OTG_ERR_NOT_TREE", 5: "OTG_ERR_CYCLE", 6: "OTG_ERR_TIMEOUT", 7: "OTG_ERR_TOO_LARGE",
    8: "OTG_ERR_WORKSPACE", 9: "OTG_ERR_ADMISSION",
}

# Every symbol include/otg.h declares (checked by the CPU test suite).
C_SYMBOLS = [
    "otg_rc_workspace_size", "otg_rc_timing", "otg_rc_status",
    "otg_levelize_workspace_size", "otg_levelize", "otg_levelize_status",
    "otg_rc_timing_host", "otg_levelize_host", "otg_release_host_context",
    "otg_status_string", "otg_kernel_launches",
    "otg_synth_rc_forest", "otg_synth_rc_sinks", "otg_synth_rc_forest_host",
    "otg_rc_timing_noalloc", "otg_rc_timing_subset",
    "otg_server_create", "otg_server_destroy", "otg_server_add_design",
    "otg_server_remove_design", "otg_server_submit", "otg_server_wait",
    "otg_server_update_sync", "otg_server_read", "otg_server_replay", "otg_server_stats",
    "otg_rc_get_tuning", "otg_rc_set_tuning", "otg_rc_autotune",
    "otg_spef_read", "otg_spef_sizes", "otg_spef_fill", "otg_spef_pins", "otg_spef_net_name",
    "otg_spef_pin_name", "otg_spef_free", "otg_prop_workspace_size", "otg_propagate",
    "otg_prop_status", "otg_rc_move_nets", "otg_spef_names", "otg_apply_updates",
    "otg_worst_slack", "otg_spef_write", "otg_fanin_csr_workspace_size", "otg_fanin_csr",
    "otg_fanin_csr_status", "otg_propagate_groups", "otg_worst_slack_groups",
    "otg_propagate_items", "otg_prop_arc_delays", "otg_report_paths",
]
# The reference-compatible C++ entry points (include/otg_compat.hpp), by
# their Itanium-mangled names.
CXX_SYMBOLS = {
    "rct_bfs_and_compute_cuda": "_Z24rct_bfs_and_compute_cuda16RctEdgeArrayCUDA",
    "rct_compute_cuda": "_Z16rct_compute_cuda7RctCUDA",
    "toposort_compute_cuda": "_Z21toposort_compute_cudaiiiPiS_S_S_RSt6vectorIiSaIiEE",
}


class OtgError(RuntimeError):
    def __init__(self, where, code):
        super().__init__(f"{where}: {STATUS.get(code, code)}")
        self.code = code


class RcForest(ctypes.Structure):
    _fields_ = [
        ("num_nets", ctypes.c_int32), ("total_nodes", ctypes.c_int32),
        ("nodes_start", ctypes.c_void_p), ("edges", ctypes.c_void_p),
        ("roots", ctypes.c_void_p), ("edges_res", ctypes.c_void_p),
        ("nodes_cap", ctypes.c_void_p), ("node2bfs", ctypes.c_void_p),
        ("pid", ctypes.c_void_p), ("load", ctypes.c_void_p), ("delay", ctypes.c_void_p),
        ("ldelay", ctypes.c_void_p), ("impulse", ctypes.c_void_p),
        ("sinks_start", ctypes.c_void_p), ("sink_nodes", ctypes.c_void_p),
        ("driver_slew", ctypes.c_void_p), ("sink_slew", ctypes.c_void_p),
    ]


class PathGraph(ctypes.Structure):
    """otg_path_graph: a propagated timing graph for otg_report_paths."""
    _fields_ = [("num_pins", ctypes.c_int32), ("num_arcs", ctypes.c_int32),
                ("num_endpoints", ctypes.c_int32), ("arc_from", ctypes.c_void_p),
                ("arc_to", ctypes.c_void_p), ("arc_is_test", ctypes.c_void_p),
                ("pin_is_source", ctypes.c_void_p), ("endpoints", ctypes.c_void_p),
                ("arc_delay", ctypes.c_void_p), ("at", ctypes.c_void_p), ("rat", ctypes.c_void_p),
                ("slack", ctypes.c_void_p)]


class RcTuning(ctypes.Structure):
    """otg_rc_tuning: block size classes of the fused RC pass."""
    _fields_ = [("num_classes", ctypes.c_int32), ("class_max", ctypes.c_int32 * 6),
                ("class_threads", ctypes.c_int32 * 6), ("class_items", ctypes.c_int32 * 6)]


class RcResult(ctypes.Structure):
    """otg_result: one incremental request's summary."""
    _fields_ = [
        ("worst_slew", ctypes.c_float * 4), ("worst_delay", ctypes.c_float * 4),
        ("status", ctypes.c_int32), ("dirty_nets", ctypes.c_int32),
        ("t_submit_ns", ctypes.c_int64), ("t_done_ns", ctypes.c_int64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m opentimer_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        I32, P, S, U64 = ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64
        PS = ctypes.POINTER(ctypes.c_size_t)
        L.otg_rc_workspace_size.argtypes = [I32, I32, PS]
        L.otg_rc_timing.argtypes = [ctypes.POINTER(RcForest), I32, P, S, P]
        L.otg_rc_status.argtypes = [P, P, ctypes.POINTER(I32)]
        L.otg_rc_timing_subset.argtypes = [ctypes.POINTER(RcForest), I32, P, P, I32, P, S, P]
        L.otg_levelize_workspace_size.argtypes = [I32, I32, PS]
        L.otg_levelize.argtypes = [I32, I32, P, P, P, P, I32, P, P, P, P, P, S, P]
        L.otg_levelize_status.argtypes = [P, P]
        L.otg_rc_timing_host.argtypes = [ctypes.POINTER(RcForest)]
        L.otg_levelize_host.argtypes = [I32, I32, P, P, P, P, I32, P, P, P, P]
        L.otg_release_host_context.argtypes = []
        L.otg_release_host_context.restype = None
        L.otg_status_string.argtypes = [ctypes.c_int]
        L.otg_status_string.restype = ctypes.c_char_p
        L.otg_kernel_launches.argtypes = []
        L.otg_kernel_launches.restype = U64
        L.otg_synth_rc_forest.argtypes = [U64, I32, P, P, P, P, P, P, P, P, P]
        L.otg_synth_rc_sinks.argtypes = [I32, P, P, P, P, P, P, P]
        L.otg_synth_rc_forest_host.argtypes = [U64, I32, P, P, P, P, P, P, P]
        L.otg_rc_timing_noalloc.argtypes = [ctypes.POINTER(RcForest), I32, P]
        I64 = ctypes.c_int64
        PR = ctypes.POINTER(RcResult)
        L.otg_server_create.argtypes = [S, I32, I32, I32, ctypes.POINTER(P)]
        L.otg_server_destroy.argtypes = [P]
        L.otg_server_destroy.restype = None
        L.otg_server_add_design.argtypes = [P, ctypes.POINTER(RcForest), ctypes.POINTER(I32), PS]
        L.otg_server_remove_design.argtypes = [P, I32]
        L.otg_server_submit.argtypes = [P, I32, I32, P, P, P, I32, P, P, ctypes.POINTER(I64)]
        L.otg_server_wait.argtypes = [P, I64, I32, PR]
        L.otg_server_update_sync.argtypes = [P, I32, I32, P, P, P, I32, P, P, PR]
        L.otg_server_read.argtypes = [P, I32, P, P, P, P, P, P]
        L.otg_server_replay.argtypes = [P, I32, P, P, P, P, P, P, P, P, P, I32, P, P]
        L.otg_server_stats.argtypes = [P, P, P]
        L.otg_rc_get_tuning.argtypes = [ctypes.POINTER(RcTuning)]
        L.otg_rc_set_tuning.argtypes = [ctypes.POINTER(RcTuning)]
        L.otg_rc_autotune.argtypes = [ctypes.POINTER(RcForest), I32, P, ctypes.POINTER(RcTuning)]
        L.otg_spef_read.argtypes = [ctypes.c_char_p, I32, ctypes.c_float, ctypes.c_float,
                                    ctypes.POINTER(P)]
        L.otg_spef_sizes.argtypes = [P, P, P, P, P]
        L.otg_spef_fill.argtypes = [P, P, P, P, P, P, P]
        L.otg_spef_pins.argtypes = [P, P, P, P, P]
        L.otg_spef_net_name.argtypes = [P, I32]
        L.otg_spef_net_name.restype = ctypes.c_char_p
        L.otg_spef_pin_name.argtypes = [P, I32, I32]
        L.otg_spef_pin_name.restype = ctypes.c_char_p
        L.otg_spef_free.argtypes = [P]
        L.otg_prop_workspace_size.argtypes = [I32, I32, I32, PS]
        L.otg_propagate.argtypes = [P, P, P, P, P, P, P, P, P, S, P]
        L.otg_prop_status.argtypes = [P, P]
        L.otg_rc_move_nets.argtypes = [P, P, P, I32, P, P]
        L.otg_apply_updates.argtypes = [I32, P, P, P, I32, I32, P, P, P, I32, P, P]
        L.otg_worst_slack.argtypes = [P, I32, P, P, P]
        L.otg_spef_write.argtypes = [ctypes.c_char_p, I32, ctypes.c_char_p] + [P] * 10 + [I32]
        L.otg_fanin_csr_workspace_size.argtypes = [I32, I32, I32, PS]
        L.otg_fanin_csr.argtypes = [I32, I32, P, P, P, P, I32, P, I32, P, P, P, P, P, P, S, P]
        L.otg_fanin_csr_status.argtypes = [P, P]
        L.otg_propagate_groups.argtypes = [P, P, P, P, P, P, P, P, P, P, P, S, P]
        L.otg_propagate_items.argtypes = [P, P, P, I32, P, P, P, P, P, S, P]
        L.otg_prop_arc_delays.argtypes = [P, S, I32, ctypes.POINTER(P)]
        L.otg_report_paths.argtypes = [ctypes.POINTER(PathGraph), I32, I32, I32, P, P, P, P, I32,
                                       P, P, P, P]
        L.otg_worst_slack_groups.argtypes = [P, I32, P, P, I32, P, P, P]
        L.otg_spef_names.argtypes = [P, P, PS]
        L.otg_spef_free.restype = None
        for name in ["otg_rc_workspace_size", "otg_rc_timing", "otg_rc_status", "otg_rc_timing_subset",
                     "otg_levelize_workspace_size", "otg_levelize", "otg_levelize_status",
                     "otg_rc_timing_host", "otg_levelize_host", "otg_synth_rc_forest",
                     "otg_synth_rc_sinks", "otg_synth_rc_forest_host", "otg_rc_timing_noalloc",
                     "otg_server_create", "otg_server_add_design", "otg_server_remove_design",
                     "otg_server_submit", "otg_server_wait", "otg_server_update_sync",
                     "otg_server_read", "otg_server_replay", "otg_server_stats",
                     "otg_rc_get_tuning", "otg_rc_set_tuning", "otg_rc_autotune",
                     "otg_spef_read", "otg_spef_sizes", "otg_spef_fill", "otg_spef_pins",
                     "otg_prop_workspace_size", "otg_propagate", "otg_prop_status",
                     "otg_rc_move_nets", "otg_spef_names", "otg_apply_updates",
                     "otg_worst_slack", "otg_spef_write", "otg_fanin_csr_workspace_size",
                     "otg_fanin_csr", "otg_fanin_csr_status", "otg_propagate_groups",
                     "otg_worst_slack_groups", "otg_propagate_items", "otg_prop_arc_delays",
                     "otg_report_paths"]:
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def check(where, code):
    if code != OK:
        raise OtgError(where, code)
