"""SPEF to the flat RC layout (otg_spef_* in include/otg.h).

    f = read_spef("design.spef", r_scale=1e-3)
    f["nodes_start"], f["edges"], f["roots"], f["res"], f["cap"]   # numpy
    f["net_names"], f["pins_start"], f["pin_node"], ...

The arrays are the inputs of the fused RC pass (otg_rc_forest) with the
reference's flattening rules (ot/timer/net.cpp:370-461); pin caps are the
caller's to add (cap[nodes_start[net] + pin_node] += pin cap for every pin
but the root).
"""
import ctypes

import numpy as np

from ._lib import check, lib


def read_spef(path, threads=0, r_scale=1.0, c_scale=1.0, names=True):
    L = lib()
    h = ctypes.c_void_p()
    check("otg_spef_read", L.otg_spef_read(str(path).encode(), threads, r_scale, c_scale,
                                           ctypes.byref(h)))
    try:
        N, V, P = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        units = (ctypes.c_double * 3)()
        check("otg_spef_sizes", L.otg_spef_sizes(h, ctypes.byref(N), ctypes.byref(V),
                                                 ctypes.byref(P), units))
        N, V, P = N.value, V.value, P.value
        out = {"nodes_start": np.empty(N + 1, np.int32), "edges": np.empty((V - N, 2), np.int32),
               "roots": np.empty(N, np.int32), "res": np.empty(V - N, np.float32),
               "cap": np.empty((V, 4), np.float32), "net_flags": np.empty(N, np.uint8),
               "pins_start": np.empty(N + 1, np.int32), "pin_node": np.empty(P, np.int32),
               "pin_dir": np.empty(P, np.int8), "pin_port": np.empty(P, np.int8),
               "units": {"ohm": units[0], "farad": units[1], "second": units[2]}}
        a = lambda k: out[k].ctypes.data  # noqa: E731
        check("otg_spef_fill", L.otg_spef_fill(h, a("nodes_start"), a("edges"), a("roots"),
                                               a("res"), a("cap"), a("net_flags")))
        check("otg_spef_pins", L.otg_spef_pins(h, a("pins_start"), a("pin_node"), a("pin_dir"),
                                               a("pin_port")))
        if names:  # all names in one call: nets, then pins in net order
            size = ctypes.c_size_t()
            check("otg_spef_names", L.otg_spef_names(h, None, ctypes.byref(size)))
            buf = ctypes.create_string_buffer(max(size.value, 1))
            check("otg_spef_names", L.otg_spef_names(h, buf, ctypes.byref(size)))
            allnames = buf.raw[:size.value].decode().split("\0")[:-1] if size.value else []
            out["net_names"] = allnames[:N]
            out["pin_names"] = allnames[N:]
        return out
    finally:
        L.otg_spef_free(h)
