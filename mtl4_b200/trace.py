"""Tracing hooks of the library (the reference's vampir_trace<N> events,
boost/numeric/mtl/interface/vpt.hpp:37-78): every traced entry point pushes
an NVTX range "<id> <name>" and, while tracing is enabled, adds its host wall
time to a per-event tally."""
from __future__ import annotations

import ctypes as C

from . import _lib


def enable(on: bool = True):
    _lib.check(_lib.lib().mtlg_trace_enable(1 if on else 0), "trace_enable")


def reset():
    _lib.check(_lib.lib().mtlg_trace_reset(), "trace_reset")


def report() -> dict:
    """{event id: (name, calls, total milliseconds)}"""
    L = _lib.lib()
    need = C.c_size_t()
    _lib.check(L.mtlg_trace_report(None, 0, C.byref(need)), "trace_report")
    buf = C.create_string_buffer(need.value)
    _lib.check(L.mtlg_trace_report(buf, need.value, None), "trace_report")
    out = {}
    for line in buf.value.decode().splitlines():
        f = line.split()
        out[int(f[0])] = (" ".join(f[1:-2]), int(f[-2]), float(f[-1]))
    return out
