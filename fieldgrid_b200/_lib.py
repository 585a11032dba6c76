"""Loads the engine's shared library (libfieldgrid.so, built in-tree next to this file) and
declares the C ABI of include/fieldgrid.h for ctypes.

There is no fallback: if the library is missing or fails to load, every entry point that needs
it raises, naming the build step.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfieldgrid.so")

_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib():
    """The loaded libfieldgrid.so; raises LibraryMissing when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibraryMissing(
            f"{LIB_PATH} is not built: run `python -c 'import __graft_entry__ as g; g.build()'` "
            "(the CUDA engine has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    _declare(L)
    _lib = L
    return L


def _declare(L):
    P = C.POINTER
    u64, u32, i32, dbl = C.c_uint64, C.c_uint32, C.c_int32, C.c_double
    vp, cp, sz = C.c_void_p, C.c_char_p, C.c_size_t
    sig = {
        "fg_version": (cp, []),
        "fg_last_error": (cp, []),
        "fg_gpu_open": (C.c_int, [C.c_int, P(vp), cp, sz]),
        "fg_gpu_close": (None, [vp]),
        "fg_gpu_name": (C.c_int, [vp, cp, sz]),
        "fg_sim_try_new": (C.c_int, [P(A.fg_sim_spec), P(vp), cp, sz]),
        "fg_sim_free": (None, [vp]),
        "fg_sim_dt": (dbl, [vp]),
        "fg_sim_dims": (None, [vp, P(u64)]),
        "fg_sim_count": (u64, [vp, cp]),
        "fg_sim_coefs": (C.c_int, [vp, u32, P(C.c_float), P(C.c_float)]),
        "fg_sim_wires": (C.c_int, [vp, P(u32), u64]),
        "fg_sim_coef_classes": (u64, [vp]),
        "fg_time_step": (dbl, [P(dbl), u64, P(dbl), u64, P(dbl), u64]),
        "fg_run": (C.c_int, [vp, vp, u64, P(A.fg_pulse), P(A.fg_extras), A.PROGRESS_FN, vp, P(vp), cp, sz]),
        "fg_record_steps": (u64, [vp]),
        "fg_record_ports": (u64, [vp]),
        "fg_record_decay_db": (dbl, [vp]),
        "fg_record_series": (P(C.c_float), [vp, P(u64)]),
        "fg_record_plane": (P(C.c_float), [vp, P(u64)]),
        "fg_record_ntff": (P(C.c_float), [vp, P(u64)]),
        "fg_record_e": (P(C.c_float), [vp, P(u64)]),
        "fg_record_h": (P(C.c_float), [vp, P(u64)]),
        "fg_record_transfer": (None, [vp, P(u64), P(u64)]),
        "fg_record_free": (None, [vp]),
        "fg_session_kernel_times": (C.c_int, [vp, u64, cp, P(dbl), u64, P(u64)]),
        "fg_session_new": (C.c_int, [vp, vp, u64, P(A.fg_pulse), P(A.fg_extras), P(vp), cp, sz]),
        "fg_session_step": (C.c_int, [vp, u64]),
        "fg_session_sync": (C.c_int, [vp]),
        "fg_session_energy": (C.c_int, [vp, P(dbl)]),
        "fg_session_steps": (u64, [vp]),
        "fg_session_read": (C.c_int, [vp, cp, P(C.c_float), u64]),
        "fg_session_stream": (vp, [vp]),
        "fg_session_launches_per_step": (u64, [vp]),
        "fg_session_device_bytes": (u64, [vp]),
        "fg_session_variant": (cp, [vp]),
        "fg_session_free": (None, [vp]),
        "fg_patches": (C.c_int, [vp, u64, P(u32), P(dbl), P(dbl), P(u64)]),
        "fg_far_load": (C.c_int, [P(dbl), P(dbl), u64, P(C.c_float), u64, u64, dbl, dbl, dbl, P(vp)]),
        "fg_far_free": (None, [vp]),
        "fg_far_field": (C.c_int, [vp, vp, P(dbl), u64, P(dbl)]),
        "fg_far_intensity": (C.c_int, [vp, vp, P(dbl), u64, P(dbl)]),
        "fg_far_radiated": (C.c_int, [vp, vp, u64, P(dbl), P(dbl)]),
        "fg_batch_new": (C.c_int, [vp, P(vp), P(u64), P(A.fg_pulse), u64, u64, P(A.fg_batch_options), P(vp), cp, sz]),
        "fg_batch_step": (C.c_int, [vp, u64, cp, sz]),
        "fg_batch_sync": (C.c_int, [vp]),
        "fg_batch_read": (C.c_int, [vp, u64, cp, P(C.c_float), u64, cp, sz]),
        "fg_batch_info": (C.c_int, [vp, P(A.fg_batch_options), P(C.c_int), P(dbl), P(u64)]),
        "fg_batch_free": (None, [vp]),
        "fg_flux_gradient": (C.c_int, [vp, vp, u64, P(A.fg_pulse), P(A.fg_flux_spec), P(A.fg_flux_result), P(dbl),
                                       P(dbl), cp, sz]),
        "fg_energy_noalloc": (C.c_int, [vp, vp, u64, vp, vp]),
        "fg_port_spectra": (C.c_int, [P(C.c_float), u64, u64, u64, dbl, P(dbl), u64, P(dbl), P(dbl)]),
        "fg_raster_fill": (C.c_int, [vp, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(dbl), u64, C.c_int, P(C.c_uint8), P(C.c_uint8), cp, sz]),
        "fg_raster_solid_edges": (C.c_int, [vp, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(C.c_uint8), cp, sz]),
        "fg_raster_solid_cells": (C.c_int, [vp, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(C.c_uint8), cp, sz]),
        "fg_raster_sheet_edges": (C.c_int, [vp, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(dbl), u64, P(C.c_uint8), cp, sz]),
        "fg_raster_closed": (C.c_int, [P(dbl), u64]),
        "fg_flux_gradient_batch": (C.c_int, [vp, vp, P(u64), P(A.fg_pulse), P(A.fg_flux_spec), u64, C.c_int,
                                             P(A.fg_flux_result), vp, vp, cp, sz]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def exported_symbols():
    """The fg_* names include/fieldgrid.h declares (parsed from the header)."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "fieldgrid.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(fg_[a-z0-9_]+)\s*\(", text)))
