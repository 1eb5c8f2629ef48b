"""Loads libppcb.so (built in-tree by ppc_b200/build.py) and declares the C ABI of
include/ppc_b200.h.  There is no fallback: without the native library every call fails."""
import ctypes as C
import os

from . import types as T

LIBDIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIBPATH = os.path.join(LIBDIR, "libppcb.so")

_lib = None


class PPCError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ppcb error {code}: {msg}")
        self.code = code


class RunInfo(C.Structure):
    _fields_ = [("photons", C.c_uint64), ("hits", C.c_uint64), ("kept", C.c_uint64), ("steps", C.c_uint64),
                ("nan_steps", C.c_uint32), ("capped", C.c_uint32), ("device_ms", C.c_double)]


class Info(C.Structure):
    _fields_ = [("max_bunch_size", C.c_uint64), ("workgroup_size", C.c_uint64), ("total_device_ms", C.c_double),
                ("max_photons", C.c_uint64), ("hit_capacity", C.c_uint64), ("devices", C.c_int32),
                ("threads", C.c_int32), ("blocks", C.c_int32), ("regs", C.c_int32), ("gsize", C.c_int32),
                ("size", C.c_int32), ("nstr", C.c_int32), ("rsize", C.c_int32), ("eff", C.c_float),
                ("ovr", C.c_uint32), ("seed", C.c_uint32), ("nextgen", C.c_int32)]


class BatchInfo(C.Structure):
    _fields_ = [("photons", C.c_uint64), ("steps", C.c_uint64), ("hits", C.c_uint64), ("kept", C.c_uint64),
                ("overflowed", C.c_uint32), ("pad_", C.c_uint32), ("device_ms", C.c_double), ("graph_ms", C.c_double)]


class TuneInfo(C.Structure):
    _fields_ = [("threads", C.c_int32), ("blocks_per_sm", C.c_int32), ("refill_below", C.c_int32),
                ("pad_", C.c_int32), ("photons_per_s", C.c_double)]


class GradInfo(C.Structure):
    _fields_ = [("ll", C.c_double), ("photons", C.c_uint64), ("hits", C.c_uint64), ("replayed", C.c_uint64),
                ("unmatched", C.c_uint64), ("steps", C.c_uint64), ("forward_ms", C.c_double),
                ("backward_ms", C.c_double)]


class LlhOpts(C.Structure):
    _fields_ = [("lbin", C.c_double), ("sig", C.c_double), ("qmin", C.c_double), ("qsat", C.c_double),
                ("drep", C.c_double), ("peak", C.c_int32), ("mono", C.c_int32), ("norm", C.c_int32),
                ("unh", C.c_int32), ("flasher", C.c_int32), ("fla_str", C.c_int32), ("fla_om", C.c_int32),
                ("fsep", C.c_int32)]


class LlhInfo(C.Structure):
    _fields_ = [("lbin", C.c_double), ("t0", C.c_double), ("ndof", C.c_int32), ("doms", C.c_int32),
                ("blocks", C.c_int32), ("errors", C.c_int32)]


class Dom(C.Structure):
    _fields_ = [("R", C.c_float), ("F", C.c_float), ("r", C.c_float * 3)]


# ppcb_hitz_rec: 76 bytes of fields, padded to 80 by the C compiler (8-byte alignment)
HITZ_DTYPE = __import__("numpy").dtype([
    ("track_first", "<i4"), ("frame", "<i4"), ("track_second", "<u8"), ("t0", "<f8"),
    ("str", "<i4"), ("om", "<i4"), ("pmt", "<i4"), ("dir", "<f4"), ("time", "<f4"),
    ("r", "<f4", 4), ("n", "<f4", 4), ("pad_", "<u4")])

# exported C symbols (kept in sync with include/ppc_b200.h; tests check every one loads)
EXPORTS = [
    "ppcb_last_error", "ppcb_create", "ppcb_destroy", "ppcb_initialize", "ppcb_choose", "ppcb_set_seed",
    "ppcb_set_options", "ppcb_ini", "ppcb_fin", "ppcb_get_info", "ppcb_flset", "ppcb_fldir", "ppcb_flshift",
    "ppcb_sett", "ppcb_addp", "ppcb_addp_clst", "ppcb_addp_mopo", "ppcb_flone", "ppcb_eout", "ppcb_efin",
    "ppcb_set_res", "ppcb_xrnd", "ppcb_hitz_count", "ppcb_hitz_copy", "ppcb_keep_raw", "ppcb_raw_count",
    "ppcb_raw_copy", "ppcb_last_run", "ppcb_propagate", "ppcb_propagate_device", "ppcb_rng_get", "ppcb_rng_set",
    "ppcb_rng_reset", "ppcb_table", "ppcb_generate_device", "ppcb_index_probe_device", "ppcb_propagate_noalloc",
    "ppcb_batch_create", "ppcb_batch_destroy", "ppcb_batch_set_graph", "ppcb_batch_run", "ppcb_batch_counts",
    "ppcb_batch_hits", "ppcb_batch_autotune", "ppcb_set_ice", "ppcb_get_ice", "ppcb_gradient",
    "ppcb_fp32_peak", "ppcb_accept_device", "ppcb_accept", "ppcb_llh_default_opts", "ppcb_llh_create",
    "ppcb_llh_destroy", "ppcb_llh_get_info", "ppcb_llh_blocks", "ppcb_llh_eval_device", "ppcb_llh_eval",
    "ppcb_sources_device", "ppcb_sources", "ppcb_f2k_sources", "ppcb_back_end", "ppcb_sfu_peak",
    "ppcb_string_grid_probe", "ppcb_gradgraph_create", "ppcb_gradgraph_run", "ppcb_gradgraph_destroy",
]


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(f"native library missing: {LIBPATH} (run `python ppc_b200/build.py`)")
    L = C.CDLL(LIBPATH)
    vp, i32, u32, u64, f32, f64 = C.c_void_p, C.c_int32, C.c_uint32, C.c_uint64, C.c_float, C.c_double
    P = C.POINTER
    sig = {
        "ppcb_last_error": (C.c_char_p, []),
        "ppcb_create": (i32, [P(vp)]),
        "ppcb_destroy": (i32, [vp]),
        "ppcb_initialize": (i32, [vp, C.c_char_p, f32]),
        "ppcb_choose": (i32, [vp, i32]),
        "ppcb_set_seed": (i32, [vp, u32]),
        "ppcb_set_options": (i32, [vp, i32, u32, i32]),
        "ppcb_ini": (i32, [vp]),
        "ppcb_fin": (i32, [vp]),
        "ppcb_get_info": (i32, [vp, P(Info)]),
        "ppcb_flset": (i32, [vp, i32, i32, P(Dom)]),
        "ppcb_fldir": (i32, [vp, vp]),
        "ppcb_flshift": (i32, [vp, vp, vp, vp]),
        "ppcb_sett": (i32, [vp, f32, f32, f32, i32, u64, i32, f64]),
        "ppcb_addp": (i32, [vp, f32, f32, f32, f32, f32, f32, i32, f32]),
        "ppcb_addp_clst": (i32, [vp, f32, f32, f32, f32, u64, f32, f32]),
        "ppcb_addp_mopo": (i32, [vp, f32, f32, f32, f32, f32, f32, f32, f32, f32]),
        "ppcb_flone": (i32, [vp, u64]),
        "ppcb_eout": (i32, [vp]),
        "ppcb_efin": (i32, [vp]),
        "ppcb_back_end": (i32, [vp, vp, u64]),
        "ppcb_set_res": (i32, [vp, f32, f32]),
        "ppcb_xrnd": (f32, [vp]),
        "ppcb_hitz_count": (i32, [vp, P(u64)]),
        "ppcb_hitz_copy": (i32, [vp, vp, u64, P(u64)]),
        "ppcb_keep_raw": (i32, [vp, i32]),
        "ppcb_raw_count": (i32, [vp, P(u64)]),
        "ppcb_raw_copy": (i32, [vp, vp, u64, P(u64)]),
        "ppcb_last_run": (i32, [vp, P(RunInfo), P(RunInfo)]),
        "ppcb_propagate": (i32, [vp, vp, i32, vp, u64, P(u64), P(RunInfo)]),
        "ppcb_propagate_device": (i32, [vp, i32, vp, vp, i32, u64, vp, u64, vp, vp]),
        "ppcb_rng_get": (i32, [vp, i32, vp, u64]),
        "ppcb_rng_set": (i32, [vp, i32, vp, u64]),
        "ppcb_rng_reset": (i32, [vp]),
        "ppcb_table": (i32, [vp, C.c_char_p, P(vp), P(u64)]),
        "ppcb_generate_device": (i32, [vp, i32, vp, vp, i32, u64, vp, vp]),
        "ppcb_index_probe_device": (i32, [vp, i32, vp, i32, vp, vp, vp]),
        "ppcb_string_grid_probe": (i32, [vp, vp, i32, vp]),
        "ppcb_gradgraph_create": (i32, [vp, vp, i32, u32, vp, f64, u64, vp]),
        "ppcb_gradgraph_run": (i32, [vp, vp, vp, vp, vp, vp, vp]),
        "ppcb_gradgraph_destroy": (i32, [vp]),
        "ppcb_propagate_noalloc": (i32, [vp, i32, vp, i32, u64, vp, u64, vp, vp]),
        "ppcb_batch_create": (i32, [vp, i32, u32, u32, u64, P(vp)]),
        "ppcb_batch_destroy": (i32, [vp]),
        "ppcb_batch_set_graph": (i32, [vp, i32]),
        "ppcb_batch_run": (i32, [vp, vp, i32, u32, f64, P(BatchInfo)]),
        "ppcb_batch_counts": (i32, [vp, vp, vp]),
        "ppcb_batch_hits": (i32, [vp, vp, u64, P(u64)]),
        "ppcb_batch_autotune": (i32, [vp, vp, i32, u32, u64, P(TuneInfo)]),
        "ppcb_set_ice": (i32, [vp, vp, vp]),
        "ppcb_get_ice": (i32, [vp, vp, vp, P(i32)]),
        "ppcb_gradient": (i32, [vp, vp, i32, u32, vp, vp, f64, u64, vp, vp, vp, P(GradInfo)]),
        "ppcb_fp32_peak": (i32, [i32, i32, P(f64), P(f64)]),
        "ppcb_sfu_peak": (i32, [i32, i32, P(f64), P(f64)]),
        "ppcb_accept_device": (i32, [vp, i32, vp, u64, u32, vp, vp, vp]),
        "ppcb_accept": (i32, [vp, vp, u64, u32, vp, u64, P(u64)]),
        "ppcb_sources_device": (i32, [vp, i32, vp, u64, u32, vp, vp, u64, vp, vp]),
        "ppcb_sources": (i32, [vp, vp, u64, u32, vp, vp, u64, P(u64), P(u64)]),
        "ppcb_f2k_sources": (i32, [C.c_char_p, u64, u32, vp, u64, P(u64), P(u64)]),
        "ppcb_llh_default_opts": (i32, [P(LlhOpts)]),
        "ppcb_llh_create": (i32, [vp, i32, vp, u64, vp, u64, vp, u64, P(LlhOpts), P(vp)]),
        "ppcb_llh_destroy": (i32, [vp]),
        "ppcb_llh_get_info": (i32, [vp, P(LlhInfo)]),
        "ppcb_llh_blocks": (i32, [vp, vp, u64, P(u64)]),
        "ppcb_llh_eval_device": (i32, [vp, vp, u64, u32, vp, i32, f64, vp, vp]),
        "ppcb_llh_eval": (i32, [vp, vp, u64, u32, vp, i32, f64, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(code):
    if code != 0:
        raise PPCError(code, lib().ppcb_last_error().decode(errors="replace"))
