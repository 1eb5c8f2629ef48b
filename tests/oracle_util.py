"""Test-side access to the oracle (oracle/libppc_oracle.so) and to the reference harness
(oracle/_ref/ref_harness).  Only tests, smoke() and bench.py's CPU-baseline leg use this.
"""
import ctypes as C
import json
import os
import subprocess

import numpy as np

from ppc_b200 import types as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libppc_oracle.so")
REF_HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
REF_PPC = os.path.join(ROOT, "oracle", "_ref", "ppc")


def _reference_dir():
    """The reference source tree as oracle/Makefile names it (its REF variable)."""
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "refdir"], capture_output=True, text=True)
    return r.stdout.strip() if r.returncode == 0 else ""


REFERENCE = _reference_dir()


class Tables(C.Structure):
    _fields_ = [("p", C.c_void_p), ("az", C.c_void_p), ("lr", C.c_void_p), ("ls", C.c_void_p),
                ("is_", C.c_void_p), ("mcol", C.c_void_p), ("sc", C.c_void_p), ("lp", C.c_void_p),
                ("absca", C.c_void_p), ("wmeta", C.c_void_p), ("oms", C.c_void_p)]


class Rng(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("a", C.c_uint32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle library missing: run `make -C oracle oracle`")
        L = C.CDLL(ORACLE_SO)
        vp, u64, u32 = C.c_void_p, C.c_uint64, C.c_uint32
        L.ppco_xrnd.restype = C.c_float
        L.ppco_xrnd.argtypes = [vp]
        L.ppco_zshift.restype = C.c_float
        L.ppco_zshift.argtypes = [vp, vp, vp]
        L.ppco_generate.argtypes = [vp, vp, vp, vp]
        L.ppco_propagate.restype = u64
        L.ppco_propagate.argtypes = [vp, vp, vp, vp, vp, u64]
        L.ppco_run_reference_order.restype = u64
        L.ppco_run_reference_order.argtypes = [vp, vp, C.c_int, u32, u32, vp, vp, u64, vp]
        L.ppco_run_fused.restype = u64
        L.ppco_run_fused.argtypes = [vp, vp, C.c_int, u64, u32, vp, vp, vp, u64, vp]
        _lib = L
    return _lib


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class OracleTables:
    """Holds a table image (dict of numpy arrays + Params) and the ppco_tables view of it."""

    def __init__(self, params, arrays):
        self.params = params
        self.a = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
        self.t = Tables(C.cast(C.pointer(self.params), C.c_void_p), ptr(self.a["az"]), ptr(self.a["lr"]),
                        ptr(self.a["ls"]), ptr(self.a["is"]), ptr(self.a["mcol"]), ptr(self.a["sc"]),
                        ptr(self.a["lp"]), ptr(self.a["absca"]), ptr(self.a["wmeta"]), ptr(self.a["oms"]))

    @property
    def tp(self):
        return C.byref(self.t)

    def zshift(self, pos):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 4)
        out = np.zeros((len(pos), 2), np.float32)
        L = lib()
        for k in range(len(pos)):
            dz = C.c_float(self.params.dh)
            out[k, 0] = L.ppco_zshift(self.tp, ptr(pos[k]), C.byref(dz))
            out[k, 1] = dz.value
        return out

    def generate(self, bunch, rng):
        out = np.zeros(1, T.PBUF_DTYPE)
        lib().ppco_generate(self.tp, ptr(bunch), C.byref(rng), ptr(out))
        return out[0]

    def run_reference_order(self, bunches, num, x, y, a, nthr=512, cap=1 << 20):
        hits = np.zeros(cap, T.HIT_DTYPE)
        pbuf = np.zeros(num, T.PBUF_DTYPE)
        s = Rng(x, y, a)
        nh = lib().ppco_run_reference_order(self.tp, ptr(bunches), len(bunches), num, nthr, C.byref(s),
                                            ptr(hits), cap, ptr(pbuf))
        return hits[:min(nh, cap)], pbuf, nh, s

    def run_fused(self, bunches, num, rs, rm, cap=1 << 20):
        """Deterministic per-thread order: len(rs) threads, thread t owns photons t, t+T, ..."""
        rs = np.ascontiguousarray(rs, np.uint64).copy()
        rm = np.ascontiguousarray(rm, np.uint32)
        hits = np.zeros(cap, T.HIT_DTYPE)
        steps = C.c_uint64(0)
        nh = lib().ppco_run_fused(self.tp, ptr(bunches), len(bunches), num, len(rs), ptr(rs), ptr(rm),
                                  ptr(hits), cap, C.byref(steps))
        return hits[:min(nh, cap)], nh, rs, steps.value


def load_dump(path):
    """Named records written by ref_harness `tables`: name[32] | esz u32 | n u64 | bytes."""
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    o = 0
    while o < len(data):
        name = data[o:o + 32].split(b"\0")[0].decode()
        esz = int.from_bytes(data[o + 32:o + 36], "little")
        n = int.from_bytes(data[o + 36:o + 44], "little")
        o += 44
        out[name] = data[o:o + esz * n]
        o += esz * n
    return out


_SCALARS_I = {"size", "tmod", "vthk", "lnum", "lpts", "l0", "gsize", "rsize"}


def tables_from_dump(raw):
    """Builds an OracleTables from a reference table dump (the reference's own values)."""
    p = T.Params()
    for name, _ in T.Params._fields_:
        if name in raw:
            b = raw[name]
            if name in ("cn", "mnum", "mcut"):
                getattr(p, name)[:] = list(np.frombuffer(b, "<i4"))
            elif name in ("cl", "crst", "cb", "mmin", "mstp", "bfr"):
                getattr(p, name)[:] = list(np.frombuffer(b, "<f4"))
            elif name in _SCALARS_I:
                v = np.frombuffer(b, "<i2" if len(b) == 2 else "<i4")[0]
                setattr(p, name, int(v))
            else:
                setattr(p, name, float(np.frombuffer(b, "<f4")[0]))
    arrays = {
        "az": np.frombuffer(raw["az"], "<f4").copy(),
        "lr": np.frombuffer(raw["lr"], "<f4").copy(),
        "ls": np.frombuffer(raw["ls"], "<u2").copy(),
        "is": np.frombuffer(raw["is"], "<u2").copy(),
        "mcol": np.frombuffer(raw["mcol"], "<i1").copy(),
        "sc": np.frombuffer(raw["sc"], T.LINE_DTYPE).copy(),
        "lp": np.frombuffer(raw["lp"], "<f4").copy(),
        "absca": np.frombuffer(raw["absca"], "<f4").copy(),
        "wmeta": np.frombuffer(raw["wmeta"], "<f4").copy(),
        "oms": np.frombuffer(raw["oms"], T.DOM_DTYPE).copy(),
    }
    # unused cells of the reference's string index are zero; the kernel never reads them
    return OracleTables(p, arrays)


def harness_available():
    return os.path.exists(REF_HARNESS)


def run_harness(args, env):
    e = dict(os.environ)
    e.update(env)
    e.setdefault("PPCB_QUIET", "1")
    r = subprocess.run([REF_HARNESS] + list(args), env=e, capture_output=True, text=True, check=True)
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    return json.loads(lines[-1]) if lines else None


def harness_tables(icedir, tmp, env=None):
    out = os.path.join(str(tmp), "tables.bin")
    e = {"PPCTABLESDIR": icedir}
    e.update(env or {})
    run_harness(["tables", out], e)
    return load_dump(out)


def harness_run(icedir, spec, photons, seed, prefix, env=None):
    e = {"PPCTABLESDIR": icedir}
    e.update(env or {})
    info = run_harness(["run", spec, str(photons), str(seed), prefix], e)
    hits = np.fromfile(prefix + ".hits", T.HIT_DTYPE)
    pbuf = np.fromfile(prefix + ".pbuf", T.PBUF_DTYPE)
    bunch = np.fromfile(prefix + ".bunch", T.BUNCH_DTYPE)
    return info, hits, pbuf, bunch


def tables_from_product(ctx):
    """OracleTables over the product's own table image (identical values to the GPU's)."""
    t = ctx.tables()
    arrays = {k: t[k] for k in ("az", "lr", "ls", "is", "mcol", "sc", "lp", "absca", "wmeta", "oms")}
    return OracleTables(ctx.params(), arrays)


def index_probe(tb, pos):
    """pos: (n, 8) float32 rows x,y,z,t,nx,ny,nz,length -> (ints (n,8), floats (n,2))."""
    L = lib()
    L.ppco_index_probe.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    pos = np.ascontiguousarray(pos, np.float32)
    n = len(pos)
    oi = np.zeros((n, 8), np.int32)
    of = np.zeros((n, 2), np.float32)
    L.ppco_index_probe(tb.tp, ptr(pos), n, ptr(oi), ptr(of))
    return oi, of


def mwc_init(seed, rm):
    """Initial stream state of every thread: (362436069 + seed, 1234567), gpu/ini.cxx:556-571."""
    v = np.uint64((362436069 + seed) & 0xFFFFFFFF) | (np.uint64(1234567) << np.uint64(32))
    return np.full(len(rm), v, np.uint64)


# ---- DirectFit likelihood oracle (oracle/libllh_oracle.so) ----------------------------------
LLH_ORACLE_SO = os.path.join(ROOT, "oracle", "libllh_oracle.so")


class LlhoOpts(C.Structure):
    _fields_ = [("lbin", C.c_double), ("sig", C.c_double), ("qmin", C.c_double), ("qsat", C.c_double),
                ("drep", C.c_double), ("peak", C.c_int32), ("mono", C.c_int32), ("norm", C.c_int32),
                ("unh", C.c_int32), ("flasher", C.c_int32), ("fla_str", C.c_int32), ("fla_om", C.c_int32),
                ("fsep", C.c_int32)]


LLHO_DEFAULTS = dict(lbin=0.0, sig=0.10, qmin=0.1, qsat=500.0, drep=1.0, peak=0, mono=0, norm=0, unh=0, flasher=0,
                     fla_str=0, fla_om=0, fsep=1)
LLHO_SIM_DTYPE = np.dtype([("str", "<i4"), ("om", "<i4"), ("t", "<f4")])

_llh = None


def llh_lib():
    global _llh
    if _llh is None:
        if not os.path.exists(LLH_ORACLE_SO):
            raise RuntimeError("likelihood oracle missing: run `make -C oracle oracle`")
        L = C.CDLL(LLH_ORACLE_SO)
        vp, lg, i32, f64 = C.c_void_p, C.c_long, C.c_int, C.c_double
        L.llho_llf.restype = f64
        L.llho_llf.argtypes = [f64, f64, f64, f64, f64, C.POINTER(i32)]
        L.llho_setup.restype = i32
        L.llho_setup.argtypes = [vp, lg, vp, lg, vp, lg, vp, vp, lg, C.POINTER(lg), C.POINTER(f64), C.POINTER(f64),
                                 C.POINTER(i32)]
        L.llho_fllh.restype = i32
        L.llho_fllh.argtypes = [vp, lg, vp, lg, vp, lg, vp, vp, lg, vp, i32, f64, vp, C.POINTER(i32)]
        _llh = L
    return _llh


def llf(s, d, nsim, ndat, sig=0.10):
    err = C.c_int(0)
    v = llh_lib().llho_llf(float(s), float(d), float(nsim), float(ndat), float(sig), C.byref(err))
    return v, err.value


def _llh_inputs(data, windows, bad, opts):
    o = LlhoOpts(**{**LLHO_DEFAULTS, **(opts or {})})
    data = np.ascontiguousarray(data, T.LLH_HIT_DTYPE)
    win = np.ascontiguousarray(windows if windows is not None else np.zeros(0, T.LLH_WINDOW_DTYPE),
                               T.LLH_WINDOW_DTYPE)
    badk = np.ascontiguousarray(bad if bad is not None else np.zeros((0, 2)), np.int32).reshape(-1, 2)
    ptr = lambda a: C.c_void_p(a.ctypes.data) if len(a) else None
    return o, data, win, badk, ptr


def llh_setup(data, windows=None, bad=None, opts=None):
    """The oracle's observed side: (blocks, lbin, t0, ndof), or None where it reports an error."""
    o, data, win, badk, ptr = _llh_inputs(data, windows, bad, opts)
    cap = 200 * (len(np.unique(data[["str", "om"]])) + len(win) + 1)
    out = np.zeros(cap, T.LLH_BLOCK_DTYPE)
    nb, lbin, t0, ndof = C.c_long(), C.c_double(), C.c_double(), C.c_int()
    r = llh_lib().llho_setup(ptr(data), len(data), ptr(win), len(win), ptr(badk), len(badk), C.byref(o),
                             C.c_void_p(out.ctypes.data), cap, C.byref(nb), C.byref(lbin), C.byref(t0),
                             C.byref(ndof))
    if r != 0:
        return None
    return out[:nb.value], lbin.value, t0.value, ndof.value


def llh_fllh(data, sim, dts, nsim, windows=None, bad=None, opts=None):
    """fllh(dt, nsim) for every dt over the accepted simulated hits `sim` (str, om, t)."""
    o, data, win, badk, ptr = _llh_inputs(data, windows, bad, opts)
    s = np.zeros(len(sim), LLHO_SIM_DTYPE)
    if len(sim):
        s["str"], s["om"], s["t"] = sim["str"], sim["om"], sim["t"]
    dts = np.ascontiguousarray(np.atleast_1d(dts), np.float64)
    out = np.zeros(len(dts))
    err = C.c_int()
    r = llh_lib().llho_fllh(ptr(data), len(data), ptr(win), len(win), ptr(badk), len(badk), C.byref(o), ptr(s),
                            len(s), C.c_void_p(dts.ctypes.data), len(dts), float(nsim),
                            C.c_void_p(out.ctypes.data), C.byref(err))
    assert r == 0
    return out, err.value
