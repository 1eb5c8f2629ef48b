"""Python face of the propagator, mirroring the reference's library interface
(namespace xppc in llh/ppc.h; definitions in gpu/ppc.cu and gpu/f2k.cxx) over the C ABI.

    ctx = PPC()                       # start()
    ctx.initialize(1.0, "ice/dir")    # initialize(enh); directory or PPCTABLESDIR
    ctx.choose(0); ctx.ini()          # choose(device), ini()
    ctx.flset(63, 20)                 # flset(str, om)
    ctx.sett(0, 0, 1, (1, 7), 0)      # sett(nx, ny, nz, id, frame)
    ctx.flone(10**7); ctx.eout()      # flone(num), eout()
    ctx.hitz()                        # the binned hit map, flattened
    ctx.efin(); ctx.fin()             # efin(), fin()

Errors raise PPCError with the reference's exit status as `.code`.
"""
import ctypes as C
import weakref

import numpy as np

from . import types as T
from ._lib import HITZ_DTYPE, Dom, Info, PPCError, RunInfo, check, lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class PPC:
    def __init__(self):
        self._c = C.c_void_p()
        self._children = weakref.WeakSet()  # handles made from this context, closed before it
        check(lib().ppcb_create(C.byref(self._c)))

    # ---- lifecycle -------------------------------------------------------------
    def initialize(self, enh=1.0, tables_dir=None):
        check(lib().ppcb_initialize(self._c, tables_dir.encode() if tables_dir else None, float(enh)))

    def choose(self, device=0):
        check(lib().ppcb_choose(self._c, int(device)))

    def set_seed(self, seed):
        check(lib().ppcb_set_seed(self._c, int(seed) & 0xFFFFFFFF))

    def set_options(self, deterministic=False, max_steps=1_000_000, blocks_per_sm=0, photon_streams=False):
        """deterministic: photon i on thread i mod T (the reference's order).  photon_streams:
        each photon draws from its own stream keyed by (seed, i), whatever thread runs it, so
        runs that differ only in the ice share every photon's random numbers.  i counts the
        photons of one launch: launches that should be independent need different seeds."""
        mode = 2 if photon_streams else int(bool(deterministic))
        check(lib().ppcb_set_options(self._c, mode, int(max_steps), int(blocks_per_sm)))

    def ini(self):
        check(lib().ppcb_ini(self._c))

    def fin(self):
        check(lib().ppcb_fin(self._c))

    def close(self):
        for h in list(getattr(self, "_children", ())):
            h.close()
        if self._c:
            lib().ppcb_destroy(self._c)
            self._c = C.c_void_p()

    stop = close

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        i = Info()
        check(lib().ppcb_get_info(self._c, C.byref(i)))
        return {k: getattr(i, k) for k, _ in Info._fields_}

    def getMaxBunchSize(self):
        return self.info()["max_bunch_size"]

    def getWorkgroupSize(self):
        return self.info()["workgroup_size"]

    def getTotalDeviceTime(self):
        return self.info()["total_device_ms"]

    # ---- sources -------------------------------------------------------------------
    def flset(self, str_, om):
        d = Dom()
        check(lib().ppcb_flset(self._c, int(str_), int(om), C.byref(d)))
        return {"R": d.R, "F": d.F, "r": list(d.r)}

    def fldir(self):
        a = np.zeros(3, np.float32)
        check(lib().ppcb_fldir(self._c, _p(a)))
        return a

    def flshift(self, m, n, r=None):
        m = np.ascontiguousarray(m, np.float32).copy()
        n = np.ascontiguousarray(n, np.float32).copy()
        rr = None if r is None else np.ascontiguousarray(r, np.float32).copy()
        check(lib().ppcb_flshift(self._c, _p(m), _p(n), _p(rr)))
        return (n, rr) if r is not None else n

    def sett(self, nx, ny, nz, id_, frame, t0=0.0):
        check(lib().ppcb_sett(self._c, nx, ny, nz, int(id_[0]), int(id_[1]), int(frame), float(t0)))

    def addp(self, x, y, z, t, E, dr, type_, scale=1.0):
        check(lib().ppcb_addp(self._c, x, y, z, t, E, dr, int(type_), scale))

    def addp_clst(self, x, y, z, t, n, dr, beta):
        check(lib().ppcb_addp_clst(self._c, x, y, z, t, int(n), dr, beta))

    def addp_mopo(self, x, y, z, t, light, length, beta, tau, fr):
        check(lib().ppcb_addp_mopo(self._c, x, y, z, t, light, length, beta, tau, fr))

    def flone(self, num):
        check(lib().ppcb_flone(self._c, int(num)))

    def eout(self):
        check(lib().ppcb_eout(self._c))

    def efin(self):
        check(lib().ppcb_efin(self._c))

    def back_end(self, hits):
        """The host back end over kernel-level hits computed elsewhere (ppcb_back_end): hits
        of the segments started with sett go into hitz, in segment order."""
        hits = np.ascontiguousarray(hits, T.HIT_DTYPE)
        check(lib().ppcb_back_end(self._c, _p(hits) if len(hits) else None, len(hits)))

    def set_res(self, t, c=0.0):
        check(lib().ppcb_set_res(self._c, float(t), float(c)))

    def xrnd(self):
        return lib().ppcb_xrnd(self._c)

    # ---- results -------------------------------------------------------------------
    def hitz(self):
        n = C.c_uint64()
        check(lib().ppcb_hitz_count(self._c, C.byref(n)))
        out = np.zeros(n.value, HITZ_DTYPE)
        w = C.c_uint64()
        check(lib().ppcb_hitz_copy(self._c, _p(out), n.value, C.byref(w)))
        return out

    def keep_raw(self, keep=True):
        check(lib().ppcb_keep_raw(self._c, int(bool(keep))))

    def raw_hits(self):
        n = C.c_uint64()
        check(lib().ppcb_raw_count(self._c, C.byref(n)))
        out = np.zeros(n.value, T.HIT_DTYPE)
        w = C.c_uint64()
        check(lib().ppcb_raw_copy(self._c, _p(out), n.value, C.byref(w)))
        return out

    def last_run(self):
        a, b = RunInfo(), RunInfo()
        check(lib().ppcb_last_run(self._c, C.byref(a), C.byref(b)))
        f = lambda r: {k: getattr(r, k) for k, _ in RunInfo._fields_}
        return f(a), f(b)

    # ---- direct hot path -----------------------------------------------------------
    def propagate(self, bunches, cap=1 << 22, out=None):
        """Host bunches in, kernel-level hits out (copies included).  `out`: a caller-owned
        HIT_DTYPE array that receives the hits (its length is the capacity); the result is
        a view of it."""
        bunches = np.ascontiguousarray(bunches, T.BUNCH_DTYPE)
        if out is not None:
            if out.dtype != T.HIT_DTYPE or not out.flags.c_contiguous:
                raise TypeError("out must be a contiguous HIT_DTYPE array")
            hits, cap = out, len(out)
        else:
            hits = np.empty(cap, T.HIT_DTYPE)  # only the first min(produced, cap) records are written
        nh = C.c_uint64()
        info = RunInfo()
        check(lib().ppcb_propagate(self._c, _p(bunches), len(bunches), _p(hits), cap, C.byref(nh), C.byref(info)))
        return hits[:min(nh.value, cap)], {k: getattr(info, k) for k, _ in RunInfo._fields_}

    def propagate_device(self, bunches_ptr, bstart_ptr, nb, num, hits_ptr, hcap, ctrl_ptr, stream=0, device=0):
        """One asynchronous launch over caller-owned device memory (raw pointers)."""
        check(lib().ppcb_propagate_device(self._c, device, C.c_void_p(bunches_ptr), C.c_void_p(bstart_ptr), nb,
                                          num, C.c_void_p(hits_ptr), hcap, C.c_void_p(ctrl_ptr),
                                          C.c_void_p(stream) if stream else None))

    def generate_device(self, bunches_ptr, bstart_ptr, nb, num, out_ptr, stream=0, device=0):
        check(lib().ppcb_generate_device(self._c, device, C.c_void_p(bunches_ptr), C.c_void_p(bstart_ptr), nb, num,
                                         C.c_void_p(out_ptr), C.c_void_p(stream) if stream else None))

    def index_probe_device(self, pos_ptr, n, oi_ptr, of_ptr, stream=0, device=0):
        check(lib().ppcb_index_probe_device(self._c, device, C.c_void_p(pos_ptr), n, C.c_void_p(oi_ptr),
                                            C.c_void_p(of_ptr), C.c_void_p(stream) if stream else None))

    def rng_get(self, device=0):
        n = self.info()["threads"]
        a = np.zeros(n, np.uint64)
        check(lib().ppcb_rng_get(self._c, device, _p(a), n))
        return a

    def rng_set(self, rs, device=0):
        rs = np.ascontiguousarray(rs, np.uint64)
        check(lib().ppcb_rng_set(self._c, device, _p(rs), len(rs)))

    def rng_reset(self):
        check(lib().ppcb_rng_reset(self._c))

    # ---- tables --------------------------------------------------------------------
    def table(self, name):
        ptr = C.c_void_p()
        n = C.c_uint64()
        check(lib().ppcb_table(self._c, name.encode(), C.byref(ptr), C.byref(n)))
        return bytes(C.string_at(ptr, n.value)) if n.value else b""

    def params(self):
        p = T.Params()
        C.memmove(C.byref(p), self.table("params"), C.sizeof(p))
        return p

    def tables(self):
        """The kernel-facing table image as numpy arrays (copies)."""
        b = lambda k, dt: np.frombuffer(self.table(k), dt).copy()
        return {
            "az": b("az", "<f4"), "lr": b("lr", "<f4"), "ls": b("ls", "<u2"), "is": b("is", "<u2"),
            "mcol": b("mcol", "<i1"), "sc": b("sc", T.LINE_DTYPE), "lp": b("lp", "<f4"),
            "absca": b("absca", "<f4"), "wmeta": b("wmeta", "<f4"), "oms": b("oms", T.DOM_DTYPE),
            "rm": b("rm", "<u4"), "wvs": b("wvs", "<f4"), "eff": b("eff", "<f4"),
        }


class Batch:
    """Many events in one launch (ppcb_batch_*): bunch .q = event index in [0, events)."""

    def __init__(self, ctx, max_events, max_bunches, hit_capacity, device=0):
        from ._lib import BatchInfo, TuneInfo  # noqa: F401
        self._ctx = ctx
        self._b = C.c_void_p()
        check(lib().ppcb_batch_create(ctx._c, device, int(max_events), int(max_bunches), int(hit_capacity),
                                      C.byref(self._b)))
        self.events = 0
        ctx._children.add(self)

    def set_graph(self, use):
        check(lib().ppcb_batch_set_graph(self._b, int(bool(use))))

    def run(self, bunches, events, hits_per_photon=0.02):
        from ._lib import BatchInfo
        bunches = np.ascontiguousarray(bunches, T.BUNCH_DTYPE)
        info = BatchInfo()
        check(lib().ppcb_batch_run(self._b, _p(bunches), len(bunches), int(events), float(hits_per_photon),
                                   C.byref(info)))
        self.events = int(events)
        return {k: getattr(info, k) for k, _ in BatchInfo._fields_ if k != "pad_"}

    def counts(self):
        produced = np.zeros(self.events, np.uint32)
        offsets = np.zeros(self.events + 1, np.uint64)
        check(lib().ppcb_batch_counts(self._b, _p(produced), _p(offsets)))
        return produced, offsets

    def hits(self):
        n = C.c_uint64()
        check(lib().ppcb_batch_hits(self._b, None, 0, C.byref(n)))
        out = np.zeros(n.value, T.HIT_DTYPE)
        check(lib().ppcb_batch_hits(self._b, _p(out), n.value, C.byref(n)))
        return out

    def autotune(self, bunches, events, sample_photons=20_000_000):
        from ._lib import TuneInfo
        bunches = np.ascontiguousarray(bunches, T.BUNCH_DTYPE)
        t = TuneInfo()
        check(lib().ppcb_batch_autotune(self._b, _p(bunches), len(bunches), int(events), int(sample_photons),
                                        C.byref(t)))
        return {k: getattr(t, k) for k, _ in TuneInfo._fields_ if k != "pad_"}

    def close(self):
        if self._b:
            lib().ppcb_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ice_methods():
    def set_ice(self, be=None, ba=None):
        """New per-layer be / ba at 400 nm (icemodel.dat columns 2-3, file order)."""
        b = None if be is None else np.ascontiguousarray(be, np.float32)
        a = None if ba is None else np.ascontiguousarray(ba, np.float32)
        check(lib().ppcb_set_ice(self._c, _p(b), _p(a)))

    def get_ice(self):
        n = C.c_int32()
        check(lib().ppcb_get_ice(self._c, None, None, C.byref(n)))
        be = np.zeros(n.value, np.float32)
        ba = np.zeros(n.value, np.float32)
        check(lib().ppcb_get_ice(self._c, _p(be), _p(ba), C.byref(n)))
        return be, ba

    def gradient(self, bunches, observed=None, weights=None, scale=1.0, hit_cap=None, events=0):
        """LL (or sum_d w_d mu_d) and its gradient in (be, ba), file order (ppcb_gradient).
        Charge bins: per DOM (events=0), or per (event, DOM) with the event = the bunch's q
        (observed / weights / counts then have shape (events, gsize))."""
        from ._lib import GradInfo
        bunches = np.ascontiguousarray(bunches, T.BUNCH_DTYPE)
        info_ = self.info()
        gsize, size = info_["gsize"], info_["size"]
        if hit_cap is None:
            hit_cap = int(bunches["num"].sum() * 0.02) + (1 << 16)
        nbins = gsize * (events if events else 1)
        obs = None if observed is None else np.ascontiguousarray(observed, np.float32).reshape(-1)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32).reshape(-1)
        for name, x in (("observed", obs), ("weights", w)):
            if x is not None and x.size != nbins:
                raise ValueError(f"{name}: {x.size} values for {nbins} charge bins")
        counts = np.zeros(nbins, np.uint32)
        g_be = np.zeros(size, np.float64)
        g_ba = np.zeros(size, np.float64)
        gi = GradInfo()
        check(lib().ppcb_gradient(self._c, _p(bunches), len(bunches), int(events), _p(obs), _p(w), float(scale),
                                  int(hit_cap), _p(counts), _p(g_be), _p(g_ba), C.byref(gi)))
        if events:
            counts = counts.reshape(events, gsize)
        return {"ll": gi.ll, "counts": counts, "g_be": g_be, "g_ba": g_ba,
                "info": {k: getattr(gi, k) for k, _ in GradInfo._fields_}}

    def gradient_graph(self, bunches, observed, events=0, scale=1.0, hit_cap=None):
        """One fit iteration as a CUDA graph over fixed bunches and observed charges
        (ppcb_gradgraph_*): GradGraph.run(be, ba) returns what gradient(observed=...) does."""
        return GradGraph(self, bunches, observed, events, scale, hit_cap)

    PPC.set_ice = set_ice
    PPC.get_ice = get_ice
    PPC.gradient = gradient
    PPC.gradient_graph = gradient_graph


_ice_methods()


def sfu_peak(device=0, repeats=5):
    """Measured special-function-unit throughput of `device` in tera-ops/s (ppcb_sfu_peak)."""
    t, ms = C.c_double(), C.c_double()
    check(lib().ppcb_sfu_peak(int(device), int(repeats), C.byref(t), C.byref(ms)))
    return t.value


def fp32_peak(device=0, repeats=5):
    """Measured FP32 FMA throughput of `device` in TFLOP/s (ppcb_fp32_peak)."""
    t, ms = C.c_double(), C.c_double()
    check(lib().ppcb_fp32_peak(int(device), int(repeats), C.byref(t), C.byref(ms)))
    return t.value


def _accept(self, hits, seed=0):
    """Device hit back end (ppcb_accept): the acceptance of the reference's host back end
    applied on the GPU, one random stream per hit.  Returns the accepted hits (ACC_DTYPE)
    in input order; `hit` indexes the input."""
    hits = np.ascontiguousarray(hits, T.HIT_DTYPE)
    out = np.empty(max(1, len(hits)), T.ACC_DTYPE)
    n = C.c_uint64()
    check(lib().ppcb_accept(self._c, _p(hits), len(hits), int(seed) & 0xFFFFFFFF, _p(out), len(out), C.byref(n)))
    return out[:n.value]


PPC.accept = _accept


def _accept_device(self, hits_ptr, n, seed, out_ptr, count_ptr, stream=0, device=0):
    """ppcb_accept_device over caller-owned device memory (raw pointers), asynchronous."""
    check(lib().ppcb_accept_device(self._c, int(device), C.c_void_p(hits_ptr), int(n), int(seed) & 0xFFFFFFFF,
                                   C.c_void_p(out_ptr), C.c_void_p(count_ptr), C.c_void_p(stream) if stream else None))


PPC.accept_device = _accept_device


def _sources(self, src, seed=0, cap=None):
    """Device front end (ppcb_sources): sources (SOURCE_DTYPE) to photon bunches, Poisson
    counts drawn on the GPU.  Returns (bunches, bstart, photons); bstart[k] is the first
    photon of bunch k, bstart[-1] the total, ready for propagate_device."""
    src = np.ascontiguousarray(src, T.SOURCE_DTYPE)
    cap = len(src) + 8 if cap is None else int(cap)
    while True:
        out = np.zeros(max(1, cap), T.BUNCH_DTYPE)
        bstart = np.zeros(cap + 1, np.uint64)
        nb, num = C.c_uint64(), C.c_uint64()
        check(lib().ppcb_sources(self._c, _p(src) if len(src) else None, len(src), int(seed) & 0xFFFFFFFF, _p(out),
                                 _p(bstart), cap, C.byref(nb), C.byref(num)))
        if nb.value <= cap:
            return out[:nb.value], bstart[:nb.value + 1], num.value
        cap = nb.value


PPC.sources = _sources


def _sources_device(self, src_ptr, ns, seed, out_ptr, bstart_ptr, cap, counts_ptr, stream=0, device=0):
    """ppcb_sources_device over caller-owned device memory (raw pointers), asynchronous."""
    check(lib().ppcb_sources_device(self._c, int(device), C.c_void_p(src_ptr), int(ns), int(seed) & 0xFFFFFFFF,
                                    C.c_void_p(out_ptr), C.c_void_p(bstart_ptr), int(cap), C.c_void_p(counts_ptr),
                                    C.c_void_p(stream) if stream else None))


PPC.sources_device = _sources_device


def f2k_sources(text, first_segment=1):
    """f2k text (TR records, one segment per line) to SOURCE_DTYPE records for the device
    front end; returns (sources, lines read)."""
    b = text.encode() if isinstance(text, str) else bytes(text)
    n, lines = C.c_uint64(), C.c_uint64()
    check(lib().ppcb_f2k_sources(b, len(b), int(first_segment), None, 0, C.byref(n), C.byref(lines)))
    out = np.zeros(max(1, n.value), T.SOURCE_DTYPE)
    check(lib().ppcb_f2k_sources(b, len(b), int(first_segment), _p(out), len(out), C.byref(n), C.byref(lines)))
    return out[:n.value], lines.value


class GradGraph:
    """The recording forward pass, charge histogram, Poisson weights and log-likelihood and
    the replay of the detected photons, captured once as a CUDA graph and replayed per call
    with new ice coefficients (ppcb_gradgraph_*).  Use PPC.gradient_graph to make one."""

    def __init__(self, ctx, bunches, observed, events=0, scale=1.0, hit_cap=None):
        self._ctx = ctx
        self._b = np.ascontiguousarray(bunches, T.BUNCH_DTYPE)
        info = ctx.info()
        self.gsize, self.size, self.events = info["gsize"], info["size"], int(events)
        self.nbins = self.gsize * (self.events if self.events else 1)
        obs = np.ascontiguousarray(observed, np.float32).reshape(-1)
        if obs.size != self.nbins:
            raise ValueError(f"observed: {obs.size} values for {self.nbins} charge bins")
        if hit_cap is None:
            hit_cap = int(self._b["num"].sum() * 0.02) + (1 << 16)
        self._h = C.c_void_p()
        check(lib().ppcb_gradgraph_create(ctx._c, _p(self._b), len(self._b), self.events, _p(obs), float(scale),
                                          int(hit_cap), C.byref(self._h)))
        ctx._children.add(self)

    def run(self, be=None, ba=None, counts=True):
        from ._lib import GradInfo
        b = None if be is None else np.ascontiguousarray(be, np.float32)
        a = None if ba is None else np.ascontiguousarray(ba, np.float32)
        cnt = np.zeros(self.nbins, np.uint32) if counts else None
        g_be = np.zeros(self.size, np.float64)
        g_ba = np.zeros(self.size, np.float64)
        gi = GradInfo()
        check(lib().ppcb_gradgraph_run(self._h, _p(b), _p(a), _p(cnt), _p(g_be), _p(g_ba), C.byref(gi)))
        if cnt is not None and self.events:
            cnt = cnt.reshape(self.events, self.gsize)
        return {"ll": gi.ll, "counts": cnt, "g_be": g_be, "g_ba": g_ba,
                "info": {k: getattr(gi, k) for k, _ in GradInfo._fields_}}

    def close(self):
        if self._h:
            lib().ppcb_gradgraph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def good_list_bad(data, good):
    """The DOMs that a good-DOM list turns bad: those with observed pulses that are not on
    the list (llh/llh.cxx:774-781 inserts each such DOM into the bad set when it reads its
    pulses), as (str, om) rows."""
    g = {(int(s), int(o)) for s, o in np.asarray(good, np.int32).reshape(-1, 2)}
    d = np.ascontiguousarray(data, T.LLH_HIT_DTYPE)
    keys = sorted({(int(s), int(o)) for s, o in zip(d["str"], d["om"])} - g)
    return np.array(keys, np.int32).reshape(-1, 2)


class Likelihood:
    """DirectFit's likelihood (llh/llh.cxx:419-662, 1075-1082) with the simulation side on
    the GPU (ppcb_llh_*).  `data`: observed pulses (LLH_HIT_DTYPE: str, om, t, q), prepared
    once on the host: binned per DOM, DOMs selected, each DOM's bins merged into blocks.
    `eval(hits, dts, nsim, seed)` takes kernel-level hits, applies the back end's
    acceptance (as PPC.accept with the same seed) and returns fllh(dt, nsim) for every
    shift dt.  Options (DirectFit's names and defaults): lbin (0: automatic), sig (0.10),
    qmin (0.1), qsat (500), drep (1), peak, mono, norm, unh (0), flasher, fla_str,
    fla_om (0), fsep (1).  `good`: the good-DOM list (DirectFit's `set` file,
    llh/llh.cxx:741-744): when given, pulses on other DOMs are dropped and those DOMs are
    treated as bad, as the reference does while reading the pulses (llh/llh.cxx:774-781)."""

    def __init__(self, ctx, data, windows=None, bad=None, device=0, good=None, **opts):
        from ._lib import LlhOpts
        o = LlhOpts()
        check(lib().ppcb_llh_default_opts(C.byref(o)))
        for k, v in opts.items():
            if k not in dict(LlhOpts._fields_):
                raise TypeError(f"unknown likelihood option {k!r}")
            setattr(o, k, v)
        data = np.ascontiguousarray(data, T.LLH_HIT_DTYPE)
        win = np.ascontiguousarray(windows if windows is not None else np.zeros(0, T.LLH_WINDOW_DTYPE),
                                   T.LLH_WINDOW_DTYPE)
        badk = np.ascontiguousarray(bad if bad is not None else np.zeros((0, 2)), np.int32).reshape(-1, 2)
        if good is not None and len(good):
            badk = np.concatenate([badk, good_list_bad(data, good)])
        self._ctx = ctx  # keeps the context alive
        self._h = C.c_void_p()
        check(lib().ppcb_llh_create(ctx._c, int(device), _p(data), len(data), _p(win) if len(win) else None,
                                    len(win), _p(badk) if len(badk) else None, len(badk), C.byref(o),
                                    C.byref(self._h)))
        self.opts = {k: getattr(o, k) for k, _ in LlhOpts._fields_}
        ctx._children.add(self)

    def info(self):
        from ._lib import LlhInfo
        i = LlhInfo()
        check(lib().ppcb_llh_get_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in LlhInfo._fields_}

    def blocks(self):
        n = C.c_uint64()
        check(lib().ppcb_llh_blocks(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(1, n.value), T.LLH_BLOCK_DTYPE)
        check(lib().ppcb_llh_blocks(self._h, _p(out), len(out), C.byref(n)))
        return out[:n.value]

    def eval(self, hits, dts=(0.0,), nsim=1.0, seed=0):
        hits = np.ascontiguousarray(hits, T.HIT_DTYPE)
        dts = np.ascontiguousarray(np.atleast_1d(dts), np.float64)
        out = np.zeros(len(dts), np.float64)
        check(lib().ppcb_llh_eval(self._h, _p(hits) if len(hits) else None, len(hits), int(seed) & 0xFFFFFFFF,
                                  _p(dts), len(dts), float(nsim), _p(out)))
        return out

    def eval_device(self, hits_ptr, n, dts, nsim, out_ptr, seed=0, stream=0):
        """Asynchronous evaluation over device memory (raw pointers: n kernel-level hits,
        len(dts) doubles out)."""
        dts = np.ascontiguousarray(np.atleast_1d(dts), np.float64)
        check(lib().ppcb_llh_eval_device(self._h, C.c_void_p(hits_ptr), int(n), int(seed) & 0xFFFFFFFF, _p(dts),
                                         len(dts), float(nsim), C.c_void_p(out_ptr),
                                         C.c_void_p(stream) if stream else None))

    def close(self):
        if self._h:
            lib().ppcb_llh_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
