#!/usr/bin/env python
"""Benchmark: photon propagation throughput (photons/s) on B200.

Workload (one step, per GPU): the full-detector cascade -- 5160 DOMs on 86 strings,
171 ice layers with a +-20 m 1-d tilt, absorption anisotropy and birefringence -- with
1e8 propagated photons from one EM cascade (gamma longitudinal profile) at a vertex
uniform in |x|,|y|,|z| <= 500 m and a direction uniform on the sphere, seeded per step
and rank.  Synthetic data (ppc_b200/synth.py, configuration `full`).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:       `value` = photons / device time of the propagation launches, bunches already
            in HBM (ppcb_propagate_device); `e2e` = the same workload through ppcb_propagate
            with host buffers (bunch upload, launch, hit download inside the timed region).
reference:  the reference's own CPU build (gpu/ppc.cu compiled as gpu/Makefile:10 does,
            oracle/_ref) on every host core, same workload, bounded sample per step.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
os.environ.setdefault("PPCB_QUIET", "1")

PHOTONS = 100_000_000
FCV = math.pi / 180


def _cascade_bunch(rng, photons, q=1, ppm=2450.08, fixed=None):
    """EM cascade bunch with the reference's longitudinal parameters (gpu/f2k.cxx:68-79):
    random vertex and direction, or `fixed` = (x, y, z, nx, ny, nz)."""
    from ppc_b200 import types as T
    # energy whose mean yield at xR=5 is `photons` propagated photons (gpu/f2k.cxx:68-71,
    # :502): photons = ppm * 5.321*0.910/0.9216 * E / 25
    E = photons * 25.0 / (ppm * 5.321 * 0.910 / 0.9216)
    logE = math.log(max(0.105658389, E))
    a = 2.01849 + 0.63176 * logE
    b = 0.39652 * 0.910 / 0.9216 / 0.63207
    v = rng.uniform(-500, 500, 3)
    ct = rng.uniform(-1, 1)
    ph = rng.uniform(0, 2 * math.pi)
    st = math.sqrt(1 - ct * ct)
    d = [st * math.cos(ph), st * math.sin(ph), ct]
    if fixed is not None:
        v, d = list(fixed[:3]), list(fixed[3:6])
    bunch = T.bunch_particle([v[0], v[1], v[2], 0.0], d, q, photons, -11, f=0.0, a=a, b=b)
    return bunch, E, v, d


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                x = [s.strip() for s in line.split(",")]
                if len(x) >= 9:
                    rows.append(x)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def cpu_reference_sample(photons_per_proc, procs, seed=0):
    """The reference CPU build (oracle/_ref/ref_harness_fm: gpu/ppc.cu + gpu/pro.cu compiled with
    the reference's flags) propagating cascade photons in `procs` concurrent processes."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness_fm")
    if not os.path.exists(exe):
        return None
    from ppc_b200 import synth
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    if not os.path.exists(os.path.join(ice, "cfg.txt")):
        synth.write("full", ice)
    rng = np.random.default_rng(seed)
    ps = []
    env = dict(os.environ, PPCTABLESDIR=ice, PPCB_QUIET="1")
    for k in range(procs):
        E = PHOTONS * 25.0 / (2450.08 * 5.321 * 0.910 / 0.9216)
        v = rng.uniform(-500, 500, 3)
        ct = rng.uniform(-1, 1)
        ph = rng.uniform(0, 2 * math.pi)
        st = math.sqrt(1 - ct * ct)
        spec = f"cascade:{v[0]}:{v[1]}:{v[2]}:{E}:{st * math.cos(ph)}:{st * math.sin(ph)}:{ct}:11"
        ps.append(subprocess.Popen([exe, "run", spec, str(photons_per_proc), str(seed * 1000 + k), "/tmp/ppcb_ref",
                                    "nodump"], env=env, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
    rate, photons, secs = 0.0, 0, 0.0
    for p in ps:
        out, _ = p.communicate()
        line = [l for l in out.splitlines() if l.startswith("{")][-1]
        r = json.loads(line)
        rate += r["photons"] / r["seconds"]
        photons += r["photons"]
        secs = max(secs, r["seconds"])
    return {"value": rate, "photons": photons, "seconds": secs}


def cpu_par_sample(photons, seed=0, cascades=None):
    """The reference's std::par build (oracle/_ref/ppc_par: par/ppc.cxx in CPU mode, OpenMP on
    every host core) on cascades of the same workload (one per core by default, random
    vertices and directions, `photons` in all), read as f2k records: photons/s over the run's
    wall time less an empty run's (configuration loading)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ppc_par")
    if not os.path.exists(exe):
        return None
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    rng = np.random.default_rng(seed)
    n = cascades or (os.cpu_count() or 1)
    E = photons / n * 25.0 / (2450.08 * 5.321 * 0.910 / 0.9216)
    text = ""
    for _ in range(n):
        v = rng.uniform(-500, 500, 3)
        th, ph = rng.uniform(0, 180), rng.uniform(0, 360)
        text += f"TR 1 0 e {v[0]:.2f} {v[1]:.2f} {v[2]:.2f} {th:.3f} {ph:.3f} 0 {E:.3f} 0\n"
    env = dict(os.environ, PPCTABLESDIR=ice + "/", OMP_NUM_THREADS=str(os.cpu_count() or 1))

    def run(text):
        t0 = time.perf_counter()
        r = subprocess.run([exe, "0"], input=text, env=env, capture_output=True, text=True, timeout=600)
        return time.perf_counter() - t0, r

    t_empty, _ = run("")
    t, r = run(text)
    if r.returncode != 0:
        return None
    n = sum(int(l.split()[1]) for l in r.stderr.splitlines() if l.startswith("photons:"))
    return {"value": n / max(1e-9, t - t_empty), "photons": n, "seconds": t - t_empty}


def _ref_harness_json(args, ice, exe="ref_harness_fm"):
    """One run of the reference harness (CPU build of the reference's own sources); its JSON
    line, or None when the harness is not built."""
    path = os.path.join(ROOT, "oracle", "_ref", exe)
    if not os.path.exists(path):
        return None
    env = dict(os.environ, PPCTABLESDIR=ice + "/")
    r = subprocess.run([path] + args, env=env, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        return None
    return json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])


def _event_ms(fn, stream, reps, flush=None):
    """Mean device time of fn() over reps calls, CUDA events on `stream`, L2 flushed before
    each call when `flush` (a buffer larger than L2) is given."""
    import torch
    total = 0.0
    for _ in range(reps):
        if flush is not None:
            flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total / reps


def stages_sample(local, photons=100_000_000, sources=1_000_000, shifts=64, reps=5):
    """The stages either side of the kernel, each on the GPU against the reference's (or the
    oracle's) CPU code for the same work:
      back end   ppcb_accept_device over the kernel-level hits of a 1e8-photon cascade on the
                 2-d tilt detector with cables; CPU: the reference's own print() (one core)
      likelihood ppcb_llh_eval_device, DirectFit's likelihood of those hits against the pulses
                 of a 1e7-photon run of the same cascade, 64 time shifts per evaluation; CPU:
                 the oracle's restatement (pinned bit for bit to the reference's llh.cxx,
                 which runs here only against a GSL stand-in), one core
      front end  ppcb_sources_device over 1e6 mixed sources (muon segments, EM and hadronic
                 cascades, 0.1-10 GeV); CPU: the reference's own addp() (one core)"""
    import torch
    from ppc_b200 import synth
    from ppc_b200 import types as T
    from ppc_b200.api import PPC, Likelihood

    import tempfile
    out = {}
    tmp = tempfile.mkdtemp(prefix="ppcb_stages_")
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full2d")
    if not os.path.exists(os.path.join(ice, "cfg.txt")):
        synth.write("full2d", ice)
    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(4242)
    c.choose(local)
    c.ini()
    ppm = c.tables()["eff"][0]
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    hbm = _peaks().get("hbm_gbs")
    rng = np.random.default_rng(99)
    b = _cascade_bunch(rng, photons, q=1, ppm=ppm, fixed=[0.0, 0.0, 0.0, 0.3, 0.4, 0.8660254])[0]

    def propagate(num, cap):
        bb = b.copy()
        bb["num"] = num
        d_b = torch.from_numpy(bb.view(np.uint8).reshape(-1).copy()).cuda()
        d_s = torch.tensor([0, num], dtype=torch.int64, device="cuda")
        d_h = torch.empty((cap, 32), dtype=torch.uint8, device="cuda")
        d_c = torch.zeros(56, dtype=torch.uint8, device="cuda")
        c.propagate_device(d_b.data_ptr(), d_s.data_ptr(), 1, num, d_h.data_ptr(), cap, d_c.data_ptr(),
                           stream.cuda_stream, 0)
        torch.cuda.synchronize()
        ctrl = T.Ctrl.from_buffer_copy(d_c.cpu().numpy().tobytes())
        return d_h, min(int(ctrl.hidx), cap)

    d_hits, nh = propagate(photons, 1 << 23)
    raw = d_hits[:nh].cpu().numpy().view(T.HIT_DTYPE).reshape(-1)

    # ---- back end
    d_acc = torch.empty((max(1, nh), 56), dtype=torch.uint8, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    run = lambda: c.accept_device(d_hits.data_ptr(), nh, 7, d_acc.data_ptr(), d_cnt.data_ptr(), stream.cuda_stream,
                                  0)
    run()
    torch.cuda.synchronize()
    ms = _event_ms(run, stream, reps, flush)
    acc = int(d_cnt.item())
    algo = 32 * nh + 56 * acc
    be = {"hits": nh, "accepted": acc, "device_ms": ms, "hits_per_s": nh / (ms / 1e3), "gpu_launches": 3,
          "roofline": {"bound": "hbm", "achieved": algo / (ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                       "frac": (algo / (ms / 1e3) / 1e9) / hbm if hbm else None,
                       "bytes": "32 B read per hit + 56 B written per accepted hit",
                       "peak_source": "of measured (MEASURED_PEAKS.json)"}}
    sample = raw[:100_000]
    sample = sample[np.lexsort((sample["z"], sample["t"], sample["i"], sample["n"]))]
    path = os.path.join(tmp, "hits.bin")
    sample.tofile(path)
    r = _ref_harness_json(["backend", path, "77", os.path.join(tmp, "hitz.bin")], ice)
    if r:
        be["cpu"] = {"hits_per_s": r["hits"] / r["seconds"], "cores": 1, "kind": "reference",
                     "sample": f"{r['hits']} of the same hits through the reference's print() "
                               "(oracle/_ref/ref_harness_fm backend)"}
        be["speedup_vs_cpu"] = be["hits_per_s"] / be["cpu"]["hits_per_s"]
    out["back_end"] = be

    # ---- likelihood
    d_small, ns = propagate(photons // 10, 1 << 22)
    obs = c.accept(d_small[:ns].cpu().numpy().view(T.HIT_DTYPE).reshape(-1), seed=3)
    data = np.zeros(len(obs), T.LLH_HIT_DTYPE)
    data["str"], data["om"], data["t"], data["q"] = obs["str"], obs["om"], obs["t"], 1.0
    L = Likelihood(c, data)
    dts = np.linspace(-200.0, 200.0, shifts)
    d_out = torch.empty(shifts, dtype=torch.float64, device="cuda")
    run = lambda: L.eval_device(d_hits.data_ptr(), nh, dts, 10.0, d_out.data_ptr(), seed=5, stream=stream.cuda_stream)
    run()
    torch.cuda.synchronize()
    ms = _event_ms(run, stream, reps, flush)
    lk = {"hits": nh, "shifts": shifts, "doms": L.info()["doms"], "blocks": L.info()["blocks"], "device_ms": ms,
          "evals_per_s": shifts / (ms / 1e3), "hit_shifts_per_s": nh * shifts / (ms / 1e3), "gpu_launches": 3}
    try:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_util as O  # CPU baseline leg: the oracle restatement of llh.cxx
        sim = c.accept(raw, seed=5)
        t0 = time.perf_counter()
        O.llh_fllh(data, sim, dts[:8], 10.0)
        secs = time.perf_counter() - t0
        lk["cpu"] = {"evals_per_s": 8 / secs, "cores": 1, "kind": "port",
                     "sample": "8 shifts of the same evaluation through oracle/llh_oracle.c (equal bit for "
                               "bit to DirectFit's llh.cxx on its golden vectors), accepted hits given"}
        lk["speedup_vs_cpu"] = lk["evals_per_s"] / lk["cpu"]["evals_per_s"]
    except Exception as e:  # the oracle library is a build product of oracle/Makefile
        lk["cpu"] = {"unavailable": str(e)[:120]}
    L.close()
    out["likelihood"] = lk

    # ---- front end
    kinds = np.array([0, 11, 12, 13, 14, 101, 102, 105])
    src = np.zeros(sources, T.SOURCE_DTYPE)
    src["kind"] = T.SRC_PARTICLE
    src["r"][:, :3] = rng.uniform(-400, 400, (sources, 3))
    src["n"] = [0.3, 0.4, 0.8660254]
    src["amount"] = 10 ** rng.uniform(-1, 1, sources)
    src["type"] = rng.choice(kinds, sources)
    src["dr"] = np.where(src["type"] == 0, rng.uniform(1, 20, sources), 0)
    src["scale"] = 1
    src["q"] = 1
    d_src = torch.from_numpy(src.view(np.uint8).reshape(-1).copy()).cuda()
    cap = sources + 1024
    d_bun = torch.empty((cap, 64), dtype=torch.uint8, device="cuda")
    d_bs = torch.empty(cap + 1, dtype=torch.int64, device="cuda")
    d_fc = torch.zeros(2, dtype=torch.int64, device="cuda")
    run = lambda: c.sources_device(d_src.data_ptr(), sources, 11, d_bun.data_ptr(), d_bs.data_ptr(), cap,
                                   d_fc.data_ptr(), stream.cuda_stream, 0)
    run()
    torch.cuda.synchronize()
    ms = _event_ms(run, stream, reps, flush)
    nb, nph = (int(x) for x in d_fc.cpu().numpy())
    algo = 72 * sources + 72 * nb
    fe = {"sources": sources, "bunches": nb, "photons": nph, "device_ms": ms, "sources_per_s": sources / (ms / 1e3),
          "gpu_launches": 3,
          "roofline": {"bound": "hbm", "achieved": algo / (ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                       "frac": (algo / (ms / 1e3) / 1e9) / hbm if hbm else None,
                       "bytes": "72 B read per source + 64 B bunch and 8 B start written per bunch",
                       "peak_source": "of measured (MEASURED_PEAKS.json)"}}
    fsrc = np.zeros(sources, [("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("t", "<f4"), ("E", "<f4"), ("dr", "<f4"),
                              ("type", "<i4")])
    fsrc["x"], fsrc["y"], fsrc["z"] = src["r"][:, 0], src["r"][:, 1], src["r"][:, 2]
    fsrc["E"], fsrc["dr"], fsrc["type"] = src["amount"], src["dr"], src["type"]
    fsrc.tofile(os.path.join(tmp, "sources.bin"))
    r = _ref_harness_json(["frontend", os.path.join(tmp, "sources.bin"), "5"], ice)
    if r:
        fe["cpu"] = {"sources_per_s": r["sources"] / r["seconds"], "cores": 1, "kind": "reference",
                     "sample": f"the same {r['sources']} sources through the reference's addp() "
                               "(oracle/_ref/ref_harness_fm frontend)"}
        fe["speedup_vs_cpu"] = fe["sources_per_s"] / fe["cpu"]["sources_per_s"]
    out["front_end"] = fe
    c.close()
    import shutil
    shutil.rmtree(tmp, ignore_errors=True)
    return out


def plain_kernel_sample(cascades, photons, local):
    """The reference's own CUDA kernel (gpu/pro.cu built for sm_100a with gpu/Makefile's
    flags, oracle/_ref/ref_gpu_harness) on the same cascades as the timed steps (vertex,
    direction, energy), one eout() per cascade; device time from the reference's own CUDA
    events (gpu/ppc.cu:296-304)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_harness")
    if not os.path.exists(exe) or not cascades:
        return None
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    path = os.path.join(tempfile.mkdtemp(), "cascades.txt")
    with open(path, "w") as f:
        for v, d, E in cascades:
            f.write("C %.9g %.9g %.9g %.9g %.9g %.9g %.9g %d\n" % (v[0], v[1], v[2], E, d[0], d[1], d[2], photons))
    env = dict(os.environ, PPCTABLESDIR=ice, CUDA_VISIBLE_DEVICES=str(local))
    r = subprocess.run([exe, "file:" + path, "0", "0", "1"], env=env, capture_output=True, text=True, timeout=600)
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not lines:
        return None
    x = json.loads(lines[-1])
    x["value"] = x["photons"] / (x["device_ms"] / 1000.0)
    return x


def gradient_sample(local, events=64, photons=10_000_000, steps=3, plain_kernel=True):
    """Ice gradient over the 342 per-layer coefficients: 64 flasher events of 1e7 photons
    (12-fold LEDs at 30 degrees on distinct random DOMs), Poisson log-likelihood of the
    per-(event, DOM) charges against charges drawn from a hidden ice (each layer's be and ba
    scaled by U(0.9, 1.1)).  One evaluation = recording forward + replay, through
    PPC.gradient with host buffers.  The comparison is a central finite-difference gradient,
    2 x 342 forward runs, with the reference's CUDA kernel (one eout() per event)."""
    from ppc_b200 import workloads as W
    from ppc_b200.api import PPC

    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(4242)
    c.choose(local)
    c.ini()
    oms = c.tables()["oms"]
    rng = np.random.default_rng(64)
    doms = rng.choice(len(oms), events, replace=False)
    b = np.concatenate([W.flasher(int(k), oms["r"][k], photons, q=i) for i, k in enumerate(doms)])
    be0, ba0 = c.get_ice()
    n = len(be0)
    c.set_ice((be0 * rng.uniform(0.9, 1.1, n)).astype(np.float32), (ba0 * rng.uniform(0.9, 1.1, n)).astype(np.float32))
    gs = c.info()["gsize"]
    mu = c.gradient(b, weights=np.zeros(events * gs, np.float32), events=events)["counts"]
    obs = rng.poisson(mu).astype(np.float32)
    c.set_ice(be0, ba0)
    c.gradient(b, observed=obs, events=events)  # warm-up
    wall, fwd, bwd, hits = [], [], [], 0
    for _ in range(steps):
        t0 = time.perf_counter()
        r = c.gradient(b, observed=obs, events=events)
        wall.append(time.perf_counter() - t0)
        fwd.append(r["info"]["forward_ms"])
        bwd.append(r["info"]["backward_ms"])
        hits = r["info"]["hits"]
        unmatched = r["info"]["unmatched"]
    c.close()
    out = {
        "evals_per_s": steps / sum(wall), "unit": "gradient evals/s (342 parameters)",
        "workload": f"{events} flasher events x {photons:.0e} photons, 12-fold LEDs at 30 deg, per-(event, DOM) "
                    "Poisson log-likelihood, hidden ice +-10% per layer",
        "forward_ms": statistics.median(fwd), "backward_ms": statistics.median(bwd),
        "backward_over_forward": statistics.median(bwd) / statistics.median(fwd),
        "wall_s": statistics.median(wall), "hits": hits, "unmatched_replays": unmatched,
    }
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_harness")
    if plain_kernel and os.path.exists(exe):
        path = os.path.join(tempfile.mkdtemp(), "flashers.txt")
        with open(path, "w") as f:
            for k in doms:
                f.write(f"F {int(k) // 60 + 1} {int(k) % 60 + 1} {photons}\n")
        env = dict(os.environ, PPCTABLESDIR=ice, CUDA_VISIBLE_DEVICES=str(local), FLDR="3960", ELEV="30")
        p = subprocess.run([exe, "file:" + path, "0", "0", "1"], env=env, capture_output=True, text=True, timeout=900)
        lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
        if p.returncode == 0 and lines:
            x = json.loads(lines[-1])
            fd_s = 2 * 2 * n * x["wall_s"]
            out["fd_plain_kernel"] = {"forward_wall_s": x["wall_s"], "forward_device_ms": x["device_ms"],
                                      "fd_gradient_s": fd_s, "evals_per_s": 1.0 / fd_s,
                                      "kind": "central differences, 2 x 342 forward runs of the reference CUDA "
                                              "kernel (gpu/pro.cu, sm_100a), one eout() per event"}
            out["speedup_vs_fd_plain_kernel"] = out["evals_per_s"] * fd_s
    # the same 64 flasher events through the drop-in API (llh/ppc.h semantics: flset, sett,
    # flone, eout with the host back end, hitz, efin), wall time, against the reference's
    # own host code doing the same (the plain-kernel forward above)
    old = {k: os.environ.get(k) for k in ("FLDR", "ELEV")}
    os.environ.update(FLDR="3960", ELEV="30")
    try:
        c = PPC()
        c.initialize(1.0, ice)
        c.set_seed(4243)
        c.choose(local)
        c.ini()
        inf = c.info()
        # flone(n) propagates n x (ppm / 2450.08) / xR^2 photons (gpu/f2k.cxx:586-588)
        nsrc = int(round(photons * inf["ovr"] * 2450.08 / inf["eff"]))
        kept = 0
        for rep in range(2):  # the first pass warms up
            p0 = c.last_run()[1]["photons"]
            t0 = time.perf_counter()
            for e, k in enumerate(doms):
                c.flset(int(k) // 60 + 1, int(k) % 60 + 1)
                c.sett(0.0, 0.0, 1.0, (e, 0), 0)
                c.flone(nsrc)
                c.eout()
                kept += len(c.hitz())
                c.efin()
            wall = time.perf_counter() - t0
            propagated = c.last_run()[1]["photons"] - p0
        c.close()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    x = {"events": events, "photons": propagated, "wall_s": wall, "photons_per_s": propagated / wall,
         "hitz_records": kept // 2,
         "kind": "flset/sett/flone/eout/hitz/efin per event, the reference's host back end included"}
    if "fd_plain_kernel" in out:
        rw = out["fd_plain_kernel"]["forward_wall_s"]
        x["reference_photons_per_s"] = events * photons / rw
        x["reference_wall_s"] = rw
        x["speedup"] = x["photons_per_s"] / x["reference_photons_per_s"]
    out["xppc_e2e"] = x
    return out


def fit_sample(local, iters=10, scale=1.0, plain_kernel=True):
    """Ice fit: 1024 flashers (log-uniform 1e5-1e7 photons, 12-fold LEDs at 30 degrees on
    distinct random DOMs) and 256 EM cascades (log-uniform 1e6-1e8 photons, vertex in
    |x|,|y|,|z| <= 500 m, isotropic directions); charges simulated with a hidden ice (be and
    ba scaled by exp(0.1 x a smooth depth profile)) and other random numbers; L-BFGS over
    the 342 coefficients on the adjoint gradient with a smoothness penalty.  Compared with an iteration that takes its
    gradient from central differences of the reference's CUDA kernel (2 x 342 forward runs)."""
    import torch
    from ppc_b200 import synth
    from ppc_b200 import workloads as W
    from ppc_b200.api import PPC
    from ppc_b200.fit import fit_ice

    torch.cuda.set_device(local)
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    if not os.path.exists(os.path.join(ice, "cfg.txt")):
        synth.write("full", ice)
    rng = np.random.default_rng(55)
    s = scale

    def ctx(seed):
        c = PPC()
        c.initialize(1.0, ice)
        c.set_seed(seed)
        c.set_options(photon_streams=True)
        c.choose(local)
        c.ini()
        return c

    truth = ctx(901)
    oms = truth.tables()["oms"]
    be0, ba0 = truth.get_ice()
    n = len(be0)
    nf, nc = 1024, 256
    doms = rng.choice(len(oms), nf, replace=False)
    nfl = np.exp(rng.uniform(np.log(1e5), np.log(1e7), nf)) * s
    ncs = np.exp(rng.uniform(np.log(1e6), np.log(1e8), nc)) * s
    parts = [W.flasher(int(k), oms["r"][k], int(nfl[i]), q=i) for i, k in enumerate(doms)]
    cas = []
    for j in range(nc):
        v = rng.uniform(-500, 500, 3)
        ct = rng.uniform(-1, 1)
        ph = rng.uniform(0, 2 * math.pi)
        st = math.sqrt(1 - ct * ct)
        d = [st * math.cos(ph), st * math.sin(ph), ct]
        parts.append(W.cascade(v, d, int(ncs[j]), q=nf + j))
        cas.append((v, d, int(ncs[j])))
    b = np.concatenate(parts)
    events = nf + nc
    photons = int(b["num"].sum())
    hit_cap = int(photons * 0.004) + (1 << 20)
    def field():  # smooth unit-variance depth profile (Gaussian kernel, 4 layers)
        x = rng.normal(size=n + 20)
        k = np.exp(-0.5 * (np.arange(-10, 11) / 4.0) ** 2)
        f = np.convolve(x, k / k.sum(), mode="same")[10:10 + n]
        return f / f.std()

    be_t = (be0 * np.exp(0.1 * field())).astype(np.float32)
    ba_t = (ba0 * np.exp(0.1 * field())).astype(np.float32)
    truth.set_ice(be_t, ba_t)
    gs = truth.info()["gsize"]
    obs = truth.gradient(b, weights=np.zeros(events * gs, np.float32), events=events,
                         hit_cap=hit_cap)["counts"].astype(np.float32)
    truth.close()
    c = ctx(17)
    g0 = c.gradient(b, observed=obs, events=events, hit_cap=hit_cap)
    lit_be = np.abs(g0["g_be"] * be0) > 0.05 * np.abs(g0["g_be"] * be0).max()
    lit_ba = np.abs(g0["g_ba"] * ba0) > 0.05 * np.abs(g0["g_ba"] * ba0).max()
    clk = Clocks(local)
    smooth = 3e-3 * float(obs.sum())  # penalty on layer-to-layer differences, scaled with the data
    r = fit_ice(c, b, obs, events, iters=iters, hit_cap=hit_cap, smooth=smooth)
    clocks = clk.stop()
    # one evaluation at the fitted ice through the graph and through the eager path
    G = c.gradient_graph(b, obs, events=events, hit_cap=hit_cap)
    t0 = time.perf_counter()
    G.run(r["be"].astype(np.float32), r["ba"].astype(np.float32), counts=False)
    eval_graph = time.perf_counter() - t0
    G.close()
    t0 = time.perf_counter()
    c.gradient(b, observed=obs, events=events, hit_cap=hit_cap)
    eval_eager = time.perf_counter() - t0
    c.close()

    def rms(x, t, m):
        return float(np.sqrt(np.mean((x[m] / t[m] - 1) ** 2)))

    line = {
        "metric": "ice-fit seconds per L-BFGS iteration", "value": r["seconds_per_iteration"],
        "unit": "s/iteration", "n_gpus": 1, "steps": r["iterations"], "warmup": 1,
        "ms_per_step": 1000 * r["seconds_per_iteration"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP64 gradient sums)", "data": "synthetic",
        "config": {"workload": f"{nf} flashers (1e5-1e7 photons) + {nc} cascades (1e6-1e8), full detector, "
                               "per-(event, DOM) Poisson LL, hidden ice = start x exp(0.1 x smooth unit field) "
                               "in be and ba, 342 parameters, smoothness penalty 3e-3 x total charge",
                   "photons_per_evaluation": photons, "photon_scale": s, "observed_charge": float(obs.sum())},
        "evaluations": r["evaluations"], "ll_first": r["history"][0]["ll"], "ll_final": r["ll"],
        "forward_ms_median": statistics.median(h["forward_ms"] for h in r["history"]),
        "backward_ms_median": statistics.median(h["backward_ms"] for h in r["history"]),
        "recovery": {"lit_layers_be": int(lit_be.sum()), "lit_layers_ba": int(lit_ba.sum()),
                     "rms_rel_error_be": [rms(be0, be_t, lit_be), rms(r["be"], be_t, lit_be)],
                     "rms_rel_error_ba": [rms(ba0, ba_t, lit_ba), rms(r["ba"], ba_t, lit_ba)]},
        "gpu_launches": 5 * r["evaluations"], "clocks": clocks, "accepted_steps": r["accepted"],
        "evaluation_s": {"graph": eval_graph, "eager": eval_eager,
                         "kind": "one likelihood-and-gradient evaluation at the fitted ice: the CUDA graph "
                                 "(forward, histogram, weights, replay) against the eager calls"},
    }
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_harness")
    if plain_kernel and os.path.exists(exe):
        path = os.path.join(tempfile.mkdtemp(), "fit_events.txt")
        with open(path, "w") as f:
            for i, k in enumerate(doms):
                f.write(f"F {int(k) // 60 + 1} {int(k) % 60 + 1} {int(nfl[i])}\n")
            for v, d, num in cas:
                E = num * 25.0 / (2450.08 * 5.321 * 0.910 / 0.9216)
                f.write("C %f %f %f %f %f %f %f %d\n" % (v[0], v[1], v[2], E, d[0], d[1], d[2], num))
        env = dict(os.environ, PPCTABLESDIR=ice, CUDA_VISIBLE_DEVICES=str(local), FLDR="3960", ELEV="30")
        p = subprocess.run([exe, "file:" + path, "0", "0", "1"], env=env, capture_output=True, text=True,
                           timeout=1800)
        lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
        if p.returncode == 0 and lines:
            x = json.loads(lines[-1])
            fd_s = 2 * 2 * n * x["wall_s"]
            line["fd_plain_kernel"] = {"forward_wall_s": x["wall_s"], "seconds_per_iteration": fd_s,
                                       "kind": "gradient by central differences, 2 x 342 forward runs of the "
                                               "reference CUDA kernel, one eout() per event (one forward timed, "
                                               "x 684)"}
            line["speedup_vs_fd_plain_kernel"] = fd_s / r["seconds_per_iteration"]
    return line


def run_fit(args, local):
    print(json.dumps(fit_sample(local, args.fit_iters, args.fit_scale, not args.no_plain_kernel)))


def _plain_kernel_events(ev, local, timeout=1800):
    """The reference's CUDA kernel on the same events, one eout() per event (file mode of
    oracle/_ref/ref_gpu_harness): events/s over its wall time, which includes the
    reference's per-event host work."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_harness")
    if not os.path.exists(exe):
        return None
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    path = os.path.join(tempfile.mkdtemp(), "events.txt")
    with open(path, "w") as f:
        for x in ev:
            if x["type"] > 0:
                k = int(np.int16(x["u"][3] & 0xFFFF))  # flasher DOM index: string-major, 60 per string
                f.write(f"F {k // 60 + 1} {k % 60 + 1} {int(x['num'])}\n")
            else:
                E = int(x["num"]) * 25.0 / (2450.08 * 5.321 * 0.910 / 0.9216)
                f.write("C %.9g %.9g %.9g %.9g %.9g %.9g %.9g %d\n" % (x["r"][0], x["r"][1], x["r"][2], E, x["n"][0],
                                                                       x["n"][1], x["n"][2], int(x["num"])))
    env = dict(os.environ, PPCTABLESDIR=ice, CUDA_VISIBLE_DEVICES=str(local), FLDR="3960", ELEV="30")
    r = subprocess.run([exe, "file:" + path, "0", "0", "1"], env=env, capture_output=True, text=True, timeout=timeout)
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not lines:
        return None
    x = json.loads(lines[-1])
    return {"events_per_s": x["events"] / x["wall_s"], "device_ms": x["device_ms"], "wall_s": x["wall_s"],
            "photons": x["photons"], "kind": "reference CUDA kernel gpu/pro.cu, sm_100a, one eout() per event"}


def batched_sample(local, events=4096, steps=3, warmup=3, plain_kernel=True):
    """4096 events (log-uniform 1e3-1e7 photons; half flashers on random DOMs, 12-fold at
    30 degrees, half cascades) in one graph-replayed launch, against the reference's CUDA
    kernel propagating the same events one eout() at a time.  `by_decade` repeats the
    comparison on 512 events per decade of photon count."""
    import torch
    from ppc_b200 import synth
    from ppc_b200 import workloads as W
    from ppc_b200.api import PPC, Batch

    torch.cuda.set_device(local)
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    if not os.path.exists(os.path.join(ice, "cfg.txt")):
        synth.write("full", ice)
    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(2024)
    c.choose(local)
    c.ini()
    oms = c.tables()["oms"]
    ev = W.batched_events(oms, n_events=events, seed=11)
    photons = int(ev["num"].sum())
    # the per-decade comparisons below reuse the batch: size it for the largest of the runs
    dec_ev = {lo: W.batched_events(oms, n_events=512, lo=lo, hi=10 * lo, seed=int(lo)) for lo in (1e3, 1e4, 1e5, 1e6)}
    most = max([photons] + [int(e["num"].sum()) for e in dec_ev.values()])
    nmax = max(events, 512)
    b = Batch(c, max_events=nmax, max_bunches=nmax, hit_capacity=int(most * 0.02) + 66 * nmax)
    tune = b.autotune(ev, events, sample_photons=50_000_000)
    for _ in range(max(1, warmup - 2)):
        b.run(ev, events, hits_per_photon=0.02)
    runs = []
    clk = Clocks(local)
    for _ in range(steps):
        runs.append(b.run(ev, events, hits_per_photon=0.02))
    clocks = clk.stop()
    graph_s = sum(r["graph_ms"] for r in runs) / 1000.0
    line = {
        "metric": "events/s", "value": events * len(runs) / graph_s, "unit": "events/s", "n_gpus": 1,
        "steps": steps, "warmup": warmup, "ms_per_step": 1000.0 * graph_s / len(runs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{events} events, log-uniform 1e3-1e7 photons, 50% flashers (12-fold, 30 deg) "
                               f"50% EM cascades, full detector", "photons_per_step": photons,
                   "launch": f"graph replay, autotuned {tune['threads']}x{tune['blocks_per_sm']} "
                             f"refill {tune['refill_below']}"},
        "photons_per_s": photons * len(runs) / graph_s,
        "overflowed_events": max(r["overflowed"] for r in runs),
        "gpu_launches": 3 * steps,
        "clocks": clocks,
    }
    decades = []
    for lo, ed in dec_ev.items():
        b.run(ed, 512, hits_per_photon=0.02)  # capture for this size
        rr = [b.run(ed, 512, hits_per_photon=0.02) for _ in range(3)]
        t = sum(r["graph_ms"] for r in rr) / 1000.0
        decades.append({"photons_per_event": [lo, 10 * lo], "events": 512, "events_per_s": 512 * len(rr) / t,
                        "photons_per_s": float(ed["num"].sum()) * len(rr) / t, "_ev": ed})
    b.close()
    c.close()
    torch.cuda.empty_cache()
    if plain_kernel:
        pk = _plain_kernel_events(ev, local)
        if pk:
            line["plain_kernel"] = pk
            line["speedup_vs_plain_kernel"] = line["value"] / pk["events_per_s"]
        for d in decades:
            pk = _plain_kernel_events(d["_ev"], local)
            if pk:
                d["plain_kernel_events_per_s"] = pk["events_per_s"]
                d["speedup_vs_plain_kernel"] = d["events_per_s"] / pk["events_per_s"]
    for d in decades:
        del d["_ev"]
    line["by_decade"] = decades
    return line


def run_batched(args, local):
    print(json.dumps(batched_sample(local, args.events, args.steps, args.warmup, not args.no_plain_kernel)))


def run_reference(args, rank, world):
    """The reference's fastest CPU path on this host: its gpu/ CPU build (the reference's own
    --fast-math flags) in one process per core.  Its std::par build on every core measured
    slower on the same cascades (bench.py's cpu_baselines_other)."""
    if rank != 0:
        return
    procs = os.cpu_count() or 1
    per = args.ref_photons
    vals = []
    for s in range(args.warmup + args.steps):
        r = cpu_reference_sample(per, procs, seed=s)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) not built"}))
            return
        if s >= args.warmup:
            vals.append(r)
    v = statistics.median([r["value"] for r in vals])
    sample = f"{per} photons x {procs} processes of the reference's gpu/ CPU build per step"
    line = {
        "impl": "reference", "metric": "photons/s", "value": v, "unit": "photons/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.median([r["seconds"] for r in vals]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "full-detector EM cascade, 5160 DOMs, 171 layers, 1-d tilt, anisotropy, BFR",
                   "photons_per_step": per * procs, "l2": "n/a (host)"},
        "cpu_baseline": {"value": v, "unit": "photons/s", "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line))


def run_ours(args, rank, world, local):
    import torch
    from ppc_b200 import synth
    from ppc_b200 import types as T
    from ppc_b200.api import PPC

    torch.cuda.set_device(local)
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    if not os.path.exists(os.path.join(ice, "cfg.txt")):
        synth.write("full", ice)
    from ppc_b200.replicas import max_over_ranks
    dist = world > 1
    if dist:
        import torch.distributed as td

    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(1000 + rank)
    c.choose(local)
    c.ini()
    info = c.info()
    ppm = c.tables()["eff"][0]
    rng = np.random.default_rng(17 + 1000 * rank)
    photons = args.photons

    cap = 1 << 22
    d_hits = torch.empty((cap, 32), dtype=torch.uint8, device="cuda")
    d_ctrl = torch.zeros(56, dtype=torch.uint8, device="cuda")
    d_bunch = torch.empty(64, dtype=torch.uint8, device="cuda")
    d_bstart = torch.tensor([0, photons], dtype=torch.int64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    timed_cascades, timed_bunches = [], []

    def step(timed):
        b, E, v, d = _cascade_bunch(rng, photons, q=1, ppm=ppm, fixed=args.cascade)
        if timed:
            timed_cascades.append((v, d, E))
            timed_bunches.append(b)
        d_bunch.copy_(torch.from_numpy(b.view(np.uint8).reshape(-1)))
        d_ctrl.zero_()
        flush.fill_(1)  # evict L2 between timed iterations
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        c.propagate_device(d_bunch.data_ptr(), d_bstart.data_ptr(), 1, photons, d_hits.data_ptr(), cap,
                           d_ctrl.data_ptr(), stream.cuda_stream, 0)
        e1.record(stream)
        e1.synchronize()
        ctrl = T.Ctrl.from_buffer_copy(d_ctrl.cpu().numpy().tobytes())
        return e0.elapsed_time(e1), ctrl

    for _ in range(args.warmup):
        step(False)
    if dist:
        td.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local) if rank == 0 else None
    times, steps_done, hits = [], 0, 0
    for _ in range(args.steps):
        ms, ctrl = step(True)
        times.append(ms)
        steps_done += ctrl.steps
        hits += ctrl.hidx
    torch.cuda.synchronize()
    clocks = clk.stop() if clk else None
    total_ms = max_over_ranks(sum(times))  # the job is as slow as its slowest rank
    if dist:
        td.barrier()

    # end to end through the host API: bunch upload, launch, hit download; the timed
    # iterations replay the cascades of the device-timed steps
    e2e_times, e2e_hits, e2e_dev_ms, e2e_cpu = [], 0, 0.0, 0.0
    hbuf = np.zeros(cap, T.HIT_DTYPE)  # the host result buffer, allocated and touched once
    clk_e2e = Clocks(local) if (rank == 0 and not args.no_e2e) else None
    for k in range(0 if args.no_e2e else args.warmup + args.steps):
        if k < args.warmup:
            b = _cascade_bunch(rng, photons, q=1, ppm=ppm, fixed=args.cascade)[0]
        else:
            b = timed_bunches[k - args.warmup]
        if dist:
            td.barrier()
        torch.cuda.synchronize()
        t0, p0 = time.perf_counter(), time.process_time()
        h, inf = c.propagate(b, out=hbuf)
        t1, p1 = time.perf_counter(), time.process_time()
        if k >= args.warmup:
            e2e_times.append(t1 - t0)
            e2e_cpu += p1 - p0
            e2e_hits += len(h)
            e2e_dev_ms += inf["device_ms"]
    e2e_clocks = clk_e2e.stop() if clk_e2e else None
    e2e_total = max_over_ranks(sum(e2e_times) if e2e_times else float("nan"))

    if rank != 0:
        return
    value = world * photons * args.steps / (total_ms / 1000.0)
    e2e_value = world * photons * args.steps / e2e_total
    launch_ms = total_ms / args.steps
    steps_per_launch = steps_done / args.steps
    # roofline: the FP32/SFU issue roofline.  Algorithmic operations per photon-step (the
    # oracle's event counts on this workload times a per-event operation table counted from
    # the reference's source: oracle/algorithmic_ops.py -> profiles/k_propagate_algorithmic.json)
    # x this launch's photon-steps / its event-timed duration, against the FFMA and SFU
    # throughputs measured on this GPU by the library's own loops (the driver-measured peaks
    # have no FP32 or SFU figure).  Beside it, the same with the kernel's executed FP32 and
    # SFU instructions per step from its ncu capture (profiles/k_propagate_cascade.json).
    from ppc_b200.api import fp32_peak, sfu_peak
    alg = _profile_json("k_propagate_algorithmic.json")
    exe = _profile_json("k_propagate_cascade.json")
    props = torch.cuda.get_device_properties(local)
    pk_fp32, pk_sfu = fp32_peak(local, repeats=5), sfu_peak(local, repeats=5)
    sps = steps_per_launch / (launch_ms / 1000.0)

    def fracs(fp32_ops, sfu_ops):
        f = {"fp32": {"ops_per_photon_step": fp32_ops, "achieved": fp32_ops * sps / 1e12, "peak": pk_fp32,
                      "unit": "TFLOP/s"},
             "sfu": {"ops_per_photon_step": sfu_ops, "achieved": sfu_ops * sps / 1e12, "peak": pk_sfu, "unit": "Tops/s"}}
        for v in f.values():
            v["frac"] = v["achieved"] / v["peak"]
        return f

    algo = fracs(alg["fp32_ops_per_step"], alg["sfu_ops_per_step"]) if alg else None
    execd = fracs(exe["fp32_ops_per_step"], exe["sfu_ops_per_step"]) if exe else None
    base = algo or execd or fracs(float("nan"), float("nan"))  # the summaries are committed under profiles/
    top = base["fp32"] if base["fp32"]["frac"] > base["sfu"]["frac"] else base["sfu"]
    traffic = exe["dram_bytes_per_step"] * steps_per_launch if exe else None
    roofline = {"bound": "sfu" if top is base["sfu"] else "fp32", "achieved": top["achieved"], "peak": top["peak"],
                "unit": top["unit"], "frac": top["frac"], "traffic": traffic,
                "kind": "FP32/SFU issue roofline on algorithmic ops (oracle event counts x per-event table of "
                        "gpu/pro.cu), the larger fraction",
                "peak_source": f"measured on this GPU: FFMA and reciprocal-square-root loops on all "
                               f"{props.multi_processor_count} SMs (ppcb_fp32_peak, ppcb_sfu_peak)",
                "algorithmic": algo, "executed": execd,
                "traffic_source": (f"ncu dram bytes per photon-step ({exe['dram_bytes_per_step']:.3g} B) scaled by "
                                   "this launch's photon-steps") if exe else None}
    if exe:
        roofline["issue_ncu"] = exe.get("issue")
    h2d = 64 + 16
    d2h = 32 * (e2e_hits / max(1, args.steps)) + 56
    line = {
        "metric": "photons/s", "value": value, "unit": "photons/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": launch_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "full-detector EM cascade, 5160 DOMs, 171 layers, 1-d tilt, anisotropy, BFR",
                   "photons_per_step": photons, "l2": "flushed (256 MB write) before each timed step",
                   "parallelism": f"replicas x{world}", "threads": info["threads"], "blocks": info["blocks"]},
        "photon_steps_per_s": world * steps_done / (total_ms / 1000.0),
        "steps_per_photon": steps_per_launch / photons,
        "hits_per_step": hits / args.steps,
        "gpu_launches": args.steps,
        "e2e": {"value": e2e_value, "unit": "photons/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": int(d2h), "gpu_launches": args.steps,
                # where the end-to-end time went: the library's own launch timing (CUDA events
                # around upload, kernel and control read-back) against the wall clock
                "wall_ms_per_step": 1e3 * sum(e2e_times) / max(1, len(e2e_times)),
                "device_ms_per_step": e2e_dev_ms / max(1, len(e2e_times)),
                "host_cpu_ms_per_step": 1e3 * e2e_cpu / max(1, len(e2e_times)),
                "clocks": e2e_clocks},
        "roofline": roofline,
        "clocks": clocks,
    }
    summary = {"photons_per_s": value, "photon_steps_per_s": line["photon_steps_per_s"], "e2e_photons_per_s": e2e_value,
               "roofline_frac": top["frac"]}
    # the comparisons below are single-GPU figures: a multi-GPU run reports throughput only
    single = world == 1
    if single:
        del d_hits, flush
        torch.cuda.empty_cache()
        c.close()
    if single and not args.no_plain_kernel:
        pk = plain_kernel_sample(timed_cascades, photons, local)
        if pk:
            line["plain_kernel"] = {"value": pk["value"], "unit": "photons/s", "device_ms": pk["device_ms"],
                                    "photons": pk["photons"],
                                    "kind": "reference CUDA kernel gpu/pro.cu, sm_100a, gpu/Makefile flags, "
                                            "the timed steps' cascades, one eout() each",
                                    "speedup": value / pk["value"]}
            summary["plain_kernel_speedup"] = value / pk["value"]
    if single and not args.no_gradient:
        g = gradient_sample(local, plain_kernel=not args.no_plain_kernel)
        line["gradient"] = g
        summary["gradient_evals_per_s"] = g["evals_per_s"]
        summary["gradient_backward_over_forward"] = g["backward_over_forward"]
    if single and not args.no_batched:
        bt = batched_sample(local, events=4096, steps=2, warmup=3, plain_kernel=not args.no_plain_kernel)
        for k in ("metric", "unit", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "dtype", "data"):
            bt.pop(k, None)
        line["batched"] = bt
        summary["batched_events_per_s"] = bt["value"]
        if "speedup_vs_plain_kernel" in bt:
            summary["batched_plain_kernel_events_per_s"] = bt["plain_kernel"]["events_per_s"]
            summary["batched_speedup_vs_plain_kernel"] = bt["speedup_vs_plain_kernel"]
    if single and not args.no_fit:
        ft = fit_sample(local, iters=args.fit_iters, scale=args.fit_scale, plain_kernel=not args.no_plain_kernel)
        for k in ("n_gpus", "higher_is_better", "scaling", "vs_baseline", "dtype", "data"):
            ft.pop(k, None)
        line["fit"] = ft
        summary["fit_seconds_per_iteration"] = ft["value"]
        summary["fit_photon_scale"] = args.fit_scale
        if "speedup_vs_fd_plain_kernel" in ft:
            summary["fit_speedup_vs_fd_plain_kernel"] = ft["speedup_vs_fd_plain_kernel"]
    if single and not args.no_stages:
        line["stages"] = stages_sample(local)
    if single and not args.no_cpu_baseline:
        # the reference's CPU paths on the same workload: its std::par build on every core
        # (the baseline, its fastest), its gpu/ CPU build in one process per core and on one
        # thread
        cores = os.cpu_count() or 1
        rp = cpu_par_sample(cores * args.ref_photons)
        r = cpu_reference_sample(args.ref_photons, cores)
        r1 = cpu_reference_sample(args.ref_photons, 1, seed=1)
        gpu_build = {"value": r["value"], "unit": "photons/s", "cores": cores, "kind": "reference",
                     "sample": f"{args.ref_photons} photons x {cores} processes of the reference's gpu/ CPU "
                               "build (same cascade workload)"} if r else None
        par = {"value": rp["value"], "unit": "photons/s", "cores": cores, "kind": "reference",
               "sample": f"{rp['photons']} photons of {cores} cascades through the reference's std::par build "
                         "on every core (oracle/_ref/ppc_par, OpenMP)"} if rp else None
        # the baseline is the faster of the two all-core paths
        cands = [x for x in (gpu_build, par) if x]
        others = {}
        if cands:
            best = max(cands, key=lambda x: x["value"])
            line["cpu_baseline"] = best
            summary["cpu_baseline_photons_per_s"] = best["value"]
            if gpu_build and gpu_build is not best:
                others["gpu_cpu_build_all_cores"] = gpu_build
            if par and par is not best:
                others["par_all_cores"] = par
        if r1:
            others["gpu_cpu_build_1_thread"] = {"value": r1["value"], "unit": "photons/s", "cores": 1,
                                                "kind": "reference",
                                                "sample": f"{args.ref_photons} photons, one process of the gpu/ "
                                                          "CPU build (oracle/_ref/ref_harness_fm)"}
        if others:
            line["cpu_baselines_other"] = others
    line["summary"] = summary  # last: the headline figures at the end of the line
    print(json.dumps(line))


def _profile_json(name):
    """A committed measurement summary under profiles/ (None when absent)."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            return json.load(f)
    except Exception:
        return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--photons", type=int, default=PHOTONS)
    ap.add_argument("--ref-photons", type=int, default=200_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="device-resident timing only (profiling runs)")
    ap.add_argument("--no-plain-kernel", action="store_true", help="skip the reference CUDA kernel comparison")
    ap.add_argument("--no-gradient", action="store_true", help="skip the ice-gradient evaluation")
    ap.add_argument("--no-stages", action="store_true", help="skip the back end, likelihood and front end stages")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-events comparison (4096 events)")
    ap.add_argument("--no-fit", action="store_true", help="skip the ice-fit iterations")
    ap.add_argument("--cascade", type=lambda t: [float(x) for x in t.split(",")], default=None,
                    help="x,y,z,nx,ny,nz: one fixed cascade for every step instead of random ones (profiling)")
    ap.add_argument("--config", default="cascade", choices=["cascade", "batched", "fit"],
                    help="cascade: the headline workload; batched: 4096 events in one launch; "
                         "fit: L-BFGS ice fit over 1280 events")
    ap.add_argument("--fit-iters", type=int, default=3)
    ap.add_argument("--fit-scale", type=float, default=1.0, help="photon counts of the fit workload x this")
    ap.add_argument("--events", type=int, default=4096)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.config == "batched":
            run_batched(args, local)
        elif args.config == "fit":
            run_fit(args, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as td
            td.destroy_process_group()


if __name__ == "__main__":
    main()
