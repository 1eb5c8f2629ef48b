"""High-statistics parity fixtures from the reference's own CPU build.

Runs the reference's gpu/ppc.cu + gpu/pro.cu + gpu/ini.cxx + gpu/f2k.cxx, compiled with its
own CPU flags (`-O2 --fast-math`, gpu/Makefile:10; oracle/Makefile target
`_ref/ref_harness_fm`), on many seeds in parallel, and keeps only what the statistical
parity test compares:

  parity_<case>.npz
    photons        propagated photons (all runs)
    counts[gsize]  kernel-level hits per DOM (gpu/pro.cu:731-753, before acceptance)
    hist[gsize,B]  per-DOM hit-time histograms on the edges `edges` (ns)
    edges[B+1]     log-spaced time-bin edges
    bunch          the 64-byte bunch record the reference propagated (its own template)
    runs, seeds    the runs that made it

Cases:
  small_point     the 7-string detector, isotropic 405 nm point source at the origin
                  (FWID=-1 WFLA=405), 1e6 photons per run -- the 7-string point-source
                  workload as written; enough runs that the total hit count is known
                  to better than 0.025%
  full_cascade    the full detector (171 layers, tilt, anisotropy, birefringence), one
                  fixed EM cascade at (12.5, -40, 60) m along (0.6, 0, 0.8)

Needs the reference sources (run in the build container, where oracle/_ref is built):
    python tests/golden/make_parity_fixture.py [case ...] [--procs N]
"""
import argparse
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness_fm")

EDGES = np.concatenate([[0.0], np.logspace(0, 5, 401)])  # 0, then 1 ns .. 100 us, 400 log bins

# case: (configuration, source spec, photons per run, runs, environment)
CASES = {
    "small_point": ("small", "point:0:0:0", 1_000_000, 2800, {"FWID": "-1", "WFLA": "405"}),
    "full_cascade": ("full", "cascade:12.5:-40:60:10000:0.6:0:0.8:11", 4_000_000, 500, {}),
}

HIT_DTYPE = np.dtype([("i", "<u4"), ("n", "<u4"), ("z", "<u4"), ("t", "<f4"),
                      ("pth", "<f4"), ("pph", "<f4"), ("dth", "<f4"), ("dph", "<f4")])


def _one(job):
    icedir, spec, photons, seed, env = job
    with tempfile.TemporaryDirectory() as tmp:
        pre = os.path.join(tmp, "r")
        e = dict(os.environ, PPCTABLESDIR=icedir + "/", **env)
        r = subprocess.run([HARNESS, "run", spec, str(photons), str(seed), pre, "hits"], env=e,
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-2000:])
        h = np.fromfile(pre + ".hits", HIT_DTYPE)
    return seed, h["i"].astype(np.int64), h["t"].astype(np.float64)


def _template(icedir, spec, env):
    """The bunch record the reference builds for `spec` (one photon, full dump)."""
    with tempfile.TemporaryDirectory() as tmp:
        pre = os.path.join(tmp, "t")
        e = dict(os.environ, PPCTABLESDIR=icedir + "/", **env)
        subprocess.run([HARNESS, "run", spec, "1", "1", pre], env=e, capture_output=True, check=True)
        return np.fromfile(pre + ".bunch", np.uint8)[:64].copy()


def make(case, procs):
    kind, spec, photons, runs, env = CASES[case]
    icedir = os.path.join(ROOT, "ppc_b200", "data", "ice", kind)
    if not os.path.exists(os.path.join(icedir, "cfg.txt")):
        from ppc_b200 import synth
        synth.write(kind, icedir)
    ndom = sum(1 for _ in open(os.path.join(icedir, "geo-f2k")))
    counts = np.zeros(ndom, np.int64)
    hist = np.zeros((ndom, len(EDGES) - 1), np.int64)
    bunch = _template(icedir, spec, env)
    seeds = list(range(1000, 1000 + runs))
    jobs = [(icedir, spec, photons, s, env) for s in seeds]
    t0 = time.time()
    with mp.get_context("spawn").Pool(procs) as pool:
        for k, (seed, dom, t) in enumerate(pool.imap_unordered(_one, jobs)):
            counts += np.bincount(dom, minlength=ndom)
            b = np.clip(np.searchsorted(EDGES, t, side="right") - 1, 0, len(EDGES) - 2)
            np.add.at(hist, (dom, b), 1)
            if (k + 1) % 50 == 0:
                print(f"{case}: {k + 1}/{runs} runs, {counts.sum()} hits, {time.time() - t0:.0f} s", flush=True)
    out = os.path.join(HERE, f"parity_{case}.npz")
    np.savez_compressed(out, photons=np.int64(photons) * runs, counts=counts, hist=hist.astype(np.uint32),
                        edges=EDGES, runs=np.int64(runs), seeds=np.array(seeds, np.int64),
                        photons_per_run=np.int64(photons), spec=spec, kind=kind, bunch=bunch)
    print(f"{case}: {photons * runs:.3e} photons, {counts.sum()} hits -> {out}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*", default=list(CASES))
    ap.add_argument("--procs", type=int, default=os.cpu_count())
    a = ap.parse_args()
    for c in a.cases:
        make(c, a.procs)
