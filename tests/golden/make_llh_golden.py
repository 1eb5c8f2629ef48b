"""Golden vectors of DirectFit's likelihood from the reference's own code.

Runs oracle/_ref/llh_harness -- the reference's llh/llh.cxx compiled unmodified against the
GSL stand-in of oracle/gsl_shim and the reference's CPU library (oracle/Makefile) -- on
synthetic pulses of the full detector and stores, per option set, the inputs and what the
reference computes: the bin width, the time origin, ndof, every fitted DOM's blocks (first
and last bin, observed charge) and fllh at five time shifts.

  llh_<name>.npz   data, windows, bad, good, sim, dts, nsim, opts (JSON), lbin, t0, ndof,
                   blocks (str, om, first, last, dat), fllh

Pulse and hit times are multiples of 1/16 ns (below 2^14 ns) and charges multiples of
1/256, so that every sum of times the two sides form is exact and both bin the same way.

Needs the reference sources where oracle/Makefile's REF points (run in the build container):
    python tests/golden/make_llh_golden.py
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
os.environ.setdefault("PPCB_QUIET", "1")

from ppc_b200 import synth  # noqa: E402
from ppc_b200 import types as T  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "llh_harness")
DTS = [-40.0, -12.5, 0.0, 7.25, 30.0]
NSIM = 1.3

# name: (options, windows, bad DOMs, flasher, good-DOM list)
SETS = {
    "defaults": ({}, False, False, False, False),
    "peak": ({"peak": 1}, False, False, False, False),
    "mono": ({"mono": 1}, False, False, False, False),
    "peak_mono": ({"peak": 1, "mono": 1}, False, False, False, False),
    "drep3_qsat50": ({"drep": 3.0, "qsat": 50.0}, False, False, False, False),
    "sig020": ({"sig": 0.2}, False, False, False, False),
    "norm_unh": ({"norm": 1, "unh": 1}, False, True, False, False),
    "windows_bad_flasher": ({"unh": 1}, True, True, True, False),
    "good_list": ({}, False, False, False, True),
}


def _geo(ice):
    rows = [ln.split() for ln in open(os.path.join(ice, "geo-f2k")) if ln.strip()]
    g = np.zeros(len(rows), [("str", "<i4"), ("om", "<i4"), ("r", "<f8", 3)])
    for k, r in enumerate(rows):
        g[k] = (int(r[5]), int(r[6]), (float(r[2]), float(r[3]), float(r[4])))
    return g


def pulses(g, rng, center, n_doms, t0, scale):
    """Pulses around a point: counts falling with distance, straight-line delay plus gamma
    delays; times on a 1/16 ns grid, charges on a 1/256 grid."""
    d = np.linalg.norm(g["r"] - center, axis=1)
    near = np.argsort(d)[:n_doms]
    out = []
    for k in near:
        n = rng.poisson(scale * np.exp(-d[k] / 25.0)) + rng.integers(0, 2)
        t = t0 + d[k] / 0.2198 + rng.gamma(2.0, 15.0 + d[k] / 3.0, n)
        q = rng.uniform(0.2, 2.5, n)
        for ti, qi in zip(t, q):
            out.append((g["str"][k], g["om"][k], np.round(ti * 16) / 16, np.round(qi * 256) / 256))
    a = np.array(out, T.LLH_HIT_DTYPE)
    return a[rng.permutation(len(a))]


def main():
    ice = os.path.join(ROOT, "ppc_b200", "data", "ice", "full")
    if not os.path.exists(os.path.join(ice, "cfg.txt")):
        synth.write("full", ice)
    g = _geo(ice)
    for name, (opts, use_win, use_bad, use_fla, use_good) in SETS.items():
        rng = np.random.default_rng(7 + list(SETS).index(name))
        center = g["r"][rng.integers(len(g))] + rng.normal(0, 20, 3)
        data = pulses(g, rng, center, 70, 1000.0, 300.0)
        sim = pulses(g, rng, center + rng.normal(0, 5, 3), 90, 1000.0, 250.0)
        sim = np.array([(s, o, t) for s, o, t, _ in sim], [("str", "<i4"), ("om", "<i4"), ("t", "<f4")])
        keys = np.unique(data[["str", "om"]])
        win = np.zeros(0, T.LLH_WINDOW_DTYPE)
        bad = np.zeros((0, 2), np.int32)
        good = np.zeros((0, 2), np.int32)
        o = dict(opts)
        args = []
        if use_win:
            win = np.zeros(3, T.LLH_WINDOW_DTYPE)
            for k in range(3):
                sel = data[(data["str"] == keys[k]["str"]) & (data["om"] == keys[k]["om"])]
                ti = np.round(np.median(sel["t"]) * 16) / 16
                win[k] = (keys[k]["str"], keys[k]["om"], ti, ti + 80.0)
        if use_bad:
            bad = np.array([[keys[5]["str"], keys[5]["om"]], [keys[6]["str"], keys[6]["om"]]], np.int32)
        if use_good:  # every DOM but a few of the hit ones
            drop = {(int(k["str"]), int(k["om"])) for k in keys[[2, 9, 15, 22]]}
            good = np.array(sorted({(int(k["str"]), int(k["om"])) for k in keys} - drop), np.int32)
        if use_fla:
            fl = keys[10]
            o.update(flasher=1, fla_str=int(fl["str"]), fla_om=int(fl["om"]), fsep=2)
            args.append(f"flasher={int(fl['str'])}:{int(fl['om'])}:2")
        for k in ("norm", "mono", "peak"):
            if o.get(k):
                args.append(k)
        if "qsat" in o:
            args.append(f"qsat={o['qsat']!r}")
        if "drep" in o:
            args.append(f"drep={int(o['drep'])}")
        if "sig" in o:
            args.append(f"sig={o['sig']!r}")
        with tempfile.TemporaryDirectory() as tmp:
            with open(os.path.join(tmp, "dat"), "w") as f:
                for r in data:
                    f.write(f"{r['str']} {r['om']} {float(r['t'])!r} {float(r['q'])!r}\n")
            if len(win):
                with open(os.path.join(tmp, "ert"), "w") as f:
                    for w in win:
                        f.write(f"{w['str']} {w['om']} {float(w['ti'])!r} {float(w['tf'])!r}\n")
            if len(good):
                with open(os.path.join(tmp, "set"), "w") as f:
                    for s_, om in good:
                        f.write(f"{s_} {om}\n")
            if len(bad):
                with open(os.path.join(tmp, "bad"), "w") as f:
                    for s, om in bad:
                        f.write(f"{s} {om}\n")
            simf = os.path.join(tmp, "sim.txt")
            with open(simf, "w") as f:
                for r in sim:
                    f.write(f"{r['str']} {r['om']} {float(r['t'])!r}\n")
            env = dict(os.environ, PPCTABLESDIR=ice + "/")
            p = subprocess.run([HARNESS, tmp, simf, repr(NSIM), ",".join(repr(x) for x in DTS)] + args, env=env,
                               capture_output=True, text=True, check=True)
        res = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])
        blocks = np.array([tuple(b) for b in res["blocks"]], T.LLH_BLOCK_DTYPE)
        np.savez_compressed(os.path.join(HERE, f"llh_{name}.npz"), data=data, windows=win, bad=bad, good=good, sim=sim,
                            dts=np.array(DTS), nsim=NSIM, opts=json.dumps(o), lbin=res["lbin"], t0=res["t0"],
                            ndof=res["ndof"], blocks=blocks, fllh=np.array(res["fllh"]))
        print(name, "blocks", len(blocks), "ndof", res["ndof"], "fllh", np.round(res["fllh"], 4))


if __name__ == "__main__":
    main()
