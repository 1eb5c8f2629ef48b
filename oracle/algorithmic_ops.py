"""Algorithmic work of the propagation hot path, per photon-step (test infrastructure).

The algorithmic FP32 and special-function operation counts behind the benchmark's
algorithmic roofline: event counts from the oracle (oracle/ppc_oracle.c, which restates
gpu/pro.cu bit for bit; `ppco_counts`) on a sample of the benchmark workload, times a fixed
per-event operation table counted from the reference's source.

Counting rules (source level, gpu/pro.cu): each +, -, * of floats is one FP32 operation, so
a*b+c is two; a division is one FP32 operation plus one reciprocal (SFU); logf, expf,
sqrtf, rsqrtf, sinf, cosf, atanf, acosf, atan2f are one SFU operation each, powf two (a
logarithm and an exponential); comparisons, min/max, conversions, integer and random-
number integer arithmetic are not counted.  The DOM search's loop over the strings of a
search cell is search structure, not algorithmic work: only the strings whose cylinder test
passes and the DOMs tested behind them are counted.  Totals are therefore a lower bound on
the floating-point work the method needs.

Writes profiles/k_propagate_algorithmic.json (read by bench.py) and prints a summary:
    python oracle/algorithmic_ops.py [photons_per_cascade] [cascades]
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
os.environ.setdefault("PPCB_QUIET", "1")

# (FP32, SFU) operations per event, counted from gpu/pro.cu as stated above.
OPS = {
    # every step: layer index (:514-515, 3), direction sign (:507, 1), absorption anisotropy
    # (:517-544, new model: 2 projections 6, scaling 3, norm 5 + rsqrt + 1, TOT/nr 1 + rcp),
    # overburden start (:548, 4), first stepping iteration (:552-566: 2 divisions, 1 mul,
    # 2 adds), tot/sca split (:567-570, 2), TOT = tot*nr (:719, 1), advance (:720-725, 8)
    "step": (1 + 3 + 16 + 4 + 5 + 2 + 1 + 8, 2 + 2),
    # 1-d tilt shift (:169-191): projection 4, depth 2, interval widths and weights 5 with
    # 2 divisions, two interpolations 6, slope term 3
    "zshift_1d": (20, 2),
    # 2-d tilt shift (:192-262) on the common path (no edge extrapolation): basis change 6,
    # 2 divisions 2 + 2, barycentric weights 5, three map points 12, slope term 3
    "zshift_2d": (30, 2),
    "sca_draw": (1, 1),  # -logf(xrnd) (:501)
    # one more layer in the stepping loop (:555-561): del = ahx/anz, 2 adds, 2 fma, next
    # iteration's 2 divisions and product
    "crossing": (10, 3),
    # a string whose cylinder test passes (:601-626): the test 17, roots and window 16,
    # sqrt and 2 divisions
    "string_passed": (33, 3),
    # a DOM tested (:627-653): 3 components 25, quadratic 9, divisions and sqrt
    "dom_tested": (35, 5),
    # a hit record (:734-745): angles (4 SFU), impact point 11, normalised height 3 + rcp
    "hit": (14, 5),
    # birefringence (:757-836) without the curved path: ra/rb 2, dot 3, sin of the angle
    # 2 + sqrt, sx and sy 10 (sqrt, atan, pow, exp each), mx 8 (atan, exp), q vector 13 +
    # rsqrt, p vector 9, two gaussians 6 + (log, sqrt, sin, cos), deflection 36 (2 + rcp,
    # normalisation 8 + rsqrt)
    "bfr": (2 + 3 + 2 + 10 + 8 + 13 + 9 + 6 + 3 + 36, 1 + 10 + 2 + 1 + 4 + 2),
    # the curved path within the segment (:790-815): two more gaussians, half deflection,
    # mid direction 18, normalisation 8 + rsqrt, position correction 11
    "bfr_curved": (59, 6),
    "bfr_layer": (2, 0),  # one more layer in the ra/rb overburden (:769)
    # scattering (:838-887): draw 1, Henyey-Greenstein 16 + 3 divisions | SAM 3 + rcp and
    # pow; then stretch 23 (rcp, rsqrt), rotate 64 (sqrt, 4 rsqrt, sin, cos, one more
    # rsqrt), unstretch 23 (2 rcp, rsqrt), k1*k2 1
    "scatter_hg": (1 + 16 + 1 + 23 + 64 + 23, 3 + 2 + 8 + 3),
    "scatter_sam": (1 + 3 + 1 + 23 + 64 + 23, 3 + 2 + 8 + 3),
    # phase 1 for one cascade photon (:337-339, :430-474): wavelength 1, gamma profile
    # (Cheng's sampler, ~1.25 iterations of 16 FP32 + 5 SFU), position 9 + rcp, secondary
    # direction 7 + 6 SFU, two rotations 128 + 16, first absorption depth 1 + log
    "photon_cascade": (1 + 20 + 9 + 7 + 128 + 1, 6 + 1 + 6 + 16 + 1),
}

EVENTS = ["photons", "steps", "sca_draws", "crossings", "strings_tested", "strings_passed", "doms_tested", "hits",
          "truncated", "bfr", "bfr_curved", "bfr_layers", "scatter_hg", "scatter_sam"]


def sample(photons_per_cascade=20000, cascades=8, seed=17):
    """Oracle event counts on cascades of the benchmark workload (full detector, random
    vertices and directions, the benchmark's longitudinal profile)."""
    import ctypes as C

    import oracle_util as O
    from ppc_b200 import types as T
    from ppc_b200.api import PPC

    class Counts(C.Structure):
        _fields_ = [(k, C.c_uint64) for k in EVENTS]

    c = PPC()
    c.initialize(1.0, os.path.join(ROOT, "ppc_b200", "data", "ice", "full"))
    tb = O.tables_from_product(c)
    L = O.lib()
    ppm = float(c.tables()["eff"][0])
    rng = np.random.default_rng(seed)
    rm = c.tables()["rm"][:4096]
    L.ppco_counts_reset()
    for k in range(cascades):
        E = 1e8 * 25.0 / (ppm * 5.321 * 0.910 / 0.9216)  # the benchmark's 1e8-photon cascade
        a = 2.01849 + 0.63176 * math.log(E)
        b = 0.39652 * 0.910 / 0.9216 / 0.63207
        v = rng.uniform(-500, 500, 3)
        ct = rng.uniform(-1, 1)
        ph = rng.uniform(0, 2 * math.pi)
        st = math.sqrt(1 - ct * ct)
        bun = T.bunch_particle([v[0], v[1], v[2], 0.0], [st * math.cos(ph), st * math.sin(ph), ct], 1,
                               photons_per_cascade, -11, f=0.0, a=a, b=b)
        tb.run_fused(bun, photons_per_cascade, O.mwc_init(k, rm), rm)
    cnt = Counts()
    L.ppco_counts_get(C.byref(cnt))
    p = c.params()
    c.close()
    return {k: int(getattr(cnt, k)) for k in EVENTS}, int(p.tmod)


def per_step(counts, tmod):
    s = counts["steps"]
    ev = {
        "step": 1.0,
        "zshift_1d": 1.0 if tmod == 1 else 0.0,
        "zshift_2d": 1.0 if tmod == 2 else 0.0,
        "sca_draw": counts["sca_draws"] / s,
        "crossing": counts["crossings"] / s,
        "string_passed": counts["strings_passed"] / s,
        "dom_tested": counts["doms_tested"] / s,
        "hit": counts["hits"] / s,
        "bfr": counts["bfr"] / s,
        "bfr_curved": counts["bfr_curved"] / s,
        "bfr_layer": counts["bfr_layers"] / s,
        "scatter_hg": counts["scatter_hg"] / s,
        "scatter_sam": counts["scatter_sam"] / s,
        "photon_cascade": counts["photons"] / s,
    }
    fp32 = sum(ev[k] * OPS[k][0] for k in ev)
    sfu = sum(ev[k] * OPS[k][1] for k in ev)
    return ev, fp32, sfu


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 20000
    m = int(sys.argv[2]) if len(sys.argv) > 2 else 8
    counts, tmod = sample(n, m)
    ev, fp32, sfu = per_step(counts, tmod)
    out = {"workload": f"full detector, {m} EM cascades (benchmark profile, random vertex and direction), "
                       f"{n} photons each, oracle event counts",
           "counts": counts, "events_per_step": ev, "ops_per_event": {k: list(v) for k, v in OPS.items()},
           "fp32_ops_per_step": fp32, "sfu_ops_per_step": sfu,
           "steps_per_photon": counts["steps"] / counts["photons"],
           "rules": "source-level counts from gpu/pro.cu: +,-,* one FP32 op (a*b+c two), division one FP32 + one "
                    "SFU, logf/expf/sqrtf/rsqrtf/sinf/cosf/atanf/acosf/atan2f one SFU, powf two SFU; string-loop "
                    "search structure excluded; a lower bound",
           "command": "python oracle/algorithmic_ops.py %d %d" % (n, m)}
    path = os.path.join(ROOT, "profiles", "k_propagate_algorithmic.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({"fp32_ops_per_step": fp32, "sfu_ops_per_step": sfu, "events_per_step": ev}, indent=1))


if __name__ == "__main__":
    main()
