"""Generates the golden vectors in this directory from the reference itself.

Runs the reference's own code (gpu/ppc.cu + gpu/ini.cxx + gpu/pro.cu + gpu/f2k.cxx,
compiled as its CPU build with IEEE float semantics by oracle/Makefile into
oracle/_ref/ref_harness) on the synthetic configurations of ppc_b200/synth.py and stores:

  tables_<kind>.json    sha256 of every table the reference's ini::set builds
  zshift_<kind>.npz     tilt shift and layer thickness at fixed random points
  run_<case>.npz        kernel-level hits, a digest of the phase-1 photon records and the
                        final random-stream state of a fixed-seed propagation
  backend_<case>.npz    the reference's own back end (print, gpu/f2k.cxx:247-363) over the
                        kernel-level hits of a propagation: its input hits, host seed and the
                        hit map it fills

Needs the reference sources where oracle/Makefile's REF points (run in the build container):
    python tests/golden/make_golden.py [names...]   (configurations / cases; default all)
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
os.environ.setdefault("PPCB_QUIET", "1")

import oracle_util as O  # noqa: E402
from ppc_b200 import synth  # noqa: E402

TABLES = ["az", "lr", "ls", "mcol", "sc", "lp", "absca", "wmeta", "oms", "rm", "wvs", "eff"]

# (case, configuration, source spec, photons, seed, environment)
RUNS = [
    ("small_point", "small", "point:0:0:0", 20000, 7, {"FWID": "-1", "WFLA": "405"}),
    ("full_cascade", "full", "cascade:10:20:-300:2000:0.3:0.4:0.8660254:11", 20000, 7, {}),
    ("full2d_flasher", "full2d", "flasher:40:30", 20000, 7, {}),
    ("small_tilt_led", "small_tilt", "flasher:1:30", 20000, 9, {"FWID": "9.7"}),
    ("small_hole_point", "small_hole", "point:0:0:0", 20000, 11, {"FWID": "-1", "WFLA": "405"}),
    ("full_ng_cascade", "full_ng", "cascade:-50:310:50:2000:0.3:0.4:0.8660254:11", 20000, 5, {}),
    ("small_xr1_point", "small_xr1", "point:0:0:0", 200000, 13, {"FWID": "-1", "WFLA": "405"}),
]
KINDS = ("small", "full", "full2d", "small_tilt", "small_hole", "full_ng", "small_xr1")

# (case, configuration, source spec, photons, propagation seed, back-end seed): standard
# sensors with cables and tilted axes; 24-PMT spheres, 2-PMT spheroids, shifting tubes
BACKENDS = [
    ("full2d", "full2d", "cascade:20:-60:-100:2000:0.3:0.4:0.8660254:11", 300000, 5, 77),
    ("full_ng_sphere", "full_ng", "cascade:20:-60:-100:2000:0.3:0.4:0.8660254:11", 300000, 5, 78),
    ("full_ng_spheroid", "full_ng", "cascade:-50:310:50:2000:0.3:0.4:0.8660254:11", 300000, 6, 79),
    ("full_ng_tube", "full_ng", "cascade:-360:10:0:2000:0.3:0.4:0.8660254:11", 300000, 7, 80),
]


def dtmn_order(hits):
    """The reference's deterministic back-end order (segment, DOM, time, wavelength bin;
    gpu/f2k.cxx:236-244 with DTMN)."""
    return hits[np.lexsort((hits["z"], hits["t"], hits["i"], hits["n"]))]


def reference_back_end(icedir, hits, seed, tmp):
    from ppc_b200._lib import HITZ_DTYPE
    fi, fo = os.path.join(tmp, "bh.bin"), os.path.join(tmp, "bo.bin")
    hits.tofile(fi)
    O.run_harness(["backend", fi, str(seed), fo], {"PPCTABLESDIR": icedir + "/"})
    return np.fromfile(fo, HITZ_DTYPE)


def ice(kind):
    path = os.path.join(ROOT, "ppc_b200", "data", "ice", kind)
    if not os.path.exists(os.path.join(path, "cfg.txt")):
        synth.write(kind, path)
    return path


def sha(b):
    return hashlib.sha256(b).hexdigest()


def probe_points(n, seed):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = rng.uniform(-750, 750, n)
    pos[:, 1] = rng.uniform(-750, 750, n)
    pos[:, 2] = rng.uniform(-600, 600, n)
    return pos


def main(only=()):
    """only: configuration and case names to (re)generate; all when empty."""
    if not O.harness_available():
        raise SystemExit("reference harness missing: make -C oracle ref")
    tmp = tempfile.mkdtemp()
    for kind in KINDS:
        if only and kind not in only:
            continue
        raw = O.harness_tables(ice(kind), tmp)
        with open(os.path.join(HERE, f"tables_{kind}.json"), "w") as f:
            json.dump({k: sha(raw[k]) for k in TABLES}, f, indent=1, sort_keys=True)
    for kind in ("full", "full2d", "small_tilt"):
        if only and kind not in only:
            continue
        pos = probe_points(2000, 5)
        fi, fo = os.path.join(tmp, "p.bin"), os.path.join(tmp, "z.bin")
        pos.tofile(fi)
        O.run_harness(["zshift", fi, fo], {"PPCTABLESDIR": ice(kind)})
        z = np.fromfile(fo, np.float32).reshape(-1, 3)[:, :2]
        np.savez_compressed(os.path.join(HERE, f"zshift_{kind}.npz"), pos=pos, zshift=z)
    for case, kind, spec, photons, seed, env in RUNS:
        if only and case not in only:
            continue
        info, hits, pbuf, bunch = O.harness_run(ice(kind), spec, photons, seed, os.path.join(tmp, case), env)
        np.savez_compressed(os.path.join(HERE, f"run_{case}.npz"), hits=hits, bunch=bunch,
                            pbuf_head=pbuf[:256], pbuf_sha=np.frombuffer(sha(pbuf.tobytes()).encode(), np.uint8),
                            rs=np.uint64(info["rs"]), seed=np.uint32(seed), photons=np.uint32(photons),
                            env=np.frombuffer(json.dumps(env).encode(), np.uint8))
        print(case, info)
    for case, kind, spec, photons, seed, bseed in BACKENDS:
        name = "backend_" + case
        if only and name not in only:
            continue
        info, hits, _, _ = O.harness_run(ice(kind), spec, photons, seed, os.path.join(tmp, name))
        hits = dtmn_order(hits)
        out = reference_back_end(ice(kind), hits, bseed, tmp)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), hits=hits, seed=np.uint32(bseed), hitz=out)
        print(name, len(hits), "hits ->", len(out), "records")


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
