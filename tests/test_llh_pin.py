"""The likelihood oracle (oracle/llh_oracle.c) pinned to the reference's own DirectFit code.

tests/golden/llh_*.npz hold what the reference's llh/llh.cxx computes (run through
oracle/_ref/llh_harness: its xyz::ini, dat::prep/optimize, cascade::ppc's hit assignment and
fllh, compiled unmodified against a GSL stand-in) for nine option sets: the defaults, the
peak window, monotonic blocks and both, a charge repetition of 3 with a saturation of 50,
a model error of 0.2, normalisation with a bad-DOM list (no-hit DOMs counted), errata
windows with bad DOMs and a flasher, and a good-DOM list (the reference's `set` file).  The
oracle must give the same bin width, time origin, ndof and blocks bit for bit, and the same
fllh to 1e-12 relative; the product's host preparation (good-DOM list included) must give
the same blocks bit for bit.  With oracle/_ref/llh_harness built, the
golden vectors are also re-derived from the reference on the spot."""
import glob
import json
import os
import subprocess

import numpy as np
import pytest

import oracle_util as O
from ppc_b200.api import PPC, Likelihood

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.path.basename(p)[4:-4] for p in glob.glob(os.path.join(GOLDEN, "llh_*.npz")))


def _load(name):
    g = np.load(os.path.join(GOLDEN, f"llh_{name}.npz"))
    return g, json.loads(str(g["opts"]))


def test_all_option_sets_present():
    assert len(CASES) == 9, CASES


def _bad(g):
    """The bad list the oracle gets: the golden's, plus what its good-DOM list excludes."""
    from ppc_b200.api import good_list_bad
    bad = g["bad"].reshape(-1, 2)
    if len(g["good"]):
        bad = np.concatenate([bad, good_list_bad(g["data"], g["good"])])
    return bad if len(bad) else None


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_likelihood(name):
    g, opts = _load(name)
    win = g["windows"] if len(g["windows"]) else None
    bad = _bad(g)
    blocks, lbin, t0, ndof = O.llh_setup(g["data"], windows=win, bad=bad, opts=opts)
    assert lbin == float(g["lbin"]) and t0 == float(g["t0"]) and ndof == int(g["ndof"])
    ref = g["blocks"]
    assert len(blocks) == len(ref)
    # the reference lists DOMs in its map's (string, module) order, as the oracle does
    for f in ("str", "om", "first", "last", "dat"):
        assert np.array_equal(blocks[f], ref[f]), f
    out, err = O.llh_fllh(g["data"], g["sim"], g["dts"], float(g["nsim"]), windows=win, bad=bad, opts=opts)
    assert err == 0
    assert np.allclose(out, g["fllh"], rtol=1e-12, atol=0), (out, g["fllh"])


@pytest.mark.parametrize("name", CASES)
def test_product_preparation_matches_reference(name, ice_full):
    g, opts = _load(name)
    c = PPC()
    c.initialize(1.0, ice_full)
    kw = {k: v for k, v in opts.items()}
    win = g["windows"] if len(g["windows"]) else None
    bad = g["bad"] if len(g["bad"]) else None
    good = g["good"] if len(g["good"]) else None
    L = Likelihood(c, g["data"], windows=win, bad=bad, good=good, **kw)
    info = L.info()
    assert info["lbin"] == float(g["lbin"]) and info["t0"] == float(g["t0"]) and info["ndof"] == int(g["ndof"])
    pb = L.blocks()
    for f in ("str", "om", "first", "last", "dat"):
        assert np.array_equal(pb[f], g["blocks"][f]), f
    L.close()
    c.close()


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(O.ORACLE_SO), "_ref", "llh_harness")),
                    reason="reference likelihood harness not built")
def test_golden_vectors_reproduce_from_the_reference(tmp_path):
    """The stored vectors are what the reference computes now (one option set re-run)."""
    import sys
    sys.path.insert(0, GOLDEN)
    import make_llh_golden as M
    g, opts = _load("windows_bad_flasher")
    d = tmp_path / "ev"
    d.mkdir()
    with open(d / "dat", "w") as f:
        for r in g["data"]:
            f.write(f"{r['str']} {r['om']} {float(r['t'])!r} {float(r['q'])!r}\n")
    with open(d / "ert", "w") as f:
        for w in g["windows"]:
            f.write(f"{w['str']} {w['om']} {float(w['ti'])!r} {float(w['tf'])!r}\n")
    with open(d / "bad", "w") as f:
        for s, om in g["bad"]:
            f.write(f"{s} {om}\n")
    simf = tmp_path / "sim.txt"
    with open(simf, "w") as f:
        for r in g["sim"]:
            f.write(f"{r['str']} {r['om']} {float(r['t'])!r}\n")
    ice = os.path.join(M.ROOT, "ppc_b200", "data", "ice", "full")
    env = dict(os.environ, PPCTABLESDIR=ice + "/")
    args = [f"flasher={opts['fla_str']}:{opts['fla_om']}:{opts['fsep']}"]
    cmd = [M.HARNESS, str(d), str(simf), repr(float(g["nsim"])), ",".join(repr(float(x)) for x in g["dts"])]
    p = subprocess.run(cmd + args, env=env, capture_output=True, text=True, check=True)
    res = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])
    assert res["ndof"] == int(g["ndof"]) and np.array_equal(np.array(res["fllh"]), g["fllh"])
