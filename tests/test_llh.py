"""DirectFit's likelihood without a GPU: the oracle's llf against its closed form and its
defining minimisation, the block partition against an exhaustive search, and the
product's host-side preparation (binning, DOM selection, windows, blocks) against the
oracle, bit for bit, over the reference's options."""
import math
import os

import numpy as np
import pytest

import oracle_util as O
from ppc_b200 import types as T
from ppc_b200.api import PPC, Likelihood, PPCError


def _geo(ice):
    rows = [ln.split() for ln in open(os.path.join(ice, "geo-f2k")) if ln.strip()]
    g = np.zeros(len(rows), [("str", "<i4"), ("om", "<i4"), ("r", "<f8", 3)])
    for k, r in enumerate(rows):
        g[k] = (int(r[5]), int(r[6]), (float(r[2]), float(r[3]), float(r[4])))
    return g


def synth_pulses(ice, seed, n_doms=80, t0=1000.0, scale=300.0, center=None):
    """Pulses around a point source: counts falling with distance, arrival times from the
    straight-line delay plus gamma-distributed scattering delays, charges around 1."""
    rng = np.random.default_rng(seed)
    g = _geo(ice)
    if center is None:
        center = g["r"][rng.integers(len(g))] + rng.normal(0, 20, 3)
    d = np.linalg.norm(g["r"] - center, axis=1)
    near = np.argsort(d)[:n_doms]
    out = []
    for k in near:
        n = rng.poisson(scale * math.exp(-d[k] / 25.0)) + rng.integers(0, 2)
        t = t0 + d[k] / 0.2198 + rng.gamma(2.0, 15.0 + d[k] / 3.0, n)
        q = rng.uniform(0.2, 2.5, n)
        for ti, qi in zip(t, q):
            out.append((g["str"][k], g["om"][k], ti, qi))
    a = np.array(out, T.LLH_HIT_DTYPE)
    return a[rng.permutation(len(a))]


# ---- llf ---------------------------------------------------------------------------------

def test_llf_without_model_error_is_the_two_sample_poisson_ratio():
    rng = np.random.default_rng(3)
    for _ in range(200):
        s, d = rng.integers(0, 400, 2).astype(float)
        nsim, ndat = rng.uniform(0.5, 20, 2)
        v, err = O.llf(s, d, nsim, ndat, 0.0)
        assert err == 0
        if s == 0 and d == 0:
            assert v == 0
            continue
        ls = (s + d) / (nsim + ndat)
        want = (s * math.log(s / (nsim * ls)) if s > 0 else 0) + (d * math.log(d / (ndat * ls)) if d > 0 else 0)
        assert abs(v - want) <= 1e-9 * max(1, abs(want))
        assert v >= -1e-12


def test_llf_with_model_error_is_its_profile_minimum():
    """llf(s, d) = min over the two rates of nsim ls - s ln ls + ndat ld - d ln ld
    + ln(ld/ls)^2 / (2 sig^2), minus the same at the saturated rates (llh/llh.cxx:637-662)."""
    from scipy.optimize import minimize
    rng = np.random.default_rng(4)
    for _ in range(40):
        s, d = rng.integers(1, 300, 2).astype(float)
        nsim, ndat = rng.uniform(0.5, 10, 2)
        sig = rng.uniform(0.05, 0.5)
        v, err = O.llf(s, d, nsim, ndat, sig)
        assert err == 0

        def F(x):
            ls, ld = np.exp(x)
            return nsim * ls - s * x[0] + ndat * ld - d * x[1] + (x[1] - x[0]) ** 2 / (2 * sig * sig)

        x0 = np.log([(s + d) / (nsim + ndat)] * 2)
        r = minimize(F, x0, method="BFGS", options={"gtol": 1e-11})
        sat = s - s * math.log(s / nsim) + d - d * math.log(d / ndat)
        assert abs((r.fun - sat) - v) <= 1e-6 * max(1, abs(v)), (s, d, nsim, ndat, sig, r.fun - sat, v)
    assert O.llf(0, 0, 1, 1)[0] == 0
    assert abs(O.llf(20, 10, 2, 1)[0]) < 1e-12  # equal rates


# ---- the block partition ---------------------------------------------------------------

def _score(L, D):
    return (D * math.log(D / L) if D > 0 else 0) + math.lgamma(L + 1)


def test_block_partition_is_the_best_partition():
    """With 250 ns bins the window is 7 bins wide; every partition of it is scored."""
    rng = np.random.default_rng(5)
    for trial in range(40):
        nb = rng.integers(3, 9)
        q = rng.gamma(1.5, 3.0, nb) * (rng.random(nb) < 0.8)
        q[0] = max(q[0], 0.5)
        pulses = [(1, 1, 1000.0 + 250.0 * k + rng.uniform(-100, 100) * (k > 0), q[k]) for k in range(nb) if q[k] > 0]
        data = np.array(pulses, T.LLH_HIT_DTYPE)
        res = O.llh_setup(data, opts={"lbin": 250.0, "sig": 0.1})
        blocks = res[0]
        n1, n2 = blocks["first"].min(), blocks["last"].max() + 1
        bins = np.zeros(200)
        for p in data:
            bins[int(round((float(np.float32(p["t"])) - res[2]) / 250.0))] += float(np.float32(p["q"]))
        x = bins[n1:n2]
        got = sum(_score(b["last"] - b["first"] + 1, b["dat"]) for b in blocks)
        best = -math.inf
        n = len(x)
        for mask in range(1 << (n - 1)):
            s, start = 0.0, 0
            for e in range(n):
                if e == n - 1 or mask >> e & 1:
                    s += _score(e - start + 1, x[start:e + 1].sum())
                    start = e + 1
            best = max(best, s)
        assert abs(got - best) <= 1e-9 * abs(best), (trial, got, best)


# ---- product preparation against the oracle ---------------------------------------------

OPTION_SETS = {
    "defaults": {},
    "peak": {"peak": 1},
    "mono": {"mono": 1},
    "peak_mono": {"peak": 1, "mono": 1},
    "lbin10": {"lbin": 10.0},
    "drep3_qsat50": {"drep": 3.0, "qsat": 50.0},
    "norm_unh": {"norm": 1, "unh": 1},
}


@pytest.fixture(scope="module")
def host_ctx(ice_full):
    c = PPC()
    c.initialize(1.0, ice_full)
    yield c
    c.close()


def _same_blocks(L, res):
    ob, lbin, t0, ndof = res
    pb = L.blocks()
    info = L.info()
    assert info["lbin"] == lbin and info["t0"] == t0 and info["ndof"] == ndof
    assert info["blocks"] == len(ob) == len(pb)
    for f in ("str", "om", "first", "last", "dat"):
        assert np.array_equal(pb[f], ob[f]), f
    return pb


@pytest.mark.parametrize("name", list(OPTION_SETS))
def test_preparation_matches_oracle(host_ctx, ice_full, name):
    opts = OPTION_SETS[name]
    for seed in (11, 12, 13):
        data = synth_pulses(ice_full, seed)
        L = Likelihood(host_ctx, data, **opts)
        pb = _same_blocks(L, O.llh_setup(data, opts=opts))
        assert len(np.unique(pb[["str", "om"]])) == L.info()["doms"] > 5
        L.close()


def test_preparation_with_windows_bad_doms_and_flasher(host_ctx, ice_full):
    data = synth_pulses(ice_full, 21, n_doms=60)
    keys = np.unique(data[["str", "om"]])
    win = np.zeros(4, T.LLH_WINDOW_DTYPE)
    for k in range(3):  # windows over parts of three hit DOMs' pulses
        sel = data[(data["str"] == keys[k]["str"]) & (data["om"] == keys[k]["om"])]
        win[k] = (keys[k]["str"], keys[k]["om"], np.median(sel["t"]), np.median(sel["t"]) + 80.0)
    win[3] = (1, 1, 0.0, 1e9)  # a DOM with a window and no pulses is kept out
    bad = np.array([[keys[5]["str"], keys[5]["om"]], [keys[6]["str"], keys[6]["om"]]], np.int32)
    fl = keys[10]
    opts = {"flasher": 1, "fla_str": int(fl["str"]), "fla_om": int(fl["om"]), "fsep": 2, "unh": 1}
    L = Likelihood(host_ctx, data, windows=win, bad=bad, **opts)
    pb = _same_blocks(L, O.llh_setup(data, windows=win, bad=bad, opts=opts))
    pk = {(int(s), int(o)) for s, o in zip(pb["str"], pb["om"])}
    assert (int(keys[5]["str"]), int(keys[5]["om"])) not in pk
    assert not any(s == fl["str"] and abs(o - fl["om"]) <= 2 for s, o in pk)
    L.close()


def test_likelihood_errors(host_ctx, ice_full):
    none_in_ice = np.array([(0, 5, 100.0, 1.0), (90, 70, 10.0, 0.0)], T.LLH_HIT_DTYPE)
    with pytest.raises(PPCError) as e:
        Likelihood(host_ctx, none_in_ice[:1])
    assert e.value.code == 7
    data = synth_pulses(ice_full, 31)
    with pytest.raises(PPCError) as e:
        Likelihood(host_ctx, data, lbin=3000.0)
    assert e.value.code == 7
    with pytest.raises(TypeError):
        Likelihood(host_ctx, data, sigma=0.2)
    L = Likelihood(host_ctx, data)
    with pytest.raises(PPCError) as e:  # no ini(): nothing on a device yet
        L.eval(np.zeros(1, T.HIT_DTYPE), [0.0], 1.0)
    assert e.value.code == 6
    L.close()
