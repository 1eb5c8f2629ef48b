"""Ice-model gradient: replay fidelity, agreement with central finite differences under
common random numbers (per-photon streams), the Poisson-likelihood weighting, the
torch.autograd wrapper, and its cost relative to a forward pass.

Finite-difference noise (measured with per-photon streams, 1e9 flasher photons per
evaluation, relative step 0.03 along all layers): about 0.5% for the absorption direction
and about 2% for the scattering direction, whose perturbed paths move hits in both
directions.  The photon counts below are set from those figures."""
import os

import numpy as np
import pytest

from conftest import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

from ppc_b200 import workloads as W  # noqa: E402
from ppc_b200.api import PPC  # noqa: E402

FLASHERS = [(20 * 60 + 29), (44 * 60 + 35)]  # string 21 DOM 30, string 45 DOM 36 of the `full` detector


def _ctx(ice, seed=11, **opts):
    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(seed)
    c.set_options(**(opts or {"photon_streams": True}))
    c.choose(0)
    c.ini()
    return c


def _bunches(c, photons):
    oms = c.tables()["oms"]
    return np.concatenate([W.flasher(k, oms["r"][k], photons, q=i) for i, k in enumerate(FLASHERS)])


def _dom_hits(c, b, be, ba, be0, ba0, cap=4_000_000):
    c.set_ice(be, ba)
    try:
        return c.gradient(b, weights=np.zeros(c.info()["gsize"], np.float32), hit_cap=cap)["counts"].astype(np.int64)
    finally:
        c.set_ice(be0, ba0)


def _total_hits(c, b, be, ba, be0, ba0, cap=4_000_000):
    return float(_dom_hits(c, b, be, ba, be0, ba0, cap).sum())


@pytest.mark.parametrize("opts", [{"deterministic": True}, {"deterministic": False}, {"photon_streams": True}],
                         ids=["static", "dynamic", "photon_streams"])
def test_replay_retraces_the_recorded_photons(ice_full, opts):
    """Static order replays thread streams; the dynamic photon pool records per-photon
    streams (a lane's thread stream would interleave with the sampling it does for others)."""
    c = _ctx(ice_full, **opts)
    b = _bunches(c, 5_000_000)
    r = c.gradient(b, weights=np.ones(c.info()["gsize"], np.float32))
    info = r["info"]
    assert info["hits"] > 5000
    assert info["replayed"] == info["hits"]
    assert info["unmatched"] <= 0.002 * info["replayed"], info
    c.close()


def test_photon_streams_repeat_exactly(ice_full):
    c = _ctx(ice_full)
    b = _bunches(c, 2_000_000)
    w = np.ones(c.info()["gsize"], np.float32)
    r1 = c.gradient(b, weights=w)
    r2 = c.gradient(b, weights=w)  # no stream reset: each photon's numbers depend on (seed, index) only
    assert np.array_equal(r1["counts"], r2["counts"])
    assert np.allclose(r1["g_ba"], r2["g_ba"], rtol=1e-9, atol=0) and np.allclose(r1["g_be"], r2["g_be"], rtol=1e-9)
    c.close()


def test_gradient_matches_central_differences(ice_full):
    """Directional derivatives along all layers at once (d_j = x_j sign(g_j), relative step
    0.03), absorption and scattering each within 2%: 9e9 flasher photons per evaluation, so
    that the finite differences' own noise (about 2% at 1e9 photons for scattering, whose
    perturbed paths move hits both ways) is below 0.7%."""
    c = _ctx(ice_full)
    be0, ba0 = c.get_ice()
    b = np.concatenate([_bunches(c, 2_250_000_000)] * 2)  # 9e9 photons in bunches below 2^32
    cap = 16_000_000
    r = c.gradient(b, weights=np.ones(c.info()["gsize"], np.float32), hit_cap=cap)
    assert r["info"]["unmatched"] <= 0.002 * r["info"]["replayed"], r["info"]
    h = 0.03
    report = []
    for kind, g, base in (("ba", r["g_ba"], ba0), ("be", r["g_be"], be0)):
        d = base * np.sign(g)
        adj = float(np.dot(g, d))
        xp, xm = (base + h * d).astype(np.float32), (base - h * d).astype(np.float32)
        if kind == "ba":
            fd = (_total_hits(c, b, be0, xp, be0, ba0, cap) - _total_hits(c, b, be0, xm, be0, ba0, cap)) / (2 * h)
        else:
            fd = (_total_hits(c, b, xp, ba0, be0, ba0, cap) - _total_hits(c, b, xm, ba0, be0, ba0, cap)) / (2 * h)
        report.append((kind, adj, fd))
    print("adjoint vs central differences along all layers (sum_j x_j |dN/dx_j|):", report)
    for kind, adj, fd in report:
        assert abs(adj - fd) <= 0.02 * abs(fd), (kind, adj, fd)
    c.close()


def test_gradient_matches_per_layer_central_differences(ice_full):
    """Per parameter: central differences of the hit count with common random numbers
    (per-photon streams: both sides see every photon's random numbers) on the 8 absorption
    and 8 scattering layers with the largest effect, 2e9 flasher photons per evaluation in
    16 independent batches, at a relative step of 0.03 and of 1e-3 (the gradient's
    specification).  At a relative step h the difference counts the photons whose fate flips
    between the two sides, about 2h x_j dN/dx_j of them: a Poisson number.  Its standard
    error is the square root of that count for absorption (raising an absorption coefficient
    only removes hits, so the count is the difference itself) and, for scattering (hits move
    both ways), the larger of the spread over the 16 batches and the per-DOM count changes.
    Each layer, and the sum over the 8 layers of each kind, must agree within 2% plus three
    standard errors: at h = 0.03 that is within about 4% for absorption, at h = 1e-3 (about
    a thousand flips per layer) within about 12%."""
    c = _ctx(ice_full)
    be0, ba0 = c.get_ice()
    K = 16
    oms = c.tables()["oms"]
    b = np.concatenate([W.flasher(k, oms["r"][k], 1_000_000_000 // K, q=q) for q in range(K) for k in FLASHERS])
    gs = c.info()["gsize"]
    cap = 8_000_000
    r = c.gradient(b, weights=np.ones(K * gs, np.float32), events=K, hit_cap=cap)

    def counts(be, ba):  # hits per (batch, DOM)
        c.set_ice(be, ba)
        try:
            n = c.gradient(b, weights=np.zeros(K * gs, np.float32), events=K, hit_cap=cap)["counts"]
            return n.reshape(K, gs).astype(np.float64)
        finally:
            c.set_ice(be0, ba0)

    rows, fails = [], []
    for h in (0.03, 1e-3):
        for kind, g, x0 in (("ba", r["g_ba"], ba0), ("be", r["g_be"], be0)):
            adj_s, fd_s, var_s = 0.0, 0.0, 0.0
            for j in np.argsort(-np.abs(g * x0))[:8]:
                xp, xm = x0.copy(), x0.copy()
                xp[j] = np.float32(x0[j] * (1 + h))
                xm[j] = np.float32(x0[j] * (1 - h))
                step = (float(xp[j]) - float(xm[j])) / float(x0[j])  # the step as float32 rounds it
                if kind == "ba":
                    cp, cm = counts(be0, xp), counts(be0, xm)
                else:
                    cp, cm = counts(xp, ba0), counts(xm, ba0)
                d = cp - cm
                fd = d.sum() / step
                if kind == "ba":
                    var = max(abs(d.sum()), 1.0) / step ** 2
                else:
                    var = max(K * d.sum(1).var(ddof=1), np.abs(d.sum(0)).sum()) / step ** 2
                adj = float(g[j] * x0[j])
                rows.append((h, kind, int(j), round(adj), round(fd), round(np.sqrt(var))))
                if abs(adj - fd) > 0.02 * abs(fd) + 3 * np.sqrt(var):
                    fails.append(rows[-1])
                adj_s += adj
                fd_s += fd
                var_s += var
            rows.append((h, kind, "sum", round(adj_s), round(fd_s), round(np.sqrt(var_s))))
            if abs(adj_s - fd_s) > 0.02 * abs(fd_s) + 3 * np.sqrt(var_s):
                fails.append(rows[-1])
    print("per-layer adjoint vs central differences (h, kind, layer, x_j dN/dx_j, FD, standard error):", rows)
    assert not fails, fails
    c.close()


def test_gradient_graph_matches_eager_gradient(ice_full):
    """One fit iteration as a CUDA graph gives what the eager gradient gives, for the starting
    ice and after new coefficients: the same charges (per-photon streams: the same photons),
    the log-likelihood and gradient to rounding (sums in another order)."""
    c = _ctx(ice_full)
    be0, ba0 = c.get_ice()
    b = _bunches(c, 20_000_000)
    b["q"] = [0, 1]
    gs = c.info()["gsize"]
    obs = c.gradient(b, weights=np.zeros(2 * gs, np.float32), events=2)["counts"].astype(np.float32) * 1.05
    G = c.gradient_graph(b, obs, events=2)
    rng = np.random.default_rng(8)
    for be, ba in ((be0, ba0), ((be0 * rng.uniform(0.95, 1.05, len(be0))).astype(np.float32),
                                (ba0 * rng.uniform(0.95, 1.05, len(ba0))).astype(np.float32))):
        rg = G.run(be, ba)
        c.set_ice(be, ba)
        re = c.gradient(b, observed=obs, events=2)
        assert np.array_equal(rg["counts"], re["counts"])
        assert abs(rg["ll"] - re["ll"]) <= 1e-9 * abs(re["ll"])
        for k in ("g_be", "g_ba"):
            assert np.allclose(rg[k], re[k], rtol=1e-9, atol=1e-9 * np.abs(re[k]).max()), k
        assert rg["info"]["hits"] == re["info"]["hits"] and rg["info"]["replayed"] == re["info"]["replayed"]
    G.close()
    c.close()


def test_likelihood_weights(ice_full):
    """observed counts -> LL = sum k log mu - mu and w_d = k_d/mu_d - 1, the gradient equal
    to the one with those weights given explicitly."""
    c = _ctx(ice_full)
    be0, ba0 = c.get_ice()
    b = _bunches(c, 20_000_000)
    rng = np.random.default_rng(3)
    c.set_ice(be0 * (1 + 0.1 * rng.standard_normal(len(be0))).astype(np.float32),
              ba0 * (1 + 0.1 * rng.standard_normal(len(ba0))).astype(np.float32))
    obs = c.gradient(b, weights=np.zeros(c.info()["gsize"], np.float32))["counts"].astype(np.float32)
    c.set_ice(be0, ba0)
    r = c.gradient(b, observed=obs)
    mu = r["counts"].astype(np.float64)
    m = mu > 0
    ll = float(np.sum(obs[m] * np.log(mu[m]) - mu[m]))
    assert abs(r["ll"] - ll) <= 1e-9 * abs(ll)
    w = np.where(m, obs / np.where(m, mu, 1) - 1, 0).astype(np.float32)
    rw = c.gradient(b, weights=w)
    assert np.array_equal(rw["counts"], r["counts"])
    assert np.allclose(rw["g_ba"], r["g_ba"], rtol=1e-6, atol=1e-9 * np.abs(r["g_ba"]).max())
    assert np.allclose(rw["g_be"], r["g_be"], rtol=1e-6, atol=1e-9 * np.abs(r["g_be"]).max())
    c.close()


def test_autograd_function_returns_the_gradient(ice_full):
    import torch

    from ppc_b200.adjoint import IceLikelihood
    c = _ctx(ice_full)
    be0, ba0 = c.get_ice()
    b = _bunches(c, 5_000_000)
    obs = c.gradient(b, weights=np.zeros(c.info()["gsize"], np.float32))["counts"].astype(np.float32) * 1.1
    params = torch.tensor(np.stack([be0, ba0]).astype(np.float64), requires_grad=True)
    ll = IceLikelihood.apply(params, c, b, obs, 1.0)
    ll.backward()
    r = c.gradient(b, observed=obs)
    assert abs(float(ll.detach()) - r["ll"]) <= 1e-9 * abs(r["ll"])
    assert np.allclose(params.grad[0].numpy(), r["g_be"]) and np.allclose(params.grad[1].numpy(), r["g_ba"])
    c.close()


def test_gradient_costs_at_most_three_forward_passes(ice_full):
    c = _ctx(ice_full, deterministic=False)
    b = _bunches(c, 50_000_000)
    r = c.gradient(b, weights=np.ones(c.info()["gsize"], np.float32))
    i = r["info"]
    print("forward ms", i["forward_ms"], "backward ms", i["backward_ms"])
    assert i["forward_ms"] + i["backward_ms"] <= 3 * i["forward_ms"], i
    c.close()


def test_per_event_charge_bins(ice_full):
    """events > 0: charges binned per (event, DOM) with the event = the bunch's q; their sum
    over events is the per-DOM histogram, and event-independent weights give the per-DOM
    gradient (per-photon streams make the two runs identical)."""
    c = _ctx(ice_full)
    b = _bunches(c, 5_000_000)
    gs = c.info()["gsize"]
    v = np.random.default_rng(5).uniform(-1, 1, gs).astype(np.float32)
    r0 = c.gradient(b, weights=v)
    r1 = c.gradient(b, weights=np.tile(v, (len(FLASHERS), 1)), events=len(FLASHERS))
    assert r1["counts"].shape == (len(FLASHERS), gs)
    assert np.array_equal(r1["counts"].sum(axis=0), r0["counts"])
    assert r1["counts"][0].sum() > 0 and r1["counts"][1].sum() > 0
    assert np.allclose(r1["g_ba"], r0["g_ba"], rtol=1e-6, atol=1e-9 * np.abs(r0["g_ba"]).max())
    assert np.allclose(r1["g_be"], r0["g_be"], rtol=1e-6, atol=1e-9 * np.abs(r0["g_be"]).max())
    with pytest.raises(ValueError):
        c.gradient(b, weights=v, events=len(FLASHERS))
    c.close()


def _smooth_field(rng, n, corr=4.0):
    x = rng.normal(size=n + 20)
    k = np.exp(-0.5 * (np.arange(-10, 11) / corr) ** 2)
    f = np.convolve(x, k / k.sum(), mode="same")[10:10 + n]
    return f / f.std()


def test_lbfgs_fit_recovers_absorption(ice_full):
    """L-BFGS on the adjoint gradient, with a smoothness penalty between neighbouring layers,
    moves the absorption of the illuminated layers towards a hidden ice (ba scaled by
    exp(0.1 x a smooth unit-variance field in depth)) whose charges were simulated with other
    random numbers.  Without the penalty the 10 m layers trade off against each other and
    the fit chases noise."""
    from ppc_b200.fit import fit_ice
    rng = np.random.default_rng(21)
    truth = _ctx(ice_full, seed=99)
    be0, ba0 = truth.get_ice()
    oms = truth.tables()["oms"]
    ne = 64
    doms = rng.choice(len(oms), ne, replace=False)
    b = np.concatenate([W.flasher(int(k), oms["r"][k], 3_000_000, q=i) for i, k in enumerate(doms)])
    ba_true = (ba0 * np.exp(0.1 * _smooth_field(rng, len(ba0)))).astype(np.float32)
    truth.set_ice(be0, ba_true)
    gs = truth.info()["gsize"]
    obs = truth.gradient(b, weights=np.zeros(ne * gs, np.float32), events=ne)["counts"].astype(np.float32)
    truth.close()
    c = _ctx(ice_full, seed=7)
    g0 = c.gradient(b, observed=obs, events=ne)
    lit = np.abs(g0["g_ba"] * ba0) > 0.1 * np.abs(g0["g_ba"] * ba0).max()
    r = fit_ice(c, b, obs, ne, iters=15, fit=("ba",), smooth=1e3)
    err0 = np.sqrt(np.mean((ba0[lit] / ba_true[lit] - 1) ** 2))
    err1 = np.sqrt(np.mean((r["ba"][lit] / ba_true[lit] - 1) ** 2))
    lls = [h["ll"] for h in r["history"]]
    print(f"fit: {lit.sum()} lit layers, rms error {err0:.4f} -> {err1:.4f}, LL {lls[0]:.1f} -> {r['ll']:.1f}, "
          f"{r['accepted']}/{r['iterations']} steps kept, {r['seconds_per_iteration']:.2f} s/iteration")
    assert r["ll"] > lls[0]
    assert err1 < 0.85 * err0
    c.close()


def _scaled_ice(src, dst, ba_scale):
    """A copy of ice directory `src` with every layer's absorption (icemodel.dat column 3)
    scaled by ba_scale."""
    import shutil
    shutil.copytree(src, dst)
    rows = open(os.path.join(src, "icemodel.dat")).read().split("\n")
    out = []
    for line in rows:
        f = line.split()
        if len(f) >= 3:
            f[2] = "%.9g" % (float(f[2]) * ba_scale)
        out.append(" ".join(f))
    open(os.path.join(dst, "icemodel.dat"), "w").write("\n".join(out))


def _reference_cpu_hits(ice, spec, photons, procs, seed0, env):
    """Kernel-level hits of the reference's own CPU build (oracle/_ref/ref_harness_fm),
    `procs` processes with distinct seeds sharing `photons`."""
    import json
    import subprocess
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness_fm")
    e = dict(os.environ, PPCTABLESDIR=ice, PPCB_QUIET="1", **env)
    ps = [subprocess.Popen([exe, "run", spec, str(photons // procs), str(seed0 + k), "/tmp/ppcb_fd", "nodump"], env=e,
                           stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for k in range(procs)]
    hits = 0
    for p in ps:
        out, _ = p.communicate()
        hits += json.loads([l for l in out.splitlines() if l.startswith("{")][-1])["hits"]
    return hits, procs * (photons // procs)


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_harness_fm")),
                    reason="reference CPU build not present")
def test_gradient_agrees_with_reference_cpu_finite_differences(ice_full, tmp_path):
    """The adjoint's derivative of the expected hit count along all absorption coefficients
    (d/dt of N at ba x (1 + t)) against a central difference of the reference's own CPU
    build (gpu/ppc.cu compiled with its flags) at t = +-0.1, one flasher (string 21, DOM 30,
    12-fold LEDs at 30 degrees), 6e7 photons per side on the host cores.  The CPU side has
    no common random numbers, so the tolerance is 3.5 Poisson standard deviations plus 3%
    for the curvature of exp(-absorption) over the step."""
    h = 0.1
    k = 20 * 60 + 29
    cpus = max(1, min(32, os.cpu_count() or 1))
    env = {"FLDR": "3960", "ELEV": "30", "FWID": "9.7"}
    n_ref = 60_000_000
    plus, minus = str(tmp_path / "plus"), str(tmp_path / "minus")
    _scaled_ice(ice_full, plus, 1 + h)
    _scaled_ice(ice_full, minus, 1 - h)
    hp, n1 = _reference_cpu_hits(plus, "flasher:21:30", n_ref, cpus, 100, env)
    hm, n2 = _reference_cpu_hits(minus, "flasher:21:30", n_ref, cpus, 200, env)
    fd = (hp - hm) / (2 * h) / n1
    sigma = np.sqrt(hp + hm) / (2 * h) / n1
    c = _ctx(ice_full)
    be0, ba0 = c.get_ice()
    oms = c.tables()["oms"]
    b = W.flasher(k, oms["r"][k], 200_000_000, q=0)
    r = c.gradient(b, weights=np.ones(c.info()["gsize"], np.float32), hit_cap=2_000_000)
    adj = float(np.dot(r["g_ba"], ba0)) / 200_000_000
    print(f"dN/dt per photon: adjoint {adj:.4e}, reference CPU central difference {fd:.4e} +- {sigma:.1e} "
          f"({hp} / {hm} hits of {n1} photons per side, {cpus} processes)")
    assert np.sign(adj) == np.sign(fd)
    assert abs(adj - fd) <= 3.5 * sigma + 0.03 * abs(fd), (adj, fd, sigma)
    c.close()
