"""DirectFit's likelihood on the GPU (ppcb_llh_eval) against the oracle.  The observed
pulses come from one flasher event through the host back end; the simulated side is the
kernel-level hits of a second, larger run.  The device applies the back end's acceptance
itself; the oracle gets the hits that PPC.accept accepts with the same seed, so both see
the same simulated hits and must agree to rounding."""
import os

import numpy as np
import pytest

from conftest import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

import oracle_util as O  # noqa: E402
from ppc_b200 import types as T  # noqa: E402
from ppc_b200.api import PPC, Likelihood, PPCError  # noqa: E402


@pytest.fixture(scope="module")
def runs(ice_full2d):
    env = {k: os.environ.get(k) for k in ("FLDR", "ELEV")}
    os.environ.update(FLDR="3960", ELEV="30")
    try:
        c = PPC()
        c.initialize(1.0, ice_full2d)
        c.set_seed(5)
        c.choose(0)
        c.ini()
        c.keep_raw(True)
        c.flset(40, 30)
        c.sett(0.0, 0.0, 1.0, (0, 7), 0)
        c.flone(300_000_000)
        c.eout()
        obs = c.hitz()
        c.efin()
        c.flset(40, 30)
        c.sett(0.0, 0.0, 1.0, (1, 7), 0)
        c.flone(600_000_000)
        c.eout()
        raw = c.raw_hits()
        c.efin()
    finally:
        for k, v in env.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    data = np.zeros(len(obs), T.LLH_HIT_DTYPE)
    data["str"], data["om"], data["t"], data["q"] = obs["str"], obs["om"], obs["r"][:, 3], 1.0
    yield c, data, raw
    c.close()


def _windows(data):
    keys = np.unique(data[["str", "om"]])
    w = np.zeros(3, T.LLH_WINDOW_DTYPE)
    for k in range(3):
        sel = data[(data["str"] == keys[k]["str"]) & (data["om"] == keys[k]["om"])]
        w[k] = (keys[k]["str"], keys[k]["om"], np.median(sel["t"]) - 30.0, np.median(sel["t"]) + 30.0)
    return w


CASES = {
    "defaults": ({}, False, False),
    # norm divides by each DOM's observed charge inside the 200 bins: pulses within 4000 ns
    # keep every DOM's charge inside them
    "norm": ({"norm": 1}, False, False),
    "peak_mono": ({"peak": 1, "mono": 1}, False, False),
    "no_model_error": ({"sig": 0.0}, False, False),
    "drep2_lbin20": ({"drep": 2.0, "lbin": 20.0}, False, False),
    "unh_bad_windows": ({"unh": 1}, True, True),
    "flasher": ({"flasher": 1, "fla_str": 40, "fla_om": 30, "fsep": 1, "unh": 1}, False, False),
}


@pytest.mark.parametrize("name", list(CASES))
def test_device_likelihood_matches_oracle(runs, name):
    c, data, raw = runs
    opts, use_bad, use_win = CASES[name]
    if opts.get("norm"):
        data = data[data["t"] < data["t"].min() + 4000.0]
    keys = np.unique(data[["str", "om"]])
    bad = np.array([[keys[4]["str"], keys[4]["om"]], [keys[9]["str"], keys[9]["om"]]], np.int32) if use_bad else None
    win = _windows(data) if use_win else None
    L = Likelihood(c, data, windows=win, bad=bad, **opts)
    assert len(data) > 2000 and len(raw) > 20000, (len(data), len(raw))
    info = L.info()
    assert info["doms"] > 10
    ob = O.llh_setup(data, windows=win, bad=bad, opts=opts)
    assert np.array_equal(L.blocks()["dat"], ob[0]["dat"]) and info["ndof"] == ob[3]
    dts = np.linspace(-150.0, 150.0, 13)
    out = L.eval(raw, dts, nsim=2.0, seed=17)
    acc = c.accept(raw, seed=17)
    ref, err = O.llh_fllh(data, acc, dts, 2.0, windows=win, bad=bad, opts=opts)
    assert err == 0 and L.info()["errors"] == 0
    assert np.all(np.isfinite(out))
    np.testing.assert_allclose(out, ref, rtol=1e-10, atol=1e-13)
    again = L.eval(raw, dts, nsim=2.0, seed=17)
    assert np.array_equal(out, again)  # fixed-order sums: bit for bit
    L.close()


def test_time_shift_scan_finds_the_true_offset(runs):
    """Observed and simulated hits come from the same flasher, so the best shift is near 0;
    hits moved by +120 ns move the minimum to -120 ns."""
    c, data, raw = runs
    L = Likelihood(c, data)
    dts = np.arange(-300.0, 301.0, 10.0)[:61]
    assert len(dts) <= 64
    out = L.eval(raw, dts, nsim=2.0, seed=3)
    assert abs(dts[np.argmin(out)]) <= 30.0, (dts[np.argmin(out)], out.min())
    moved = raw.copy()
    moved["t"] += np.float32(120.0)
    out2 = L.eval(moved, dts, nsim=2.0, seed=3)
    assert abs(dts[np.argmin(out2)] + 120.0) <= 30.0, dts[np.argmin(out2)]
    with pytest.raises(PPCError) as e:
        L.eval(raw, np.zeros(65), nsim=2.0)
    assert e.value.code == 7
    L.close()


def test_no_simulated_hits(runs):
    """Without simulated hits every block compares 0 against its observed charge."""
    c, data, _ = runs
    L = Likelihood(c, data)
    out = L.eval(np.zeros(0, T.HIT_DTYPE), [0.0, 7.0], nsim=2.0)
    ref, err = O.llh_fllh(data, np.zeros(0, O.LLHO_SIM_DTYPE), [0.0, 7.0], 2.0)
    assert err == 0 and out[0] == out[1]
    np.testing.assert_allclose(out, ref, rtol=1e-10)
    assert len(c.accept(np.zeros(0, T.HIT_DTYPE))) == 0  # the back end on no hits
    L.close()
