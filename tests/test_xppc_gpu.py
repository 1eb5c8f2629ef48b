"""The drop-in path end to end on the GPU: the reference's library API (llh/ppc.h
semantics: flset, sett, flone, eout, hitz, efin) from Python and from a C++ program linked
against libxppc.so, with the host back end (acceptance, PMT assignment, time binning)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

from ppc_b200.api import PPC  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_eout_fills_hitz_with_accepted_hits(ice_full, monkeypatch):
    monkeypatch.setenv("FLDR", "3960")
    monkeypatch.setenv("ELEV", "30")
    c = PPC()
    c.initialize(1.0, ice_full)
    c.set_seed(21)
    c.choose(0)
    c.ini()
    c.keep_raw(True)
    c.set_res(10.0)  # 10 ns time bins
    total, nraw = 0, 0
    for e, (s, om) in enumerate([(21, 30), (45, 36), (60, 10)]):
        c.flset(s, om)
        c.sett(0.0, 0.0, 1.0, (e, 7), 0)
        c.flone(5_000_000)
        c.eout()
        h = c.hitz()
        assert len(h) > 0
        assert set(h["track_first"]) == {e} and set(h["track_second"]) == {7}
        assert h["str"].min() >= 1 and h["str"].max() <= 86 and h["om"].min() >= 1 and h["om"].max() <= 60
        assert np.allclose(h["time"] / 10.0 - np.floor(h["time"] / 10.0), 0.5)  # bin centres
        assert np.all(np.isfinite(h["r"])) and np.all(np.isfinite(h["n"]))
        assert np.allclose(np.linalg.norm(h["n"][:, :3], axis=1), 1, atol=1e-4)
        raw = c.raw_hits()
        assert set(raw["n"]) == {e + 1}  # this event's segment
        assert len(h) <= len(raw)  # acceptance keeps a fraction of the kernel-level hits
        total += len(h)
        nraw += len(raw)
        c.efin()  # clears the event's hit map and kernel-level hits
        assert len(c.hitz()) == 0 and len(c.raw_hits()) == 0
    assert 0 < total < nraw
    last, tot = c.last_run()
    assert tot["photons"] > 0 and tot["hits"] >= nraw
    c.close()


LLH_LIKE = r"""
#include <cmath>
#include <cstdio>
#include <map>
#include <vector>
#include "xppc.h"
int main() {
  xppc::start();
  xppc::initialize(1.f);
  xppc::choose(0);
  xppc::ini();
  xppc::flset(21, 30);
  xppc::sett(0, 0, 1, std::make_pair(3, 9ULL), 0);
  xppc::flone(40000000);
  xppc::eout();
  size_t n = 0;
  for (xppc::outz::const_iterator i = xppc::hitz.begin(); i != xppc::hitz.end(); ++i) n += i->second.size();
  printf("hitz %zu\n", n);
  xppc::efin();
  xppc::fin();
  printf("device %g\n", xppc::getTotalDeviceTime());
  xppc::stop();
  return n > 0 ? 0 : 1;
}
"""


def test_program_linked_against_libxppc_runs(ice_full, tmp_path, monkeypatch):
    lib = os.path.join(ROOT, "ppc_b200", "lib")
    src = tmp_path / "llh_like.cxx"
    src.write_text(LLH_LIKE)
    exe = tmp_path / "llh_like"
    r = subprocess.run(["g++", "-O1", "-std=c++11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L" + lib, "-lxppc", "-Wl,-rpath," + lib], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    env = dict(os.environ, PPCTABLESDIR=ice_full, FLDR="3960", ELEV="30")
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, (r.stdout[-500:], r.stderr[-2000:])
    n = int([l for l in r.stdout.splitlines() if l.startswith("hitz")][0].split()[1])
    # the same flasher through the Python path of the same library: the two counts are
    # independent Poisson-like samples of one mean, so they agree within 5 sigma
    monkeypatch.setenv("FLDR", "3960")
    monkeypatch.setenv("ELEV", "30")
    c = PPC()
    c.initialize(1.0, ice_full)
    c.choose(0)
    c.ini()
    c.flset(21, 30)
    c.sett(0.0, 0.0, 1.0, (3, 9), 0)
    c.flone(40_000_000)
    c.eout()
    m = len(c.hitz())
    c.efin()
    c.close()
    assert m > 300, m  # the mean is about 1000 hits: this floor is more than 20 sigma below it
    assert abs(n - m) < 5 * np.sqrt(n + m), (n, m)


def test_device_back_end_matches_host_back_end(ice_full2d, monkeypatch):
    """ppcb_accept (the back end on the GPU) against eout()'s host back end on the same
    kernel-level hits, on a detector with tilted sensor axes and cable azimuths: the two draw
    different random numbers, so the accepted fraction, the per-DOM counts and the
    wavelength and time distributions agree statistically, and a hit both accept carries
    the same impact point and direction."""
    from scipy import stats
    monkeypatch.setenv("FLDR", "3960")
    monkeypatch.setenv("ELEV", "30")
    c = PPC()
    c.initialize(1.0, ice_full2d)
    c.set_seed(5)
    c.set_options(deterministic=True)  # photon i on thread i mod T: a fixed sample for a given build
    c.choose(0)
    c.ini()
    c.keep_raw(True)
    raws, hosts = [], []
    for e, (s, om) in enumerate([(40, 30), (21, 20), (60, 40), (5, 50)]):
        c.flset(s, om)
        c.sett(0.0, 0.0, 1.0, (e, 7), 0)
        c.flone(600_000_000)
        c.eout()
        hosts.append(c.hitz())
        raws.append(c.raw_hits())
        c.efin()
    raw = np.concatenate(raws)
    host = np.concatenate(hosts)
    dev = c.accept(raw, seed=11)
    c.close()
    n = len(raw)
    assert n > 50000 and len(host) > 5000, (n, len(host))
    assert np.all(np.diff(dev["hit"].astype(np.int64)) > 0)  # input order
    p_host, p_dev = len(host) / n, len(dev) / n
    sd = np.sqrt(2 * p_host * (1 - p_host) / n)
    assert abs(p_host - p_dev) < 4 * sd, (p_host, p_dev, sd)
    # per-DOM counts (two-sample chi-square over DOMs with enough hits)
    key_h = host["str"].astype(np.int64) * 100 + host["om"]
    key_d = dev["str"].astype(np.int64) * 100 + dev["om"]
    doms = np.union1d(key_h, key_d)
    ch = np.array([np.count_nonzero(key_h == k) for k in doms])
    cd = np.array([np.count_nonzero(key_d == k) for k in doms])
    m = ch + cd >= 30
    assert m.sum() >= 10
    p_chi = stats.chi2_contingency(np.vstack([ch[m], cd[m]]))[1]
    assert p_chi > 1e-3, p_chi
    assert stats.ks_2samp(host["n"][:, 3], dev["wv"]).pvalue > 0.01
    assert stats.ks_2samp(host["r"][:, 3], dev["t"]).pvalue > 0.01
    # hits both back ends accepted: same geometry.  A host record is traced to its
    # kernel-level hit by (event, arrival time); times two hits share are left out.
    index = {}
    base = 0
    for e, r in enumerate(raws):
        for j, t in enumerate(r["t"]):
            key = (e + 1, float(t))
            index[key] = -1 if key in index else base + j
        base += len(r)
    at = {int(k): j for j, k in enumerate(dev["hit"])}
    both = ambiguous = 0
    for h in host:
        k = index.get((int(h["track_first"]) + 1, float(h["r"][3])))
        assert k is not None
        if k < 0:
            ambiguous += 1
            continue
        j = at.get(k)
        if j is None:
            continue
        both += 1
        d = dev[j]
        assert d["str"] == h["str"] and d["om"] == h["om"]
        assert np.allclose(d["r"], h["r"][:3], atol=2e-5) and np.allclose(d["d"], h["n"][:3], atol=2e-5)
    assert ambiguous < 0.05 * len(host)
    assert both > 0.5 * min(len(host), len(dev)) * p_dev, (both, len(host), len(dev), p_dev)


def _module_kind(s):
    return np.where(s <= 20, 1, np.where(s <= 35, 2, np.where(s <= 45, 3, 0)))


def test_device_back_end_multi_pmt_matches_host_back_end(ice_full_ng):
    """Multi-PMT sensors on the device (24-PMT spheres, 2-PMT spheroids, shifting tubes)
    against the host back end, which is pinned bit for bit to the reference's: accepted
    fraction per module type, counts per (module type, PMT), and the tubes' transit delays."""
    from scipy import stats
    c = PPC()
    c.initialize(1.0, ice_full_ng)
    c.set_seed(8)
    c.set_options(deterministic=True)  # photon i on thread i mod T: a fixed sample for a given build
    c.choose(0)
    c.ini()
    c.keep_raw(True)
    raws, hosts = [], []
    for e, (x, y, z) in enumerate([(20.0, -60.0, -100.0), (-50.0, 310.0, 50.0), (-360.0, 10.0, 0.0)] * 2):
        c.sett(0.3, 0.4, 0.8660254, (e, 7), 0)
        c.addp(x, y, z, 0.0, 20000.0, 0.0, 11)
        c.eout()
        hosts.append(c.hitz())
        raws.append(c.raw_hits())
        c.efin()
    raw = np.concatenate(raws)
    host = np.concatenate(hosts)
    dev = c.accept(raw, seed=13)
    c.close()
    rs = raw["i"].astype(np.int64) // 60 + 1
    rk, hk, dk = _module_kind(rs), _module_kind(host["str"]), _module_kind(dev["str"])
    for k in (1, 2, 3):
        n = int((rk == k).sum())
        nh, nd = int((hk == k).sum()), int((dk == k).sum())
        assert n > 3000 and nh > 500, (k, n, nh)
        p = (nh + nd) / (2 * n)
        assert abs(nh - nd) / n < 4 * np.sqrt(2 * p * (1 - p) / n), (k, n, nh, nd)
    # PMT choice: counts per (module type, PMT)
    cat_h = hk * 100 + host["pmt"]
    cat_d = dk * 100 + dev["pmt"]
    cats = np.union1d(cat_h, cat_d)
    ch = np.array([np.count_nonzero(cat_h == x) for x in cats])
    cd = np.array([np.count_nonzero(cat_d == x) for x in cats])
    m = ch + cd >= 30
    assert m.sum() >= 20
    assert stats.chi2_contingency(np.vstack([ch[m], cd[m]]))[1] > 1e-3
    # tubes: transit delays added to the hit time
    tube = dk == 3
    d_shift = dev["t"][tube] - raw["t"][dev["hit"][tube]]
    assert np.all(d_shift > 0)
    key = {}
    for e, r in enumerate(raws):
        s = r["i"].astype(np.int64) // 60 + 1
        nz = np.cos(r["pth"]).astype(np.float32)
        for j in np.nonzero(_module_kind(s) == 3)[0]:
            key.setdefault((e, int(r["i"][j]), round(float(nz[j]), 4)), []).append(float(r["t"][j]))
    h_shift = []
    for h in host[hk == 3]:
        ts = key.get((int(h["track_first"]), (int(h["str"]) - 1) * 60 + int(h["om"]) - 1, round(float(h["n"][2]), 4)))
        if ts is not None and len(ts) == 1:
            h_shift.append(float(h["r"][3]) - ts[0])
    h_shift = np.array(h_shift)
    assert len(h_shift) > 0.7 * (hk == 3).sum()
    assert stats.ks_2samp(h_shift, d_shift).pvalue > 0.01
