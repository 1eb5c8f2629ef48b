"""Statistical parity with the reference (totals within 0.1%, per-DOM counts within 3
sigma, hit-time KS p > 0.01), against high-statistics
fixtures made by the reference's own CPU build (tests/golden/make_parity_fixture.py:
gpu/ppc.cu + gpu/pro.cu compiled with its --fast-math flags, thousands of seeds).

Workloads:
  small_point   the 7-string detector, isotropic 405 nm point source at the origin, 1e6
                photons per reference run (2.8e9 photons, ~2e7 kernel-level hits);
  full_cascade  the full detector (tilt, anisotropy, birefringence), one EM cascade at
                (12.5, -40, 60) m along (0.6, 0, 0.8) (2e9 photons).

The GPU propagates the reference's own bunch record (stored in the fixture) with per-photon
random streams from a fixed seed (a fixed sample for a given build, so that the test gives
the same answer every run), and the kernel-level hits are compared:
  * total hits per photon within 0.1% of the reference's (small_point, where the two
    samples resolve it: 0.1% is more than 3.5 combined standard deviations), and within
    4 standard deviations for both workloads;
  * per-DOM counts within 3 Poisson standard deviations: the number of DOMs beyond 3 sigma
    is what chance gives for that many DOMs (0.27% of them, plus 4 binomial standard
    deviations), and no DOM is beyond the Bonferroni bound for a family-wise ALPHA (1e-4);
  * per-DOM hit-time distributions: two-sample KS test on the fixture's time bins (binning
    only lowers the statistic, so the p-values are conservative) for every DOM with at
    least 1000 hits on each side; p > 0.01 for all but the fraction chance gives (1%, plus
    4 binomial standard deviations), none below the Bonferroni bound ALPHA/DOMs, and the
    pooled time distribution at p > ALPHA.
"""
import os

import numpy as np
import pytest

from conftest import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

from ppc_b200 import types as T  # noqa: E402
from ppc_b200.api import PPC  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# False-alarm probability of each family-wise check (the largest |z|, the smallest KS p-value
# over the DOMs, the pooled KS): a deviation the checks must catch gives p-values many orders
# of magnitude below it at these sample sizes.
ALPHA = 1e-4


def _ks_binned(h1, h2):
    """Two-sample KS statistic on binned counts and its asymptotic p-value."""
    from scipy import stats
    n1, n2 = h1.sum(), h2.sum()
    d = np.abs(np.cumsum(h1) / n1 - np.cumsum(h2) / n2).max()
    ne = n1 * n2 / (n1 + n2)
    return d, stats.kstwobign.sf(d * np.sqrt(ne))


def _gpu_histograms(ice, bunch, photons, edges, env, monkeypatch, chunk=200_000_000, seed=97):
    import torch
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(seed)
    c.set_options(photon_streams=True)  # a fixed sample for a given build: the test does not flicker
    c.choose(0)
    c.ini()
    ndom = c.params().gsize
    b = bunch.copy()
    cap = 1 << 24
    d_h = torch.empty((cap, 32), dtype=torch.uint8, device="cuda")
    d_c = torch.zeros(56, dtype=torch.uint8, device="cuda")
    d_e = torch.from_numpy(edges).cuda()
    counts = torch.zeros(ndom, dtype=torch.int64, device="cuda")
    hist = torch.zeros(ndom * (len(edges) - 1), dtype=torch.int64, device="cuda")
    done = 0
    while done < photons:
        num = min(chunk, photons - done)
        c.set_seed(seed + done // chunk)  # per-photon streams are keyed by (seed, photon index in the launch)
        b["num"] = num
        d_b = torch.from_numpy(b.view(np.uint8).copy()).cuda()
        d_s = torch.tensor([0, num], dtype=torch.int64, device="cuda")
        d_c.zero_()
        c.propagate_device(d_b.data_ptr(), d_s.data_ptr(), 1, num, d_h.data_ptr(), cap, d_c.data_ptr())
        torch.cuda.synchronize()
        ctrl = T.Ctrl.from_buffer_copy(d_c.cpu().numpy().tobytes())
        assert ctrl.hidx <= cap and ctrl.nan_steps == 0
        h = d_h[:ctrl.hidx]
        dom = h[:, 0:4].contiguous().view(torch.int32).reshape(-1).long()
        t = h[:, 12:16].contiguous().view(torch.float32).reshape(-1).double()
        counts += torch.bincount(dom, minlength=ndom)
        tb = (torch.bucketize(t, d_e, right=True) - 1).clamp(0, len(edges) - 2)
        hist += torch.bincount(dom * (len(edges) - 1) + tb, minlength=hist.numel())
        done += num
    c.close()
    return counts.cpu().numpy(), hist.cpu().numpy().reshape(ndom, len(edges) - 1)


@pytest.mark.parametrize("case,gpu_photons", [("small_point", 6_000_000_000), ("full_cascade", 8_000_000_000)])
def test_high_statistics_parity(case, gpu_photons, request, monkeypatch):
    from scipy import stats
    fx = np.load(os.path.join(GOLDEN, f"parity_{case}.npz"))
    kind = str(fx["kind"])
    ice = request.getfixturevalue("ice_" + kind)
    env = {"FWID": "-1", "WFLA": "405"} if case == "small_point" else {}
    bunch = fx["bunch"].view(T.BUNCH_DTYPE).copy()
    edges = fx["edges"]
    cg, hg = _gpu_histograms(ice, bunch, gpu_photons, edges, env, monkeypatch)
    cr, hr = fx["counts"].astype(np.int64), fx["hist"].astype(np.int64)
    nr = int(fx["photons"])
    # totals
    rg, rr = cg.sum() / gpu_photons, cr.sum() / nr
    sig = np.sqrt(cg.sum() / gpu_photons ** 2 + cr.sum() / nr ** 2)
    print(f"{case}: GPU {cg.sum()} hits / {gpu_photons:.2e}, reference {cr.sum()} / {nr:.2e}; "
          f"ratio {rg / rr:.5f} ({(rg - rr) / sig:+.2f} sigma, sigma {sig / rr:.2e})")
    assert abs(rg - rr) < 4 * sig
    if case == "small_point":
        assert 3 * sig / rr < 1e-3  # the samples resolve 0.1% ...
        assert abs(rg / rr - 1) < 1e-3  # ... and the totals agree within it
    # per DOM, at 3 Poisson sigma
    s = nr / gpu_photons
    sel = cr >= 25
    z = (cg[sel] * s - cr[sel]) / np.sqrt(cg[sel] * s * s + cr[sel])
    m = int(sel.sum())
    beyond = int((np.abs(z) > 3).sum())
    expect = 0.0027 * m
    zmax = stats.norm.isf(ALPHA / (2 * m))
    print(f"{case}: {m} DOMs, {beyond} beyond 3 sigma (chance {expect:.1f}), max |z| {np.abs(z).max():.2f} "
          f"(bound {zmax:.2f})")
    assert beyond <= expect + 4 * np.sqrt(expect * (1 - 0.0027)) + 1
    assert np.abs(z).max() < zmax
    # hit times per DOM
    ps = []
    for d in np.flatnonzero((cr >= 1000) & (cg >= 1000)):
        ps.append(_ks_binned(hg[d], hr[d])[1])
    ps = np.array(ps)
    low = int((ps < 0.01).sum())
    print(f"{case}: KS on {len(ps)} DOMs, {low} below p 0.01, min p {ps.min():.2e}")
    assert len(ps) >= 10
    assert low <= 0.01 * len(ps) + 4 * np.sqrt(0.01 * 0.99 * len(ps)) + 1
    assert ps.min() > ALPHA / len(ps)
    D, p = _ks_binned(hg.sum(0), hr.sum(0))
    print(f"{case}: pooled times KS D={D:.2e} p={p:.3f}")
    assert p > ALPHA
