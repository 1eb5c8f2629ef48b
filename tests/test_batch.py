"""Batched events: one persistent launch, per-event hit regions, graph replay, autotuner.
Every event's hits must be its own, and per-event hit counts must agree with propagating
the events one by one (the reference's way, one eout() per source)."""
import numpy as np
import pytest

from conftest import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

from ppc_b200 import workloads as W  # noqa: E402
from ppc_b200.api import PPC, Batch  # noqa: E402


def _ctx(ice, seed=31):
    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(seed)
    c.choose(0)
    c.ini()
    return c


def test_batch_events_keep_their_hits(ice_full):
    c = _ctx(ice_full)
    ev = W.batched_events(c.tables()["oms"], n_events=300, lo=1e3, hi=3e5, seed=4)
    b = Batch(c, max_events=512, max_bunches=1024, hit_capacity=1 << 24)
    info = b.run(ev, len(ev), hits_per_photon=0.05)
    assert info["photons"] == int(ev["num"].sum())
    assert info["overflowed"] == 0 and info["kept"] == info["hits"]
    produced, off = b.counts()
    hits = b.hits()
    assert len(hits) == off[-1] == produced.sum()
    for e in range(len(ev)):
        seg = hits[off[e]:off[e + 1]]
        assert np.all(seg["n"] == e)
    # graph replay and direct launch agree statistically
    b.set_graph(False)
    info2 = b.run(ev, len(ev), hits_per_photon=0.05)
    assert abs(info2["hits"] - info["hits"]) < 5 * np.sqrt(info["hits"] + 1)
    b.close()
    c.close()


def test_batch_matches_one_event_at_a_time(ice_full):
    """Per-event hit counts: batched vs separate launches (chi-square over events)."""
    from scipy import stats
    c = _ctx(ice_full, seed=77)
    ev = W.batched_events(c.tables()["oms"], n_events=60, lo=2e5, hi=2e6, seed=8)
    b = Batch(c, max_events=64, max_bunches=64, hit_capacity=1 << 24)
    b.run(ev, len(ev), hits_per_photon=0.05)
    pb, _ = b.counts()
    single = np.zeros(len(ev))
    for e in range(len(ev)):
        x = ev[e:e + 1].copy()
        h, info = c.propagate(x)
        single[e] = info["hits"]
    sel = (single + pb) >= 20
    chi2 = (((pb[sel] - single[sel]) ** 2) / (pb[sel] + single[sel])).sum()
    p = stats.chi2.sf(chi2, sel.sum())
    assert p > 1e-3, (chi2, sel.sum(), p)
    b.close()
    c.close()


def test_batch_overflow_is_counted_not_written(ice_full):
    c = _ctx(ice_full, seed=3)
    ev = W.batched_events(c.tables()["oms"], n_events=40, lo=1e5, hi=1e6, seed=2)
    b = Batch(c, max_events=64, max_bunches=64, hit_capacity=1 << 20)
    info = b.run(ev, len(ev), hits_per_photon=0.0)   # 64 slots per event
    produced, off = b.counts()
    assert info["overflowed"] == int((produced > 64).sum()) > 0
    assert np.all(np.diff(off) == np.minimum(produced, 64))
    b.close()
    c.close()


def test_autotune_picks_a_working_shape(ice_full):
    c = _ctx(ice_full, seed=9)
    ev = W.batched_events(c.tables()["oms"], n_events=200, lo=1e3, hi=1e6, seed=1)
    b = Batch(c, max_events=256, max_bunches=256, hit_capacity=1 << 24)
    t = b.autotune(ev, len(ev), sample_photons=5_000_000)
    assert t["threads"] in (128, 256, 768, 864) and t["photons_per_s"] > 0
    info = b.run(ev, len(ev), hits_per_photon=0.05)
    assert info["photons"] == int(ev["num"].sum()) and info["overflowed"] == 0
    b.close()
    c.close()
