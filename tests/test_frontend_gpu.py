"""The source front end on the GPU (ppcb_sources) against the reference and the host front
end.  Bunch templates: the reference's own addp/yield (oracle/_ref/ref_harness, built from
the reference sources).  Photon counts: Poisson statistics, the hadronic light fluctuation,
exact counts and bunch splitting.  End to end: f2k muon segments and cascades through the
device front end and the kernel against the same sources through the host front end."""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

from ppc_b200 import types as T  # noqa: E402
from ppc_b200.api import PPC, f2k_sources  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
TYPES = [0, 1, 10, 11, 12, 13, 14, 101, 102, 103, 104, 105, 106, 107]


@pytest.fixture(scope="module")
def ctx(ice_full):
    c = PPC()
    c.initialize(1.0, ice_full)
    c.set_seed(9)
    c.choose(0)
    c.ini()
    yield c
    c.close()


def _particles(specs):
    src = np.zeros(len(specs), T.SOURCE_DTYPE)
    for k, (E, dr, type_, scale) in enumerate(specs):
        src[k] = T.source(T.SRC_PARTICLE, (1.0 * k, -2.0, 3.0, 4.0 * k), (0.6, 0.0, 0.8), E, dr, type_, scale,
                          q=k + 1)[0]
    return src


def _reference_yield(ice, specs, tmp_path):
    if not os.path.exists(HARNESS):
        pytest.skip("reference harness not built")
    a = np.array(specs, [("E", "<f4"), ("dr", "<f4"), ("type", "<i4"), ("scale", "<f4")])
    a.tofile(tmp_path / "src.bin")
    env = dict(os.environ, PPCTABLESDIR=ice + "/")
    subprocess.run([HARNESS, "yield", str(tmp_path / "src.bin"), str(tmp_path / "out.bin")], env=env, check=True,
                   capture_output=True, timeout=120)
    return np.fromfile(tmp_path / "out.bin", np.float32).reshape(-1, 6)  # mean, f, a, b, length, yield


def test_bunch_templates_match_the_reference(ctx, ice_full, tmp_path):
    specs = [(E, dr, t, s) for t in TYPES for E, dr, s in [(0.05, 0.0, 1.0), (3.0, 0.0, 1.0), (250.0, 0.0, 0.5),
                                                         (4e4, 12.5, 2.0)]]
    ref = _reference_yield(ice_full, specs, tmp_path)
    src = _particles(specs)
    b, bstart, num = ctx.sources(src, seed=1)
    # every source with photons made exactly one bunch, in source order
    assert np.array_equal(bstart[1:] - bstart[:-1], b["num"]) and bstart[-1] == num
    k = b["q"] - 1
    u = b["u"].view(np.float32)
    assert np.array_equal(b["type"], -np.array([s[2] for s in specs])[k])
    np.testing.assert_allclose(b["f"], ref[k, 1], rtol=2e-6, atol=0)
    np.testing.assert_allclose(u[:, 0], ref[k, 2], rtol=2e-6, atol=1e-7)  # a
    np.testing.assert_allclose(u[:, 1], ref[k, 3], rtol=2e-6, atol=0)     # b
    np.testing.assert_allclose(b["n"][:, 3], ref[k, 4], rtol=0, atol=0)   # length
    assert np.all(u[:, 2] == 1) and np.all(u[:, 3] == 0)                 # beta, tau
    assert np.array_equal(b["r"], src["r"][k]) and np.allclose(b["n"][:, :3], [0.6, 0.0, 0.8])


def _poisson_chi2(x, mu):
    from scipy import stats
    lo, hi = int(max(0, mu - 5 * math.sqrt(mu) - 2)), int(mu + 5 * math.sqrt(mu) + 3)
    edges = np.arange(lo, hi + 2) - 0.5
    obs, _ = np.histogram(x, edges)
    cdf = stats.poisson.cdf(edges[1:] - 0.5, mu) - stats.poisson.cdf(edges[:-1] - 0.5, mu)
    exp = cdf * len(x)
    m = exp > 5
    return stats.chisquare(obs[m], exp[m] * obs[m].sum() / exp[m].sum()).pvalue


@pytest.mark.parametrize("target", [3.0, 9.5, 40.0, 900.0])
def test_photon_counts_are_poisson(ctx, ice_full, tmp_path, target):
    """Both branches of the sampler (below 12: products of uniforms; above: rejection)."""
    base = _reference_yield(ice_full, [(1.0, 0.0, 11, 1.0)], tmp_path)[0, 0]  # mean per GeV
    E = target / base
    mu = float(_reference_yield(ice_full, [(E, 0.0, 11, 1.0)], tmp_path)[0, 0])
    n = 20000
    src = _particles([(E, 0.0, 11, 1.0)] * n)
    src["q"] = np.arange(1, n + 1)
    b, bstart, num = ctx.sources(src, seed=int(target * 7))
    counts = np.zeros(n, np.int64)
    counts[b["q"] - 1] = b["num"]
    assert num == counts.sum()
    assert abs(counts.mean() - mu) < 5 * math.sqrt(mu / n), (counts.mean(), mu)
    assert abs(counts.var() / mu - 1) < 5 * math.sqrt(2.0 / n) + 0.01
    assert _poisson_chi2(counts, mu) > 1e-4


def test_hadronic_light_fluctuation(ctx, ice_full, tmp_path):
    """Counts of a 30 GeV hadron: Poisson of mu0 f, f ~ N(F, dF) truncated to [0, 1.1]
    (gpu/f2k.cxx:150-156), mu0 the EM yield of the same energy."""
    from scipy import stats
    E = 30.0
    mu0 = float(_reference_yield(ice_full, [(E, 0.0, 11, 1.0)], tmp_path)[0, 0]) / 1000.0
    n = 20000
    src = _particles([(E, 0.0, 101, 1e-3)] * n)  # scaled down to keep the Poisson part visible
    src["q"] = np.arange(1, n + 1)
    b, _, _ = ctx.sources(src, seed=5)
    counts = np.zeros(n)
    counts[b["q"] - 1] = b["num"]
    e = max(np.float32(2.71828183), np.float32(E))
    E0, m, f0, rms0, gamma = 0.18791678, 0.16267529, 0.30974123, 0.95899551, 1.35589541
    F = 1 - (e / E0) ** -m * (1 - f0)
    dF = F * rms0 * math.log(e) ** -gamma
    tn = stats.truncnorm((0 - F) / dF, (1.1 - F) / dF, loc=F, scale=dF)
    mean = mu0 * tn.mean()
    var = mu0 * tn.mean() + mu0 ** 2 * tn.var()
    assert abs(counts.mean() - mean) < 5 * math.sqrt(var / n), (counts.mean(), mean)
    assert abs(counts.var() / var - 1) < 0.06, (counts.var(), var)


def test_exact_counts_split_bunches_and_empty_sources(ctx):
    src = np.concatenate([
        T.source(T.SRC_CLST, (0, 0, 0, 0), amount=5e9, dr=3.0, beta=0.9, q=1),
        T.source(T.SRC_POINT, (1, 1, 1, 2), amount=12345, q=2),
        T.source(T.SRC_PARTICLE, (0, 0, 0, 0), amount=100.0, dr=0.0, type_=0, q=3),  # muon without length: none
        T.source(T.SRC_MOPO, (2, 2, 2, 0), amount=2000.0, dr=7.0, beta=0.8, tau=3.0, fr=0.25, q=4),
    ])
    b, bstart, num = ctx.sources(src, seed=3)
    assert list(b["q"][:3]) == [1, 1, 1] and list(b["num"][:3]) == [2 ** 31, 2 ** 31, 5_000_000_000 - 2 ** 32]
    assert b["q"][3] == 2 and b["num"][3] == 12345 and b["type"][3] == 1 and b["n"][3, 3] == 1
    u = b["u"].view(np.float32)
    assert b["type"][0] == 0 and b["f"][0] == 1 and u[0, 2] == np.float32(0.9) and b["n"][0, 3] == 3
    assert 3 not in set(b["q"])
    m = b[b["q"] == 4]
    assert len(m) == 1 and m["f"][0] == np.float32(0.25) and m["n"][0, 3] == 7
    assert u[b["q"] == 4][0, 2] == np.float32(0.8) and u[b["q"] == 4][0, 3] == 3
    assert np.array_equal(np.diff(bstart.astype(np.int64)), b["num"].astype(np.int64)) and bstart[-1] == num
    assert num == 5_000_000_000 + 12345 + int(b["num"][4])
    with pytest.raises(Exception):  # flasher types need the host front end (flset)
        ctx.sources(T.source(T.SRC_PARTICLE, (0, 0, 0, 0), amount=1.0, type_=-1), seed=1)


F2K_EVENT = """TR 1 0 amu 10.0 -30.0 120.0 60.0 40.0 300.0 2000.0 0.0
TR 1 0 brems 60.0 0.0 100.0 60.0 40.0 0.0 800.0 150.0
TR 1 0 epair -20.0 -40.0 200.0 60.0 40.0 0.0 300.0 450.0
TR 1 0 hadr 0.0 -50.0 50.0 30.0 200.0 0.0 500.0 20.0
TR 1 0 e- -60.0 40.0 -80.0 120.0 100.0 0.0 1200.0 35.0
"""


def test_f2k_event_device_front_end_matches_host_front_end(ctx):
    """Five f2k sources, 40 repetitions each: photons and kernel-level hits from the device
    front end agree with the same sources through the host front end (addp + eout)."""
    src, _ = f2k_sources(F2K_EVENT)
    reps = 40
    many = np.tile(src, reps)
    b, bstart, num = ctx.sources(many, seed=77)
    hits_dev, info = ctx.propagate(b, cap=1 << 24)
    assert info["photons"] == num
    ctx.keep_raw(True)
    before = ctx.last_run()[1]["photons"]
    host_hits = 0
    for r in range(reps):
        for s in src:
            ctx.sett(float(s["n"][0]), float(s["n"][1]), float(s["n"][2]), (r, int(s["q"])), 0)
            ctx.addp(float(s["r"][0]), float(s["r"][1]), float(s["r"][2]), float(s["r"][3]), float(s["amount"]),
                     float(s["dr"]), int(s["type"]))
        ctx.eout()
        host_hits += len(ctx.raw_hits())
        ctx.efin()
    host_ph = ctx.last_run()[1]["photons"] - before  # photons of the host front end's runs
    ctx.keep_raw(False)
    assert abs(host_ph - num) < 6 * math.sqrt(2 * num) + 0.03 * num, (host_ph, num)
    assert abs(len(hits_dev) - host_hits) < 6 * math.sqrt(2 * host_hits) + 0.03 * host_hits, (len(hits_dev), host_hits)


def test_no_sources(ctx):
    b, bstart, num = ctx.sources(np.zeros(0, T.SOURCE_DTYPE), seed=1)
    assert len(b) == 0 and bstart.tolist() == [0] and num == 0
