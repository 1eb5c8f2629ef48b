"""Source lists for the benchmark and tests, as bunch records (ppc_b200/types.py).

* cascade(...): one EM cascade (gamma longitudinal profile, gpu/f2k.cxx:68-79) whose mean
  yield at oversize xR is `photons` propagated photons.
* flasher(...): a flasher LED on an in-ice DOM set up like flset() with FLDR/ELEV
  (gpu/f2k.cxx:630-759): N-fold azimuthal pattern, 2-d Gaussian beam of 9.7 degrees.
* batched_events(...): N events, photon counts log-uniform in [lo, hi], half flashers on
  random DOMs (12-fold, 30 degrees elevation), half cascades at random vertices in
  |x|,|y|,|z| <= 500 m with random directions; one bunch per event, .q = event index.
"""
import math

import numpy as np

from . import types as T

FCV = math.pi / 180


def cascade(vertex, direction, photons, q=0, ppm=2450.08, xR=5, etype=11):
    E = photons * xR * xR / (ppm * 5.321 * 0.910 / 0.9216)
    logE = math.log(max(0.105658389, E))
    a = 2.01849 + 0.63176 * logE
    b = 0.39652 * 0.910 / 0.9216 / 0.63207
    return T.bunch_particle([vertex[0], vertex[1], vertex[2], 0.0], direction, q, photons, -etype, f=0.0, a=a, b=b)


def flasher(dom_index, dom_pos, photons, q=0, fldr=11 * 360.0, elev=30.0, fwid=9.7):
    up = np.float32(elev * FCV)
    xi = np.float32(fldr * FCV)
    n = [math.cos(up) * math.cos(xi), math.cos(up) * math.sin(xi), math.sin(up)]
    ka = np.float32(FCV * fwid) ** 2
    return T.bunch_led([dom_pos[0], dom_pos[1], dom_pos[2], 0.0], n, q, photons, 1, ka=ka, up=up, fldr=fldr,
                       fla=dom_index, ofla=dom_index)


def batched_events(oms, n_events=4096, lo=1e3, hi=1e7, seed=0, ppm=2450.08):
    """oms: the DOM table (structured array with field r) of the configuration."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(math.log(lo), math.log(hi), n_events)).astype(np.uint32)
    out = np.zeros(n_events, T.BUNCH_DTYPE)
    for e in range(n_events):
        if e % 2 == 0:
            k = int(rng.integers(0, len(oms)))
            out[e] = flasher(k, oms["r"][k], int(counts[e]), q=e)[0]
        else:
            v = rng.uniform(-500, 500, 3)
            ct = rng.uniform(-1, 1)
            ph = rng.uniform(0, 2 * math.pi)
            st = math.sqrt(1 - ct * ct)
            out[e] = cascade(v, [st * math.cos(ph), st * math.sin(ph), ct], int(counts[e]), q=e, ppm=ppm)[0]
    return out
