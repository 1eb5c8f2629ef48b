"""Synthetic detector / ice configurations written in the reference's file formats
(doc/index.rst "Configuration files"; parsed by gpu/ini.cxx:578-1700).

Every configuration is generated from a fixed seed, so a directory is reproducible.
Workloads (sizes as used by the tests and the benchmark):

  small   7 strings (1 centre + 6 on a 125 m hexagon), 60 DOMs at 17 m from z=+503 to
          -500 m, 100 layers of 10 m, b_e(400) ~ U[0.02,0.08]/m, a_dust(400) ~
          U[0.005,0.02]/m (numpy default_rng(1)), HG g=0.9, no tilt, no anisotropy, no
          birefringence; isotropic 405 nm point source at the origin.
  small_xr1 `small` with DOMs at their true size (xR = 1 in cfg.txt instead of 5).
  full    86 strings (78 on a 125 m hexagonal lattice + 8 infill strings at ~70 m), 60
          DOMs each (5160), 171 layers of 10 m with smooth log-normal (sigma 0.3) b_e and
          a_dust profiles, 1-d tilt with a +-20 m sinusoidal dust-layer shift, absorption
          anisotropy of strength 0.08, birefringence diffusion; HG/SAM mix as in SPICE.
  full2d  the `full` detector and ice with a 2-d tilt map (tilt.set/tilt.map) instead,
          sensor axes a few degrees off vertical (cx.dat) and cable azimuths (dx.dat).
  full_ng the `full` configuration with multi-PMT sensors on strings 1-45 (om.conf,
          om.map, om.dirs, om.wv_*): 24-PMT spheres, 2-PMT spheroids and wavelength-
          shifting tubes, plus sensor axes and cable azimuths.

The ice-model constants (alpha, kappa, A, B of icemodel.par, the 12 birefringence
parameters of cfg.txt) are values of the same form and magnitude as the published SPICE
fits, chosen for these synthetic workloads.
"""
import math
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ZOFF = 1948.07
DATA = os.path.join(HERE, "data")


def multipliers_file(count=131072):
    """Path of rnd.txt with `count` MWC multipliers (generated once, cached)."""
    os.makedirs(DATA, exist_ok=True)
    out = os.path.join(DATA, f"rnd_{count}.txt")
    if os.path.exists(out):
        return out
    exe = os.path.join(HERE, "bin", "mwc_multipliers")
    if not os.path.exists(exe):
        os.makedirs(os.path.dirname(exe), exist_ok=True)
        subprocess.run(["gcc", "-O2", "-fopenmp", os.path.join(HERE, "csrc", "mwc_multipliers.c"), "-o", exe],
                       check=True)
    tmp = out + ".tmp"
    with open(tmp, "w") as f:
        subprocess.run([exe, str(count)], stdout=f, check=True)
    os.replace(tmp, out)
    return out


def _geo(path, strings, zs):
    with open(path, "w") as f:
        for s, (x, y) in strings:
            for k, z in enumerate(zs, start=1):
                f.write(f"SYN{s:03d}{k:02d}\t0x{(s << 8) | k:012x}\t{x:.2f}\t{y:.2f}\t{z - ZOFF:.2f}\t{s}\t{k}\n")


def _hexagon7():
    pts = [(0.0, 0.0)]
    for i in range(6):
        a = math.radians(60 * i)
        pts.append((125 * math.cos(a), 125 * math.sin(a)))
    return [(i + 1, p) for i, p in enumerate(pts)]


def _lattice86():
    """78 strings on a 125 m triangular lattice inside a hexagonal footprint, plus 8 infill."""
    pts = []
    for i in range(-6, 7):
        for j in range(-6, 7):
            x = 125 * (i + 0.5 * j)
            y = 125 * (math.sqrt(3) / 2) * j
            pts.append((math.hypot(x, y), x, y))
    pts.sort()
    main = [(x, y) for _, x, y in pts[:78]]
    infill = []
    for i in range(8):
        a = math.radians(45 * i + 10)
        infill.append((35 + 70 * math.cos(a) * (0.5 + 0.5 * (i % 2)), 25 + 70 * math.sin(a) * (0.5 + 0.5 * (i % 2))))
    return [(i + 1, p) for i, p in enumerate(main + infill)]


def _smooth(rng, n, sigma, corr=8):
    w = rng.normal(size=n + 4 * corr)
    k = np.exp(-0.5 * (np.arange(-2 * corr, 2 * corr + 1) / corr) ** 2)
    s = np.convolve(w, k / np.sqrt((k ** 2).sum()), mode="same")[2 * corr:2 * corr + n]
    return np.exp(sigma * s - sigma ** 2 / 2)


def _wv(path, lo=300.0, hi=600.0, step=10.0):
    """Cumulative emission x acceptance in wavelength (Cherenkov 1/lambda^2 times a smooth
    acceptance bump), tabulated as `fraction wavelength` from 0 to 1."""
    w = np.arange(lo, hi + step / 2, step)
    acc = np.exp(-0.5 * ((w - 420.0) / 70.0) ** 2)
    dens = acc / w ** 2
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (dens[1:] + dens[:-1]) * step)])
    cum /= cum[-1]
    with open(path, "w") as f:
        for c, x in zip(cum, w):
            f.write(f"{c:.8f} {x:.1f}\n")


_BFR = [0.0768, 5.4e5, 2.23, 0.00262, 0.0774, 1.55e6, 2.45, 0.00250, 0.00100, 0.248, 2.35, 1.68]


def write(kind, path, count=131072, xR=5):
    """Writes configuration `kind` (small | small_xr1 | small_tilt | small_hole | full |
    full2d | full_ng) into directory `path`."""
    if kind == "small_xr1":  # the 7-string detector with DOMs at their true size
        kind, xR = "small", 1
    os.makedirs(path, exist_ok=True)
    shutil.copyfile(multipliers_file(count), os.path.join(path, "rnd.txt"))
    with open(os.path.join(path, "icemodel.par"), "w") as f:
        f.write("0.90 0.03\n1.08 0.02\n6950.0 970.0\n6620.0 70.0\n")
    _wv(os.path.join(path, "wv.dat"))
    rng = np.random.default_rng(1)
    if kind in ("small", "small_tilt", "small_hole"):
        _geo(os.path.join(path, "geo-f2k"), _hexagon7(), [503.0 - 17.0 * k for k in range(60)])
        # 100 layers of 10 m covering z in [-500, 503]: depth = 1948.07 - z
        dp = 1445.0 + 10.0 * np.arange(100)
        be = rng.uniform(0.02, 0.08, 100)
        ba = rng.uniform(0.005, 0.02, 100)
        with open(os.path.join(path, "icemodel.dat"), "w") as f:
            for d, b, a in zip(dp, be, ba):
                f.write(f"{d:.2f} {b:.6f} {a:.6f} 0\n")
        with open(os.path.join(path, "cfg.txt"), "w") as f:
            if kind == "small_hole":
                # hole-ice column of 8 DOM radii around each string: effective scattering
                # length 0.5 m, absorption length 100 m, SAM fraction 0.35, g = 0.5
                f.write(f"{xR}\n1.0\n0\n0.9\n130\n0\n0\n8.0\n0.5\n100.0\n0.35\n0.5\n")
            else:
                f.write(f"{xR}\n1.0\n0\n0.9\n")
        with open(os.path.join(path, "as.dat"), "w") as f:
            f.write("1\n1\n")
        if kind == "small_tilt":
            _tilt1d(path, rng)
        return path
    # full detector
    _geo(os.path.join(path, "geo-f2k"), _lattice86(), [500.0 - 17.0 * k for k in range(60)])
    n = 171
    dp = 1100.0 + 10.0 * np.arange(n)
    base_be = 0.03 + 0.02 * np.exp(-0.5 * ((dp - 2000.0) / 40.0) ** 2)
    base_ba = 0.008 + 0.004 * np.exp(-0.5 * ((dp - 2000.0) / 40.0) ** 2)
    be = base_be * _smooth(rng, n, 0.3)
    ba = base_ba * _smooth(rng, n, 0.3)
    td = rng.normal(0, 3, n)
    with open(os.path.join(path, "icemodel.dat"), "w") as f:
        for d, b, a, t in zip(dp, be, ba, td):
            f.write(f"{d:.2f} {b:.6f} {a:.6f} {t:.4f} 0 0 1 1\n")
    with open(os.path.join(path, "cfg.txt"), "w") as f:
        vals = [xR, 1.0, 0.35, 0.9, 130.0, 0.0, 0.0, 0.0, 0.03, 100, 0.35, 0.9, 0.08, -0.04, -0.04, 0.0] + _BFR
        f.write("# synthetic configuration, reference cfg.txt order\n")
        for v in vals:
            f.write(f"{v}\n")
    with open(os.path.join(path, "as.dat"), "w") as f:
        f.write("1.0\n0.35\n0.5\n0.15\n")
    if kind == "full2d":
        _tilt2d(path)
        _sensor_axes_and_cables(path, np.random.default_rng(7))
    else:
        _tilt1d(path, rng)
    if kind == "full_ng":
        _sensor_axes_and_cables(path, np.random.default_rng(8))
        _nextgen(path)
    return path


def _nextgen(path):
    """Multi-PMT sensors (om.conf, om.map, om.dirs, om.wv_<type>.0): strings 1-20 carry a
    24-PMT sphere, 21-35 a 2-PMT elongated spheroid, 36-45 a wavelength-shifting tube
    (a cylinder read out at both ends); the other strings keep standard DOMs."""
    with open(os.path.join(path, "om.conf"), "w") as f:
        f.write("msphere 1 0.0044 0.33 0.178 0.178 24 33.0 0.0 0.0\n")
        first = True
        for th, off in ((33.0, 0.0), (72.0, 30.0), (108.0, 0.0), (147.0, 30.0)):
            for k in range(6):
                if first:
                    first = False
                    continue
                f.write(f"{th} {off + 60.0 * k}\n")
        f.write("spheroid 2 0.010 0.33 0.15 0.27 2 0.0 0.0 15.0\n180.0 0.0\n")
        f.write("tube 3 0.020 -2 0.057 -0.45 1 0.0 0.0\n")
    with open(os.path.join(path, "om.map"), "w") as f:
        for s in range(1, 46):
            m = 1 if s <= 20 else 2 if s <= 35 else 3
            for om in range(1, 61):
                f.write(f"{s} {om} {m}\n")
    n = 642  # Fibonacci sphere
    k = np.arange(n) + 0.5
    z = 1 - 2 * k / n
    phi = np.pi * (1 + 5 ** 0.5) * k
    rxy = np.sqrt(1 - z * z)
    with open(os.path.join(path, "om.dirs"), "w") as f:
        for i in range(n):
            f.write(f"{i} {rxy[i] * np.cos(phi[i]):.7f} {rxy[i] * np.sin(phi[i]):.7f} {z[i]:.7f}\n")
    # acceptance curves scaled so that each module type registers a fraction of the light
    # comparable to a standard DOM's (integrated acceptance about 0.4-0.8 of it)
    for m, (peak, width, top) in {1: (400.0, 90.0, 18000.0), 2: (390.0, 80.0, 3600.0),
                                  3: (360.0, 60.0, 2100.0)}.items():
        with open(os.path.join(path, f"om.wv_{m}.0"), "w") as f:
            for w in np.arange(300.0, 601.0, 10.0):
                f.write(f"{w:.1f} {top * np.exp(-0.5 * ((w - peak) / width) ** 2):.4f}\n")


def _sensor_axes_and_cables(path, rng):
    """cx.dat: each DOM's axis, a few degrees off vertical (string om nx ny nz r);
    dx.dat: each DOM's cable azimuth in degrees (string om azimuth r)."""
    rows = [ln.split() for ln in open(os.path.join(path, "geo-f2k")) if ln.strip()]
    keys = [(int(r[5]), int(r[6])) for r in rows]
    with open(os.path.join(path, "cx.dat"), "w") as f:
        for s, om in keys:
            nx, ny = rng.normal(0.0, 0.03, 2)
            f.write(f"{s} {om} {nx:.6f} {ny:.6f} {np.sqrt(1.0 - nx * nx - ny * ny):.6f} 0.5\n")
    with open(os.path.join(path, "dx.dat"), "w") as f:
        for s, om in keys:
            f.write(f"{s} {om} {rng.uniform(-180.0, 180.0):.3f} 1.0\n")


def _tilt_shift(depth, r):
    return 20.0 * np.sin(2 * np.pi * (depth - 1200.0) / 500.0 + r / 400.0)


def _tilt1d(path, rng):
    """tilt.par: (string, distance along 225 deg); tilt.dat: depth + shift per map."""
    rs = [-500.0, -250.0, 0.0, 250.0, 500.0, 750.0]
    with open(os.path.join(path, "tilt.par"), "w") as f:
        for k, r in enumerate(rs):
            f.write(f"{k + 1} {r}\n")
    depths = 1200.0 + 10.0 * np.arange(125)
    with open(os.path.join(path, "tilt.dat"), "w") as f:
        for d in depths:
            f.write(f"{d:.2f} " + " ".join(f"{_tilt_shift(d, r):.4f}" for r in rs) + "\n")


def _tilt2d(path):
    """tilt.set: the two grid axes (9.3 and 129.3 deg); tilt.map: depth + shift per map."""
    mnum, mcut = (11, 10), (6, 5)
    with open(os.path.join(path, "tilt.set"), "w") as f:
        f.write(f"9.3 -610.0 125.0 {mnum[0]} {mcut[0]}\n129.3 -550.0 125.0 {mnum[1]} {mcut[1]}\n")
    size = sum(1 for j in range(mnum[1]) for i in range(mnum[0]) if i < j + mcut[0] and j < i + mcut[1])
    depths = 1200.0 + 10.0 * np.arange(125)
    with open(os.path.join(path, "tilt.map"), "w") as f:
        for d in depths:
            f.write(f"{d:.2f} " + " ".join(f"{_tilt_shift(d, 60.0 * m - 700.0):.4f}" for m in range(size)) + "\n")
