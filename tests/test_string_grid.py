"""The string-proximity pre-test of the DOM search (ppc_b200/csrc/strgrid.h) never skips a
search that could find something.

For random segments, the oracle runs the reference's string loop (gpu/pro.cu:577-672: the
search cells a segment touches, the cylinder test of each of their strings, and the
hole-ice column test); whenever a string passes either test, the product's pre-test
(the kernel's code, compiled for the host and called through ppcb_string_grid_probe) must
answer "may reach".  Segments are drawn near strings (where the tests matter), uniformly
over the detector, and near-vertical (the pre-test's distance-bound branch).  The
pre-test's selectivity is checked too: far from strings it lets almost every step skip
the search."""
import ctypes as C

import numpy as np
import pytest

import oracle_util as O
from ppc_b200._lib import lib
from ppc_b200.api import PPC


def _segments(rng, sc, n, mode):
    pos = np.zeros((n, 8), np.float32)
    if mode == "near":
        m = rng.integers(0, len(sc), n)
        rho = rng.uniform(0, 25, n)
        phi = rng.uniform(0, 2 * np.pi, n)
        pos[:, 0] = sc["x"][m] + rho * np.cos(phi)
        pos[:, 1] = sc["y"][m] + rho * np.sin(phi)
    else:
        pos[:, 0] = rng.uniform(-800, 800, n)
        pos[:, 1] = rng.uniform(-800, 800, n)
    pos[:, 2] = rng.uniform(-520, 520, n)
    d = rng.normal(size=(n, 3))
    if mode == "vertical":
        d[:, :2] *= 10.0 ** rng.uniform(-4, -1.5, (n, 1))
    d /= np.linalg.norm(d, axis=1)[:, None]
    pos[:, 4:7] = d
    L = rng.exponential(5.0, n)
    L[rng.random(n) < 0.1] *= 8  # a tail of long steps (the grid walk's size limits)
    pos[:, 7] = L
    return pos


def _probe(c, pos):
    out = np.zeros(len(pos), np.int32)
    r = lib().ppcb_string_grid_probe(c._c, pos.ctypes.data_as(C.c_void_p), len(pos), out.ctypes.data_as(C.c_void_p))
    assert r == 0, lib().ppcb_last_error()
    return out


@pytest.mark.parametrize("kind", ["small", "full", "full2d", "full_ng", "small_hole", "small_xr1"])
def test_pretest_never_skips_a_reachable_string(kind, request):
    c = PPC()
    c.initialize(1.0, request.getfixturevalue("ice_" + kind))
    tb = O.tables_from_product(c)
    L = O.lib()
    L.ppco_string_pass.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    sc = c.tables()["sc"][:c.params().nstr]
    rng = np.random.default_rng(2024)
    rates = {}
    for mode in ("near", "uniform", "vertical"):
        pos = _segments(rng, sc, 100_000, mode)
        exact = np.zeros((len(pos), 2), np.int32)
        L.ppco_string_pass(tb.tp, O.ptr(pos), len(pos), O.ptr(exact))
        may = _probe(c, pos)
        reach = (exact[:, 0] > 0) | (exact[:, 1] > 0)
        missed = np.flatnonzero(reach & (may == 0))
        assert len(missed) == 0, (mode, pos[missed[:3]], exact[missed[:3]])
        rates[mode] = (reach.mean(), may.mean())
        if mode == "near":
            assert reach.sum() > 100, "too few reachable segments to be discriminating"
    print(kind, {k: (round(a, 5), round(b, 5)) for k, (a, b) in rates.items()})
    # far from strings almost nothing goes to the full search
    assert rates["uniform"][1] < 0.02, rates
    c.close()
