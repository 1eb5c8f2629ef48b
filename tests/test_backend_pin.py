"""The host back end (Session::print, the reference's print() of gpu/f2k.cxx:247-363) against
the reference's own back end, record for record and bit for bit: golden hit maps made by
tests/golden/make_golden.py from the reference compiled as its CPU build, over kernel-level
hits of the reference's own propagation.  Same hits, same host seed, so every random draw
(acceptance, PMT choice, the shifting tube's transit delay, wavelength) is shared.  Covers
standard sensors with cables and tilted axes, and the multi-PMT sensors of the nextgen
configuration: 24-PMT spheres, 2-PMT spheroids and wavelength-shifting tubes."""
import os

import numpy as np
import pytest

from ppc_b200.api import PPC

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {"full2d": "full2d", "full_ng_sphere": "full_ng", "full_ng_spheroid": "full_ng", "full_ng_tube": "full_ng"}
FIELDS = ("track_first", "track_second", "frame", "t0", "str", "om", "pmt", "dir", "time", "r", "n")


@pytest.mark.parametrize("case", list(CASES))
def test_host_back_end_matches_reference(case, request):
    g = np.load(os.path.join(GOLD, f"backend_{case}.npz"))
    c = PPC()
    c.initialize(1.0, request.getfixturevalue("ice_" + CASES[case]))
    c.set_seed(int(g["seed"]))
    c.sett(0.0, 0.0, 1.0, (3, 9), 0)
    c.back_end(g["hits"])
    got = c.hitz()
    want = g["hitz"]
    assert len(got) == len(want) > 50
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f
    if case != "full2d":
        assert len(np.unique(want["pmt"])) > 1  # several PMTs of a multi-PMT sensor
    if case == "full_ng_tube":
        tube = want[(want["str"] >= 36) & (want["str"] <= 45)]
        assert len(tube) > 30 and set(np.unique(tube["pmt"])) == {0, 1}  # the two ends of the tube
    c.close()


def test_back_end_drops_hits_of_earlier_segments():
    """As in print(): once hits of segment 2 went through, hits of segment 1 are dropped
    (the reference reports them as out of range); hits of the current segment still count."""
    g = np.load(os.path.join(GOLD, "backend_full2d.npz"))
    from conftest import _ice
    c = PPC()
    c.initialize(1.0, _ice("full2d"))
    c.set_seed(int(g["seed"]))
    c.sett(0.0, 0.0, 1.0, (3, 8), 0)
    c.sett(0.0, 0.0, 1.0, (3, 9), 0)
    h2 = g["hits"].copy()
    h2["n"] = 2
    c.back_end(h2[:300])
    n1 = len(c.hitz())
    assert n1 > 0 and set(c.hitz()["track_second"]) == {9}
    c.back_end(g["hits"])  # segment 1: dropped
    assert len(c.hitz()) == n1
    c.back_end(h2[300:])  # segment 2 again: accepted
    assert len(c.hitz()) > n1
    c.close()
